"""ctypes binding of libgpufem_b200.so (the C-ABI in include/gpufem_b200.h).

The shared library is the only compute path: if it is missing and cannot be
built, importing this module raises — there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libgpufem_b200.so"

GF_OK, GF_ERR_INVALID_ARG, GF_ERR_OOM, GF_ERR_NOT_CONVERGED = 0, 1, 2, 3
GF_ERR_STALLED, GF_ERR_CUDA, GF_ERR_STATE, GF_ERR_UNSUPPORTED = 4, 5, 6, 7
STATUS_NAMES = {0: "GF_OK", 1: "GF_ERR_INVALID_ARG", 2: "GF_ERR_OOM", 3: "GF_ERR_NOT_CONVERGED",
                4: "GF_ERR_STALLED", 5: "GF_ERR_CUDA", 6: "GF_ERR_STATE", 7: "GF_ERR_UNSUPPORTED"}

GF_Q4, GF_Q8, GF_BRICK8, GF_BRICK20 = 0, 1, 2, 3
GF_PLANE_STRESS, GF_PLANE_STRAIN = 0, 1
GF_F64, GF_F32 = 0, 1
GF_SCATTER_COLOR, GF_SCATTER_ATOMIC, GF_SCATTER_OWNER, GF_SCATTER_AUTO = 0, 1, 2, 3
GF_ENGINE_CUDA_CORE, GF_ENGINE_TF32_MMA = 0, 1
GF_BC_PENALTY, GF_BC_ELIMINATION = 0, 1
GF_SOLVER_CG, GF_SOLVER_PCG, GF_SOLVER_MIXED_PCG, GF_SOLVER_LEARNED_FCG, GF_SOLVER_MIXED_PCG32 = 0, 1, 2, 3, 4
GF_SOLVER_TWOLEVEL_PCG, GF_SOLVER_TWOLEVEL_PCG32 = 5, 6
GF_LP_LOSS_ERROR, GF_LP_LOSS_RESIDUAL = 0, 1


class SolveOpts(C.Structure):
    _fields_ = [("solver", C.c_int32), ("matrix", C.c_int32), ("max_iter", C.c_int32),
                ("tol", C.c_double), ("inner_tol", C.c_double), ("max_outer", C.c_int32),
                ("check_every", C.c_int32), ("max_seconds", C.c_double)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("outer", C.c_int32), ("fallback", C.c_int32),
                ("status", C.c_int32), ("rel_residual", C.c_double), ("seconds", C.c_double)]


P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
D = C.c_double

# name -> (restype, argtypes); kept in the order of include/gpufem_b200.h
# callbacks of the sharded solve (gf_dist_pcg): collectives enqueued on the given stream
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p)
HALO_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p)

SIGNATURES = {
    "gf_create": (I32, [C.POINTER(P), I32]),
    "gf_destroy": (I32, [P]),
    "gf_last_error": (C.c_char_p, [P]),
    "gf_version": (C.c_char_p, []),
    "gf_last_device_seconds": (D, [P]),
    "gf_last_assembly_split": (I32, [P, C.POINTER(D), C.POINTER(D)]),
    "gf_kernel_launches": (I64, [P]),
    "gf_sync": (I32, [P]),
    "gf_stream": (I32, [P, C.POINTER(C.c_void_p)]),
    "gf_mesh_create": (I32, [P, I32, I32, P, I32, P, I32, D, P, D, I32]),
    "gf_mesh_set_modulus": (I32, [P, D, P]),
    "gf_mesh_color": (I32, [P, P, C.POINTER(I32)]),
    "gf_mesh_color_device": (I32, [P, C.c_uint64, C.POINTER(I32)]),
    "gf_mesh_get_colors": (I32, [P, P]),
    "gf_ell_build_pattern": (I32, [P, C.POINTER(I32), C.POINTER(I32), C.POINTER(I64)]),
    "gf_assemble": (I32, [P, I32, I32, I32]),
    "gf_ell_convert_f64_to_f32": (I32, [P]),
    "gf_ell_view": (I32, [P, I32, C.POINTER(I32), C.POINTER(I32), C.POINTER(P), C.POINTER(P),
                          C.POINTER(P)]),
    "gf_ell_version": (I32, [P, I32, C.POINTER(I64)]),
    "gf_ell_download": (I32, [P, I32, P, P, P]),
    "gf_ell_upload": (I32, [P, I32, I32, P, P, P]),
    "gf_ell_diagonal": (I32, [P, I32, P]),
    "gf_set_supports": (I32, [P, I32, P]),
    "gf_set_nodal_loads": (I32, [P, I32, P]),
    "gf_set_force": (I32, [P, P]),
    "gf_get_force": (I32, [P, P]),
    "gf_apply_constraints": (I32, [P, I32]),
    "gf_spmv": (I32, [P, I32, P, P]),
    "gf_spmv_host": (I32, [P, I32, P, P]),
    "gf_solve": (I32, [P, C.POINTER(SolveOpts), C.POINTER(SolveInfo)]),
    "gf_dist_set_halo": (I32, [P, I32, I32, P, I32, P]),
    # the callbacks pass as plain pointers: C.cast(ALLREDUCE_FN(f), C.c_void_p)
    "gf_dist_pcg": (I32, [P, C.POINTER(SolveOpts), P, P, P, C.POINTER(SolveInfo)]),
    "gf_get_solution": (I32, [P, P]),
    "gf_residual_dd": (I32, [P, P, P, P, C.POINTER(D)]),
    "gf_solution_view": (I32, [P, C.POINTER(P)]),
    "gf_lp_num_params": (I64, [I32]),
    "gf_lp_init": (I32, [P, I32, C.c_uint64]),
    "gf_lp_get_weights": (I32, [P, P]),
    "gf_lp_set_weights": (I32, [P, P]),
    "gf_lp_collect": (I32, [P, I32, I32, D, I32]),
    "gf_lp_train": (I32, [P, I32, I32, C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "gf_lp_apply": (I32, [P, P, P]),
    "gf_lp_set_coarse": (I32, [P, I32]),
    "gf_lp_set_loss": (I32, [P, I32]),
    "gf_lp_collect_random": (I32, [P, I32, C.c_uint64]),
    "gf_lp_loss_grad": (I32, [P, P, P, C.POINTER(C.c_float), P]),
    "gf_twolevel_setup": (I32, [P, I32, C.POINTER(I32)]),
    "gf_twolevel_apply": (I32, [P, P, P]),
    "gf_twolevel_aggregates": (I32, [P, P, C.POINTER(D)]),
    "gf_pcg_noalloc": (I32, [I32, I32, P, P, P, P, P, D, I32, P, C.POINTER(I32),
                             C.POINTER(D)]),
}
GF_PCG_NOALLOC_MAX_N = 262144


def _load() -> C.CDLL:
    if not LIB_PATH.exists() or os.environ.get("GPUFEM_REBUILD"):
        from . import build as _build  # compiles with nvcc; raises if the toolkit is absent
        _build.build()
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class GpufemError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def check(status: int, ctx=None) -> None:
    if status != GF_OK:
        msg = lib.gf_last_error(ctx).decode() if ctx else ""
        raise GpufemError(status, msg)
