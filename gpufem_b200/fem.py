"""Host-side mirror of the reference's FEM / StiffAlgo / SPRmatrix interface for
the hot path, over the C-ABI (include/gpufem_b200.h).

Reference interface mirrored (fpaboim/gpufem):
  FEM            src/FEM/fem.h:34-86      Init, CalcStiffnessMat, ApplyConstraint,
                                           SetDeviceMode, SetUseColoring, GetFemData
  FemData        src/FEM/FemData.h:43-105 Init(format, n_gpts, E, Nu, fileIO) -> here
                                           Init from arrays (coords, connectivity,
                                           supports, loads)
  StiffAlgo      src/FEM/StiffAlgo.h:40-84 CalcGlobalStiffness(femdata) -> seconds,
                                           SetParallelColoring, SetMakeAssembly
  SPRmatrix/ELL  src/SPRmatrix/SPRmatrix.h:71-89, ELLmatrix.h:46-72
                                           GetElem, GetNNZ, GetMatSize, Axy, CG

Everything computes on the GPU through libgpufem_b200.so.  `Context` is the thin
owner of one gf_ctx; the reference-named classes sit on top of it.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import check, lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Context:
    """One gf_ctx: a CUDA stream plus all device memory of one problem."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = lib.gf_create(C.byref(h), device)
        if st != _lib.GF_OK:
            raise _lib.GpufemError(st, f"gf_create(device={device}) failed")
        self.h = h
        self.dim = 0
        self.n = 0

    def close(self) -> None:
        if getattr(self, "h", None):
            lib.gf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _c(self, st: int) -> None:
        check(st, self.h)

    # ---- mesh -----------------------------------------------------------
    def mesh_create(self, elem_type: int, coords: np.ndarray, conn: np.ndarray, ngauss: int,
                    E: float, E_elem: Optional[np.ndarray] = None, nu: float = 0.3,
                    analysis: int = _lib.GF_PLANE_STRESS) -> None:
        coords = np.ascontiguousarray(coords, np.float64)
        conn = np.ascontiguousarray(conn, np.int32)
        E_elem = None if E_elem is None else np.ascontiguousarray(E_elem, np.float64)
        nnodes = coords.shape[0]
        self._c(lib.gf_mesh_create(self.h, elem_type, nnodes, _ptr(coords), conn.shape[0],
                                   _ptr(conn), ngauss, float(E), _ptr(E_elem), float(nu),
                                   analysis))
        self.dim = coords.shape[1] if coords.ndim == 2 else (2 if elem_type < 2 else 3)
        self.n = nnodes * self.dim

    def set_modulus(self, E: float, E_elem: Optional[np.ndarray] = None) -> None:
        E_elem = None if E_elem is None else np.ascontiguousarray(E_elem, np.float64)
        self._c(lib.gf_mesh_set_modulus(self.h, float(E), _ptr(E_elem)))

    def color(self, colors: Optional[np.ndarray] = None) -> int:
        colors = None if colors is None else np.ascontiguousarray(colors, np.int32)
        nc = C.c_int32()
        self._c(lib.gf_mesh_color(self.h, _ptr(colors), C.byref(nc)))
        return nc.value

    def color_device(self, seed: int = 0) -> int:
        """Jones–Plassmann colouring on the device; returns the number of colours."""
        nc = C.c_int32(0)
        self._c(lib.gf_mesh_color_device(self.h, seed, C.byref(nc)))
        return nc.value

    def colors(self, nelem: int) -> np.ndarray:
        out = np.empty(nelem, np.int32)
        self._c(lib.gf_mesh_get_colors(self.h, _ptr(out)))
        return out

    def build_pattern(self):
        n, w, nnz = C.c_int32(), C.c_int32(), C.c_int64()
        self._c(lib.gf_ell_build_pattern(self.h, C.byref(n), C.byref(w), C.byref(nnz)))
        self.n = n.value
        return n.value, w.value, nnz.value

    def assemble(self, dtype: int = _lib.GF_F64, scatter: int = _lib.GF_SCATTER_COLOR,
                 engine: int = _lib.GF_ENGINE_CUDA_CORE) -> float:
        self._c(lib.gf_assemble(self.h, dtype, scatter, engine))
        return lib.gf_last_device_seconds(self.h)

    def convert_f64_to_f32(self) -> None:
        self._c(lib.gf_ell_convert_f64_to_f32(self.h))

    def ell_shape(self):
        n, w = C.c_int32(), C.c_int32()
        self._c(lib.gf_ell_view(self.h, _lib.GF_F64, C.byref(n), C.byref(w), None, None, None))
        return n.value, w.value

    def ell_download(self, dtype: int = _lib.GF_F64):
        n, w = self.ell_shape()
        rownnz = np.empty(n, np.int32)
        colidx = np.empty(n * w, np.int32)
        vals = np.empty(n * w, np.float64 if dtype == _lib.GF_F64 else np.float32)
        self._c(lib.gf_ell_download(self.h, dtype, _ptr(rownnz), _ptr(colidx), _ptr(vals)))
        return rownnz, colidx.reshape(w, n), vals.reshape(w, n)

    def ell_diagonal(self, dtype: int = _lib.GF_F64) -> np.ndarray:
        d = np.empty(self.n, np.float64)
        self._c(lib.gf_ell_diagonal(self.h, dtype, _ptr(d)))
        return d

    def ell_upload(self, rownnz: np.ndarray, colidx: np.ndarray, vals: np.ndarray) -> None:
        """colidx / vals: (width, n) column-major ELL as the reference stores it."""
        rownnz = np.ascontiguousarray(rownnz, np.int32)
        colidx = np.ascontiguousarray(colidx, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        w, n = colidx.shape
        self._c(lib.gf_ell_upload(self.h, n, w, _ptr(rownnz), _ptr(colidx), _ptr(vals)))
        self.n = n

    # ---- loads / constraints -------------------------------------------
    def set_supports(self, supports: np.ndarray) -> None:
        supports = np.ascontiguousarray(supports, np.int32)
        self._c(lib.gf_set_supports(self.h, supports.shape[0], _ptr(supports)))

    def set_nodal_loads(self, loads: np.ndarray) -> None:
        loads = np.ascontiguousarray(loads, np.float64)
        self._c(lib.gf_set_nodal_loads(self.h, loads.shape[0], _ptr(loads)))

    def set_force(self, f: np.ndarray) -> None:
        f = np.ascontiguousarray(f, np.float64)
        self._c(lib.gf_set_force(self.h, _ptr(f)))

    def get_force(self) -> np.ndarray:
        f = np.empty(self.n, np.float64)
        self._c(lib.gf_get_force(self.h, _ptr(f)))
        return f

    def apply_constraints(self, mode: int) -> None:
        self._c(lib.gf_apply_constraints(self.h, mode))

    # ---- solve ----------------------------------------------------------
    def spmv(self, x: np.ndarray, dtype: int = _lib.GF_F64) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(x)
        self._c(lib.gf_spmv_host(self.h, dtype, _ptr(x), _ptr(y)))
        return y

    def solve(self, solver: int = _lib.GF_SOLVER_PCG, matrix: int = _lib.GF_F64,
              tol: float = 1e-10, max_iter: int = 10000, inner_tol: float = 0.0,
              max_outer: int = 0, check_every: int = 0, max_seconds: float = 0.0,
              raise_on_error: bool = True) -> _lib.SolveInfo:
        o = _lib.SolveOpts(solver=solver, matrix=matrix, max_iter=max_iter, tol=tol,
                           inner_tol=inner_tol, max_outer=max_outer, check_every=check_every,
                           max_seconds=max_seconds)
        info = _lib.SolveInfo()
        st = lib.gf_solve(self.h, C.byref(o), C.byref(info))
        if raise_on_error:
            self._c(st)
        return info

    def solution(self) -> np.ndarray:
        u = np.empty(self.n, np.float64)
        self._c(lib.gf_get_solution(self.h, _ptr(u)))
        return u

    def residual_dd(self, u_hi: np.ndarray, u_lo: np.ndarray):
        """r = f - K64 (u_hi + u_lo) in double-double on the device (gf_residual_dd);
        returns (r rounded to FP64, ||r|| / ||f||)."""
        import torch
        dev = lambda a: torch.tensor(np.ascontiguousarray(a, np.float64), device="cuda")
        uh, ul = dev(u_hi), dev(u_lo)
        r = torch.empty_like(uh)
        rel = C.c_double()
        torch.cuda.synchronize()
        self._c(lib.gf_residual_dd(self.h, C.c_void_p(uh.data_ptr()), C.c_void_p(ul.data_ptr()),
                                   C.c_void_p(r.data_ptr()), C.byref(rel)))
        return r.cpu().numpy(), rel.value

    def refine_dd(self, solver: int = _lib.GF_SOLVER_PCG, matrix: int = _lib.GF_F64,
                  inner_tol: float = 1e-8, target: float = 1e-16, max_steps: int = 8,
                  max_iter: int = 400000):
        """Iterative refinement of K64 u = f with the solution held in double-double:
        r = f - K (u_hi + u_lo) exactly enough (gf_residual_dd), K d = r solved by `solver`
        to `inner_tol`, (u_hi, u_lo) += d by exact two-sums, until ||r|| / ||f|| <= target
        or the residual stops falling.  The context's force vector is restored afterwards.
        Returns (u_hi, u_lo, info) with the residual history, the relative size of the last
        correction and the inner iterations."""
        f = self.get_force()
        u_hi = np.zeros(self.n)
        u_lo = np.zeros(self.n)
        hist, inner, corr = [], [], []
        try:
            for _ in range(max_steps + 1):
                if hist:
                    self.set_force(f)             # the residual is always against f
                r, rel = self.residual_dd(u_hi, u_lo)
                hist.append(rel)
                if rel <= target or (len(hist) > 2 and rel >= 0.5 * hist[-2]):
                    break
                if len(hist) > max_steps:
                    break
                self.set_force(r)
                info = self.solve(solver, matrix, tol=inner_tol, max_iter=max_iter,
                                  raise_on_error=False)
                d = self.solution()
                inner.append(int(info.iterations))
                s = u_hi + d                      # TwoSum(u_hi, d) = s + e exactly
                bb = s - u_hi
                e = (u_hi - (s - bb)) + (d - bb)
                lo = u_lo + e
                u_hi = s + lo                     # renormalise (FastTwoSum, |s| >= |lo|)
                u_lo = lo - (u_hi - s)
                nu = np.linalg.norm(u_hi)
                corr.append(float(np.linalg.norm(d) / nu) if nu > 0 else 0.0)
        finally:
            self.set_force(f)
        return u_hi, u_lo, {"rel_residual_history": hist, "inner_iterations": inner,
                            "correction_history": corr}

    # ---- learned preconditioner ------------------------------------------
    def lp_init(self, dim: int, seed: int = 0) -> None:
        self._c(lib.gf_lp_init(self.h, dim, seed))
        self.lp_dim = dim

    def lp_num_params(self, dim: int) -> int:
        return int(lib.gf_lp_num_params(dim))

    def lp_get_weights(self) -> np.ndarray:
        w = np.empty(self.lp_num_params(self.lp_dim), np.float32)
        self._c(lib.gf_lp_get_weights(self.h, _ptr(w)))
        return w

    def lp_set_weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, np.float32)
        self._c(lib.gf_lp_set_weights(self.h, _ptr(w)))

    def lp_set_coarse(self, on: bool) -> None:
        self._c(lib.gf_lp_set_coarse(self.h, 1 if on else 0))

    def lp_set_loss(self, loss: int) -> None:
        """GF_LP_LOSS_ERROR or GF_LP_LOSS_RESIDUAL."""
        self._c(lib.gf_lp_set_loss(self.h, loss))

    def lp_collect(self, npairs: int, every: int, tol: float = 1e-6, max_iter: int = 100000) -> None:
        self._c(lib.gf_lp_collect(self.h, npairs, every, tol, max_iter))

    def lp_collect_random(self, npairs: int, seed: int = 0) -> None:
        self._c(lib.gf_lp_collect_random(self.h, npairs, seed))

    def lp_train(self, steps: int, batch: int = 4, lr: float = 1e-3, seed: int = 0) -> float:
        loss = C.c_float()
        self._c(lib.gf_lp_train(self.h, steps, batch, lr, seed, C.byref(loss)))
        return loss.value

    def _dev(self, a: np.ndarray):
        import torch
        return torch.tensor(np.ascontiguousarray(a, np.float32), device="cuda")

    def lp_apply(self, r: np.ndarray) -> np.ndarray:
        import torch
        rd = self._dev(r)
        zd = torch.empty_like(rd)
        torch.cuda.synchronize()
        self._c(lib.gf_lp_apply(self.h, C.c_void_p(rd.data_ptr()), C.c_void_p(zd.data_ptr())))
        return zd.cpu().numpy()

    def lp_loss_grad(self, r: np.ndarray, e: np.ndarray):
        import torch
        rd, ed = self._dev(r), self._dev(e)
        g = np.empty(self.lp_num_params(self.lp_dim), np.float32)
        loss = C.c_float()
        torch.cuda.synchronize()
        self._c(lib.gf_lp_loss_grad(self.h, C.c_void_p(rd.data_ptr()), C.c_void_p(ed.data_ptr()),
                                    C.byref(loss), _ptr(g)))
        return loss.value, g

    # ---- two-level preconditioner -----------------------------------------
    def twolevel_setup(self, target_coarse: int = 0) -> int:
        nc = C.c_int32()
        self._c(lib.gf_twolevel_setup(self.h, target_coarse, C.byref(nc)))
        return nc.value

    def twolevel_apply(self, r: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(r, np.float64)
        z = np.empty_like(r)
        self._c(lib.gf_twolevel_apply(self.h, _ptr(r), _ptr(z)))
        return z

    def twolevel_aggregates(self):
        agg = np.empty(self.n // self.dim, np.int32)
        s = C.c_double()
        self._c(lib.gf_twolevel_aggregates(self.h, _ptr(agg), C.byref(s)))
        return agg, s.value

    def launches(self) -> int:
        return int(lib.gf_kernel_launches(self.h))

    def sync(self) -> None:
        self._c(lib.gf_sync(self.h))

    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer (torch.cuda.ExternalStream takes it)."""
        h = C.c_void_p()
        self._c(lib.gf_stream(self.h, C.byref(h)))
        return int(h.value or 0)


# ---------------------------------------------------------------------------
# Reference-named mirror
# ---------------------------------------------------------------------------
class FemData:
    """Mesh, material, Gauss rule, supports and loads (FemData::Init,
    src/FEM/FemData.cc:122-194), from arrays instead of a FileIO."""

    def Init(self, elem_type: int, coords, conn, n_gpts: int, E: float, Nu: float,
             supports=None, nodal_loads=None, E_elem=None,
             analysis: int = _lib.GF_PLANE_STRESS) -> None:
        self.elem_type = elem_type
        self.coords = np.ascontiguousarray(coords, np.float64)
        self.conn = np.ascontiguousarray(conn, np.int32)
        self.n_gpts = n_gpts
        self.E = E
        self.Nu = Nu
        self.E_elem = E_elem
        self.analysis = analysis
        self.supports = supports
        self.nodal_loads = nodal_loads
        self.stiffness: Optional[ELLmatrixCUDA] = None
        self.displacements: Optional[np.ndarray] = None

    def InitFromFile(self, nf_path: str, n_gpts: int, E: float, Nu: float,
                     E_elem=None) -> None:
        """FemData::Init with a FileIO that has read a neutral file (FileIO::ReadNF,
        src/Utils/fileIO.cc:73-404); see gpufem_b200.nf."""
        from .nf import read_nf
        m = read_nf(nf_path)
        loads = m.loads if m.loads.shape[0] else None
        self.Init(m.elem_type, m.coords, m.conn, n_gpts, E, Nu, supports=m.supports,
                  nodal_loads=loads, E_elem=E_elem)

    def GetStiffnessMatrix(self) -> "ELLmatrixCUDA":
        return self.stiffness

    def GetDisplVector(self) -> Optional[np.ndarray]:
        return self.displacements


class ELLmatrixCUDA:
    """Device-resident ELL matrix (SPRmatrix interface, ELLmatrix.h:46-72)."""

    def __init__(self, ctx: Context, dtype: int = _lib.GF_F64):
        self.ctx = ctx
        self.dtype = dtype
        self._host = None

    def _download(self):
        if self._host is None:
            self._host = self.ctx.ell_download(self.dtype)
        return self._host

    def invalidate(self) -> None:
        self._host = None

    def GetMatDim(self) -> int:
        return self.ctx.ell_shape()[0]

    def GetElem(self, row: int, col: int) -> float:
        n, w = self.ctx.ell_shape()
        if row < 0 or row >= n or col < 0 or col >= n:
            return 0.0
        rownnz, colidx, vals = self._download()
        for s in range(rownnz[row]):
            if colidx[s, row] == col:
                return float(vals[s, row])
        return 0.0

    def GetNNZ(self) -> int:
        rownnz, colidx, vals = self._download()
        mask = np.arange(colidx.shape[0])[:, None] < rownnz[None, :]
        return int(np.count_nonzero(vals[mask]))

    def GetMatSize(self) -> int:
        n, w = self.ctx.ell_shape()
        return n * w * (8 if self.dtype == _lib.GF_F64 else 4) + n * w * 4

    def Axy(self, x: np.ndarray) -> np.ndarray:
        return self.ctx.spmv(x, self.dtype)

    def CG(self, vector_B: np.ndarray, n_iterations: int = 10000, epsilon: float = 1e-4,
           preconditioned: bool = False) -> np.ndarray:
        """Plain CG from x0 = 0, stop at ||r|| <= eps ||b|| (SPRmatrix::CPU_CG,
        SPRmatrix.cc:405-480); Jacobi-preconditioned when asked."""
        self.ctx.set_force(np.asarray(vector_B, np.float64))
        solver = _lib.GF_SOLVER_PCG if preconditioned else _lib.GF_SOLVER_CG
        info = self.ctx.solve(solver=solver, matrix=self.dtype, tol=epsilon,
                              max_iter=n_iterations, raise_on_error=False)
        if info.status not in (_lib.GF_OK, _lib.GF_ERR_NOT_CONVERGED):
            check(info.status, self.ctx.h)
        self.last_info = info
        return self.ctx.solution()


class StiffAlgoCUDA:
    """StiffAlgo strategy that assembles on the GPU (StiffAlgo.h:40-84)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.m_assemble = True
        self.m_usecoloring = True
        self.dtype = _lib.GF_F64

    def SetParallelColoring(self, usecoloring: bool) -> None:
        self.m_usecoloring = bool(usecoloring)

    def GetParallelColoring(self) -> bool:
        return self.m_usecoloring

    def SetMakeAssembly(self, assemble: bool) -> None:
        self.m_assemble = bool(assemble)

    def GetMakeAssembly(self) -> bool:
        return self.m_assemble

    def CalcGlobalStiffness(self, femdata: FemData) -> float:
        scatter = _lib.GF_SCATTER_COLOR if self.m_usecoloring else _lib.GF_SCATTER_ATOMIC
        secs = self.ctx.assemble(self.dtype, scatter)
        femdata.stiffness = ELLmatrixCUDA(self.ctx, self.dtype)
        return secs


class FEM:
    """FEM facade (src/FEM/fem.h:34-86).  DeviceMode GPU maps to StiffAlgoCUDA."""
    CPU, OMP, GPUOMP, GPU = 0, 1, 2, 3
    PEN, SUB = 0, 1

    def __init__(self, device: int = 0):
        self.ctx = Context(device)
        self.m_femdata: Optional[FemData] = None
        self.m_stiffnessalgo: Optional[StiffAlgoCUDA] = None

    def Init(self, assemble: bool = True, devicemode: int = 3) -> None:
        if devicemode != FEM.GPU:
            raise ValueError("this implementation provides only the GPU strategy; the CPU "
                             "strategies are the reference's own code")
        self.m_femdata = FemData()
        self.m_stiffnessalgo = StiffAlgoCUDA(self.ctx)
        self.m_stiffnessalgo.SetMakeAssembly(assemble)

    def GetFemData(self) -> FemData:
        return self.m_femdata

    def SetUseColoring(self, usecolor: bool) -> None:
        self.m_stiffnessalgo.SetParallelColoring(usecolor)

    def SetPrecision(self, dtype: int) -> None:
        self.m_stiffnessalgo.dtype = dtype

    def _upload(self) -> None:
        fd = self.m_femdata
        self.ctx.mesh_create(fd.elem_type, fd.coords, fd.conn, fd.n_gpts, fd.E, fd.E_elem,
                             fd.Nu, fd.analysis)
        if fd.supports is not None:
            self.ctx.set_supports(fd.supports)
        if fd.nodal_loads is not None:
            self.ctx.set_nodal_loads(fd.nodal_loads)
        self._uploaded = True

    def CalcStiffnessMat(self) -> float:
        if not getattr(self, "_uploaded", False):
            self._upload()
        return self.m_stiffnessalgo.CalcGlobalStiffness(self.m_femdata)

    def ApplyConstraint(self, conmode: int) -> None:
        mode = _lib.GF_BC_PENALTY if conmode == FEM.PEN else _lib.GF_BC_ELIMINATION
        self.ctx.apply_constraints(mode)
        if self.m_femdata.stiffness is not None:
            self.m_femdata.stiffness.invalidate()

    def Solve(self, n_iterations: int = 3000, epsilon: float = 1e-3,
              preconditioned: bool = False) -> np.ndarray:
        """CG on the assembled matrix with the force vector (interface.cpp:304-328)."""
        f = self.ctx.get_force()
        u = self.m_femdata.stiffness.CG(f, n_iterations, epsilon, preconditioned)
        self.m_femdata.displacements = u
        return u
