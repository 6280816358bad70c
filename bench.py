"""Benchmark of the hot path on B200: stiffness assembly throughput (elements/s)
on the Q8 512x512 workload, plus the time to solve it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--config q8_512]
  python bench.py --impl reference ...     # the reference's CPU path on host cores

One JSON line on rank 0.  `value` = elements assembled per second with inputs
resident in HBM (device time of gf_assemble with the owner-computes schedule: the
per-element geometry kernel and the owner kernel that writes every K entry once, FP32),
L2 flushed between steps; the colour, atomic and TF32 tensor-core variants are timed
beside it.  `e2e` = the same metric through the public C-ABI from pinned host buffers:
mesh upload, pattern, assembly and download of the ELL matrix, every step.  For N > 1 each
rank assembles its own replica of the workload (weak scaling; the assembly needs
no exchange) and the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "elems/s assembled"
SOLVERS = ["pcg_fp64", "mixed_pcg", "mixed_pcg32", "twolevel_pcg", "twolevel_pcg_k32",
           "twolevel_pcg32", "learned"]
UNIT = "elements/s"
WORKLOADS = {
    # name: (description, dtype of the timed assembly)
    "q8_512": "Q8 512x512 plane stress, jitter 0.15h, 3x3 Gauss, log-normal E (sigma 0.5), "
              "FP32 owner-computes assembly into ELL",
    "q4_64": "Q4 64x64 plane stress, jitter 0.2h, 2x2 Gauss, FP64 assembly",
    "brick8_128": "Brick8 128^3, jitter 0.1h, 2x2x2 Gauss, FP32 assembly",
    "brick20_64": "Brick20 64^3, jitter 0.05h, 3x3x3 Gauss, correlated log-normal E, FP32",
}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML every 5 ms while the timed
    region runs (read-only queries; nothing about the GPU is changed)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = None
        self._thread = None
        self.error = None

    def __enter__(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            dev_index = self.device
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            if vis:
                try:
                    dev_index = int(vis.split(",")[self.device])
                except ValueError:
                    pass
            h = pynvml.nvmlDeviceGetHandleByIndex(dev_index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        except Exception as exc:  # NVML unavailable: report it, keep benchmarking
            self.error = str(exc)
            return self
        self._stop = threading.Event()

        def loop():
            while not self._stop.is_set():
                try:
                    self.samples.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                    r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    for nm, bit in self.REASONS.items():
                        if r & bit:
                            self.reasons.add(nm)
                except Exception:
                    pass
                self._stop.wait(0.005)

        self._thread = threading.Thread(target=loop, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=2)

    def summary(self):
        if self.error:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [f"nvml: {self.error}"]}
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own CPU assembly on a bounded sample
# ---------------------------------------------------------------------------
class stdout_to_stderr:
    """The reference's C code reports progress with printf: fd 1 goes to stderr while it
    runs, so that stdout carries the bench's JSON line alone."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *exc):
        C.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def reference_sample(config: str, steps: int, warmup: int, scale: float = 1.0):
    """Time the reference's StiffAlgoCPU (naive, OpenMP critical scatter, FP32 as
    shipped) on the workload mesh (scale 1: the full mesh); elements/s per step.  Falls
    back to the single-threaded C oracle port when the reference build is absent."""
    from gpufem_b200 import meshgen as mg
    from oracle.oracle import Oracle, Reference
    m = mg.workload(config, scale=scale)
    cores = os.cpu_count() or 1
    times = []
    if Reference.available("fp32"):
        kind = "reference"
        R = Reference("fp32")
        s = R.open_mesh(m)
        for i in range(warmup + steps):
            t = s.assemble(coloring=False, nthreads=cores)
            if i >= warmup:
                times.append(t)
        s.close()
        sample = (f"{mg.NAMES[m.elem_type]} {'x'.join(map(str, m.n))} ({m.nelem} elements): "
                  f"reference StiffAlgoCPU naive, FP32, {cores} OpenMP threads, {steps} steps "
                  f"after {warmup} warm-up; E scalar (the reference's FemData holds one "
                  f"modulus; Ke scales linearly in E, so the work per element is the same)")
    else:
        kind = "port"
        cores = 1
        O = Oracle()
        pat = O.pattern(m.elem_type, m.nnodes, m.conn)
        for i in range(warmup + steps):
            t0 = time.perf_counter()
            O.assemble(m.elem_type, m.ngauss, m.coords, m.conn, m.E0, m.nu, E_elem=m.E, pattern=pat)
            if i >= warmup:
                times.append(time.perf_counter() - t0)
        sample = (f"{mg.NAMES[m.elem_type]} {'x'.join(map(str, m.n))} ({m.nelem} elements): "
                  f"C oracle port, FP64, 1 thread")
    t = float(np.mean(times))   # whole-run throughput, as the GPU arm reports it
    return {"value": m.nelem / t, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
            "cpu": cpu_model(), "seconds_per_step": t}


def reference_cg_sample(m, iters: int = 20):
    """The reference's own flow on the full workload mesh (FP32 build as shipped):
    ReadNF -> StiffAlgoCPU (naive, all cores) -> ApplyConstraint(PEN) -> CPU_CG in
    DEV_OMP for `iters` iterations.  Returns the full-size assembly rate and the CG time
    per iteration; None without the reference build."""
    from oracle.oracle import Reference
    if not Reference.available("fp32"):
        return None
    cores = os.cpu_count() or 1
    s = Reference("fp32").open_mesh(m)
    try:
        t_asm = s.assemble(coloring=False, nthreads=cores)
        s.penalty()
        _, t_cg = s.cg(iters, 1e-30, nthreads=cores)   # eps far below reach: exactly iters
    finally:
        s.close()
    return {"assembly_elements_per_s": m.nelem / t_asm, "cg_us_per_iteration": t_cg / iters * 1e6,
            "cg_iterations_timed": iters, "threads": cores, "cpu": cpu_model()}


def workload_config(cfg: str, m, world: int) -> dict:
    """The `config` object both arms print for workload `cfg` (mesh-derived only)."""
    return {"workload": cfg, "description": WORKLOADS[cfg], "elements": m.nelem,
            "nodes": m.nnodes, "dofs": m.ndof, "parallelism": f"replicas x{world}"}


def run_reference_arm(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return
    from gpufem_b200 import meshgen as mg
    steps, warm = args.steps, args.warmup
    with stdout_to_stderr():
        cb = reference_sample(args.config, steps, warm)
    m = mg.workload(args.config)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": cb["seconds_per_step"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.config, m, args.gpus),
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def host_recheck(ctx, u_hi, u_lo):
    """Host-side check of the device-certified solution u* = u_hi + u_lo on the full
    system: the oracle's double-double residual (C restatement, one thread) and the
    reference's own FP64 ELLmatrix::Axy (ELLmatrix.cc:194-204, FP64 build, all cores) on
    the downloaded K64.  The FP64 residual of fl(u*) cannot fall below the FP64 rounding
    of K u (about eps * || |K| |u| || / ||f||), which is reported beside it."""
    from gpufem_b200 import _lib
    from oracle.oracle import Oracle, Reference
    t0 = time.perf_counter()
    rn, ci, v = ctx.ell_download(_lib.GF_F64)
    f = ctx.get_force()
    fn = float(np.linalg.norm(f))
    out = {"download_seconds": time.perf_counter() - t0}
    _, nrm = Oracle().residual_dd(rn, ci, v, f, u_hi, u_lo)
    out["oracle_dd_rel_residual"] = nrm / fn
    if Reference.available("fp64"):
        cores = os.cpu_count() or 1
        with stdout_to_stderr():
            y, t = Reference("fp64").ell_axy(rn, ci, v, u_hi, nthreads=cores)
        out["reference_axy_fp64_rel_residual"] = float(np.linalg.norm(f - y) / fn)
        out["reference_axy_seconds"] = t
        ku = np.zeros(rn.size)
        au = np.abs(u_hi)
        for j in range(ci.shape[0]):       # || |K| |u| || by slots, for the FP64 floor
            live = np.nonzero(j < rn)[0]
            ku[live] += np.abs(v[j, live]) * au[ci[j, live]]
        out["fp64_roundoff_floor"] = float(np.finfo(np.float64).eps * np.linalg.norm(ku) / fn)
    out["seconds"] = time.perf_counter() - t0
    return out


# ---------------------------------------------------------------------------
# solves to an error target against a certified solution
# ---------------------------------------------------------------------------
SOLVER_TABLE = {
    # name: (solver, matrix dtype, uses the two-level set-up, label)
    "pcg_fp64": ("GF_SOLVER_PCG", "GF_F64", False, "FP64 Jacobi-PCG"),
    "mixed_pcg": ("GF_SOLVER_MIXED_PCG", "GF_F32", False,
                  "Jacobi-PCG on K32, FP64 vectors, FP64 reliable updates on K64"),
    "mixed_pcg32": ("GF_SOLVER_MIXED_PCG32", "GF_F32", False,
                    "Jacobi-PCG on K32, FP32 vectors, FP64 reliable updates on K64"),
    "twolevel_pcg": ("GF_SOLVER_TWOLEVEL_PCG", "GF_F64", True,
                     "FP64 PCG, M = Jacobi + rigid-body modes of box aggregates"),
    "twolevel_pcg_k32": ("GF_SOLVER_TWOLEVEL_PCG", "GF_F32", True,
                         "two-level PCG with K32 SpMVs, FP64 vectors, reliable updates on K64"),
    "twolevel_pcg32": ("GF_SOLVER_TWOLEVEL_PCG32", "GF_F32", True,
                       "two-level PCG with K32 SpMVs and FP32 vectors, FP64 dot products, "
                       "reliable updates on K64"),
}


def time_to_error(ctx, solver, matrix, ustar, target, max_iter=400000):
    """Solve with stopping tolerances target x (1, 0.3, 0.1, ...) until the relative
    error against the certified solution is <= target; the run that first meets it is
    the result (its device time and iterations).  Returns the result and every run."""
    from gpufem_b200 import _lib
    nrm = float(np.linalg.norm(ustar))
    runs = []
    for fac in (1.0, 0.3, 0.1, 0.03, 0.01, 3e-3, 1e-3, 3e-4, 1e-4, 3e-5, 1e-5):
        tol = max(target * fac, 1e-14)
        info = ctx.solve(solver, matrix, tol=tol, max_iter=max_iter, inner_tol=1e-4,
                         raise_on_error=False)
        err = float(np.linalg.norm(ctx.solution() - ustar) / nrm)
        runs.append({"tol": tol, "seconds": info.seconds, "iterations": info.iterations,
                     "rel_err": err, "rel_residual": info.rel_residual, "status": info.status,
                     "outer": info.outer, "fallback": info.fallback})
        if (err <= target and info.status == _lib.GF_OK) or tol <= 1e-14:
            break
    best = dict(runs[-1])
    best["met"] = bool(best["rel_err"] <= target and best["status"] == _lib.GF_OK)
    best["runs"] = runs
    return best


def solve_study(ctx, target, solvers, asm_seconds):
    """Every solver on the context's constrained system (K64 and K32, f set), to a
    relative error <= target against u* = the double-double refined solution (two-level
    FP64 PCG corrections, residual certified by gf_residual_dd and rechecked on the host).
    Totals add the assembly (asm_seconds: {"f64": s, "f32": s}), the solver layout build,
    the two-level set-up where used, and the solve."""
    from gpufem_b200 import _lib
    out = {"target_rel_error": target}
    # the solver layout (sliced copies of K64 and K32) is built by the first product;
    # build it once here, from device vectors (no host copies in the figure), so that every
    # solve below is timed alike
    import torch
    x64 = torch.zeros(ctx.n, dtype=torch.float64, device="cuda")
    x32 = torch.zeros(ctx.n, dtype=torch.float32, device="cuda")
    y64, y32 = torch.empty_like(x64), torch.empty_like(x32)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for dt, xx, yy in ((_lib.GF_F64, x64, y64), (_lib.GF_F32, x32, y32)):
        _lib.check(_lib.lib.gf_spmv(ctx.h, dt, C.c_void_p(xx.data_ptr()),
                                    C.c_void_p(yy.data_ptr())), ctx.h)
    ctx.sync()
    layout_s = time.perf_counter() - t0
    del x64, x32, y64, y32
    t0 = time.perf_counter()
    nc = ctx.twolevel_setup(0)
    setup_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    u_hi, u_lo, rinfo = ctx.refine_dd(_lib.GF_SOLVER_TWOLEVEL_PCG, inner_tol=1e-9, target=1e-17)
    out["reference_solution"] = {
        "how": "double-double iterative refinement: r = f - K64 (u_hi + u_lo) by "
               "gf_residual_dd, corrections by FP64 two-level PCG to 1e-9",
        "rel_residual_dd": rinfo["rel_residual_history"][-1],
        "rel_residual_history": rinfo["rel_residual_history"],
        "last_correction_rel": rinfo["correction_history"][-1] if rinfo["correction_history"]
        else None,
        "seconds": time.perf_counter() - t0}
    out["layout_seconds"] = layout_s
    out["twolevel_setup_seconds"] = setup_s
    out["coarse_unknowns"] = nc
    ustar = u_hi
    rank, world, _ = dist_info()
    if rank == 0 and world == 1:
        out["reference_solution"]["host_recheck"] = host_recheck(ctx, u_hi, u_lo)
    base = None
    for name in solvers:
        sv, mt, tl, label = SOLVER_TABLE[name]
        mt_v = getattr(_lib, mt)
        r = time_to_error(ctx, getattr(_lib, sv), mt_v, ustar, target)
        asm = asm_seconds["f64"] + (asm_seconds.get("convert", 0.0) if mt_v == _lib.GF_F32 else 0)
        r["label"] = label
        r["total_seconds"] = asm + layout_s + (setup_s if tl else 0.0) + r["seconds"]
        r["total_includes"] = ("FP64 assembly" + (" + FP32 copy" if mt_v == _lib.GF_F32 else "")
                               + " + solver layout" + (" + two-level set-up" if tl else "")
                               + " + solve")
        out[name] = r
        if name == "pcg_fp64":
            base = r["total_seconds"]
    if base:
        out["speedup_total_vs_pcg_fp64"] = {k: base / out[k]["total_seconds"]
                                            for k in solvers if k != "pcg_fp64"}
    return out


def brick20_study(args, flush):
    """Brick20 64^3 (the solve-time target workload): FP32 and FP64 assembly in every schedule,
    then every solver to FP64-oracle relative error 1e-6 with totals against FP64
    Jacobi-PCG."""
    import torch
    from gpufem_b200 import _lib
    from gpufem_b200 import meshgen as mg
    from gpufem_b200.fem import Context
    m = mg.workload("brick20_64")
    ctx = Context(0)
    lib_stream = torch.cuda.ExternalStream(ctx.stream_handle())
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    n, W, nnz = ctx.build_pattern()
    ctx.color(None)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)

    def timed(dtype, scatter, engine=0, reps=3):
        ctx.assemble(dtype, scatter, engine)
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            with torch.cuda.stream(lib_stream):
                flush.zero_()
            ts.append(ctx.assemble(dtype, scatter, engine))
        return float(np.median(ts))

    asm = {}
    for dname, dt in (("f32", _lib.GF_F32), ("f64", _lib.GF_F64)):
        for sname, sc in (("auto", _lib.GF_SCATTER_AUTO), ("owner", _lib.GF_SCATTER_OWNER),
                          ("atomic", _lib.GF_SCATTER_ATOMIC), ("colour", _lib.GF_SCATTER_COLOR)):
            t = timed(dt, sc)
            asm[f"{dname}_{sname}"] = {"ms": t * 1e3, "elements_per_s": m.nelem / t}
    # the tcgen05 engine (FP32): element Gram matrices on the tensor cores, scattered by
    # atomics, or stored and gathered by the owner kernel (split: tensor kernel, gather)
    for sname, sc in (("atomic", _lib.GF_SCATTER_ATOMIC), ("owner", _lib.GF_SCATTER_OWNER)):
        t = timed(_lib.GF_F32, sc, _lib.GF_ENGINE_TF32_MMA)
        g_s, s_s = C.c_double(), C.c_double()
        _lib.lib.gf_last_assembly_split(ctx.h, C.byref(g_s), C.byref(s_s))
        asm[f"f32_tcgen05_{sname}"] = {"ms": t * 1e3, "elements_per_s": m.nelem / t,
                                       "split_ms": [g_s.value * 1e3, s_s.value * 1e3]}
    # the system solved: FP64 assembly (AUTO), its FP32 rounding, elimination BCs
    t_f64 = asm["f64_auto"]["ms"] * 1e-3
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_AUTO)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.convert_f64_to_f32()
    ctx.sync()
    t_conv = time.perf_counter() - t0
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    solvers = [x for x in args.solvers.split(",") if x in SOLVER_TABLE]
    study = solve_study(ctx, 1e-6, solvers, {"f64": t_f64, "convert": t_conv})
    ctx.close()
    return {"workload": "brick20_64", "description": WORKLOADS["brick20_64"],
            "elements": m.nelem, "dofs": n, "nnz": nnz, "ell_width": W,
            "assembly": asm, "fp32_copy_seconds": t_conv, "solve": study,
            "l2": "flushed (256 MB write) before each timed assembly"}


# ---------------------------------------------------------------------------
# learned preconditioner vs plain Jacobi-PCG (multi-mesh Brick8 workload)
# ---------------------------------------------------------------------------
def _preconditioner_diagnostic(ctx, ustar):
    """How the learned preconditioner M acts on residuals r_k of Jacobi-PCG after k
    iterations, against Jacobi (D^-1 r): the cosine between the two corrections, and the
    energy norm of the error left after the best multiple of each correction,
    ||e - a z||_K / ||e||_K (1.0 = no reduction)."""
    import scipy.sparse as sp
    from gpufem_b200 import _lib
    rn, ci, v = ctx.ell_download(_lib.GF_F64)
    W, n = ci.shape
    mask = np.arange(W)[:, None] < rn[None, :]
    rows = np.broadcast_to(np.arange(n)[None, :], (W, n))
    K = sp.csr_matrix((v[mask], (rows[mask], ci[mask])), shape=(n, n))
    f = ctx.get_force()
    d = K.diagonal()
    out = []
    for it in (1, 20, 100):
        ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-14, max_iter=it, raise_on_error=False)
        u = ctx.solution()
        r = f - K @ u
        e = ustar - u
        eKe = float(e @ (K @ e))
        row = {"pcg_iterations": it}
        zs = {"jacobi": r / d, "learned": ctx.lp_apply(r)}
        for k, z in zs.items():
            Kz = K @ z
            a = float(z @ (K @ e)) / float(z @ Kz)
            w = e - a * z
            row[f"energy_error_after_{k}"] = float(np.sqrt(max(w @ (K @ w), 0.0) / eKe))
        zj, zl = zs["jacobi"], zs["learned"]
        row["cosine_learned_jacobi"] = float(zj @ zl / (np.linalg.norm(zj) * np.linalg.norm(zl)))
        out.append(row)
    return out


def learned_application(edge: int = 48, ctx_lp=None, reps: int = 7):
    """Device time of one learned-preconditioner application (features with two products
    with K, three message-passing layers, output) on the largest training-set mesh, a
    Brick8 cube of edge 48 (117,649 nodes, 352,947 dofs; correlated log-normal E), against
    one FP64 SpMV of the same matrix; L2 flushed before each call, median of `reps`.
    Uses the network of ctx_lp (trained) when given, else a seeded untrained one."""
    import torch
    from gpufem_b200 import _lib
    from gpufem_b200 import meshgen as mg
    from gpufem_b200.fem import Context
    m = mg.clamp_and_load(mg.structured(mg.BRICK8, (edge,) * 3, jitter=0.1, seed=48))
    m.E = mg.lognormal_correlated(m, 1.0, 0.2, 48)
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    ctx.lp_init(3, seed=1)
    if ctx_lp is not None:
        ctx.lp_set_weights(ctx_lp.lp_get_weights())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ls = torch.cuda.ExternalStream(ctx.stream_handle())
    r = torch.randn(m.ndof, device="cuda", dtype=torch.float32)
    z = torch.empty_like(r)
    x = torch.randn(m.ndof, device="cuda", dtype=torch.float64)
    y = torch.empty_like(x)
    ta, ts = [], []
    for _ in range(reps + 1):
        torch.cuda.synchronize()
        with torch.cuda.stream(ls):
            flush.zero_()
        _lib.check(_lib.lib.gf_lp_apply(ctx.h, C.c_void_p(r.data_ptr()), C.c_void_p(z.data_ptr())),
                   ctx.h)
        ta.append(_lib.lib.gf_last_device_seconds(ctx.h))
        torch.cuda.synchronize()
        with torch.cuda.stream(ls):
            flush.zero_()
        _lib.check(_lib.lib.gf_spmv(ctx.h, _lib.GF_F64, C.c_void_p(x.data_ptr()),
                                    C.c_void_p(y.data_ptr())), ctx.h)
        ts.append(_lib.lib.gf_last_device_seconds(ctx.h))
    ctx.close()
    a, sp = float(np.median(ta[1:])), float(np.median(ts[1:]))
    return {"mesh": f"Brick8 {edge}^3", "nodes": m.nnodes, "dofs": m.ndof,
            "application_us": a * 1e6, "spmv_fp64_us": sp * 1e6, "application_over_spmv": a / sp,
            "timing": "device time, L2 flushed before each call, median of %d" % reps}


def learned_comparison(seed_base: int = 20260105, n_train: int = 24, n_test: int = 16,
                       steps: int = 120, lr: float = 1e-3):
    """Brick8 cubes with edge n uniform in 16..48 elements, correlated log-normal E (sigma
    U(0.5, 2), correlation length U(0.05, 0.3)) and nu U(0.2, 0.4), z = 0 clamped,
    pressure on z = 1; n_train seeded training meshes and n_test held-out ones.  The
    network runs beside the two-level coarse correction (M = D^-1 + c y(r) + P Ac^-1 P^T:
    the coarse space takes the smooth error, which no local network can represent) and is
    trained with the residual loss on pairs from two-level PCG runs on the training meshes
    (one pass, `steps` Adam steps per mesh).  On the held-out meshes: time and iterations to
    a true relative residual of 1e-8, and the error against an FP64 PCG solution to 1e-12,
    for FP64 Jacobi-PCG, mixed-precision PCG, two-level PCG (the same method without the
    network) and learned FCG (with its fallback to the network-free preconditioner)."""
    from gpufem_b200 import _lib
    from gpufem_b200 import meshgen as mg
    from gpufem_b200.fem import Context

    def make(seed):
        rs = np.random.default_rng(seed)
        nn = int(rs.integers(16, 49))
        m = mg.clamp_and_load(mg.structured(mg.BRICK8, (nn,) * 3, jitter=0.1, seed=seed))
        m.E = mg.lognormal_correlated(m, rs.uniform(0.5, 2.0), rs.uniform(0.05, 0.3), seed)
        m.nu = float(rs.uniform(0.2, 0.4))
        return nn, m

    def setup(ctx, m):
        ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
        ctx.set_supports(m.supports)
        ctx.set_force(m.f)
        ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)
        ctx.convert_f64_to_f32()
        ctx.apply_constraints(_lib.GF_BC_ELIMINATION)

    ctx = Context(0)
    ctx.lp_init(3, seed=seed_base)
    ctx.lp_set_loss(_lib.GF_LP_LOSS_RESIDUAL)
    ctx.lp_set_coarse(True)
    t0 = time.perf_counter()
    losses = []
    for k in range(n_train):
        _, m = make(seed_base + 100 + k)
        setup(ctx, m)
        ctx.lp_collect(npairs=32, every=8, tol=1e-8)
        losses.append(ctx.lp_train(steps=steps, batch=8, lr=lr, seed=seed_base + k))
    train_s = time.perf_counter() - t0
    results = []
    names = (("pcg_fp64", _lib.GF_SOLVER_PCG), ("mixed_pcg", _lib.GF_SOLVER_MIXED_PCG),
             ("twolevel_pcg", _lib.GF_SOLVER_TWOLEVEL_PCG),
             ("learned_fcg", _lib.GF_SOLVER_LEARNED_FCG))
    for k in range(n_test):
        nn, m = make(seed_base + 900 + k)
        setup(ctx, m)
        ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-12, max_iter=400000, raise_on_error=False)
        ustar = ctx.solution()
        nrm = np.linalg.norm(ustar)
        row = {"edge": nn, "dofs": m.ndof}
        for name, solver in names:
            info = ctx.solve(solver, _lib.GF_F64, tol=1e-8, max_iter=400000, raise_on_error=False)
            err = float(np.linalg.norm(ctx.solution() - ustar) / nrm)
            row[name] = {"seconds": info.seconds, "iterations": info.iterations,
                         "rel_err_vs_reference": err, "status": info.status,
                         **({"fallback": info.fallback} if name == "learned_fcg" else {})}
        if k == 0:
            row["diagnostic"] = _preconditioner_diagnostic(ctx, ustar)
        # device time of one network application (features, three message-passing layers,
        # output) against one FP64 SpMV of the same matrix (median of 5 each)
        rr = np.random.default_rng(k).standard_normal(m.ndof)
        ta, ts = [], []
        for _ in range(5):
            ctx.lp_apply(rr)
            ta.append(_lib.lib.gf_last_device_seconds(ctx.h))
            ctx.spmv(rr, _lib.GF_F64)
            ts.append(_lib.lib.gf_last_device_seconds(ctx.h))
        row["application_us"] = float(np.median(ta)) * 1e6
        row["spmv_fp64_us"] = float(np.median(ts)) * 1e6
        results.append(row)

    app48 = learned_application(ctx_lp=ctx)
    ctx.close()

    def ratio(a, b, key):
        return float(np.median([r[a][key] / r[b][key] for r in results]))

    summary = {f"median_{key}_ratio_{a}_over_{b}": ratio(a, b, key)
               for a, b in (("learned_fcg", "pcg_fp64"), ("twolevel_pcg", "pcg_fp64"),
                            ("learned_fcg", "twolevel_pcg"))
               for key in ("iterations", "seconds")}
    summary["learned_fcg_fallbacks"] = int(sum(r["learned_fcg"]["fallback"] for r in results))
    summary["learned_fcg_fewer_iterations_than_twolevel"] = int(
        sum(r["learned_fcg"]["iterations"] < r["twolevel_pcg"]["iterations"] for r in results))
    summary["application_brick8_48"] = app48
    return {"train_meshes": n_train, "held_out_meshes": n_test, "train_seconds": train_s,
            "final_train_loss": losses[-1], "first_train_loss": losses[0],
            "loss": "residual", "coarse_correction": True,
            "tol_rel_residual": 1e-8, "summary": summary, "held_out": results}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_sharded_arm(args):
    """--sharded: the workload split into node slabs over the ranks (one halo layer of
    elements each, gpufem_b200.shard).  Every rank assembles its local mesh (owner
    schedule, FP32 K for the metric; FP64 K for the solve) and all ranks run the
    device-resident sharded Jacobi-PCG (gf_dist_pcg, NCCL on the library stream) to a
    relative residual of 1e-8.  value = workload elements / max-over-ranks assembly time
    (strong scaling: the total work is fixed)."""
    import datetime
    import torch
    import torch.distributed as dist
    from gpufem_b200 import _lib
    from gpufem_b200 import meshgen as mg
    from gpufem_b200 import shard as sd
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    if not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29533")
        dist.init_process_group("nccl", rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=300))
    cfg = args.config
    m = mg.workload(cfg)
    solver = sd.ShardedSolver(m, rank, world, device=local, scatter=_lib.GF_SCATTER_OWNER)
    ctx = solver.ctx
    # assembly throughput of the local meshes (FP32, owner schedule), max over ranks
    for _ in range(args.warmup):
        ctx.assemble(_lib.GF_F32, _lib.GF_SCATTER_OWNER)
    dist.barrier()
    torch.cuda.synchronize()
    ts = [ctx.assemble(_lib.GF_F32, _lib.GF_SCATTER_OWNER) for _ in range(args.steps)]
    t = torch.tensor([float(sum(ts))], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    per_step = float(t.item()) / args.steps
    # the solve: the FP64 system the solver holds (assembled and constrained at set-up)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    solver.solve_device(tol=1e-8, max_iter=400000)          # warm: solver layout built
    x, info = solver.solve_device(tol=1e-8, max_iter=400000)
    st = torch.tensor([info.seconds], device="cuda", dtype=torch.float64)
    dist.all_reduce(st, op=dist.ReduceOp.MAX)
    if rank == 0:
        line = {"metric": METRIC, "value": m.nelem / per_step, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": dict(workload_config(cfg, m, world), parallelism=f"node slabs x{world}"),
                "sharded_solve": {"solver": "gf_dist_pcg (Jacobi-PCG, FP64, NCCL halo exchange "
                                            "and all-reduces on the library stream)",
                                  "iterations": info.iterations, "seconds_max_over_ranks":
                                  float(st.item()), "us_per_iteration":
                                  float(st.item()) / max(1, info.iterations) * 1e6,
                                  "status": info.status},
                "local_dofs": solver.shard.n_local, "owned_dofs": solver.shard.n_owned}
        print(json.dumps(line), flush=True)
    solver.close()
    dist.barrier()
    dist.destroy_process_group()


def run_gpu_arm(args):
    import torch
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from gpufem_b200 import _lib
    from gpufem_b200 import meshgen as mg
    from gpufem_b200.fem import Context

    cfg = args.config
    m = mg.workload(cfg, scale=args.scale)
    dtype = _lib.GF_F64 if cfg == "q4_64" else _lib.GF_F32
    esize = 8 if dtype == _lib.GF_F64 else 4
    ctx = Context(local)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    n, W, nnz = ctx.build_pattern()
    ctx.color(None)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    # "auto" resolves as the library's GF_SCATTER_AUTO does: atomic in 3-D, owner in 2-D
    sname = args.scatter if args.scatter != "auto" else ("atomic" if m.dim == 3 else "owner")
    scatter = {"owner": _lib.GF_SCATTER_OWNER, "colour": _lib.GF_SCATTER_COLOR,
               "atomic": _lib.GF_SCATTER_ATOMIC}[sname]
    for _ in range(args.warmup):
        ctx.assemble(dtype, scatter)
    barrier()
    # L2 flushes go on the library's stream right before each timed call: its start event
    # then waits on the flush kernel instead of on the host's first launch of the call
    lib_stream = torch.cuda.ExternalStream(ctx.stream_handle())
    launches0 = ctx.launches()
    dev_s = []
    split = []   # (geometry kernel, scatter kernel) seconds of each step
    g_s, s_s = C.c_double(), C.c_double()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            with torch.cuda.stream(lib_stream):
                flush.zero_()
            dev_s.append(ctx.assemble(dtype, scatter))
            _lib.lib.gf_last_assembly_split(ctx.h, C.byref(g_s), C.byref(s_s))
            split.append((g_s.value, s_s.value))
        barrier()
    launches = ctx.launches() - launches0
    total = float(sum(dev_s))
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([total], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    per_step = total / args.steps
    value = world * m.nelem / per_step

    # the same metric with the symbolic phase inside each step: pattern build (node
    # incidence, adjacency, ELL columns) + assembly, host wall time around both with the
    # device synchronised, as the reference's timed StiffAlgoCPU inserts its entries
    pat_t = []
    for _ in range(max(3, min(args.steps, 10))):
        torch.cuda.synchronize()
        with torch.cuda.stream(lib_stream):
            flush.zero_()
        ctx.sync()
        t0 = time.perf_counter()
        ctx.build_pattern()
        ctx.assemble(dtype, scatter)
        ctx.sync()
        pat_t.append(time.perf_counter() - t0)
    with_pattern = {"value": world * m.nelem / float(np.median(pat_t)), "unit": UNIT,
                    "ms_per_step": float(np.median(pat_t)) * 1e3,
                    "includes": "gf_ell_build_pattern + gf_assemble, host wall time"}

    # the three scatter schedules side by side (median of a few steps each)
    variants = {}
    runs = [("owner", _lib.GF_SCATTER_OWNER, 0), ("colour", _lib.GF_SCATTER_COLOR, 0),
            ("atomic", _lib.GF_SCATTER_ATOMIC, 0)]
    if esize == 4:   # the tcgen05 tensor-core engine assembles FP32 only
        runs += [("atomic_tcgen05", _lib.GF_SCATTER_ATOMIC, _lib.GF_ENGINE_TF32_MMA),
                 ("owner_tcgen05", _lib.GF_SCATTER_OWNER, _lib.GF_ENGINE_TF32_MMA)]
    for name, sc, eng in runs:
        ts = []
        for _ in range(max(3, min(args.steps, 10))):
            torch.cuda.synchronize()
            with torch.cuda.stream(lib_stream):
                flush.zero_()
            ts.append(ctx.assemble(dtype, sc, eng))
        variants[name] = {"value": m.nelem / float(np.median(ts)), "unit": UNIT,
                          "ms": float(np.median(ts)) * 1e3}

    # roofline of the whole assembly: algorithmic bytes = K values written once + node
    # coordinates, connectivity and moduli read once
    hbm, peak_kind = peaks()
    alg_bytes = nnz * esize + m.nnodes * m.dim * esize + m.nelem * (m.nen * 4 + esize)
    achieved = alg_bytes / per_step / 1e9
    # dominant kernel (owner schedule: k_assemble_owner_node for 2-D FP32, else
    # k_assemble_owner): K values written once, plus what it must read — J^-1 and w*detJ
    # per element and Gauss point (the 2-D FP32 kernel reads w*detJ*E, the modulus folded
    # in; the other reads the moduli apart), and per incidence the element id, local node
    # index and nen neighbour slots
    ngp = m.ngauss ** m.dim
    t_geo = float(np.mean([a for a, _ in split]))
    t_dom = float(np.mean([b for _, b in split]))
    if sname == "owner":
        ninc = m.nelem * m.nen
        node_kernel = m.dim == 2 and esize == 4
        dom_bytes = (nnz * esize + m.nelem * ngp * (m.dim * m.dim + 1) * esize
                     + (0 if node_kernel else m.nelem * esize)
                     + ninc * (4 + 1 + 2 * m.nen) + (m.nnodes + 1) * 4)
        dom_name = "k_assemble_owner_node" if node_kernel else "k_assemble_owner"
    else:
        dom_bytes = alg_bytes
        dom_name = ("k_assemble (all colour passes)" if sname == "colour" else
                    "k_assemble (atomic)") + " + K zero-fill"
    traffic = traffic_asm = None
    tfile = ROOT / "profiles" / "ncu_traffic.json"
    if tfile.exists() and sname == "owner":
        tr = json.loads(tfile.read_text()).get(f"{cfg}/assemble")
        if tr is not None:
            traffic_asm = tr.get("bytes_per_assembly")
            traffic = tr.get("kernels", {}).get(dom_name)

    # SpMV roofline: node-block slices, i.e. the values, one int32 column per dim x dim
    # block, x read once and y written once
    ctx.assemble(dtype, scatter)
    xs = torch.randn(n, device="cuda", dtype=torch.float32 if esize == 4 else torch.float64)
    ys = torch.empty_like(xs)
    sp = []
    torch.cuda.synchronize()
    for _ in range(10):
        # the flush runs on the library's stream just before the SpMV, so the SpMV's start
        # event waits on the flush, not on the host's launch of the SpMV
        with torch.cuda.stream(lib_stream):
            flush.zero_()
        _lib.check(_lib.lib.gf_spmv(ctx.h, dtype, xs.data_ptr(), ys.data_ptr()), ctx.h)
        sp.append(_lib.lib.gf_last_device_seconds(ctx.h))
    t_spmv = float(np.median(sp))
    spmv_bytes = nnz * esize + (nnz // (m.dim * m.dim)) * 4 + n * 2 * esize

    # e2e through the public API from pinned host buffers, every step
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    h_coords, h_conn = pin(m.coords), pin(m.conn)
    h_E = pin(m.E) if m.E is not None else None
    h_rownnz = torch.empty(n, dtype=torch.int32).pin_memory()
    h_colidx = torch.empty(n * W, dtype=torch.int32).pin_memory()
    h_vals = torch.empty(n * W, dtype=torch.float32 if esize == 4 else torch.float64).pin_memory()
    lib = _lib.lib

    def e2e_step():
        _lib.check(lib.gf_mesh_create(ctx.h, m.elem_type, m.nnodes, C.c_void_p(h_coords.data_ptr()),
                                      m.nelem, C.c_void_p(h_conn.data_ptr()), m.ngauss, m.E0,
                                      None if h_E is None else C.c_void_p(h_E.data_ptr()), m.nu, 0),
                   ctx.h)
        _lib.check(lib.gf_assemble(ctx.h, dtype, scatter, 0), ctx.h)
        _lib.check(lib.gf_ell_download(ctx.h, dtype, C.c_void_p(h_rownnz.data_ptr()),
                                       C.c_void_p(h_colidx.data_ptr()),
                                       C.c_void_p(h_vals.data_ptr())), ctx.h)

    e2e_step()
    barrier()
    e2e_t = []
    for _ in range(max(2, min(args.steps, 5))):
        t0 = time.perf_counter()
        e2e_step()
        e2e_t.append(time.perf_counter() - t0)
    e2e_per = float(np.median(e2e_t))
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([e2e_per], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_per = float(t.item())
    h2d = m.coords.nbytes + m.conn.nbytes + (m.E.nbytes if m.E is not None else 0)
    d2h = n * 4 + n * W * 4 + n * W * esize

    # solve: every solver on the same problem, to a relative error against the certified
    # solution (1e-8 for the 2-D workloads, 1e-6 for the 3-D ones)
    solve = None
    solvers = [x for x in args.solvers.split(",") if x]
    unknown = set(solvers) - set(SOLVERS)
    if unknown:
        raise SystemExit(f"unknown solver(s) {sorted(unknown)}; choose from {SOLVERS}")
    if not args.no_solve and any(x in SOLVER_TABLE for x in solvers):
        ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
        ctx.set_supports(m.supports)
        ctx.set_force(m.f)
        t_f64 = ctx.assemble(_lib.GF_F64, scatter)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.convert_f64_to_f32()     # symmetric FP32 copy for the mixed solvers
        ctx.sync()
        t_conv = time.perf_counter() - t0
        ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
        target = 1e-8 if m.dim == 2 else 1e-6
        solve = solve_study(ctx, target, [x for x in solvers if x in SOLVER_TABLE],
                            {"f64": t_f64, "convert": t_conv})
        if (rank == 0 and world == 1 and not args.no_cpu and "pcg_fp64" in solve
                and cfg in ("q4_64", "q8_512")):
            # (the reference's assembly of the full 3-D meshes alone takes minutes)
            with stdout_to_stderr():
                rc = reference_cg_sample(m)
            if rc is not None:
                its = solve["pcg_fp64"]["iterations"]
                rc["extrapolated_seconds"] = rc["cg_us_per_iteration"] * 1e-6 * its
                rc["label"] = ("extrapolated: reference CPU_CG (unpreconditioned CG, FP32, OpenMP) "
                               "time per iteration on the full system x the FP64 Jacobi-PCG "
                               "iteration count above; assembly timed once on the full mesh")
                solve["cpu_reference"] = rc

    learned = None
    if not args.no_solve and rank == 0 and "learned" in solvers:
        learned = learned_comparison()

    brick20 = None
    if (not args.no_solve and not args.no_brick20 and rank == 0 and world == 1
            and cfg == "q8_512"):
        ctx.close()                  # free the Q8 matrices before the Brick20 64^3 study
        brick20 = brick20_study(args, flush)

    cpu_baseline = None
    if rank == 0 and world == 1 and not args.no_cpu:
        with stdout_to_stderr():
            cb = reference_sample(cfg, steps=2, warmup=1)
        cpu_baseline = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if esize == 4 else "f64", "data": "synthetic",
            "config": dict(workload_config(cfg, m, world),
                           **({"scale": args.scale} if args.scale != 1.0 else {})),
            "matrix": {"dofs": n, "nnz": nnz, "ell_width": W},
            "timing": "device time (CUDA events on the library's stream); L2 flushed (256 MB "
                      "write) before every timed step",
            "value_with_pattern": with_pattern,
            "roofline": {"bound": "hbm", "achieved": dom_bytes / t_dom / 1e9, "peak": hbm,
                         "unit": "GB/s", "frac": dom_bytes / t_dom / 1e9 / hbm,
                         "traffic": traffic, "kernel": dom_name,
                         "us_per_launch": t_dom * 1e6, "algorithmic_bytes": dom_bytes,
                         "peak_source": peak_kind},
            "roofline_assembly": {"bound": "hbm", "achieved": achieved, "peak": hbm,
                                  "unit": "GB/s", "frac": achieved / hbm,
                                  "traffic": traffic_asm, "algorithmic_bytes": alg_bytes,
                                  "kernels_us": {"k_elem_geometry": t_geo * 1e6,
                                                 dom_name: t_dom * 1e6}},
            "roofline_spmv": {"bound": "hbm", "achieved": spmv_bytes / t_spmv / 1e9, "peak": hbm,
                              "unit": "GB/s", "frac": spmv_bytes / t_spmv / 1e9 / hbm,
                              "us_per_launch": t_spmv * 1e6, "algorithmic_bytes": spmv_bytes},
            "scatter": sname,
            "scatter_variants": variants,
            "e2e": {"value": world * m.nelem / e2e_per, "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "includes": "mesh upload, pattern, assembly, ELL download"},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "solve": solve,
            "brick20_64": brick20,
            "learned": learned,
            "cpu_baseline": cpu_baseline,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="q8_512", choices=sorted(WORKLOADS))
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--solvers", default=",".join(SOLVERS),
                    help="comma list of the solve block's entries (default: all)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="mesh edge scale of the workload (1 = the full workload; smaller "
                         "cases for profiler captures)")
    ap.add_argument("--sharded", action="store_true",
                    help="split the workload over the ranks (node slabs) and solve with the "
                         "device-resident sharded PCG instead of running replicas")
    ap.add_argument("--learned-application", action="store_true",
                    help="time only one learned-preconditioner application against one FP64 "
                         "SpMV on the Brick8 48^3 mesh (untrained network) and print it")
    ap.add_argument("--no-brick20", action="store_true",
                    help="skip the Brick20 64^3 assembly + solve study of the default run")
    ap.add_argument("--scatter", default="auto", choices=["owner", "colour", "atomic", "auto"])
    args = ap.parse_args()
    if args.warmup < 3:     # both arms: at least 3 warm-up steps
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.sharded:
        run_sharded_arm(args)
    elif args.learned_application:
        print(json.dumps(learned_application()), flush=True)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
