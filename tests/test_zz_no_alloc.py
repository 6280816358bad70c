"""gf_pcg_noalloc: the Jacobi-PCG entry point for callers that cannot allocate GPU
memory (their framework owns every device byte, or a cudaMalloc and the device
synchronisation it may cause is not allowed where they solve).  It is called
through the C-ABI on caller-owned device buffers and must give the same solution
as the allocating solver (gf_solve with GF_SOLVER_PCG) on two calls in a row.
Collected last on purpose: a run that stops at the first failure has then already
run every other test."""
import ctypes as C

import numpy as np
import pytest

from gpufem_b200 import _lib
from gpufem_b200 import meshgen as mg

pytestmark = pytest.mark.gpu

TOL = 1e-10          # solver tolerance, as the other FP64 PCG tests use
SOL_RTOL = 1e-8      # solution agreement, as tests/test_solver_gpu.py


def _problem():
    import torch
    from gpufem_b200.fem import Context
    m = mg.workload("q4_64", scale=0.5)        # Q4 32x32, jittered, 2178 dofs
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_COLOR)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    return torch, ctx


def test_pcg_noalloc_matches_allocating_solver_twice():
    torch, ctx = _problem()
    info = ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=TOL, max_iter=100000)
    u_ref = ctx.solution()
    n, W = C.c_int32(), C.c_int32()
    rn, ci, vals = C.c_void_p(), C.c_void_p(), C.c_void_p()
    _lib.check(_lib.lib.gf_ell_view(ctx.h, _lib.GF_F64, C.byref(n), C.byref(W), C.byref(rn),
                                    C.byref(ci), C.byref(vals)), ctx.h)
    b = torch.tensor(ctx.get_force(), device="cuda", dtype=torch.float64)
    x = torch.empty(n.value, device="cuda", dtype=torch.float64)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        x.fill_(float("nan"))          # the output must be fully rewritten
        it, rel = C.c_int32(-1), C.c_double(-1.0)
        st = _lib.lib.gf_pcg_noalloc(n.value, W.value, rn, ci, vals, C.c_void_p(b.data_ptr()),
                                     C.c_void_p(x.data_ptr()), TOL, 100000, stream,
                                     C.byref(it), C.byref(rel))
        torch.cuda.synchronize()
        assert st == _lib.GF_OK, f"call {call}: status {st}"
        u = x.cpu().numpy()
        assert np.all(np.isfinite(u))
        assert np.linalg.norm(u - u_ref) <= SOL_RTOL * np.linalg.norm(u_ref), f"call {call}"
        assert 0 < it.value <= 100000 and abs(it.value - info.iterations) <= 2
        assert 0.0 <= rel.value <= 1e-8


def _view(ctx):
    n, W = C.c_int32(), C.c_int32()
    rn, ci, vals = C.c_void_p(), C.c_void_p(), C.c_void_p()
    _lib.check(_lib.lib.gf_ell_view(ctx.h, _lib.GF_F64, C.byref(n), C.byref(W), C.byref(rn),
                                    C.byref(ci), C.byref(vals)), ctx.h)
    return n.value, W.value, rn, ci, vals


def test_pcg_noalloc_iteration_cap_zero_rhs_and_null_outputs():
    torch, ctx = _problem()
    n, W, rn, ci, vals = _view(ctx)
    b = torch.tensor(ctx.get_force(), device="cuda", dtype=torch.float64)
    x = torch.empty(n, device="cuda", dtype=torch.float64)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # an iteration cap below what the tolerance needs: NOT_CONVERGED after exactly 3
    it, rel = C.c_int32(-1), C.c_double(-1.0)
    st = _lib.lib.gf_pcg_noalloc(n, W, rn, ci, vals, C.c_void_p(b.data_ptr()),
                                 C.c_void_p(x.data_ptr()), TOL, 3, stream, C.byref(it),
                                 C.byref(rel))
    torch.cuda.synchronize()
    assert st == _lib.GF_ERR_NOT_CONVERGED and it.value == 3
    # (the CG residual norm is not monotone: after 3 steps it may sit just above 1)
    assert TOL < rel.value < 10.0
    # a zero right-hand side: converged at once, x = 0
    z = torch.zeros_like(b)
    x.fill_(float("nan"))
    st = _lib.lib.gf_pcg_noalloc(n, W, rn, ci, vals, C.c_void_p(z.data_ptr()),
                                 C.c_void_p(x.data_ptr()), TOL, 100, stream, C.byref(it),
                                 C.byref(rel))
    torch.cuda.synchronize()
    assert st == _lib.GF_OK and it.value == 0 and rel.value == 0.0
    assert torch.count_nonzero(x).item() == 0
    # a real solve with both optional outputs NULL
    info = ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=TOL, max_iter=100000)
    u_ref = ctx.solution()
    st = _lib.lib.gf_pcg_noalloc(n, W, rn, ci, vals, C.c_void_p(b.data_ptr()),
                                 C.c_void_p(x.data_ptr()), TOL, 100000, stream, None, None)
    torch.cuda.synchronize()
    assert st == _lib.GF_OK and info.status == _lib.GF_OK
    u = x.cpu().numpy()
    assert np.linalg.norm(u - u_ref) <= SOL_RTOL * np.linalg.norm(u_ref)


def test_pcg_noalloc_rejects_an_inconsistent_ell():
    import torch
    n, W = 4, 2
    rownnz = torch.tensor([1, 1, 1, 1], device="cuda", dtype=torch.int32)
    colidx = torch.tensor([0, 1, 2, 3, 0, 1, 2, 3], device="cuda", dtype=torch.int32)
    vals = torch.tensor([2.0] * 4 + [0.0] * 4, device="cuda", dtype=torch.float64)
    b = torch.ones(n, device="cuda", dtype=torch.float64)
    x = torch.zeros(n, device="cuda", dtype=torch.float64)
    args = lambda rn, ci: (n, W, C.c_void_p(rn.data_ptr()), C.c_void_p(ci.data_ptr()),
                           C.c_void_p(vals.data_ptr()), C.c_void_p(b.data_ptr()),
                           C.c_void_p(x.data_ptr()), TOL, 100, None, None, None)
    assert _lib.lib.gf_pcg_noalloc(*args(rownnz, colidx)) == _lib.GF_OK   # diagonal 2I
    torch.cuda.synchronize()
    assert torch.allclose(x, torch.full_like(x, 0.5))
    long_row = rownnz.clone()
    long_row[2] = W + 1                      # a row longer than the stored width
    assert _lib.lib.gf_pcg_noalloc(*args(long_row, colidx)) == _lib.GF_ERR_INVALID_ARG
    bad_col = colidx.clone()
    bad_col[1] = n                           # a stored column outside [0, n)
    assert _lib.lib.gf_pcg_noalloc(*args(rownnz, bad_col)) == _lib.GF_ERR_INVALID_ARG
    bad_col[1] = -1
    assert _lib.lib.gf_pcg_noalloc(*args(rownnz, bad_col)) == _lib.GF_ERR_INVALID_ARG


def test_pcg_noalloc_rejects_sizes_beyond_its_maximum():
    import torch
    big = _lib.GF_PCG_NOALLOC_MAX_N + 1
    # valid device buffers, so only the size decides; nothing is launched
    buf_i = torch.zeros(16, device="cuda", dtype=torch.int32)
    buf_d = torch.zeros(16, device="cuda", dtype=torch.float64)
    pi, pd = C.c_void_p(buf_i.data_ptr()), C.c_void_p(buf_d.data_ptr())
    st = _lib.lib.gf_pcg_noalloc(big, 1, pi, pi, pd, pd, pd, 1e-8, 10, None, None, None)
    assert st == _lib.GF_ERR_INVALID_ARG
    st = _lib.lib.gf_pcg_noalloc(0, 1, pi, pi, pd, pd, pd, 1e-8, 10, None, None, None)
    assert st == _lib.GF_ERR_INVALID_ARG
