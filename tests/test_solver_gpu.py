"""Device SpMV, constraints and the CG family through the C-ABI, against the
reference's known answers, its golden vectors and the oracle."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from ellutil import ell_from_entries, ell_to_dense
from gpufem_b200 import _lib
from gpufem_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Context():
    from gpufem_b200.fem import Context
    return Context


def upload(Context, n, entries):
    ctx = Context(0)
    rn, ci, v = ell_from_entries(n, entries)
    ctx.ell_upload(rn, ci, v)
    return ctx, (rn, ci, v)


@pytest.mark.parametrize("dtype", [_lib.GF_F64, _lib.GF_F32])
def test_kat_cg_8x8(Context, dtype):
    """LAopsTest.cpp:108-137."""
    from gpufem_b200.fem import ELLmatrixCUDA
    n = 8
    e = {(i, i): float((i + 1) ** 2) for i in range(n)}
    e[(0, 0)] = 2.0
    e[(0, 1)] = 2.0
    e[(1, 0)] = 2.0
    ctx, _ = upload(Context, n, e)
    K = ELLmatrixCUDA(ctx, dtype)
    x = K.CG(np.array([(i + 1) ** 2 for i in range(n)], float), 3000, 1e-5)
    assert np.allclose(x, [-1, 1.5] + [1] * 6, atol=1e-3)


@pytest.mark.parametrize("dtype", [_lib.GF_F64, _lib.GF_F32])
def test_kat_cg_tridiagonal_and_ones(Context, dtype):
    """AxyGPUTest.cpp:288-318 and 334-358."""
    from gpufem_b200.fem import ELLmatrixCUDA
    e = {}
    for i in range(4):
        e[(i, i)] = 2.0
        if i + 1 < 4:
            e[(i, i + 1)] = -1.0
        if i > 0:
            e[(i, i - 1)] = -1.0
    ctx, _ = upload(Context, 4, e)
    x = ELLmatrixCUDA(ctx, dtype).CG(np.ones(4), 200, 1e-5)
    assert np.allclose(x, [2, 3, 3, 2], atol=1e-3)
    n = 32
    ctx, _ = upload(Context, n, {(i, j): (2.0 if i == j else 1.0) for i in range(n) for j in range(n)})
    x = ELLmatrixCUDA(ctx, dtype).CG(np.ones(n), 500, 1e-5)
    assert np.allclose(x, 0.0303, atol=1e-3)


@pytest.mark.parametrize("dtype", [_lib.GF_F64, _lib.GF_F32])
def test_kat_spmv(Context, dtype):
    """AxyGPUTest.cpp:44-187: diagonal, band, band near the last rows, 64k rows."""
    from gpufem_b200.fem import ELLmatrixCUDA
    n = 4096
    ctx, _ = upload(Context, n, {(i, i): float(i + 1) for i in range(n)})
    x = np.arange(1, n + 1, dtype=float)
    assert np.allclose(ELLmatrixCUDA(ctx, dtype).Axy(x), x * x, rtol=1e-6)
    n, band = 64, 8
    ctx, _ = upload(Context, n, {(i, j): 1.0 for i in range(n) for j in range(band)})
    assert np.allclose(ELLmatrixCUDA(ctx, dtype).Axy(np.full(n, 2.0)), 2.0 * band)
    band = 4
    ctx, _ = upload(Context, n, {(i, i + j): 1.0 for i in range(n) for j in range(band) if i + j < n})
    y = ELLmatrixCUDA(ctx, dtype).Axy(np.full(n, 2.0))
    yres = np.full(n, 2.0 * band)
    for i in range(1, band):
        yres[n - band + i] -= 2 * i
    assert np.allclose(y, yres)
    n = 64 * 1024
    ctx, _ = upload(Context, n, {(i, j): 1.0 for i in range(n) for j in range(8)})
    assert np.allclose(ELLmatrixCUDA(ctx, dtype).Axy(np.ones(n)), 8.0)


def _fixed(g):
    dim = g["coords"].shape[1]
    fixed = np.zeros(g["coords"].shape[0] * dim, np.uint8)
    for row in g["supports"]:
        for c in range(dim):
            if row[1 + c] == 1:
                fixed[(row[0] - 1) * dim + c] = 1
    return fixed


@pytest.mark.parametrize("name", golden_names())
def test_penalty_and_cg_match_reference(Context, name):
    """FEM::ApplyConstraint(PEN) then CG (eps 1e-10) in FP64 against the reference."""
    g = load_golden(name)
    ctx = Context(0)
    ctx.mesh_create(int(g["elem_type"]), g["coords"], g["conn"], int(g["ngauss"]), float(g["E"]),
                    None, float(g["nu"]))
    ctx.set_supports(g["supports"])
    ctx.set_force(g["force"])
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_COLOR)
    ctx.apply_constraints(_lib.GF_BC_PENALTY)
    rn, ci, v = ctx.ell_download(_lib.GF_F64)
    diag = np.array([v[np.nonzero(ci[: rn[r], r] == r)[0][0], r] for r in range(rn.size)])
    assert np.allclose(diag, g["diag_pen_fp64"], rtol=1e-12, atol=0)
    info = ctx.solve(_lib.GF_SOLVER_CG, _lib.GF_F64, tol=1e-10, max_iter=20000)
    u = ctx.solution()
    ref = g["u_cg_fp64"]
    assert np.linalg.norm(u - ref) <= 1e-6 * np.linalg.norm(ref)
    assert info.iterations > 0


@pytest.mark.parametrize("name", ["q4_64", "q8_512", "brick8_128", "brick20_64"])
def test_pcg_and_mixed_match_oracle(Context, oracle, name):
    """Elimination BCs; FP64 Jacobi-PCG and mixed FP32/FP64 refinement against the
    oracle's FP64 PCG solution on a down-scaled workload."""
    scale = {"q4_64": 0.25, "q8_512": 1 / 32, "brick8_128": 1 / 16, "brick20_64": 1 / 16}[name]
    m = mg.workload(name, scale=scale)
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_COLOR)
    ctx.assemble(_lib.GF_F32, _lib.GF_SCATTER_COLOR)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    rn, ci, v = oracle.assemble(m.elem_type, m.ngauss, m.coords, m.conn, m.E0, m.nu, E_elem=m.E)
    fixed = np.zeros(m.ndof, np.uint8)
    for row in m.supports:
        for c in range(m.dim):
            fixed[(row[0] - 1) * m.dim + c] = 1
    v, f = oracle.eliminate(rn, ci, v, fixed, m.f)
    ustar, _ = oracle.cg(rn, ci, v, f, maxit=200000, eps=1e-13, precond=True)
    info = ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-12, max_iter=200000)
    u = ctx.solution()
    # PCG stops on its recursive residual; the reported true FP64 residual drifts
    # a little above it in finite precision
    assert info.rel_residual <= 1e-11
    assert np.linalg.norm(u - ustar) <= 1e-8 * np.linalg.norm(ustar)
    for solver in (_lib.GF_SOLVER_MIXED_PCG, _lib.GF_SOLVER_MIXED_PCG32):
        info = ctx.solve(solver, tol=1e-12, max_iter=200000, inner_tol=1e-4)
        u2 = ctx.solution()
        assert info.rel_residual <= 1e-12 and info.outer >= 2, (solver, info)
        assert np.linalg.norm(u2 - ustar) <= 1e-8 * np.linalg.norm(ustar), solver


def test_fp32_pcg_and_spmv_vs_oracle(Context, oracle):
    m = mg.workload("q8_512", scale=1 / 16)
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)
    ctx.assemble(_lib.GF_F32, _lib.GF_SCATTER_ATOMIC)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    rn, ci, v = ctx.ell_download(_lib.GF_F32)
    x = np.random.default_rng(2).standard_normal(m.ndof)
    y = ctx.spmv(x, _lib.GF_F32)
    yo = oracle.spmv(rn, ci, v.astype(np.float64), x.astype(np.float32).astype(np.float64))
    assert np.linalg.norm(y - yo) <= 1e-6 * np.linalg.norm(yo)
    info = ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F32, tol=1e-5, max_iter=100000)
    assert info.status == _lib.GF_OK


def test_solver_caps_and_errors(Context):
    m = mg.workload("q4_64", scale=0.5)
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)
    ctx.assemble(_lib.GF_F64)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    info = ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-14, max_iter=5, raise_on_error=False)
    assert info.status == _lib.GF_ERR_NOT_CONVERGED and info.iterations == 5
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.solve(_lib.GF_SOLVER_MIXED_PCG, tol=1e-8)   # no FP32 matrix yet
    assert ei.value.status == _lib.GF_ERR_STATE
    # zero right-hand side converges immediately to zero
    ctx.set_force(np.zeros(m.ndof))
    info = ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-10)
    assert info.iterations == 0 and np.all(ctx.solution() == 0)


@pytest.mark.parametrize("dtype", [_lib.GF_F64, _lib.GF_F32])
def test_spmv_2d_node_blocks_vs_oracle_and_alignment(Context, oracle, dtype):
    """2-D meshes read x in pairs: K x through gf_spmv against the oracle's ELL SpMV, and a
    device x that is not aligned to two entries is refused before any launch."""
    import torch
    m = mg.workload("q8_512", scale=1 / 32)
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.assemble(dtype)
    rn, ci, v = ctx.ell_download(dtype)
    tdt = torch.float64 if dtype == _lib.GF_F64 else torch.float32
    x = torch.randn(m.ndof + 1, dtype=tdt, device="cuda")
    y = torch.empty(m.ndof, dtype=tdt, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib.gf_spmv(ctx.h, dtype, x.data_ptr(), y.data_ptr()), ctx.h)
    xh = x[:m.ndof].cpu().numpy().astype(np.float64)
    yo = oracle.spmv(rn, ci, v.astype(np.float64), xh)
    tol = 1e-12 if dtype == _lib.GF_F64 else 1e-5
    assert np.linalg.norm(y.cpu().numpy() - yo) <= tol * np.linalg.norm(yo)
    st = _lib.lib.gf_spmv(ctx.h, dtype, x[1:].data_ptr(), y.data_ptr())
    assert st == _lib.GF_ERR_INVALID_ARG


def test_residual_dd_and_refinement_vs_oracle(Context, oracle):
    """gf_residual_dd equals the oracle's double-double residual for a solution held as
    u_hi + u_lo, and refinement drives the true residual far below what an FP64 residual
    can show (the FP64 residual of the refined solution is bounded below by roundoff)."""
    m = mg.workload("q8_512", scale=1 / 32)
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    rn, ci, v = ctx.ell_download(_lib.GF_F64)
    f = ctx.get_force()
    ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-10, max_iter=100000)
    uh = ctx.solution()
    ul = uh * 1e-17 * np.random.default_rng(3).standard_normal(uh.size)
    r_dev, rel_dev = ctx.residual_dd(uh, ul)
    r_or, nrm = oracle.residual_dd(rn, ci, v, f, uh, ul)
    scale = np.abs(v).max() * np.abs(uh).max()
    assert np.abs(r_dev - r_or).max() <= 1e-14 * np.abs(r_or).max() + 1e-28 * scale
    assert rel_dev == pytest.approx(nrm / np.linalg.norm(f), rel=1e-10)
    u_hi, u_lo, info = ctx.refine_dd(_lib.GF_SOLVER_PCG, inner_tol=1e-9, target=1e-18)
    hist = info["rel_residual_history"]
    assert hist[0] == pytest.approx(1.0) and hist[-1] <= 1e-16, hist
    _, nrm = oracle.residual_dd(rn, ci, v, f, u_hi, u_lo)
    assert nrm / np.linalg.norm(f) <= 1e-16
    ustar, _ = oracle.cg(rn, ci, v, f, maxit=200000, eps=1e-13, precond=True)
    assert np.linalg.norm(u_hi - ustar) <= 1e-9 * np.linalg.norm(ustar)
