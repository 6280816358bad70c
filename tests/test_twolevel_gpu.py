"""Two-level preconditioner and GF_SOLVER_TWOLEVEL_PCG through the C-ABI, against the
numpy oracle (aggregates, M r) and against converged solutions of the C oracle and of
the reference's own CG."""
import numpy as np
import pytest

from conftest import load_golden
from gpufem_b200 import _lib
from gpufem_b200 import meshgen as mg
from oracle import twolevel_oracle as tl

pytestmark = pytest.mark.gpu

CASES = [("q8_512", 1 / 16), ("brick8_128", 1 / 16), ("brick20_64", 1 / 16), ("q4_64", 0.25)]


def _fixed(m):
    fixed = np.zeros(m.ndof, np.uint8)
    for row in m.supports:
        for c in range(m.dim):
            if row[1 + c] == 1:
                fixed[(row[0] - 1) * m.dim + c] = 1
    return fixed


def _ctx(m, mode=_lib.GF_BC_ELIMINATION):
    from gpufem_b200.fem import Context
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_AUTO)
    ctx.apply_constraints(mode)
    return ctx


@pytest.mark.parametrize("name,scale", CASES)
@pytest.mark.parametrize("target", [0, 200])
def test_aggregates_and_apply_match_oracle(name, scale, target):
    m = mg.workload(name, scale=scale)
    ctx = _ctx(m)
    nc = ctx.twolevel_setup(target)
    agg, side = ctx.twolevel_aggregates()
    agg_o, side_o = tl.aggregates(m.coords, target if target else tl.default_target(m.ndof))
    np.testing.assert_array_equal(agg, agg_o)
    assert side == side_o
    rn, ci, v = ctx.ell_download(_lib.GF_F64)
    pc = tl.TwoLevel(m.coords, rn, ci, v, _fixed(m), agg=agg, side=side)
    assert nc == pc.ncoarse
    rng = np.random.default_rng(5)
    for _ in range(2):
        r = rng.standard_normal(m.ndof)
        z = ctx.twolevel_apply(r)
        zo = pc.apply(r)
        assert np.linalg.norm(z - zo) <= 1e-9 * np.linalg.norm(zo)


@pytest.mark.parametrize("name,scale", CASES)
def test_twolevel_pcg_matches_oracle_solution(oracle, name, scale):
    m = mg.workload(name, scale=scale)
    ctx = _ctx(m)
    rn, ci, v = oracle.assemble(m.elem_type, m.ngauss, m.coords, m.conn, m.E0, m.nu, E_elem=m.E)
    v, f = oracle.eliminate(rn, ci, v, _fixed(m), m.f)
    ustar, it_j = oracle.cg(rn, ci, v, f, maxit=200000, eps=1e-13, precond=True)
    info = ctx.solve(_lib.GF_SOLVER_TWOLEVEL_PCG, tol=1e-12, max_iter=200000)
    u = ctx.solution()
    assert info.status == _lib.GF_OK and info.rel_residual <= 1e-11
    assert np.linalg.norm(u - ustar) <= 1e-8 * np.linalg.norm(ustar)
    info_j = ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-12, max_iter=200000)
    assert info.iterations * 2 < info_j.iterations, (info.iterations, info_j.iterations)
    # the oracle's two-level PCG takes the same number of iterations, within rounding
    rn2, ci2, v2 = ctx.ell_download(_lib.GF_F64)
    agg, side = ctx.twolevel_aggregates()
    _, it_o = tl.TwoLevel(m.coords, rn2, ci2, v2, _fixed(m), agg=agg, side=side).pcg(f, 1e-12)
    assert abs(info.iterations - it_o) <= max(2, it_o // 20), (info.iterations, it_o)


@pytest.mark.parametrize("name,scale", CASES)
def test_twolevel_on_fp32_matrix_with_reliable_updates(oracle, name, scale):
    """matrix = GF_F32: SpMVs on K32, FP64 vectors, residual replaced from K64."""
    m = mg.workload(name, scale=scale)
    ctx = _ctx(m)
    ctx.convert_f64_to_f32()
    rn, ci, v = oracle.assemble(m.elem_type, m.ngauss, m.coords, m.conn, m.E0, m.nu, E_elem=m.E)
    v, f = oracle.eliminate(rn, ci, v, _fixed(m), m.f)
    ustar, _ = oracle.cg(rn, ci, v, f, maxit=200000, eps=1e-13, precond=True)
    info = ctx.solve(_lib.GF_SOLVER_TWOLEVEL_PCG, _lib.GF_F32, tol=1e-10, max_iter=200000)
    assert info.status == _lib.GF_OK and info.rel_residual <= 1e-10 and info.outer >= 2
    u = ctx.solution()
    assert np.linalg.norm(u - ustar) <= 1e-7 * np.linalg.norm(ustar)
    info64 = ctx.solve(_lib.GF_SOLVER_TWOLEVEL_PCG, _lib.GF_F64, tol=1e-10, max_iter=200000)
    assert info.iterations <= 2 * info64.iterations + 10, (info.iterations, info64.iterations)


@pytest.mark.parametrize("name,scale", CASES)
def test_twolevel_fp32_recursion_with_reliable_updates(oracle, name, scale):
    """GF_SOLVER_TWOLEVEL_PCG32: K32 SpMVs and FP32 vectors in the recursion, FP64 dot
    products, residual replaced from K64: converges to the FP64 oracle solution."""
    m = mg.workload(name, scale=scale)
    ctx = _ctx(m)
    ctx.convert_f64_to_f32()
    rn, ci, v = oracle.assemble(m.elem_type, m.ngauss, m.coords, m.conn, m.E0, m.nu, E_elem=m.E)
    v, f = oracle.eliminate(rn, ci, v, _fixed(m), m.f)
    ustar, _ = oracle.cg(rn, ci, v, f, maxit=200000, eps=1e-13, precond=True)
    info = ctx.solve(_lib.GF_SOLVER_TWOLEVEL_PCG32, _lib.GF_F32, tol=1e-10, max_iter=200000)
    assert info.status == _lib.GF_OK and info.rel_residual <= 1e-10 and info.outer >= 2
    u = ctx.solution()
    assert np.linalg.norm(u - ustar) <= 1e-7 * np.linalg.norm(ustar)
    info64 = ctx.solve(_lib.GF_SOLVER_TWOLEVEL_PCG, _lib.GF_F64, tol=1e-10, max_iter=200000)
    assert info.iterations <= 2 * info64.iterations + 10, (info.iterations, info64.iterations)


def test_twolevel_fp32_recursion_needs_both_matrices():
    m = mg.workload("brick8_128", scale=1 / 16)
    ctx = _ctx(m)   # K64 only
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.solve(_lib.GF_SOLVER_TWOLEVEL_PCG32, _lib.GF_F32, tol=1e-8)
    assert ei.value.status == _lib.GF_ERR_STATE


@pytest.mark.parametrize("name", ["ref_Q8", "ref_brick8", "ref_2bricks20", "ref_placa16_Q4"])
def test_penalty_twolevel_matches_reference(name):
    """FEM::ApplyConstraint(PEN), then two-level PCG, against the reference's CG
    solution (eps 1e-10) stored in the golden fixture."""
    from gpufem_b200.fem import Context
    g = load_golden(name)
    ctx = Context(0)
    ctx.mesh_create(int(g["elem_type"]), g["coords"], g["conn"], int(g["ngauss"]), float(g["E"]),
                    None, float(g["nu"]))
    ctx.set_supports(g["supports"])
    ctx.set_force(g["force"])
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_COLOR)
    ctx.apply_constraints(_lib.GF_BC_PENALTY)
    info = ctx.solve(_lib.GF_SOLVER_TWOLEVEL_PCG, tol=1e-12, max_iter=20000)
    ref = g["u_cg_fp64"]
    assert info.status == _lib.GF_OK
    assert np.linalg.norm(ctx.solution() - ref) <= 1e-6 * np.linalg.norm(ref)


def test_twolevel_state_errors_and_rebuild():
    from gpufem_b200.fem import Context
    m = mg.workload("q8_512", scale=1 / 32)
    ctx = _ctx(m)
    assert ctx.twolevel_setup(100000) <= tl.MAX_COARSE     # capped
    assert ctx.twolevel_setup(3) == 3                       # one aggregate: 3 modes in 2-D
    info = ctx.solve(_lib.GF_SOLVER_TWOLEVEL_PCG, tol=1e-10, max_iter=100000)
    assert info.status == _lib.GF_OK
    u1 = ctx.solution()
    # new values: the next solve rebuilds the coarse space for them
    ctx.set_modulus(2.0 * m.E0, 2.0 * m.E)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_AUTO)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    info = ctx.solve(_lib.GF_SOLVER_TWOLEVEL_PCG, tol=1e-10, max_iter=100000)
    assert info.status == _lib.GF_OK
    assert np.linalg.norm(ctx.solution() - 0.5 * u1) <= 1e-8 * np.linalg.norm(u1)
    # an uploaded matrix has no mesh: the two-level solver refuses it
    ctx2 = Context(0)
    ctx2.ell_upload(np.array([1, 1], np.int32), np.array([[0, 1]], np.int32),
                    np.array([[2.0, 3.0]]))
    with pytest.raises(_lib.GpufemError) as ei:
        ctx2.solve(_lib.GF_SOLVER_TWOLEVEL_PCG, tol=1e-8)
    assert ei.value.status == _lib.GF_ERR_STATE
    with pytest.raises(_lib.GpufemError):
        ctx.twolevel_setup(-1)
