"""The TF32 tensor-core engine (GF_ENGINE_TF32_MMA): element Gram matrices on the
tcgen05 tensor cores (TMEM accumulators, three TF32 products of split operands), against
the oracle and the reference's golden vectors with the FP32 tolerance (row-relative
1e-6), on the colour and atomic schedules."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from ellutil import ell_to_dense, row_rel_err
from gpufem_b200 import _lib
from gpufem_b200 import meshgen as mg

pytestmark = pytest.mark.gpu

TOL32 = 1e-6
TF32 = _lib.GF_ENGINE_TF32_MMA
SCATTERS = [_lib.GF_SCATTER_COLOR, _lib.GF_SCATTER_ATOMIC, _lib.GF_SCATTER_OWNER,
            _lib.GF_SCATTER_AUTO]


def _ctx(mesh, E_elem=None):
    from gpufem_b200.fem import Context
    ctx = Context(0)
    ctx.mesh_create(mesh.elem_type, mesh.coords, mesh.conn, mesh.ngauss, mesh.E0,
                    mesh.E if E_elem is None else E_elem, mesh.nu)
    return ctx


@pytest.mark.parametrize("et,n,ng", [(mg.Q4, (9, 7), 2), (mg.Q8, (6, 5), 3), (mg.Q8, (5, 4), 2),
                                     (mg.BRICK8, (5, 4, 3), 2), (mg.BRICK8, (3, 3, 3), 3),
                                     (mg.BRICK20, (3, 3, 2), 3), (mg.BRICK20, (3, 2, 2), 2)])
def test_tf32_engine_matches_oracle(oracle, et, n, ng):
    m = mg.structured(et, n, jitter=0.2, seed=31, ngauss=ng)
    E = mg.lognormal_iid(m, 1.0, seed=5)
    ctx = _ctx(m, E)
    ro, co, vo = oracle.assemble(et, ng, m.coords, m.conn, 210e3, m.nu, E_elem=E)
    A = ell_to_dense(ro, co, vo)
    for scatter in SCATTERS:
        ctx.assemble(_lib.GF_F32, scatter, TF32)
        rn, ci, v = ctx.ell_download(_lib.GF_F32)
        assert np.array_equal(ci, co) and np.array_equal(rn, ro)
        assert row_rel_err(A, ell_to_dense(rn, ci, v.astype(np.float64))) <= TOL32, scatter


@pytest.mark.parametrize("name", golden_names())
def test_tf32_engine_matches_reference(name):
    g = load_golden(name)
    from gpufem_b200.fem import Context
    ctx = Context(0)
    ctx.mesh_create(int(g["elem_type"]), g["coords"], g["conn"], int(g["ngauss"]), float(g["E"]),
                    None, float(g["nu"]))
    ctx.assemble(_lib.GF_F32, _lib.GF_SCATTER_ATOMIC, TF32)
    rn, ci, v = ctx.ell_download(_lib.GF_F32)
    n = rn.size
    B = ell_to_dense(rn, ci, v.astype(np.float64), n)
    A64 = ell_to_dense(g["rownnz_fp64"], g["colidx_fp64"], g["vals_fp64"], n)
    assert row_rel_err(A64, B) <= TOL32


def test_tf32_engine_distorted_element(oracle):
    """max/min detJ > 10: the gradients come from the FP64 Jacobian as on CUDA cores."""
    m = mg.structured(mg.BRICK20, (1, 1, 1), ngauss=3)
    X = m.coords.copy()
    s = 1.0 - 0.95 * X[:, 2]
    X[:, 0] = (X[:, 0] - 0.5) * s + 0.5
    X[:, 1] = (X[:, 1] - 0.5) * s + 0.5
    m.coords = X
    ctx = _ctx(m)
    ro, co, vo = oracle.assemble(mg.BRICK20, 3, X, m.conn, 210e3, 0.3)
    for scatter in SCATTERS:
        ctx.assemble(_lib.GF_F32, scatter, TF32)
        rn, ci, v = ctx.ell_download(_lib.GF_F32)
        assert row_rel_err(ell_to_dense(ro, co, vo), ell_to_dense(rn, ci, v.astype(np.float64))) <= TOL32


@pytest.mark.parametrize("scatter", [_lib.GF_SCATTER_ATOMIC, _lib.GF_SCATTER_OWNER])
def test_tf32_engine_full_size_brick20_agrees_with_cuda_cores(scatter):
    m = mg.workload("brick20_64", scale=1 / 4)
    ctx = _ctx(m)
    ctx.assemble(_lib.GF_F32, _lib.GF_SCATTER_ATOMIC)
    x = np.random.default_rng(3).standard_normal(m.ndof)
    y0 = ctx.spmv(x, _lib.GF_F32)
    ctx.assemble(_lib.GF_F32, scatter, TF32)
    y1 = ctx.spmv(x, _lib.GF_F32)
    assert np.linalg.norm(y1 - y0) <= 1e-6 * np.linalg.norm(y0)


def test_tf32_engine_argument_errors():
    m = mg.structured(mg.Q8, (2, 2), ngauss=3)
    ctx = _ctx(m)
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_ATOMIC, TF32)
    assert ei.value.status == _lib.GF_ERR_INVALID_ARG


@pytest.mark.parametrize("et,n,ng,swap", [(mg.BRICK8, (3, 2, 2), 2, [(0, 4), (1, 5), (2, 6), (3, 7)]),
                                          (mg.BRICK20, (2, 2, 1), 3, None),
                                          (mg.Q8, (3, 3), 3, [(1, 7), (2, 6), (3, 5)])])
def test_tf32_engine_inverted_element(oracle, et, n, ng, swap):
    """An element whose node order is mirrored (detJ < 0 at every Gauss point: the
    reference assembles it with the negative weights as they come).  Its group forms M on
    the CUDA cores from the operand tiles; the others stay on the tensor cores.  The
    mirrored element's Ke cancels against its neighbours' in the assembled rows, which
    amplifies FP32 rounding relative to max|row| for either engine (the CUDA-core kernel
    measures 9.1e-7 on the Brick20 case), so the bound is the FP32 tolerance or 1.25x the
    CUDA-core engine's own error on the same mesh, whichever is larger."""
    m = mg.structured(et, n, jitter=0.1, seed=4, ngauss=ng)
    conn = m.conn.copy()
    if swap is None:   # Brick20: mirror r -> -r (corner and mid-side nodes on r = +1 / -1)
        swap = [(0, 12), (1, 13), (2, 14), (3, 15), (4, 16), (5, 17), (6, 18), (7, 19)]
    for a, b in swap:
        conn[1, [a, b]] = conn[1, [b, a]]
    m.conn = conn
    ro, co, vo = oracle.assemble(et, ng, m.coords, m.conn, 210e3, m.nu)
    A = ell_to_dense(ro, co, vo)
    ctx = _ctx(m)
    for scatter in SCATTERS:
        ctx.assemble(_lib.GF_F32, scatter)
        rn, ci, v = ctx.ell_download(_lib.GF_F32)
        cc = row_rel_err(A, ell_to_dense(rn, ci, v.astype(np.float64)))
        ctx.assemble(_lib.GF_F32, scatter, TF32)
        rn, ci, v = ctx.ell_download(_lib.GF_F32)
        tc = row_rel_err(A, ell_to_dense(rn, ci, v.astype(np.float64)))
        assert tc <= max(TOL32, 1.25 * cc), (scatter, tc, cc)
