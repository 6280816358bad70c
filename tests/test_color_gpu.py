"""Device colouring (Jones–Plassmann): a valid colouring of the element dual graph
for every element type, including shuffled (unstructured-order) meshes, and colour-
scheduled assembly on it equals the owner-computes assembly."""
import numpy as np
import pytest

from gpufem_b200 import meshgen as mg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def Context():
    from gpufem_b200.fem import Context
    return Context

CASES = [
    (mg.Q4, (9, 7), 2),
    (mg.Q8, (8, 6), 3),
    (mg.BRICK8, (5, 4, 3), 2),
    (mg.BRICK20, (3, 3, 2), 3),
]


def _shuffled(m, seed):
    """Same geometry, element order and node ids permuted."""
    rs = np.random.default_rng(seed)
    ep = rs.permutation(m.nelem)
    npm = rs.permutation(m.nnodes)            # old node -> new node
    inv = np.empty_like(npm)
    inv[npm] = np.arange(m.nnodes)
    coords = m.coords[inv]
    conn = (npm[m.conn[ep] - 1] + 1).astype(np.int32)
    return coords, conn


def _valid(conn, colors):
    nen = conn.shape[1]
    nnodes = conn.max()
    for a in range(1, nnodes + 1):
        els = np.nonzero((conn == a).any(axis=1))[0]
        c = colors[els]
        assert np.unique(c).size == c.size, f"node {a}: colours {c}"


@pytest.mark.parametrize("shuffle", [False, True])
@pytest.mark.parametrize("et,n,ngauss", CASES)
def test_device_colouring_valid_and_assembles(Context, et, n, ngauss, shuffle):
    from gpufem_b200 import _lib
    m = mg.structured(et, n, jitter=0.2, seed=11, ngauss=ngauss)
    coords, conn = _shuffled(m, 5) if shuffle else (m.coords, m.conn)
    ctx = Context(0)
    ctx.mesh_create(et, coords, conn, ngauss, 210e3, None, 0.3)
    ncol = ctx.color_device(seed=1234)
    colors = ctx.colors(conn.shape[0])
    assert colors.min() == 0 and colors.max() == ncol - 1
    _valid(conn, colors)
    assert ncol <= (8 if mg.DIM[et] == 2 else 27) + 8
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)
    _, _, v_owner = ctx.ell_download(_lib.GF_F64)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_COLOR)
    _, _, v_col = ctx.ell_download(_lib.GF_F64)
    assert np.abs(v_col - v_owner).max() <= 1e-12 * np.abs(v_owner).max()


def test_device_colouring_depends_only_on_seed(Context):
    m = mg.structured(mg.Q8, (16, 16), jitter=0.1, seed=3, ngauss=2)
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, 2, 210e3, None, 0.3)
    n1 = ctx.color_device(seed=7)
    c1 = ctx.colors(m.nelem)
    n2 = ctx.color_device(seed=7)
    c2 = ctx.colors(m.nelem)
    assert n1 == n2 and np.array_equal(c1, c2)
