"""Parity of the CUDA assembly (through the C-ABI) with the reference's golden
vectors and with the oracle.  Tolerances (row-relative: max|A-B| / max|A_row|):
FP64 1e-12, FP32 1e-6; ELL column indices and row lengths bit-exact against the
topological pattern."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from ellutil import ell_to_dense, row_rel_err
from gpufem_b200 import _lib
from gpufem_b200 import meshgen as mg

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-6
SCATTERS = [_lib.GF_SCATTER_COLOR, _lib.GF_SCATTER_ATOMIC, _lib.GF_SCATTER_OWNER,
            _lib.GF_SCATTER_AUTO]


@pytest.fixture(scope="module")
def fem():
    from gpufem_b200.fem import Context
    return Context


def make_ctx(Context, g=None, mesh=None, E_elem=None):
    ctx = Context(0)
    if g is not None:
        ctx.mesh_create(int(g["elem_type"]), g["coords"], g["conn"], int(g["ngauss"]),
                        float(g["E"]), None, float(g["nu"]))
    else:
        ctx.mesh_create(mesh.elem_type, mesh.coords, mesh.conn, mesh.ngauss, mesh.E0,
                        mesh.E if E_elem is None else E_elem, mesh.nu)
    return ctx


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("scatter", SCATTERS)
def test_fp64_assembly_matches_reference(fem, oracle, name, scatter):
    g = load_golden(name)
    ctx = make_ctx(fem, g)
    ctx.assemble(_lib.GF_F64, scatter)
    rn, ci, v = ctx.ell_download(_lib.GF_F64)
    # pattern: bit-exact against the topological oracle pattern
    orn, oci = oracle.pattern(int(g["elem_type"]), g["coords"].shape[0], g["conn"])
    assert np.array_equal(rn, orn)
    assert np.array_equal(ci, oci)
    # reference rows are subsets of ours (value-dependent pattern, zeros dropped)
    for r in range(rn.size):
        assert set(g["colidx_fp64"][: g["rownnz_fp64"][r], r]) <= set(ci[: rn[r], r])
    n = rn.size
    A = ell_to_dense(g["rownnz_fp64"], g["colidx_fp64"], g["vals_fp64"], n)
    B = ell_to_dense(rn, ci, v, n)
    assert row_rel_err(A, B) <= TOL64
    # padding slots hold col = row and value 0
    W = ci.shape[0]
    pad = np.arange(W)[:, None] >= rn[None, :]
    assert np.all(v[pad] == 0) and np.all(ci[pad] == np.broadcast_to(np.arange(n), (W, n))[pad])


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("scatter", SCATTERS)
def test_fp32_assembly_matches_reference(fem, name, scatter):
    g = load_golden(name)
    ctx = make_ctx(fem, g)
    ctx.assemble(_lib.GF_F32, scatter)
    rn, ci, v = ctx.ell_download(_lib.GF_F32)
    n = rn.size
    A = ell_to_dense(g["rownnz_fp32"], g["colidx_fp32"], g["vals_fp32"].astype(np.float64), n)
    B = ell_to_dense(rn, ci, v.astype(np.float64), n)
    assert row_rel_err(A, B) <= TOL32
    A64 = ell_to_dense(g["rownnz_fp64"], g["colidx_fp64"], g["vals_fp64"], n)
    assert row_rel_err(A64, B) <= TOL32


@pytest.mark.parametrize("et,n,ng", [(mg.Q4, (9, 7), 2), (mg.Q8, (6, 5), 3), (mg.Q8, (5, 4), 2),
                                     (mg.BRICK8, (5, 4, 3), 2), (mg.BRICK8, (3, 3, 3), 3),
                                     (mg.BRICK20, (3, 3, 2), 3), (mg.BRICK20, (3, 2, 2), 2)])
def test_per_element_modulus_matches_oracle(fem, oracle, et, n, ng):
    m = mg.structured(et, n, jitter=0.2, seed=31, ngauss=ng)
    E = mg.lognormal_iid(m, 1.0, seed=5)
    ctx = make_ctx(fem, mesh=m, E_elem=E)
    ro, co, vo = oracle.assemble(et, ng, m.coords, m.conn, 210e3, m.nu, E_elem=E)
    A = ell_to_dense(ro, co, vo)
    for dtype, tol in ((_lib.GF_F64, TOL64), (_lib.GF_F32, TOL32)):
        for scatter in SCATTERS:
            ctx.assemble(dtype, scatter)
            rn, ci, v = ctx.ell_download(dtype)
            assert np.array_equal(ci, co)
            assert row_rel_err(A, ell_to_dense(rn, ci, v.astype(np.float64))) <= tol


def _fan_mesh(et, k, R=2.5):
    """k quadrilaterals around one centre node (the centre has k elements; every other
    node one or two): spoke nodes at radius 1, outer corners at radius R between the
    spokes, counter-clockwise in the reference's node order; Q8 adds the edge midpoints."""
    th = 2 * np.pi * np.arange(k) / k
    xy = [[0.0, 0.0]] + [[np.cos(t), np.sin(t)] for t in th] + \
         [[R * np.cos(t + np.pi / k), R * np.sin(t + np.pi / k)] for t in th]
    conn = [[1, 2 + j, 2 + k + j, 2 + (j + 1) % k] for j in range(k)]   # 1-based
    if et == mg.Q8:
        mids = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in mids:
                xy.append([(xy[a - 1][0] + xy[b - 1][0]) / 2, (xy[a - 1][1] + xy[b - 1][1]) / 2])
                mids[key] = len(xy)
            return mids[key]
        conn = [c + [mid(c[0], c[1]), mid(c[1], c[2]), mid(c[2], c[3]), mid(c[3], c[0])]
                for c in conn]
    return np.array(xy), np.array(conn, np.int32)


# (R keeps the elements well enough shaped for the FP32 tolerance: a numpy FP32
# restatement of Ke gives 2-3e-7 of max|row| on these, against 1e-5 for a Q8 fan of 5
# elements with R = 1.6)
@pytest.mark.parametrize("et,k,R,fp32", [(mg.Q4, 5, 2.5, True), (mg.Q4, 7, 2.5, True),
                                         (mg.Q8, 3, 1.6, True), (mg.Q8, 5, 2.5, True),
                                         (mg.Q8, 9, 3.0, True), (mg.Q8, 11, 3.0, True),
                                         (mg.Q4, 34, 2.0, False)])
def test_irregular_node_degree_matches_oracle(fem, oracle, et, k, R, fp32):
    """A node shared by k elements, through each per-node pattern pass: 32 register keys
    (at most 32 element-node slots per node: Q4 k = 5, 7, Q8 k = 3), 64 (Q8 k = 5: 40
    slots), the warp's shared-memory sort (Q8 k = 9: 72 slots) and the general passes
    (Q4 k = 34: more than 32 elements at a node; FP64 only, its 34 slivers are beyond the
    FP32 tolerance); then the owner kernels (Q8 k = 11: rows of 112 slots, too wide for the
    thread-per-node row tile, take the task kernel in FP32 too) and every schedule against
    the oracle."""
    xy, conn = _fan_mesh(et, k, R)
    ctx = fem(0)
    ctx.mesh_create(et, xy, conn, 3, 210e3, None, 0.3)
    ro, co, vo = oracle.assemble(et, 3, xy, conn, 210e3, 0.3)
    A = ell_to_dense(ro, co, vo)
    for dtype, tol in ((_lib.GF_F64, TOL64), (_lib.GF_F32, TOL32))[:2 if fp32 else 1]:
        for scatter in SCATTERS:
            ctx.assemble(dtype, scatter)
            rn, ci, v = ctx.ell_download(dtype)
            assert np.array_equal(rn, ro) and np.array_equal(ci, co)
            assert row_rel_err(A, ell_to_dense(rn, ci, v.astype(np.float64))) <= tol


class _I32View:
    """A device int32 buffer as __cuda_array_interface__ (zero-copy)."""

    def __init__(self, ptr, count):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<i4",
                                         "data": (int(ptr), False), "version": 3,
                                         "strides": None, "stream": None}


@pytest.mark.parametrize("name,scale", [("q8_512", 1.0), ("brick8_128", 0.25),
                                        ("brick20_64", 0.25)])
def test_download_expands_pattern_exactly(fem, name, scale):
    """gf_ell_download sends a mesh-built pattern as its node adjacency and expands rownnz
    and colidx on host threads: bit-equal to the device arrays (read through gf_ell_view)."""
    import ctypes as C
    import torch
    m = mg.workload(name, scale=scale)
    ctx = make_ctx(fem, mesh=m)
    ctx.assemble(_lib.GF_F32)
    rn, ci, v = ctx.ell_download(_lib.GF_F32)
    n, W = C.c_int32(), C.c_int32()
    drn, dci, dv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    _lib.check(_lib.lib.gf_ell_view(ctx.h, _lib.GF_F32, C.byref(n), C.byref(W), C.byref(drn),
                                    C.byref(dci), C.byref(dv)), ctx.h)
    rn_dev = torch.as_tensor(_I32View(drn.value, n.value), device="cuda").cpu().numpy()
    ci_dev = torch.as_tensor(_I32View(dci.value, n.value * W.value), device="cuda").cpu().numpy()
    assert np.array_equal(rn, rn_dev)
    assert np.array_equal(ci.ravel(), ci_dev)


def test_colour_and_atomic_agree_and_parity_colouring(fem):
    m = mg.workload("brick20_64", scale=1 / 8)
    ctx = make_ctx(fem, mesh=m)
    nc = ctx.color(m.colors)
    assert nc == 8
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_COLOR)
    _, _, v1 = ctx.ell_download(_lib.GF_F64)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_ATOMIC)
    _, _, v2 = ctx.ell_download(_lib.GF_F64)
    assert np.abs(v1 - v2).max() <= 1e-13 * np.abs(v1).max()
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)
    _, _, v3 = ctx.ell_download(_lib.GF_F64)
    assert np.abs(v1 - v3).max() <= 1e-13 * np.abs(v1).max()
    # library greedy colouring equals the oracle's (reference femColor rule)
    ctx2 = make_ctx(fem, mesh=m)
    nc2 = ctx2.color(None)
    from oracle.oracle import Oracle
    col, ncol = Oracle().greedy_color(m.elem_type, m.nnodes, m.conn)
    assert nc2 == ncol
    assert np.array_equal(ctx2.colors(m.nelem), col)


def test_invalid_colouring_rejected(fem):
    m = mg.structured(mg.Q4, (4, 4))
    ctx = make_ctx(fem, mesh=m)
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.color(np.zeros(m.nelem, np.int32))
    assert ei.value.status == _lib.GF_ERR_INVALID_ARG


def test_distorted_element_fp32_uses_fp64_jacobian(fem, oracle):
    """An element with max/min detJ > 10 over its Gauss points: FP32 stays within
    tolerance of the FP64 oracle (the FP32 path switches J, J^-1 to FP64)."""
    m = mg.structured(mg.BRICK20, (1, 1, 1), ngauss=3)
    # taper: the cross-section shrinks linearly with z to 5% at the top face; the
    # map is linear along every edge, so mid-side nodes stay at edge midpoints
    X = m.coords.copy()
    s = 1.0 - 0.95 * X[:, 2]
    X[:, 0] = (X[:, 0] - 0.5) * s + 0.5
    X[:, 1] = (X[:, 1] - 0.5) * s + 0.5
    m.coords = X
    e = m.conn[0] - 1
    ctx = make_ctx(fem, mesh=m)
    ro, co, vo = oracle.assemble(mg.BRICK20, 3, X, m.conn, 210e3, 0.3)
    pts, _ = oracle.gauss(3, 3)
    dets = [np.linalg.det(oracle.dshape(mg.BRICK20, p) @ X[e]) for p in pts]
    assert min(dets) > 0 and max(dets) / min(dets) > 10
    for scatter in SCATTERS:
        ctx.assemble(_lib.GF_F32, scatter)
        rn, ci, v = ctx.ell_download(_lib.GF_F32)
        B = ell_to_dense(rn, ci, v.astype(np.float64))
        assert row_rel_err(ell_to_dense(ro, co, vo), B) <= TOL32


def test_single_element_and_isolated_node(fem, oracle):
    m = mg.structured(mg.Q8, (1, 1), ngauss=3)
    coords = np.vstack([m.coords, [[5.0, 5.0]]])      # node 9 belongs to no element
    ctx = fem(0)
    ctx.mesh_create(mg.Q8, coords, m.conn, 3, 210e3, None, 0.3)
    ro, co, vo = oracle.assemble(mg.Q8, 3, m.coords, m.conn, 210e3, 0.3)
    A = ell_to_dense(ro, co, vo)
    for scatter in SCATTERS:
        ctx.assemble(_lib.GF_F64, scatter)
        rn, ci, v = ctx.ell_download(_lib.GF_F64)
        assert rn[-1] == 0 and rn[-2] == 0
        assert np.all(v[:, -2:] == 0)
        B = ell_to_dense(rn, ci, v)[:16, :16]
        assert row_rel_err(A, B) <= TOL64


@pytest.mark.parametrize("bad", ["zero_id", "too_big", "repeat", "ngauss", "nu", "modulus"])
def test_invalid_mesh_rejected(fem, bad):
    m = mg.structured(mg.Q4, (2, 2))
    conn = m.conn.copy()
    ng, nu, E = 2, 0.3, 210e3
    if bad == "zero_id":
        conn[0, 0] = 0
    elif bad == "too_big":
        conn[0, 0] = m.nnodes + 1
    elif bad == "repeat":
        conn[0, 1] = conn[0, 0]
    elif bad == "ngauss":
        ng = 4
    elif bad == "nu":
        nu = 0.5
    elif bad == "modulus":
        E = -1.0
    ctx = fem(0)
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.mesh_create(mg.Q4, m.coords, conn, ng, E, None, nu)
    assert ei.value.status == _lib.GF_ERR_INVALID_ARG


def test_state_errors(fem):
    ctx = fem(0)
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.assemble()
    assert ei.value.status == _lib.GF_ERR_STATE


@pytest.mark.parametrize("name", ["q8_512", "brick20_64"])
def test_full_size_rigid_translation(fem, name):
    """Size-independent property at the full workload size: K annihilates rigid
    translations (before constraints), checked with the device SpMV."""
    m = mg.workload(name)
    ctx = make_ctx(fem, mesh=m)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_COLOR)
    n = m.ndof
    _, W = ctx.ell_shape()
    x = np.random.default_rng(0).standard_normal(n)
    scale = np.abs(ctx.spmv(x, _lib.GF_F64)).max()     # ~ max|K| * sqrt(W)
    for c in range(m.dim):
        u = np.zeros((m.nnodes, m.dim))
        u[:, c] = 1.0
        y = ctx.spmv(u.ravel(), _lib.GF_F64)
        assert np.abs(y).max() <= 1e-13 * W * scale
    ctx.assemble(_lib.GF_F32, _lib.GF_SCATTER_COLOR)
    y32 = ctx.spmv(x, _lib.GF_F32)
    y64 = ctx.spmv(x, _lib.GF_F64)
    assert np.linalg.norm(y32 - y64) <= 1e-5 * np.linalg.norm(y64)


def test_rejected_mesh_keeps_current_and_reuse_is_exact(fem, oracle):
    """A mesh that fails validation leaves the current one usable; re-creating meshes
    (same shape, then another shape, then the first again) reuses pooled buffers and
    gives the same matrix every time."""
    m = mg.structured(mg.Q8, (6, 5), jitter=0.2, seed=4, ngauss=3)
    other = mg.structured(mg.BRICK8, (3, 3, 2), jitter=0.1, seed=5, ngauss=2)
    ctx = fem(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, 3, 210e3, None, 0.3)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)
    first = ctx.ell_download(_lib.GF_F64)
    bad = m.conn.copy()
    bad[2, 3] = bad[2, 0]
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.mesh_create(m.elem_type, m.coords, bad, 3, 210e3, None, 0.3)
    assert ei.value.status == _lib.GF_ERR_INVALID_ARG
    assert "repeats node" in str(ei.value)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)      # the current mesh still works
    again = ctx.ell_download(_lib.GF_F64)
    for a, b in zip(first, again):
        assert np.array_equal(a, b)
    ctx.mesh_create(other.elem_type, other.coords, other.conn, 2, 210e3, None, 0.3)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)
    rn, ci, v = ctx.ell_download(_lib.GF_F64)
    rno, cio, vo = oracle.assemble(other.elem_type, 2, other.coords, other.conn, 210e3, 0.3)
    assert np.array_equal(rn, rno)
    for _ in range(2):
        ctx.mesh_create(m.elem_type, m.coords, m.conn, 3, 210e3, None, 0.3)
        ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)
        third = ctx.ell_download(_lib.GF_F64)
        for a, b in zip(first, third):
            assert np.array_equal(a, b)
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.set_modulus(-5.0)
    assert ei.value.status == _lib.GF_ERR_INVALID_ARG
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)      # modulus unchanged
    for a, b in zip(first, ctx.ell_download(_lib.GF_F64)):
        assert np.array_equal(a, b)
