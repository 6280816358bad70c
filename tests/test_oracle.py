"""The oracle pinned against the reference: committed golden vectors (made by the
reference's own compiled CPU code) and, where the reference build is present, the
live reference library.  CPU only."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from ellutil import ell_from_entries, ell_to_dense, row_rel_err
from gpufem_b200 import meshgen as mg
from oracle.oracle import Reference


def _topology_subset(ref_rn, ref_ci, rn, ci):
    """Reference rows (value-dependent, H3) must be subsets of the topological rows."""
    missing = 0
    for r in range(len(rn)):
        ours = set(ci[: rn[r], r].tolist())
        theirs = set(ref_ci[: ref_rn[r], r].tolist())
        if not theirs <= ours:
            return False, r
        missing += len(ours - theirs)
    return True, missing


@pytest.mark.parametrize("name", golden_names())
def test_oracle_assembly_matches_reference_fp64(oracle, name):
    g = load_golden(name)
    et, ng = int(g["elem_type"]), int(g["ngauss"])
    rn, ci, v = oracle.assemble(et, ng, g["coords"], g["conn"], float(g["E"]), float(g["nu"]))
    ok, info = _topology_subset(g["rownnz_fp64"], g["colidx_fp64"], rn, ci)
    assert ok, f"reference column outside the topological pattern in row {info}"
    n = rn.size
    A = ell_to_dense(g["rownnz_fp64"], g["colidx_fp64"], g["vals_fp64"], n)
    B = ell_to_dense(rn, ci, v, n)
    assert row_rel_err(A, B) <= 1e-12
    # entries the reference omitted (exact zeros, H3) are zero or roundoff here
    omitted = (A == 0) & (B != 0)
    if omitted.any():
        assert np.abs(B[omitted]).max() <= 1e-12 * np.abs(B).max()


@pytest.mark.parametrize("name", golden_names())
def test_oracle_fp32_reference_within_tolerance(oracle, name):
    """The reference's FP32 K sits within 1e-6 (row-relative) of the FP64 oracle."""
    g = load_golden(name)
    et, ng = int(g["elem_type"]), int(g["ngauss"])
    rn, ci, v = oracle.assemble(et, ng, g["coords"], g["conn"], float(g["E"]), float(g["nu"]))
    n = rn.size
    A = ell_to_dense(g["rownnz_fp32"], g["colidx_fp32"], g["vals_fp32"].astype(np.float64), n)
    B = ell_to_dense(rn, ci, v, n)
    assert row_rel_err(B, A) <= 1e-6


@pytest.mark.parametrize("name", golden_names())
def test_oracle_penalty_matches_reference(oracle, name):
    g = load_golden(name)
    et, ng = int(g["elem_type"]), int(g["ngauss"])
    rn, ci, v = oracle.assemble(et, ng, g["coords"], g["conn"], float(g["E"]), float(g["nu"]))
    dim = g["coords"].shape[1]
    fixed = np.zeros(rn.size, np.uint8)
    for row in g["supports"]:
        for c in range(dim):
            if row[1 + c] == 1:
                fixed[(row[0] - 1) * dim + c] = 1
    vp = oracle.penalty(rn, ci, v, fixed)
    diag = np.array([vp[np.nonzero(ci[: rn[r], r] == r)[0][0], r] for r in range(rn.size)])
    ref = g["diag_pen_fp64"]
    assert np.allclose(diag, ref, rtol=1e-12, atol=0)


@pytest.mark.parametrize("name", golden_names())
def test_oracle_cg_matches_reference(oracle, name):
    """Plain CG (x0 = 0, stop at ||r|| <= eps ||b||) on the penalty-modified K."""
    g = load_golden(name)
    et, ng = int(g["elem_type"]), int(g["ngauss"])
    rn, ci, v = oracle.assemble(et, ng, g["coords"], g["conn"], float(g["E"]), float(g["nu"]))
    dim = g["coords"].shape[1]
    fixed = np.zeros(rn.size, np.uint8)
    for row in g["supports"]:
        for c in range(dim):
            if row[1 + c] == 1:
                fixed[(row[0] - 1) * dim + c] = 1
    vp = oracle.penalty(rn, ci, v, fixed)
    x, it = oracle.cg(rn, ci, vp, g["force"], maxit=20000, eps=1e-10, precond=False)
    ref = g["u_cg_fp64"]
    assert np.linalg.norm(x - ref) <= 1e-6 * max(np.linalg.norm(ref), 1e-300)


def test_gauss_rule_order(oracle):
    """Tensor order i (first coordinate) outermost, weights multiply (FemData.cc:226-316)."""
    pts, w = oracle.gauss(3, 3)
    a = np.sqrt(3 / 5)
    assert np.allclose(pts[0], [-a, -a, -a]) and np.allclose(pts[1], [-a, -a, 0])
    assert np.allclose(pts[9], [0, -a, -a])
    assert np.isclose(w.sum(), 8.0)
    pts2, w2 = oracle.gauss(2, 2)
    assert np.allclose(pts2[1], [-1 / np.sqrt(3), 1 / np.sqrt(3)]) and np.allclose(w2, 1.0)


@pytest.mark.parametrize("et", [mg.Q4, mg.Q8, mg.BRICK8, mg.BRICK20])
def test_partition_of_unity_derivatives(oracle, et):
    rng = np.random.default_rng(3)
    dim = mg.DIM[et]
    for _ in range(5):
        p = rng.uniform(-1, 1, dim)
        dN = oracle.dshape(et, p)
        assert np.allclose(dN.sum(axis=1), 0.0, atol=1e-14)
        # derivative of sum_i N_i x_i with x_i = natural coords is the identity
        nat = np.array(mg.NAT[et], float)
        assert np.allclose(dN @ nat, np.eye(dim), atol=1e-14)


@pytest.mark.parametrize("et", [mg.Q4, mg.Q8, mg.BRICK8, mg.BRICK20])
def test_element_rigid_modes_and_symmetry(oracle, et):
    m = mg.structured(et, (1,) * mg.DIM[et], jitter=0.0, ngauss=3)
    X = m.coords[m.conn[0] - 1] + 0.03 * np.random.default_rng(1).standard_normal(m.coords[m.conn[0] - 1].shape)
    D = oracle.dmatrix(m.dim, 0, 210e3, 0.3)
    Ke = oracle.element_ke(et, 3, X, D)
    assert np.abs(Ke - Ke.T).max() <= 1e-10 * np.abs(Ke).max()
    for c in range(m.dim):  # rigid translations
        u = np.zeros(X.shape)
        u[:, c] = 1.0
        assert np.abs(Ke @ u.ravel()).max() <= 1e-9 * np.abs(Ke).max()
    w = np.linalg.eigvalsh(Ke)
    nrigid = 3 if m.dim == 2 else 6
    assert np.all(w[nrigid:] > 1e-8 * w[-1]), "spurious zero-energy modes"


# ---- known answers from the reference's own tests --------------------------
def test_kat_cg_8x8(oracle):
    """LAopsTest.cpp:108-137: diag(i^2) with K00 = 2, K01 = K10 = 2 -> x = (-1, 1.5, 1, ...)."""
    n = 8
    e = {(i, i): float((i + 1) ** 2) for i in range(n)}
    e[(0, 0)] = 2.0
    e[(0, 1)] = 2.0
    e[(1, 0)] = 2.0
    b = np.array([(i + 1) ** 2 for i in range(n)], float)
    rn, ci, v = ell_from_entries(n, e)
    x, _ = oracle.cg(rn, ci, v, b, maxit=3000, eps=1e-5, precond=False)
    assert np.allclose(x, [-1, 1.5] + [1] * 6, atol=1e-3)


def test_kat_cg_tridiagonal(oracle):
    """AxyGPUTest.cpp:288-318: [-1 2 -1] 4x4, b = 1 -> (2, 3, 3, 2)."""
    n = 4
    e = {}
    for i in range(n):
        e[(i, i)] = 2.0
        if i + 1 < n:
            e[(i, i + 1)] = -1.0
        if i - 1 >= 0:
            e[(i, i - 1)] = -1.0
    rn, ci, v = ell_from_entries(n, e)
    x, _ = oracle.cg(rn, ci, v, np.ones(n), maxit=200, eps=1e-5, precond=False)
    assert np.allclose(x, [2, 3, 3, 2], atol=1e-3)


def test_kat_cg_ones_plus_identity(oracle):
    """AxyGPUTest.cpp:334-358: ones(32) + I, b = 1 -> x_i = 1/33."""
    n = 32
    e = {(i, j): (2.0 if i == j else 1.0) for i in range(n) for j in range(n)}
    rn, ci, v = ell_from_entries(n, e)
    x, _ = oracle.cg(rn, ci, v, np.ones(n), maxit=500, eps=1e-5, precond=False)
    assert np.allclose(x, 0.0303, atol=1e-3)


def test_kat_spmv_diagonal_and_band(oracle):
    """AxyGPUTest.cpp:44-160: diagonal i -> y = i^2; band of ones -> 2*band."""
    n = 4096
    rn, ci, v = ell_from_entries(n, {(i, i): float(i + 1) for i in range(n)})
    x = np.arange(1, n + 1, dtype=float)
    assert np.allclose(oracle.spmv(rn, ci, v, x), x * x)
    n, band = 64, 8
    rn, ci, v = ell_from_entries(n, {(i, j): 1.0 for i in range(n) for j in range(band)})
    assert np.allclose(oracle.spmv(rn, ci, v, np.full(n, 2.0)), 2.0 * band)
    band = 4
    e = {(i, i + j): 1.0 for i in range(n) for j in range(band) if i + j < n}
    rn, ci, v = ell_from_entries(n, e)
    y = oracle.spmv(rn, ci, v, np.full(n, 2.0))
    yres = np.full(n, 2.0 * band)
    for i in range(1, band):
        yres[n - band + i] -= 2 * i
    assert np.allclose(y, yres)


def test_greedy_coloring_valid(oracle):
    m = mg.structured(mg.BRICK20, (3, 3, 2), jitter=0.05, seed=2)
    col, nc = oracle.greedy_color(m.elem_type, m.nnodes, m.conn)
    assert nc >= 8
    for a in range(m.nnodes):
        els = np.nonzero(np.any(m.conn == a + 1, axis=1))[0]
        assert len(set(col[els].tolist())) == len(els)


# ---- live reference (present only where its sources were compiled) ---------
needs_ref = pytest.mark.skipif(not Reference.available("fp64"), reason="reference build absent")


@needs_ref
def test_reference_stepped_search_kat():
    """SPRSearchTest.cpp:160-200 on the compiled ELLmatrix::BinSearchIntStep."""
    R = Reference("fp64")
    v = np.zeros(16, np.int32)
    v[:10] = [1, 2, 3, 4, 5, 6, 11, 16, 20, 21]
    import ctypes as C
    p = v.ctypes.data_as(C.c_void_p)
    cases = [((0, 5, 0, 2), 0), ((3, 5, 0, 2), 2), ((4, 5, 0, 2), 4), ((12, 5, 0, 2), 8),
             ((22, 5, 0, 2), -1), ((1, 5, 1, 2), 1), ((3, 5, 1, 2), 3), ((5, 5, 1, 2), 5),
             ((30, 5, 1, 2), -1)]
    for args, want in cases:
        assert R.lib.ref_binsearch_step(p, *args) == want


@needs_ref
@pytest.mark.parametrize("et,n,ng", [(mg.Q4, (5, 4), 2), (mg.Q8, (4, 3), 3),
                                     (mg.BRICK8, (3, 2, 2), 2), (mg.BRICK20, (2, 2, 1), 3)])
def test_oracle_vs_live_reference_coloured(oracle, et, n, ng):
    """Colour-scheduled reference assembly (femColor + CalcStiffnessColoring) equals
    the oracle, and the reference's greedy colour count equals the oracle's."""
    R = Reference("fp64")
    m = mg.clamp_and_load(mg.structured(et, n, jitter=0.15, seed=9, ngauss=ng, E0=100.0, nu=0.25))
    s = R.open_mesh(m)
    s.assemble(coloring=True, nthreads=2)
    rn, ci, v = s.ell()
    ro, co, vo = oracle.assemble(et, ng, m.coords, m.conn, 100.0, 0.25)
    assert row_rel_err(ell_to_dense(rn, ci, v), ell_to_dense(ro, co, vo)) <= 1e-12
    _, nc = oracle.greedy_color(et, m.nnodes, m.conn)
    assert s.num_colors() == nc


def test_residual_dd_is_exact_to_double_double():
    """or_residual_dd against exact rational arithmetic on a small ELL system whose
    solution is held as u_hi + u_lo: the FP64 residual f - K u_hi loses the u_lo part and
    the rounding of K u; the compensated one keeps both."""
    from fractions import Fraction
    from oracle.oracle import Oracle
    rng = np.random.default_rng(7)
    n, W = 40, 5
    rownnz = rng.integers(1, W + 1, n).astype(np.int32)
    colidx = np.zeros((W, n), np.int32)
    vals = np.zeros((W, n))
    for i in range(n):
        cols = np.sort(rng.choice(n, rownnz[i], replace=False))
        colidx[: rownnz[i], i] = cols
        vals[: rownnz[i], i] = rng.standard_normal(rownnz[i]) * 10.0 ** rng.integers(-3, 4)
    uh = rng.standard_normal(n)
    ul = uh * 1e-17 * rng.standard_normal(n)
    f = np.zeros(n)
    for i in range(n):   # f close to K u so that the residual cancels heavily
        f[i] = sum(vals[j, i] * uh[colidx[j, i]] for j in range(rownnz[i]))
    r, nrm = Oracle().residual_dd(rownnz, colidx, vals, f, uh, ul)
    for i in range(n):
        exact = Fraction(f[i]) - sum(Fraction(vals[j, i]) * (Fraction(uh[colidx[j, i]])
                                                              + Fraction(ul[colidx[j, i]]))
                                     for j in range(rownnz[i]))
        scale = max(abs(Fraction(vals[j, i]) * Fraction(uh[colidx[j, i]]))
                    for j in range(rownnz[i]))
        assert abs(Fraction(r[i]) - exact) <= Fraction(2.0 ** -100) * scale + abs(exact) * Fraction(2.0 ** -52)
    assert np.isclose(nrm, np.linalg.norm(r))


def test_reference_axy_on_external_ell_matches_oracle_spmv():
    """The reference's own ELLmatrix::Axy lent a caller's ELL (ref_ell_axy_external)
    equals the oracle's SpMV on an assembled matrix."""
    from oracle.oracle import Oracle, Reference
    if not Reference.available("fp64"):
        pytest.skip("reference oracle build absent")
    from gpufem_b200 import meshgen as mg
    m = mg.clamp_and_load(mg.structured(mg.BRICK8, (3, 3, 2), jitter=0.1, seed=2))
    O = Oracle()
    rn, ci, v = O.assemble(m.elem_type, m.ngauss, m.coords, m.conn, m.E0, m.nu)
    x = np.random.default_rng(1).standard_normal(m.ndof)
    y, _ = Reference("fp64").ell_axy(rn, ci, v, x, nthreads=2)
    assert np.allclose(y, O.spmv(rn, ci, v, x), rtol=1e-13, atol=1e-9 * np.abs(v).max())
