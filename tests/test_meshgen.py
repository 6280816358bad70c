"""Synthetic workloads: sizes match the hot-path table, loads are consistent, the
neutral-file round trip through the reference's reader is exact.  CPU only."""
import numpy as np
import pytest

from gpufem_b200 import meshgen as mg
from oracle.oracle import Reference


def count_nodes(et, n):
    dim = mg.DIM[et]
    if et in (mg.Q4, mg.BRICK8):
        return int(np.prod([v + 1 for v in n]))
    if et == mg.Q8:
        nx, ny = n
        return (2 * nx + 1) * (2 * ny + 1) - nx * ny
    nx, ny, nz = n
    corners = (nx + 1) * (ny + 1) * (nz + 1)
    edges = nx * (ny + 1) * (nz + 1) + (nx + 1) * ny * (nz + 1) + (nx + 1) * (ny + 1) * nz
    return corners + edges


@pytest.mark.parametrize("et,n,nodes", [
    (mg.Q4, (64, 64), 4225), (mg.Q8, (512, 512), 788481), (mg.BRICK8, (128,) * 3, 2146689),
    (mg.BRICK20, (64,) * 3, 1085825)])
def test_workload_node_counts(et, n, nodes):
    assert count_nodes(et, n) == nodes


@pytest.mark.parametrize("et,n", [(mg.Q4, (5, 4)), (mg.Q8, (4, 5)), (mg.BRICK8, (3, 2, 4)),
                                  (mg.BRICK20, (2, 3, 2))])
def test_structured_counts_and_orientation(oracle, et, n):
    m = mg.structured(et, n, jitter=0.2, seed=4)
    assert m.nnodes == count_nodes(et, n)
    assert m.nelem == int(np.prod(n))
    assert m.conn.min() == 1 and m.conn.max() == m.nnodes
    # every element has positive detJ at every Gauss point
    pts, _ = oracle.gauss(m.dim, 3)
    for e in range(m.nelem):
        X = m.coords[m.conn[e] - 1]
        for p in pts:
            dN = oracle.dshape(et, p)
            assert np.linalg.det(dN @ X) > 0


@pytest.mark.parametrize("et,n,W", [(mg.Q4, (4, 4), 18), (mg.Q8, (4, 4), 42),
                                    (mg.BRICK8, (3, 3, 3), 81), (mg.BRICK20, (3, 3, 3), 243)])
def test_ell_width_matches_table(oracle, et, n, W):
    m = mg.structured(et, n)
    rn, ci = oracle.pattern(et, m.nnodes, m.conn)
    assert ci.shape[0] == W == rn.max()


def test_jitter_bounds_and_boundary_fixed():
    h = 1.0 / 8
    m0 = mg.structured(mg.BRICK20, (8, 8, 8), jitter=0.0)
    m = mg.structured(mg.BRICK20, (8, 8, 8), jitter=0.05, seed=7)
    d = m.coords - m0.coords
    assert np.abs(d).max() <= 0.05 * h + 1e-15
    on_bnd = np.any((m0.coords < 1e-12) | (m0.coords > 1 - 1e-12), axis=1)
    assert np.all(d[on_bnd] == 0)
    # mid-side nodes stay at the midpoint of their end corners
    e = m.conn[100] - 1
    assert np.allclose(m.coords[e[1]], 0.5 * (m.coords[e[0]] + m.coords[e[2]]))


def test_seeded_reproducible():
    a = mg.workload("q8_512", scale=1 / 32)
    b = mg.workload("q8_512", scale=1 / 32)
    assert np.array_equal(a.coords, b.coords) and np.array_equal(a.E, b.E)


@pytest.mark.parametrize("name,total", [("q4_64", 1.0), ("q8_512", 1.0), ("brick8_128", -1.0),
                                        ("brick20_64", -1.0)])
def test_consistent_loads_sum(name, total):
    m = mg.workload(name, scale=1 / 16)
    f = m.f.reshape(m.nnodes, m.dim)
    comp = 0 if m.dim == 2 else 2
    assert np.isclose(f[:, comp].sum(), total)
    assert np.allclose(np.delete(f, comp, axis=1), 0)


def test_correlated_field_statistics():
    m = mg.structured(mg.BRICK20, (16, 16, 16))
    E = mg.lognormal_correlated(m, 1.0, 0.1, seed=3)
    g = np.log(E / 210e3)
    assert abs(g.mean()) < 1e-12 and abs(g.std() - 1.0) < 1e-12
    # neighbours in x are correlated, far elements much less
    G = g.reshape(16, 16, 16, order="F")
    c1 = np.corrcoef(G[:-1].ravel(), G[1:].ravel())[0, 1]
    c8 = np.corrcoef(G[:-8].ravel(), G[8:].ravel())[0, 1]
    assert c1 > 0.5 and c8 < 0.2


def test_parity_colouring_is_valid():
    m = mg.structured(mg.BRICK8, (4, 3, 2))
    for a in range(1, m.nnodes + 1):
        els = np.nonzero(np.any(m.conn == a, axis=1))[0]
        assert len(set(m.colors[els].tolist())) == len(els)


@pytest.mark.skipif(not Reference.available("fp64"), reason="reference build absent")
@pytest.mark.parametrize("et", [mg.Q4, mg.Q8, mg.BRICK8, mg.BRICK20])
def test_neutral_file_round_trip(et):
    m = mg.clamp_and_load(mg.structured(et, (2,) * mg.DIM[et], jitter=0.1, seed=1))
    s = Reference("fp64").open_mesh(m)
    assert np.array_equal(s.connect(), m.conn)
    assert np.array_equal(s.coords(), m.coords)
    assert np.array_equal(s.supports(), m.supports)
    f = s.force()
    assert np.allclose(f, m.f.astype(np.float32), rtol=1e-7)
