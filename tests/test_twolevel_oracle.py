"""The two-level preconditioner's numpy oracle on the CPU: its aggregation rule, that
M is symmetric positive definite, and that PCG with it reaches the Jacobi-PCG solution
of the C oracle in far fewer iterations."""
import numpy as np
import pytest

from gpufem_b200 import meshgen as mg
from oracle import twolevel_oracle as tl


def _system(oracle, m):
    rn, ci, v = oracle.assemble(m.elem_type, m.ngauss, m.coords, m.conn, m.E0, m.nu, E_elem=m.E)
    fixed = np.zeros(m.ndof, np.uint8)
    for row in m.supports:
        for c in range(m.dim):
            if row[1 + c] == 1:
                fixed[(row[0] - 1) * m.dim + c] = 1
    v, f = oracle.eliminate(rn, ci, v, fixed, m.f)
    return rn, ci, v, f, fixed


@pytest.mark.parametrize("dim,target", [(2, 3072), (2, 48), (3, 96), (3, 4096)])
def test_aggregation_rule(dim, target):
    rng = np.random.default_rng(dim * 100 + target)
    x = rng.uniform(0.0, 1.0, (3000, dim)) * np.array([3.0, 1.0, 0.5][:dim])
    agg, side = tl.aggregates(x, target)
    nm = 3 if dim == 2 else 6
    na = agg.max() + 1
    assert na * nm <= min(target, tl.MAX_COARSE)
    assert np.all(np.bincount(agg) > 0)               # every aggregate holds nodes
    # numbering follows box order: aggregate ids ascend with the box key
    lo, hi = x.min(0), x.max(0)
    first = np.array([np.flatnonzero(agg == a)[0] for a in range(na)])
    b = np.floor((x[first] - lo) / (hi - lo) * np.maximum(1, np.round((hi - lo) / side))).astype(int)
    nb = np.maximum(1, np.floor((hi - lo) / side + 0.5)).astype(int)
    b = np.minimum(b, nb - 1)
    key = b[:, 0] + nb[0] * (b[:, 1] + (nb[1] * b[:, 2] if dim == 3 else 0))
    assert np.all(np.diff(key) > 0)


def test_degenerate_extent_single_aggregate():
    x = np.zeros((5, 2))
    x[:, 0] = np.linspace(0, 1, 5)            # all nodes on a line: zero y extent
    agg, side = tl.aggregates(x, 3)
    assert agg.max() == 0 and side > 0


@pytest.mark.parametrize("et,n", [(mg.Q8, (6, 5)), (mg.BRICK8, (3, 3, 2))])
def test_preconditioner_is_spd(oracle, et, n):
    m = mg.clamp_and_load(mg.structured(et, n, jitter=0.2, seed=3, ngauss=2))
    rn, ci, v, f, fixed = _system(oracle, m)
    pc = tl.TwoLevel(m.coords, rn, ci, v, fixed, target=6 * 4)
    M = np.stack([pc.apply(e) for e in np.eye(m.ndof)], 1)
    assert np.allclose(M, M.T, atol=1e-12 * np.abs(M).max())
    assert np.linalg.eigvalsh(0.5 * (M + M.T)).min() > 0.0


@pytest.mark.parametrize("name,scale", [("q8_512", 1 / 16), ("brick8_128", 1 / 16)])
def test_twolevel_pcg_matches_jacobi_pcg(oracle, name, scale):
    m = mg.workload(name, scale=scale)
    rn, ci, v, f, fixed = _system(oracle, m)
    ustar, it_j = oracle.cg(rn, ci, v, f, maxit=200000, eps=1e-12, precond=True)
    pc = tl.TwoLevel(m.coords, rn, ci, v, fixed, target=256)
    u, it_2 = pc.pcg(f, 1e-12)
    assert np.linalg.norm(u - ustar) <= 1e-8 * np.linalg.norm(ustar)
    assert it_2 * 2 < it_j, (it_2, it_j)


@pytest.mark.parametrize("n,expect", [(0, 192), (8450, 192), (46875, 366), (206763, 1615),
                                      (393216, 3072), (1576962, 3072)])
def test_default_coarse_target(n, expect):
    """The library's default coarse size: n / 128 within [192, 3072]."""
    assert tl.default_target(n) == expect
