"""The numpy oracle of the learned preconditioner is self-consistent: analytic
gradients of both losses agree with central finite differences (FP64, BF16 rounding
off), the untrained network (zero output layer) is Jacobi, and M is
scale-equivariant.  CPU."""
import numpy as np
import pytest

from gpufem_b200 import meshgen as mg
from oracle import gnn_oracle as G


def small_problem(seed=0):
    m = mg.structured(mg.BRICK8, (2, 2, 1), jitter=0.1, seed=seed)
    adj = G.node_adjacency(m.conn, m.nnodes)
    rng = np.random.default_rng(seed)
    d = np.exp(rng.normal(size=m.ndof))
    # a symmetric matrix on the dof graph of the node adjacency, diagonal d
    n = m.ndof
    A = np.zeros((n, n))
    for a, nbrs in enumerate(adj):
        for b in nbrs:
            A[3 * a:3 * a + 3, 3 * b:3 * b + 3] = rng.normal(scale=0.1, size=(3, 3))
    K = 0.5 * (A + A.T)
    K[np.arange(n), np.arange(n)] = d
    r = rng.normal(size=m.ndof)
    e = rng.normal(size=m.ndof)
    return m, adj, d, r, e, K


def random_weights(dim, seed=1, scale=0.3):
    n = G.offsets(dim)["total"][0]
    return np.random.default_rng(seed).normal(scale=scale, size=n)


def test_untrained_network_is_jacobi():
    m, adj, d, r, _, K = small_problem()
    w = random_weights(3)
    p, size = G.offsets(3)["Wout"]
    w[p:p + size] = 0
    pb, sb = G.offsets(3)["bout"]
    w[pb:pb + sb] = 0
    z, _ = G.forward(w, 3, adj, d, r, K)
    assert np.allclose(z, r / d)


def test_scale_equivariance():
    m, adj, d, r, _, K = small_problem()
    w = random_weights(3)
    z1, _ = G.forward(w, 3, adj, d, r, K)
    z2, _ = G.forward(w, 3, adj, d, 7.5 * r, K)
    assert np.allclose(z2, 7.5 * z1, rtol=1e-12)


@pytest.mark.parametrize("loss", ["error", "residual"])
def test_gradient_matches_finite_differences(loss):
    m, adj, d, r, e, K = small_problem()
    w = random_weights(3, scale=0.2)
    L, g, _ = G.loss_and_grad(w, 3, adj, d, r, e, K, loss, bf16=False)
    rng = np.random.default_rng(3)
    idx = rng.choice(w.size, 40, replace=False)
    o = G.offsets(3)
    # make sure every block is probed
    idx = np.concatenate([idx] + [[p] for name, (p, s) in o.items() if s])
    for k in idx:
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        Lp, _, _ = G.loss_and_grad(wp, 3, adj, d, r, e, K, loss, bf16=False)
        Lm, _, _ = G.loss_and_grad(wm, 3, adj, d, r, e, K, loss, bf16=False)
        fd = (Lp - Lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(fd)), (k, fd, g[k])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.001953125, -3.14159, 0.0], np.float32)
    b = G.to_bf16(x)
    assert b[0] == 1.0
    assert b[1] == 1.0        # 1 + 2^-8 lies half way between 1 and 1 + 2^-7: tie to even
    assert b[2] == 1.0        # below half way
    assert abs(b[3] + 3.140625) < 1e-6
    assert b[4] == 0.0
