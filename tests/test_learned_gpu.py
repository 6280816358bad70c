"""Learned preconditioner on the GPU: forward and gradients against the numpy
oracle, training on residual/error pairs, flexible CG with the Jacobi fallback."""
import numpy as np
import pytest

from gpufem_b200 import _lib
from gpufem_b200 import meshgen as mg
from oracle import gnn_oracle as G

pytestmark = pytest.mark.gpu


def brick8_problem(n=(4, 3, 3), seed=5, sigma=1.0):
    from gpufem_b200.fem import Context
    m = mg.clamp_and_load(mg.structured(mg.BRICK8, n, jitter=0.1, seed=seed))
    m.E = mg.lognormal_correlated(m, sigma, 0.2, seed)
    ctx = Context(0)
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)
    return m, ctx


def diag_of(ctx):
    rn, ci, v = ctx.ell_download(_lib.GF_F64)
    return np.array([v[np.nonzero(ci[: rn[r], r] == r)[0][0], r] for r in range(rn.size)])


def csr_of(ctx):
    import scipy.sparse as sp
    rn, ci, v = ctx.ell_download(_lib.GF_F64)
    W, n = ci.shape
    mask = np.arange(W)[:, None] < rn[None, :]
    rows = np.broadcast_to(np.arange(n)[None, :], (W, n))
    return sp.csr_matrix((v[mask], (rows[mask], ci[mask])), shape=(n, n))


def random_weights(dim, seed=2, scale=0.25):
    return np.random.default_rng(seed).normal(scale=scale, size=G.offsets(dim)["total"][0])


def test_untrained_network_is_jacobi():
    m, ctx = brick8_problem()
    ctx.lp_init(3, seed=1)
    r = np.random.default_rng(0).normal(size=m.ndof)
    z = ctx.lp_apply(r)
    d = diag_of(ctx)
    assert np.allclose(z, r / d, rtol=1e-6, atol=0)


# the 4x3x3 cube puts every node next to the boundary; the 16^3 cube (4,913 nodes,
# 14,739 dofs) is the smallest mesh of the learned-preconditioner workload, where the
# tensor-core layers run 39 full 128-node tiles and the aggregation walks interior nodes
@pytest.mark.parametrize("loss,n", [("error", (4, 3, 3)), ("residual", (4, 3, 3)),
                                    ("error", (16, 16, 16))])
def test_forward_and_gradient_match_oracle(loss, n):
    m, ctx = brick8_problem(n=n)
    ctx.lp_init(3, seed=1)
    if loss == "residual":
        ctx.lp_set_loss(_lib.GF_LP_LOSS_RESIDUAL)
    w = random_weights(3).astype(np.float32)
    ctx.lp_set_weights(w)
    assert np.array_equal(ctx.lp_get_weights(), w)
    rng = np.random.default_rng(1)
    r = rng.normal(size=m.ndof).astype(np.float32)
    e = rng.normal(size=m.ndof).astype(np.float32)
    d = diag_of(ctx)
    K = csr_of(ctx)
    adj = G.node_adjacency(m.conn, m.nnodes)
    z_gpu = ctx.lp_apply(r)
    L_ref, g_ref, z_ref = G.loss_and_grad(w.astype(np.float64), 3, adj, d, r.astype(np.float64),
                                          e.astype(np.float64), K, loss)
    assert np.linalg.norm(z_gpu - z_ref) <= 1e-4 * np.linalg.norm(z_ref)
    L_gpu, g_gpu = ctx.lp_loss_grad(r, e)
    assert abs(L_gpu - L_ref) <= 1e-4 * abs(L_ref)
    for name, (p, size) in G.offsets(3).items():
        if size == 0:
            continue
        a, b = g_gpu[p:p + size], g_ref[p:p + size]
        assert np.linalg.norm(a - b) <= 1e-3 * max(np.linalg.norm(b), 1e-12), name


@pytest.mark.parametrize("loss,pairs", [(_lib.GF_LP_LOSS_ERROR, "pcg"),
                                        (_lib.GF_LP_LOSS_RESIDUAL, "pcg"),
                                        (_lib.GF_LP_LOSS_ERROR, "random")])
def test_training_reduces_loss(loss, pairs):
    m, ctx = brick8_problem(n=(6, 6, 6))
    ctx.lp_init(3, seed=3)
    ctx.lp_set_loss(loss)
    if pairs == "random":
        ctx.lp_collect_random(24, seed=11)
    else:
        ctx.lp_collect(npairs=24, every=4, tol=1e-8)
    l0 = ctx.lp_train(steps=1, batch=8, lr=1e-3, seed=1)
    l1 = ctx.lp_train(steps=150, batch=8, lr=1e-3, seed=2)
    assert np.isfinite(l1) and l1 < 0.9 * l0, (l0, l1)


def test_learned_fcg_converges_and_matches_pcg():
    m, ctx = brick8_problem(n=(6, 6, 6))
    info = ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-10, max_iter=100000)
    u_pcg = ctx.solution()
    ctx.lp_init(3, seed=3)
    ctx.lp_collect(npairs=24, every=4, tol=1e-8)
    ctx.lp_train(steps=100, batch=8, lr=1e-3, seed=2)
    info2 = ctx.solve(_lib.GF_SOLVER_LEARNED_FCG, tol=1e-10, max_iter=100000)
    u = ctx.solution()
    assert info2.status == _lib.GF_OK and info2.rel_residual <= 1e-9
    assert np.linalg.norm(u - u_pcg) <= 1e-7 * np.linalg.norm(u_pcg)


def negating_weights(dim):
    """Weights whose network gives y = -2 rho / c, i.e. M(r) = -D^-1 r (z.r < 0 at the
    first step, whatever the rounding of the dot products): the first 2 dim hidden
    channels carry +-rho / c through the ReLUs unchanged, every other weight is 0; all
    values are exact in BF16."""
    o = G.offsets(dim)
    w = np.zeros(o["total"][0])
    F = 4 * dim
    W0 = np.zeros((G.H, F))
    Ws = np.zeros((G.H, G.H))
    Wout = np.zeros((dim, G.H))
    for k in range(dim):
        W0[2 * k, k], W0[2 * k + 1, k] = 1.0, -1.0
        Ws[2 * k, 2 * k] = Ws[2 * k + 1, 2 * k + 1] = 1.0
        Wout[k, 2 * k], Wout[k, 2 * k + 1] = -2.0, 2.0
    w[o["W0"][0]:o["W0"][0] + o["W0"][1]] = W0.ravel()
    for l in range(G.LAYERS):
        w[o[f"Ws{l}"][0]:o[f"Ws{l}"][0] + o[f"Ws{l}"][1]] = Ws.ravel()
    w[o["Wout"][0]:o["Wout"][0] + o["Wout"][1]] = Wout.ravel()
    return w


def test_fallback_to_jacobi_when_learned_preconditioner_is_bad():
    m, ctx = brick8_problem(n=(6, 6, 6))
    ctx.lp_init(3, seed=3)
    w = negating_weights(3).astype(np.float32)
    # (the oracle confirms the construction: M(r) = -D^-1 r)
    r = np.random.default_rng(4).normal(size=m.ndof)
    z_ref, _ = G.forward(w.astype(np.float64), 3, G.node_adjacency(m.conn, m.nnodes),
                         diag_of(ctx), r, csr_of(ctx))
    assert np.allclose(z_ref, -r / diag_of(ctx), rtol=1e-12, atol=0)
    ctx.lp_set_weights(w)
    info = ctx.solve(_lib.GF_SOLVER_LEARNED_FCG, tol=1e-10, max_iter=100000)
    assert info.status == _lib.GF_OK and info.rel_residual <= 1e-9
    assert info.fallback == 1


def test_learned_fcg_requires_init():
    m, ctx = brick8_problem()
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.solve(_lib.GF_SOLVER_LEARNED_FCG, tol=1e-8)
    assert ei.value.status == _lib.GF_ERR_STATE
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.lp_set_loss(_lib.GF_LP_LOSS_RESIDUAL)
    assert ei.value.status == _lib.GF_ERR_STATE
    ctx.lp_init(3, seed=1)
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.lp_set_loss(7)
    assert ei.value.status == _lib.GF_ERR_INVALID_ARG


def test_coarse_mode_untrained_is_twolevel():
    """With the coarse correction on, the untrained network (M = D^-1) gives
    M = D^-1 + P Ac^-1 P^T: flexible CG takes two-level PCG's iteration count."""
    m, ctx = brick8_problem(n=(8, 6, 6))
    info_tl = ctx.solve(_lib.GF_SOLVER_TWOLEVEL_PCG, tol=1e-10, max_iter=100000)
    u_tl = ctx.solution()
    ctx.lp_init(3, seed=3)
    ctx.lp_set_coarse(True)
    info = ctx.solve(_lib.GF_SOLVER_LEARNED_FCG, tol=1e-10, max_iter=100000)
    assert info.status == _lib.GF_OK and info.fallback == 0
    assert abs(info.iterations - info_tl.iterations) <= 2, (info.iterations, info_tl.iterations)
    assert np.linalg.norm(ctx.solution() - u_tl) <= 1e-7 * np.linalg.norm(u_tl)


def test_coarse_mode_trained_and_fallback_converge():
    m, ctx = brick8_problem(n=(8, 6, 6))
    info_j = ctx.solve(_lib.GF_SOLVER_PCG, _lib.GF_F64, tol=1e-10, max_iter=100000)
    u_pcg = ctx.solution()
    ctx.lp_init(3, seed=3)
    ctx.lp_set_coarse(True)
    ctx.lp_collect(npairs=16, every=2, tol=1e-8)
    ctx.lp_train(steps=50, batch=8, lr=1e-3, seed=2)
    info = ctx.solve(_lib.GF_SOLVER_LEARNED_FCG, tol=1e-10, max_iter=100000)
    assert info.status == _lib.GF_OK and info.rel_residual <= 1e-9
    assert np.linalg.norm(ctx.solution() - u_pcg) <= 1e-7 * np.linalg.norm(u_pcg)
    # a bad network falls back to FCG with D^-1 + P Ac^-1 P^T, far fewer iterations than Jacobi
    ctx.lp_set_weights(random_weights(3, seed=9, scale=3.0).astype(np.float32))
    info = ctx.solve(_lib.GF_SOLVER_LEARNED_FCG, tol=1e-10, max_iter=100000)
    assert info.status == _lib.GF_OK and info.rel_residual <= 1e-9 and info.fallback == 1
    assert np.linalg.norm(ctx.solution() - u_pcg) <= 1e-7 * np.linalg.norm(u_pcg)
    ctx.lp_set_coarse(False)
    info = ctx.solve(_lib.GF_SOLVER_LEARNED_FCG, tol=1e-10, max_iter=100000)
    assert info.status == _lib.GF_OK and info.fallback == 1


def test_random_pairs_are_k_times_error():
    """lp_collect_random: e white in the D-norm, r = K e.  With the zero network
    (M = D^-1) the error loss of a pair is sum d (D^-1 K e - e)^2 / sum d e^2, which the
    oracle evaluates from the same e; the sample mean of d e^2 is 1 per dof."""
    m, ctx = brick8_problem(n=(5, 4, 4))
    ctx.lp_init(3, seed=3)
    ctx.lp_collect_random(4, seed=5)
    L0 = ctx.lp_train(steps=1, batch=64, lr=1e-12, seed=1)
    d = diag_of(ctx)
    K = csr_of(ctx)
    rng = np.random.default_rng(0)
    vals = []
    for _ in range(64):
        e = rng.standard_normal(m.ndof) / np.sqrt(d)
        z = (K @ e) / d
        vals.append(np.sum(d * (z - e) ** 2) / np.sum(d * e * e))
    assert abs(L0 - np.mean(vals)) <= 0.1 * np.mean(vals), (L0, np.mean(vals))
    ctx.lp_set_coarse(True)
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.lp_collect_random(4, seed=5)
    assert ei.value.status == _lib.GF_ERR_UNSUPPORTED


def test_coarse_mode_needs_init():
    from gpufem_b200.fem import Context
    ctx = Context(0)
    with pytest.raises(_lib.GpufemError) as ei:
        ctx.lp_set_coarse(True)
    assert ei.value.status == _lib.GF_ERR_STATE


def _seeded_brick8(seed, lo, hi):
    rs = np.random.default_rng(seed)
    nn = int(rs.integers(lo, hi))
    m = mg.clamp_and_load(mg.structured(mg.BRICK8, (nn,) * 3, jitter=0.1, seed=seed))
    m.E = mg.lognormal_correlated(m, rs.uniform(0.5, 2.0), rs.uniform(0.05, 0.3), seed)
    m.nu = float(rs.uniform(0.2, 0.4))
    return m


def _load(ctx, m):
    ctx.mesh_create(m.elem_type, m.coords, m.conn, m.ngauss, m.E0, m.E, m.nu)
    ctx.set_supports(m.supports)
    ctx.set_force(m.f)
    ctx.assemble(_lib.GF_F64, _lib.GF_SCATTER_OWNER)
    ctx.apply_constraints(_lib.GF_BC_ELIMINATION)


def test_trained_network_gains_over_the_method_without_it():
    """What the trained network gains: beside the coarse correction (M = D^-1 + c y(r) +
    P Ac^-1 P^T), trained with the residual loss on pairs from two-level PCG runs on seeded
    Brick8 meshes, flexible CG takes fewer iterations on held-out meshes than two-level PCG
    (M = D^-1 + P Ac^-1 P^T: the same preconditioner without the network), with no fallback,
    and reaches the same solution."""
    from gpufem_b200.fem import Context
    ctx = Context(0)
    ctx.lp_init(3, seed=7)
    ctx.lp_set_loss(_lib.GF_LP_LOSS_RESIDUAL)
    ctx.lp_set_coarse(True)
    for k in range(16):
        _load(ctx, _seeded_brick8(1000 + k, 12, 19))
        ctx.lp_collect(npairs=32, every=8, tol=1e-8)
        ctx.lp_train(steps=120, batch=8, lr=1e-3, seed=k)
    its_l, its_t = [], []
    for k in range(4):
        _load(ctx, _seeded_brick8(9000 + k, 14, 19))
        info_t = ctx.solve(_lib.GF_SOLVER_TWOLEVEL_PCG, tol=1e-8, max_iter=100000)
        u_t = ctx.solution()
        info_l = ctx.solve(_lib.GF_SOLVER_LEARNED_FCG, tol=1e-8, max_iter=100000)
        assert info_l.status == _lib.GF_OK and info_l.fallback == 0
        assert info_l.rel_residual <= 1e-8
        assert np.linalg.norm(ctx.solution() - u_t) <= 1e-6 * np.linalg.norm(u_t)
        its_l.append(info_l.iterations)
        its_t.append(info_t.iterations)
    # measured on B200: 53 + 177 + 60 + 49 learned against 75 + 174 + 93 + 66 two-level
    assert sum(its_l) <= 0.95 * sum(its_t), (its_l, its_t)
    assert sum(a < b for a, b in zip(its_l, its_t)) >= 2, (its_l, its_t)
