"""TEST INFRASTRUCTURE ONLY — numpy restatement of the learned preconditioner
(forward, losses and backward), the checker for the CUDA kernels in
gpufem_b200/csrc/gf_learned.cu.  The reference has no learned preconditioner, so
this oracle restates the network as include/gpufem_b200.h documents it.

Network (hidden width 64, weights used as BF16, FP64 arithmetic here):
  rho = r / d, v1 = (K rho) / d, v2 = (K v1) / d, c = rms(rho)
  f_a = [rho_a / c, v1_a / c, v2_a / c, log(d_a / geomean d)]     (4 dim features)
  h0 = relu(W0 f + b0); h_{l+1} = relu(Ws_l h_l + Wn_l mean_{N(a)} h_l + b_l), l < 3
  y = Wout h3 + bout;  M(r) = rho + c y
Losses for a pair (r, e), z = M(r):
  "error":    L = sum d (z - e)^2 / sum d e^2
  "residual": L = sum (K (e - z))^2 / d / sum (K e)^2 / d
"""
from __future__ import annotations

import numpy as np

H = 64
LAYERS = 3


def offsets(dim: int) -> dict:
    F = 4 * dim
    o, p = {}, 0

    def take(name, size):
        nonlocal p
        o[name] = (p, size)
        p += size

    take("W0", H * F)
    take("b0", H)
    for l in range(LAYERS):
        take(f"Ws{l}", H * H)
        take(f"Wn{l}", H * H)
        take(f"b{l + 1}", H)
    take("Wout", dim * H)
    take("bout", dim)
    o["total"] = (p, 0)
    return o


def to_bf16(w: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), returned as float64."""
    u = np.ascontiguousarray(w, np.float32).view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = (u + 0x7FFF + lsb) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w: np.ndarray, dim: int, bf16: bool = True) -> dict:
    o = offsets(dim)
    wb = to_bf16(w) if bf16 else np.asarray(w, np.float64)
    F = 4 * dim
    out = {}
    for name, (p, size) in o.items():
        if name == "total":
            continue
        a = wb[p:p + size]
        if name == "W0":
            a = a.reshape(H, F)
        elif name.startswith("Ws") or name.startswith("Wn"):
            a = a.reshape(H, H)
        elif name == "Wout":
            a = a.reshape(dim, H)
        out[name] = a
    return out


def node_adjacency(conn1: np.ndarray, nnodes: int):
    """Sorted neighbour lists (nodes sharing an element, self included)."""
    nb = [set() for _ in range(nnodes)]
    for e in conn1 - 1:
        for a in e:
            nb[a].update(e.tolist())
    return [np.array(sorted(s), np.int64) for s in nb]


def _aggregate(adj, h):
    return np.stack([h[nbrs].mean(axis=0) for nbrs in adj])


def _aggregate_t(adj, g):
    deg_inv = np.array([1.0 / len(nbrs) for nbrs in adj])
    gs = g * deg_inv[:, None]
    return np.stack([gs[nbrs].sum(axis=0) for nbrs in adj])


def forward(w, dim, adj, d, r, K, bf16=True):
    """z = M(r); K is the matrix (anything with K @ x), d its diagonal."""
    P = unpack(w, dim, bf16)
    N = len(adj)
    rho = r / d
    v1 = (K @ rho) / d
    v2 = (K @ v1) / d
    c = np.sqrt(np.mean(rho * rho)) + 1e-30
    logd = np.log(d) - np.mean(np.log(d))
    f = np.concatenate([(rho / c).reshape(N, dim), (v1 / c).reshape(N, dim),
                        (v2 / c).reshape(N, dim), logd.reshape(N, dim)], axis=1)
    cache = {"f": f, "rho": rho, "c": c}
    pre0 = f @ P["W0"].T + P["b0"]
    h = np.maximum(pre0, 0)
    cache["pre0"], cache["h0"] = pre0, h
    for l in range(LAYERS):
        agg = _aggregate(adj, h)
        pre = h @ P[f"Ws{l}"].T + agg @ P[f"Wn{l}"].T + P[f"b{l + 1}"]
        cache[f"agg{l}"] = agg
        h = np.maximum(pre, 0)
        cache[f"pre{l + 1}"], cache[f"h{l + 1}"] = pre, h
    y = (h @ P["Wout"].T + P["bout"]).reshape(-1)
    cache["y"] = y
    return rho + c * y, cache


def loss_and_grad(w, dim, adj, d, r, e, K, loss="error", bf16=True):
    P = unpack(w, dim, bf16)
    z, cache = forward(w, dim, adj, d, r, K, bf16)
    c = cache["c"]
    if loss == "error":
        S = np.sum(d * e * e)
        diff = z - e
        L = np.sum(d * diff * diff) / S
        dz = 2.0 * d * diff / S
    elif loss == "residual":
        t = K @ e
        S = np.sum(t * t / d)
        s_ = K @ (e - z)
        L = np.sum(s_ * s_ / d) / S
        dz = -2.0 * (K @ (s_ / d)) / S
    else:
        raise ValueError(loss)
    dy = (c * dz).reshape(-1, dim)
    o = offsets(dim)
    g = np.zeros(o["total"][0])

    def put(name, val):
        p, size = o[name]
        g[p:p + size] += val.reshape(-1)

    h3 = cache[f"h{LAYERS}"]
    put("Wout", dy.T @ h3)
    put("bout", dy.sum(axis=0))
    dh = dy @ P["Wout"]
    for l in reversed(range(LAYERS)):
        dpre = dh * (cache[f"pre{l + 1}"] > 0)
        put(f"Ws{l}", dpre.T @ cache[f"h{l}"])
        put(f"Wn{l}", dpre.T @ cache[f"agg{l}"])
        put(f"b{l + 1}", dpre.sum(axis=0))
        dh = dpre @ P[f"Ws{l}"] + _aggregate_t(adj, dpre @ P[f"Wn{l}"])
    dpre0 = dh * (cache["pre0"] > 0)
    put("W0", dpre0.T @ cache["f"])
    put("b0", dpre0.sum(axis=0))
    return L, g, z
