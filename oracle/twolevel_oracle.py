"""TEST INFRASTRUCTURE ONLY — numpy restatement of the two-level preconditioner, the
checker for gpufem_b200/csrc/gf_twolevel.cu.  The reference has no preconditioner
(SPRmatrix::CPU_CG, src/SPRmatrix/SPRmatrix.cc:405-480, is plain CG), so this oracle
restates the method as include/gpufem_b200.h documents it; the solver built on it is
checked against the reference's own converged solutions.

  M r = D^-1 r + P (P^T K P)^-1 P^T r

Aggregates: boxes of a regular grid over the nodes' bounding box.  With nm rigid-body
modes per aggregate (3 in 2-D, 6 in 3-D) and cap = min(max(target, nm), 4096), the box
side starts at s = (volume / (cap / nm))^(1/k) over the k axes of positive extent; the
grid has min(cap, max(1, round(extent / s))) boxes per axis, and s grows by 5 % until
boxes * nm <= cap.  Occupied boxes, in box order
(x fastest), are the aggregates.  Columns of P per aggregate A: translations t_c, then
rotations (2-D: rot_z = (-d_y, d_x); 3-D: rot_x = (0, -d_z, d_y), rot_y = (d_z, 0, -d_x),
rot_z = (-d_y, d_x, 0)) with d = (x - centroid_A) / s; rows of constrained dofs are zero.
Ac is regularised: a zero diagonal entry becomes 1, every other gets + 1e-10 max diag.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

MAX_COARSE = 4096
DEFAULT_COARSE = 3072


def default_target(n: int) -> int:
    """The library's default coarse size for n dofs: n // 128 within [192, 3072]."""
    return min(DEFAULT_COARSE, max(192, n // 128))


def _lround(v: float) -> int:
    return int(math.floor(v + 0.5)) if v >= 0 else -int(math.floor(-v + 0.5))


def aggregates(coords: np.ndarray, target: int = DEFAULT_COARSE):
    """Node -> aggregate (0-based) and the box side."""
    x = np.asarray(coords, np.float64)
    nnodes, dim = x.shape
    nm = 3 if dim == 2 else 6
    lo = x.min(0)
    ext = x.max(0) - lo
    pos = [c for c in range(dim) if ext[c] > 0.0]
    vol = 1.0
    for c in pos:
        vol *= float(ext[c])
    cap = min(max(target, nm), MAX_COARSE)
    side = math.pow(vol / max(1.0, cap / nm), 1.0 / len(pos)) if pos else 1.0
    for _ in range(100000):
        nb = []
        for c in range(dim):
            q = float(ext[c]) / side
            nb.append(cap if q >= cap else max(1, _lround(q)))
        if int(np.prod(nb)) * nm <= cap:
            break
        side *= 1.05
    key = np.zeros(nnodes, np.int64)
    mul = 1
    for c in range(dim):
        if ext[c] > 0.0:
            b = np.floor((x[:, c] - lo[c]) / ext[c] * nb[c]).astype(np.int64)
        else:
            b = np.zeros(nnodes, np.int64)
        b = np.clip(b, 0, nb[c] - 1)
        key += b * mul
        mul *= nb[c]
    _, agg = np.unique(key, return_inverse=True)
    return agg.astype(np.int32), side


def prolongation(coords: np.ndarray, agg: np.ndarray, side: float, fixed: np.ndarray):
    x = np.asarray(coords, np.float64)
    nnodes, dim = x.shape
    nm = 3 if dim == 2 else 6
    na = int(agg.max()) + 1
    cnt = np.bincount(agg, minlength=na).astype(np.float64)
    cen = np.zeros((na, dim))
    np.add.at(cen, agg, x)
    cen /= np.maximum(cnt, 1.0)[:, None]
    d = (x - cen[agg]) / side
    rows, cols, vals = [], [], []

    def put(c, m, v):
        r = np.arange(nnodes) * dim + c
        rows.append(r)
        cols.append(agg * nm + m)
        vals.append(np.broadcast_to(v, (nnodes,)).astype(np.float64))

    for c in range(dim):
        put(c, c, 1.0)
    if dim == 2:
        put(0, 2, -d[:, 1])
        put(1, 2, d[:, 0])
    else:
        put(1, 3, -d[:, 2]); put(2, 3, d[:, 1])
        put(0, 4, d[:, 2]);  put(2, 4, -d[:, 0])
        put(0, 5, -d[:, 1]); put(1, 5, d[:, 0])
    r = np.concatenate(rows)
    cc = np.concatenate(cols)
    v = np.concatenate(vals)
    keep = fixed[r] == 0
    return sp.csr_matrix((v[keep], (r[keep], cc[keep])), shape=(nnodes * dim, na * nm))


def ell_to_csr(rownnz, colidx, vals):
    W, n = colidx.shape
    mask = np.arange(W)[:, None] < rownnz[None, :]
    rows = np.broadcast_to(np.arange(n)[None, :], (W, n))
    return sp.csr_matrix((vals[mask], (rows[mask], colidx[mask])), shape=(n, n))


def coarse_inverse(K: sp.spmatrix, P: sp.spmatrix) -> np.ndarray:
    Ac = (P.T @ (K @ P)).toarray()
    dmax = max(float(np.diag(Ac).max()), 0.0)
    for i in range(Ac.shape[0]):
        Ac[i, i] = Ac[i, i] + 1e-10 * dmax if Ac[i, i] > 0.0 else 1.0
    Ai = np.linalg.inv(Ac)
    return 0.5 * (Ai + Ai.T)


class TwoLevel:
    """M for the ELL matrix (column-major (width, n) arrays) of a mesh."""

    def __init__(self, coords, rownnz, colidx, vals, fixed, target=DEFAULT_COARSE,
                 agg=None, side=None):
        if agg is None:
            agg, side = aggregates(coords, target)
        self.agg, self.side = agg, side
        self.K = ell_to_csr(rownnz, colidx, vals)
        d = self.K.diagonal()
        self.dinv = np.where(d != 0.0, 1.0 / np.where(d != 0.0, d, 1.0), 1.0)
        self.P = prolongation(coords, agg, side, np.asarray(fixed))
        self.Ainv = coarse_inverse(self.K, self.P)

    @property
    def ncoarse(self) -> int:
        return self.Ainv.shape[0]

    def apply(self, r: np.ndarray) -> np.ndarray:
        return self.dinv * r + self.P @ (self.Ainv @ (self.P.T @ r))

    def pcg(self, b: np.ndarray, tol: float, maxit: int = 100000):
        """PCG with M (x0 = 0, stop on r.r <= tol^2 b.b); returns x, iterations."""
        x = np.zeros_like(b)
        r = b.copy()
        z = self.apply(r)
        p = z.copy()
        rz = r @ z
        tol2 = tol * tol * (b @ b)
        it = 0
        while it < maxit and r @ r > tol2:
            q = self.K @ p
            a = rz / (p @ q)
            x += a * p
            r -= a * q
            z = self.apply(r)
            rzn = r @ z
            p = z + (rzn / rz) * p
            rz = rzn
            it += 1
        return x, it
