"""Helpers shared by the tests: column-major ELL <-> dense / dict, tolerances."""
from __future__ import annotations

import numpy as np


def ell_to_dict(rownnz, colidx, vals):
    """{(row, col): value} over the stored entries (slots < rownnz)."""
    out = {}
    W, n = colidx.shape
    for r in range(n):
        for s in range(int(rownnz[r])):
            out[(r, int(colidx[s, r]))] = float(vals[s, r])
    return out


def ell_to_dense(rownnz, colidx, vals, n=None):
    W, nn = colidx.shape
    n = nn if n is None else n
    A = np.zeros((n, n))
    mask = np.arange(W)[:, None] < np.asarray(rownnz)[None, :]
    rows = np.broadcast_to(np.arange(nn)[None, :], (W, nn))[mask]
    np.add.at(A, (rows, colidx[mask]), np.asarray(vals, np.float64)[mask])
    return A


def row_rel_err(A, B):
    """max over rows of max|A - B| / max|A_row| (rows with max|A| = 0 use 1)."""
    scale = np.abs(A).max(axis=1)
    scale[scale == 0] = 1.0
    return float((np.abs(A - B).max(axis=1) / scale).max())


def ell_from_entries(n, entries):
    """Build a column-major ELL (rownnz, colidx (W, n), vals (W, n)) from
    {(row, col): value}; columns sorted per row."""
    rows = [[] for _ in range(n)]
    for (r, c), v in entries.items():
        rows[r].append((c, v))
    W = max(1, max(len(x) for x in rows))
    rownnz = np.zeros(n, np.int32)
    colidx = np.tile(np.arange(n, dtype=np.int32), (W, 1))
    vals = np.zeros((W, n))
    for r, x in enumerate(rows):
        x.sort()
        rownnz[r] = len(x)
        for s, (c, v) in enumerate(x):
            colidx[s, r] = c
            vals[s, r] = v
    return rownnz, colidx, vals
