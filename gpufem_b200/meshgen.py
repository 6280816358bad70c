"""Seeded structured meshes, material fields and loads for the hot-path workloads.

Meshes are structured grids on the unit square / cube with h = 1/n.  Interior
corner nodes are jittered by U(-a h, a h) per coordinate; boundary nodes stay in
place; mid-side nodes of Q8 / Brick20 sit at the midpoint of their (jittered)
end corners, so edges stay straight and no element inverts.  Element-local node
order is the reference's natural-coordinate order (src/FEM/StiffAlgo.cc:47-202)
and connectivity is 1-based, as FileIO/FemData store it
(src/Utils/fileIO.cc:117-239).

Random numbers come from numpy's counter-based Philox generator, one named
sub-stream per purpose (jitter, modulus field), keyed by (seed, stream id).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

Q4, Q8, BRICK8, BRICK20 = 0, 1, 2, 3
NEN = {Q4: 4, Q8: 8, BRICK8: 8, BRICK20: 20}
DIM = {Q4: 2, Q8: 2, BRICK8: 3, BRICK20: 3}
NAMES = {Q4: "Q4", Q8: "Q8", BRICK8: "BRICK8", BRICK20: "BRICK20"}

# natural coordinates of element nodes, reference order
NAT = {
    Q4: [(-1, -1), (1, -1), (1, 1), (-1, 1)],
    Q8: [(-1, -1), (0, -1), (1, -1), (1, 0), (1, 1), (0, 1), (-1, 1), (-1, 0)],
    BRICK8: [(1, -1, -1), (1, 1, -1), (1, 1, 1), (1, -1, 1),
             (-1, -1, -1), (-1, 1, -1), (-1, 1, 1), (-1, -1, 1)],
    BRICK20: [(1, -1, -1), (1, 0, -1), (1, 1, -1), (1, 1, 0), (1, 1, 1), (1, 0, 1), (1, -1, 1),
              (1, -1, 0), (0, -1, -1), (0, 1, -1), (0, 1, 1), (0, -1, 1), (-1, -1, -1),
              (-1, 0, -1), (-1, 1, -1), (-1, 1, 0), (-1, 1, 1), (-1, 0, 1), (-1, -1, 1),
              (-1, -1, 0)],
}

STREAM_JITTER = 1
STREAM_MODULUS = 2


def rng(seed: int, stream: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(key=[seed & 0xFFFFFFFFFFFFFFFF, stream]))


@dataclass
class Mesh:
    elem_type: int
    n: tuple                      # elements per direction
    coords: np.ndarray            # (nnodes, dim) float64
    conn: np.ndarray              # (nelem, nen) int32, 1-based
    E: Optional[np.ndarray]       # (nelem,) float64 or None (scalar E0)
    E0: float = 210e3
    nu: float = 0.3
    ngauss: int = 2
    supports: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    f: Optional[np.ndarray] = None  # (ndof,) float64
    colors: Optional[np.ndarray] = None  # (nelem,) int32, parity colouring

    @property
    def dim(self) -> int:
        return DIM[self.elem_type]

    @property
    def nen(self) -> int:
        return NEN[self.elem_type]

    @property
    def nnodes(self) -> int:
        return self.coords.shape[0]

    @property
    def nelem(self) -> int:
        return self.conn.shape[0]

    @property
    def ndof(self) -> int:
        return self.nnodes * self.dim

    def nodal_loads(self) -> np.ndarray:
        """Rows (node id 1-based, f_x, f_y[, f_z]) for every loaded node."""
        f = self.f.reshape(self.nnodes, self.dim)
        nodes = np.nonzero(np.any(f != 0.0, axis=1))[0]
        return np.column_stack([nodes + 1.0, f[nodes]]).astype(np.float64)


def structured(elem_type: int, n, jitter: float = 0.0, seed: int = 0, ngauss: int = 2,
               E0: float = 210e3, nu: float = 0.3) -> Mesh:
    """Structured mesh of the unit square (n = (nx, ny)) or cube (n = (nx, ny, nz))."""
    dim = DIM[elem_type]
    if np.isscalar(n):
        n = (int(n),) * dim
    n = tuple(int(v) for v in n)
    quadratic = elem_type in (Q8, BRICK20)
    step = 2 if quadratic else 1
    fine = tuple(step * v + 1 for v in n)                # points per direction
    grids = np.meshgrid(*[np.arange(m) for m in fine], indexing="ij")
    idx = np.stack([g.ravel(order="F") for g in grids], axis=1)  # x fastest
    if quadratic:
        odd = (idx % 2).sum(axis=1)
        keep = odd <= 1                                    # corners and edge mid-points
    else:
        keep = np.ones(idx.shape[0], bool)
    node_of = -np.ones(idx.shape[0], np.int64)
    node_of[keep] = np.arange(int(keep.sum()))
    pts = idx[keep]
    h = np.array([1.0 / v for v in n])
    x = pts.astype(np.float64) / step * h                 # exact grid positions

    # jitter interior corner nodes
    if jitter > 0.0:
        corner = np.all(pts % step == 0, axis=1)
        interior = np.all((pts > 0) & (pts < np.array(fine) - 1), axis=1)
        sel = np.nonzero(corner & interior)[0]
        g = rng(seed, STREAM_JITTER)
        d = g.uniform(-jitter, jitter, size=(sel.size, dim)) * h
        x[sel] += d
        if quadratic:
            # mid-side nodes: midpoint of the two end corners along the odd axis
            mids = np.nonzero(~corner)[0]
            mp = pts[mids]
            ax = np.argmax(mp % 2, axis=1)
            lo = mp.copy()
            hi = mp.copy()
            lo[np.arange(mids.size), ax] -= 1
            hi[np.arange(mids.size), ax] += 1
            def flat(p):
                mult = np.cumprod((1,) + fine[:-1])
                return (p * mult).sum(axis=1)
            x[mids] = 0.5 * (x[node_of[flat(lo)]] + x[node_of[flat(hi)]])

    # connectivity
    ecoords = np.meshgrid(*[np.arange(v) for v in n], indexing="ij")
    eidx = np.stack([g.ravel(order="F") for g in ecoords], axis=1)  # element (ex, ey[, ez]), x fastest
    nat = np.array(NAT[elem_type])
    mult = np.cumprod((1,) + fine[:-1])
    conn = np.empty((eidx.shape[0], nat.shape[0]), np.int64)
    for k, xi in enumerate(nat):
        if quadratic:
            p = 2 * eidx + 1 + xi
        else:
            p = eidx + (xi + 1) // 2
        conn[:, k] = node_of[(p * mult).sum(axis=1)]
    assert np.all(conn >= 0)
    # parity colouring: elements with the same (ex%2, ey%2[, ez%2]) share no node
    colors = np.zeros(eidx.shape[0], np.int32)
    for a in range(dim):
        colors += (eidx[:, a] % 2).astype(np.int32) << a
    return Mesh(elem_type=elem_type, n=n, coords=x, conn=(conn + 1).astype(np.int32), E=None,
                E0=E0, nu=nu, ngauss=ngauss, colors=colors)


# ---------------------------------------------------------------------------
# modulus fields
# ---------------------------------------------------------------------------
def lognormal_iid(mesh: Mesh, sigma: float, seed: int, E0: float = 210e3) -> np.ndarray:
    z = rng(seed, STREAM_MODULUS).standard_normal(mesh.nelem)
    return np.exp(np.log(E0) + sigma * z)


def lognormal_correlated(mesh: Mesh, sigma: float, corr_len: float, seed: int,
                         E0: float = 210e3) -> np.ndarray:
    """E = exp(ln E0 + sigma g), g a zero-mean unit-variance Gaussian field with
    covariance exp(-r^2 / (2 l^2)) at element centroids, by FFT filtering of white
    noise on the (periodic) centroid grid, then renormalised to unit variance."""
    n = mesh.n
    w = rng(seed, STREAM_MODULUS).standard_normal(n[::-1]).T  # axes (x, y[, z])
    ks = np.meshgrid(*[2 * np.pi * np.fft.fftfreq(m, d=1.0 / m) for m in n], indexing="ij")
    k2 = sum(k * k for k in ks)
    filt = np.exp(-0.25 * k2 * corr_len * corr_len)      # sqrt of the Gaussian spectrum
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    g = (g - g.mean()) / g.std()
    return np.exp(np.log(E0) + sigma * g.ravel(order="F"))


# ---------------------------------------------------------------------------
# boundary conditions and consistent loads
# ---------------------------------------------------------------------------
def _boundary_nodes(mesh: Mesh, axis: int, value: float) -> np.ndarray:
    return np.nonzero(np.abs(mesh.coords[:, axis] - value) < 1e-12)[0]


def clamp_and_load(mesh: Mesh, traction: float = 1.0, pressure: float = 1.0) -> Mesh:
    """2-D: x = 0 edge clamped, uniform x-traction on x = 1.
    3-D: z = 0 face clamped, uniform pressure on z = 1 (force along -z).
    Loads are the consistent nodal forces of the element edge/face."""
    dim = mesh.dim
    f = np.zeros((mesh.nnodes, dim))
    if dim == 2:
        fixed = _boundary_nodes(mesh, 0, 0.0)
        nx, ny = mesh.n
        hy = 1.0 / ny
        right = mesh.conn[np.arange(mesh.nelem) % nx == nx - 1] - 1
        if mesh.elem_type == Q4:
            for a, b in ((1, 2),):
                np.add.at(f[:, 0], right[:, a], traction * hy / 2)
                np.add.at(f[:, 0], right[:, b], traction * hy / 2)
        else:
            np.add.at(f[:, 0], right[:, 2], traction * hy / 6)
            np.add.at(f[:, 0], right[:, 3], traction * hy * 2 / 3)
            np.add.at(f[:, 0], right[:, 4], traction * hy / 6)
    else:
        fixed = _boundary_nodes(mesh, 2, 0.0)
        nx, ny, nz = mesh.n
        area = 1.0 / (nx * ny)
        ez = np.arange(mesh.nelem) // (nx * ny)
        top = mesh.conn[ez == nz - 1] - 1
        nat = np.array(NAT[mesh.elem_type])
        face = np.nonzero(nat[:, 2] == 1)[0]
        for k in face:
            if mesh.elem_type == BRICK8:
                wgt = 0.25
            else:
                wgt = -1.0 / 12.0 if np.all(nat[k] != 0) else 1.0 / 3.0
            np.add.at(f[:, 2], top[:, k], -pressure * area * wgt)
    sup = np.zeros((fixed.size, dim + 1), np.int32)
    sup[:, 0] = fixed + 1
    sup[:, 1:] = 1
    mesh.supports = sup
    mesh.f = f.ravel()
    return mesh


# ---------------------------------------------------------------------------
# named workloads
# ---------------------------------------------------------------------------
def workload(name: str, scale: float = 1.0, seed_base: int = 20260101) -> Mesh:
    """The five hot-path workloads; `scale` shrinks the element count per direction
    (parity runs use scale < 1; the bench uses 1)."""
    def nn(v):
        return max(2, int(round(v * scale)))
    if name == "q4_64":
        m = structured(Q4, (nn(64), nn(64)), jitter=0.2, seed=seed_base + 1, ngauss=2)
    elif name == "q8_512":
        m = structured(Q8, (nn(512), nn(512)), jitter=0.15, seed=seed_base + 2, ngauss=3)
        m.E = lognormal_iid(m, 0.5, seed_base + 2)
    elif name == "brick8_128":
        m = structured(BRICK8, (nn(128),) * 3, jitter=0.1, seed=seed_base + 3, ngauss=2)
    elif name == "brick20_64":
        m = structured(BRICK20, (nn(64),) * 3, jitter=0.05, seed=seed_base + 4, ngauss=3)
        m.E = lognormal_correlated(m, 1.0, 0.1, seed_base + 4)
    else:
        raise ValueError(f"unknown workload {name}")
    return clamp_and_load(m)


# ---------------------------------------------------------------------------
# neutral-file writer (input format of FileIO::ReadNF, src/Utils/fileIO.cc:73-404)
# ---------------------------------------------------------------------------
# FileIO renumbers Brick20 connectivity on read: stored[k] = file[NF_BRICK20[k]]
NF_BRICK20 = [0, 7, 6, 11, 18, 19, 12, 8, 1, 5, 17, 13, 2, 3, 4, 10, 16, 15, 14, 9]


def write_nf(mesh: Mesh, path: str, analysis: str = "plane_stress") -> None:
    """Write `mesh` so that ReadNF returns exactly mesh.coords / mesh.conn /
    mesh.supports / nodal loads.  Sections are ordered so the reader finds each
    one scanning forward."""
    tag = {Q4: "Q4", Q8: "Q8", BRICK8: "BRICK8", BRICK20: "BRICK20"}[mesh.elem_type]
    lines = []
    lines.append("%ELEMENT")
    lines.append(str(mesh.nelem))
    lines.append("")
    lines.append(f"%ELEMENT.{tag}")
    lines.append(str(mesh.nelem))
    # the reader skips 4 leading integers on Q4/Q8 lines and 3 on brick lines
    lead = "1\t1\t1" if mesh.dim == 2 else "1\t1"
    conn = mesh.conn
    if mesh.elem_type == BRICK20:
        filec = np.empty_like(conn)
        filec[:, NF_BRICK20] = conn
        conn = filec
    for e in range(mesh.nelem):
        lines.append(f"{e + 1}\t{lead}\t" + "\t".join(str(int(v)) for v in conn[e]))
    lines.append("")
    lines.append("%HEADER.ANALYSIS")
    lines.append(f"'{analysis}'")
    lines.append("")
    lines.append("%NODE.COORD")
    lines.append(str(mesh.nnodes))
    for i, c in enumerate(mesh.coords):
        cz = list(c) + [0.0] * (3 - mesh.dim)
        lines.append(f"{i + 1}\t" + "\t".join(repr(float(v)) for v in cz))
    lines.append("")
    lines.append("%NODE.SUPPORT")
    lines.append(str(mesh.supports.shape[0]))
    for s in mesh.supports:
        lines.append("\t".join(str(int(v)) for v in s) + "\t0" * (6 - mesh.dim))
    lines.append("")
    loads = mesh.nodal_loads() if mesh.f is not None else np.zeros((0, mesh.dim + 1))
    lines.append("%LOAD.CASE.NODAL.FORCES")
    lines.append(str(loads.shape[0]))
    for row in loads:
        lines.append(f"{int(row[0])}\t" + "\t".join(repr(float(v)) for v in row[1:]) +
                     "\t0.0" * (6 - mesh.dim))
    lines.append("")
    lines.append("%END")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")
