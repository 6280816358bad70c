"""Neutral-file (.nf) reader: the reference's mesh input format.

Follows FileIO::ReadNF (src/Utils/fileIO.cc:73-404) section by section, so that a
mesh from the reference's model library reaches the C-ABI with the same arrays the
reference's FemData receives:

* the element block is the first line containing "%ELEMENT." (FileIO::findElemString,
  fileIO.cc:797-825); its type is the rest of that line (Q4, Q8, BRICK8, BRICK20); the
  next line is the element count; each element line carries 4 (Q4, Q8) or 3 (bricks)
  leading integers before the node ids; Brick20 ids are renumbered from the file's
  order to the natural-coordinate order (fileIO.cc:184-204);
* 2-D files then give "%HEADER.ANALYSIS" and one token on the next line;
* "%NODE.COORD": count, then `id x y [z]` lines read in file order (ids ignored);
  2-D files carry a z column that is not read;
* "%NODE.SUPPORT": count, then dim + 1 integers per line (node, flags);
* "%LOAD.CASE.NODAL.FORCE": count, then dim + 1 numbers per line, each parsed as a
  32-bit float (fileIO.cc:317-323) — the reference's loads are FP32 even in an FP64
  build.

Each section is searched forward from the previous one by substring match
(FileIO::findParameter, fileIO.cc:761-793); reaching "%END" rewinds the file once.
FemData::CalcForceVector (src/FEM/FemData.cc:369-385) then *sets* (does not add)
f[dim*(node-1) + c] for every non-zero load component.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from .meshgen import BRICK8, BRICK20, DIM, NEN, NF_BRICK20, Q4, Q8, Mesh

_TYPES = {"%ELEMENT.BRICK20": BRICK20, "%ELEMENT.BRICK8": BRICK8, "%ELEMENT.Q4": Q4,
          "%ELEMENT.Q8": Q8}


class NfError(ValueError):
    pass


@dataclass
class NfModel:
    elem_type: int
    coords: np.ndarray      # (nnodes, dim) float64 (float32-rounded when read as "f32")
    conn: np.ndarray        # (nelem, nen) int32, 1-based, natural-coordinate node order
    supports: np.ndarray    # (nsup, dim + 1) int32: node (1-based), fixed flags
    loads: np.ndarray       # (nload, dim + 1) float64 holding FP32 values: node, f_x, ...
    analysis: str           # 2-D: the token after %HEADER.ANALYSIS (quotes kept); 3-D: ""

    @property
    def dim(self) -> int:
        return DIM[self.elem_type]

    def force_vector(self) -> np.ndarray:
        """FemData::CalcForceVector: f[dim*(node-1) + c] = load (set, non-zero only)."""
        f = np.zeros(self.coords.shape[0] * self.dim)
        for row in self.loads:
            node = int(row[0])
            for c in range(self.dim):
                if row[1 + c] != 0.0:
                    f[self.dim * (node - 1) + c] = row[1 + c]
        return f

    def to_mesh(self, E: float = 210e3, nu: float = 0.3, ngauss: int = 2,
                E_elem: Optional[np.ndarray] = None) -> Mesh:
        """A Mesh (the structure the hot-path API takes) with supports and loads."""
        return Mesh(elem_type=self.elem_type, n=(), coords=self.coords.copy(),
                    conn=self.conn.copy(), E=E_elem, E0=E, nu=nu, ngauss=ngauss,
                    supports=self.supports.copy(), f=self.force_vector())


class _Lines:
    """Forward line scanner with the reference's one-time rewind at %END."""

    def __init__(self, lines: List[str]):
        self.lines = lines
        self.pos = 0

    def next(self) -> str:
        if self.pos >= len(self.lines):
            return ""
        s = self.lines[self.pos]
        self.pos += 1
        return s

    def find(self, token: str) -> Optional[str]:
        rewound = False
        while True:
            while self.pos < len(self.lines):
                s = self.lines[self.pos]
                self.pos += 1
                if token in s:
                    return s
                if "%END" in s:
                    if rewound:
                        return None
                    rewound = True
                    self.pos = 0
                    break
            else:
                return None


def _ints(s: str, count: int) -> List[int]:
    tok = s.split()
    if len(tok) < count:
        raise NfError(f"expected {count} integers, got line {s!r}")
    return [int(float(t)) for t in tok[:count]]


def _count(s: str) -> int:
    tok = s.split()
    if not tok:
        raise NfError("missing count line")
    return int(tok[0])


def read_nf(path: str, precision: str = "f64") -> NfModel:
    """Read a neutral file.  `precision` "f32" rounds coordinates to FP32 as the
    reference's FP32 build stores them; "f64" keeps the decimal values."""
    if not str(path).endswith(".nf"):
        raise NfError("not a .nf file")
    with open(path, "r", errors="replace") as fh:
        lines = fh.read().splitlines()
    sc = _Lines(lines)
    head = sc.find("%ELEMENT.")
    if head is None:
        raise NfError("no %ELEMENT.<type> section")
    et = _TYPES.get(head.strip())
    if et is None:
        raise NfError(f"element type not supported: {head.strip()!r}")
    dim, nen = DIM[et], NEN[et]
    nelem = _count(sc.next())
    lead = 4 if dim == 2 else 3
    conn = np.empty((nelem, nen), np.int64)
    for e in range(nelem):
        vals = _ints(sc.next(), lead + nen)
        conn[e] = vals[lead:lead + nen]
    if et == BRICK20:
        conn = conn[:, NF_BRICK20]
    analysis = ""
    if dim == 2:
        if sc.find("%HEADER.ANALYSIS") is None:
            raise NfError("2-D file without %HEADER.ANALYSIS")
        tok = sc.next().split()
        analysis = tok[0] if tok else ""
    if sc.find("%NODE.COORD") is None:
        raise NfError("no %NODE.COORD section")
    nnodes = _count(sc.next())
    coords = np.empty((nnodes, dim), np.float64)
    for i in range(nnodes):
        tok = sc.next().split()
        if len(tok) < 1 + dim:
            raise NfError(f"node line {i + 1}: expected id and {dim} coordinates")
        coords[i] = [float(t) for t in tok[1:1 + dim]]
    if precision == "f32":
        coords = coords.astype(np.float32).astype(np.float64)
    supports = np.zeros((0, dim + 1), np.int32)
    if sc.find("%NODE.SUPPORT") is not None:
        ns = _count(sc.next())
        supports = np.array([_ints(sc.next(), dim + 1) for _ in range(ns)],
                            np.int32).reshape(ns, dim + 1)
    loads = np.zeros((0, dim + 1), np.float64)
    if sc.find("%LOAD.CASE.NODAL.FORCE") is not None:
        nl = _count(sc.next())
        rows = []
        for _ in range(nl):
            tok = sc.next().split()
            if len(tok) < dim + 1:
                raise NfError("nodal load line too short")
            rows.append([float(np.float32(t)) for t in tok[:dim + 1]])
        loads = np.array(rows, np.float64).reshape(nl, dim + 1)
    if conn.size and (conn.min() < 1 or conn.max() > nnodes):
        raise NfError("connectivity refers to a node outside 1..nnodes")
    return NfModel(elem_type=et, coords=coords, conn=conn.astype(np.int32),
                   supports=supports, loads=loads, analysis=analysis)


def write_xyz_vector(path: str, u: np.ndarray, append: bool = True) -> None:
    """Displacement dump in the reference's text format (FileIO::writeXYZVector,
    src/Utils/fileIO.cc:735-753): a header, then one line per group of three
    consecutive entries, "%3i -" followed by three " %7.2f" values.  The reference
    groups by three whatever the model dimension, and so does this writer."""
    u = np.asarray(u, np.float64).ravel()
    out = ["", "Displacement Vector Dump:", " Node+===x===+===y===+===z===+"]
    text = "\n".join(out) + "\n"
    rows = []
    for i in range(u.size // 3):
        rows.append("%3i -" % (i + 1) + "".join(" %7.2f" % u[3 * i + j] for j in range(3)))
    text += "".join(r + "\n" for r in rows)
    with open(path, "a" if append else "w") as fh:
        fh.write(text)
