"""TEST INFRASTRUCTURE ONLY — Python access to the oracle.

* `Oracle`     the plain-C restatement oracle/gf_oracle.c (liboracle.so, built from
               source here by `build_oracle()`; gcc only).
* `Reference`  the reference's own CPU path compiled by oracle/build_ref.sh into
               oracle/_ref/libref_{fp32,fp64}.so (present only where the reference
               sources were available at build time).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"


def build_oracle(force: bool = False) -> Path:
    src = HERE / "gf_oracle.c"
    if force or not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        cc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"
        tmp = LIB.with_suffix(".so.tmp")
        subprocess.run([cc, "-O2", "-shared", "-fPIC", "-std=c99", str(src), "-o", str(tmp), "-lm"],
                       check=True)
        os.replace(tmp, LIB)
    return LIB


def reference_root(ref_root: str | None = None) -> str | None:
    """Where the reference sources lie: the argument, else $GPUFEM_REFERENCE_ROOT."""
    return ref_root or os.environ.get("GPUFEM_REFERENCE_ROOT") or None


def build_reference(ref_root: str | None = None) -> bool:
    """Compile the reference CPU path into oracle/_ref (no-op without sources).
    The source tree is `ref_root`, else $GPUFEM_REFERENCE_ROOT."""
    ref_root = reference_root(ref_root)
    if ref_root is None or not Path(ref_root, "src", "FEM").exists():
        return False
    subprocess.run(["bash", str(HERE / "build_ref.sh"), ref_root], check=True)
    return (REF_DIR / "libref_fp64.so").exists()


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    def __init__(self):
        self.lib = C.CDLL(str(build_oracle()))
        L = self.lib
        v, i32, d = C.c_void_p, C.c_int, C.c_double
        L.or_gauss.argtypes = [i32, i32, v, v]
        L.or_dshape.argtypes = [i32, v, v]
        L.or_dmatrix.argtypes = [i32, i32, d, d, v]
        L.or_element_ke.argtypes = [i32, i32, v, v, v]
        L.or_pattern.argtypes = [i32, i32, i32, v, i32, v, v]
        L.or_pattern.restype = i32
        L.or_assemble.argtypes = [i32, i32, i32, i32, v, i32, v, v, d, d, i32, v, v, v]
        L.or_assemble.restype = i32
        L.or_penalty.argtypes = [i32, i32, v, v, v, v]
        L.or_eliminate.argtypes = [i32, i32, v, v, v, v, v]
        L.or_spmv.argtypes = [i32, i32, v, v, v, v, v]
        L.or_residual_dd.argtypes = [i32, i32, v, v, v, v, v, v, v]
        L.or_residual_dd.restype = d
        L.or_cg.argtypes = [i32, i32, v, v, v, v, v, i32, d, i32]
        L.or_cg.restype = i32
        L.or_greedy_color.argtypes = [i32, i32, i32, v, v]
        L.or_greedy_color.restype = i32

    def gauss(self, dim, ng):
        npt = ng ** dim
        pts = np.zeros(npt * dim)
        w = np.zeros(npt)
        self.lib.or_gauss(dim, ng, _p(pts), _p(w))
        return pts.reshape(npt, dim), w

    def dshape(self, et, p):
        nen, dim = [4, 8, 8, 20][et], [2, 2, 3, 3][et]
        p = np.ascontiguousarray(p, np.float64)
        dN = np.zeros(dim * nen)
        self.lib.or_dshape(et, _p(p), _p(dN))
        return dN.reshape(dim, nen)

    def dmatrix(self, dim, analysis, E, nu):
        s = 3 if dim == 2 else 6
        D = np.zeros(s * s)
        self.lib.or_dmatrix(dim, analysis, E, nu, _p(D))
        return D.reshape(s, s)

    def element_ke(self, et, ng, X, D):
        X = np.ascontiguousarray(X, np.float64)
        D = np.ascontiguousarray(D, np.float64)
        m = X.size
        Ke = np.zeros(m * m)
        self.lib.or_element_ke(et, ng, _p(X), _p(D), _p(Ke))
        return Ke.reshape(m, m)

    def pattern(self, et, nnodes, conn1):
        conn1 = np.ascontiguousarray(conn1, np.int32)
        dim = [2, 2, 3, 3][et]
        W = self.lib.or_pattern(et, nnodes, conn1.shape[0], _p(conn1), 0, None, None)
        n = nnodes * dim
        rownnz = np.zeros(n, np.int32)
        colidx = np.zeros(W * n, np.int32)
        self.lib.or_pattern(et, nnodes, conn1.shape[0], _p(conn1), W, _p(rownnz), _p(colidx))
        return rownnz, colidx.reshape(W, n)

    def assemble(self, et, ng, coords, conn1, E, nu, E_elem=None, analysis=0, pattern=None):
        coords = np.ascontiguousarray(coords, np.float64)
        conn1 = np.ascontiguousarray(conn1, np.int32)
        E_elem = None if E_elem is None else np.ascontiguousarray(E_elem, np.float64)
        if pattern is None:
            pattern = self.pattern(et, coords.shape[0], conn1)
        rownnz, colidx = pattern
        W, n = colidx.shape
        vals = np.zeros(W * n)
        miss = self.lib.or_assemble(et, ng, analysis, coords.shape[0], _p(coords), conn1.shape[0],
                                    _p(conn1), _p(E_elem), float(E), float(nu), W, _p(rownnz),
                                    _p(np.ascontiguousarray(colidx)), _p(vals))
        assert miss == 0, "pattern misses element entries"
        return rownnz, colidx, vals.reshape(W, n)

    def penalty(self, rownnz, colidx, vals, fixed):
        vals = np.array(vals, np.float64, copy=True)
        W, n = colidx.shape
        self.lib.or_penalty(n, W, _p(rownnz), _p(np.ascontiguousarray(colidx)), _p(vals),
                            _p(np.ascontiguousarray(fixed, np.uint8)))
        return vals

    def eliminate(self, rownnz, colidx, vals, fixed, f):
        vals = np.array(vals, np.float64, copy=True)
        f = np.array(f, np.float64, copy=True)
        W, n = colidx.shape
        self.lib.or_eliminate(n, W, _p(rownnz), _p(np.ascontiguousarray(colidx)), _p(vals),
                              _p(np.ascontiguousarray(fixed, np.uint8)), _p(f))
        return vals, f

    def spmv(self, rownnz, colidx, vals, x):
        W, n = colidx.shape
        y = np.zeros(n)
        self.lib.or_spmv(n, W, _p(rownnz), _p(np.ascontiguousarray(colidx)),
                         _p(np.ascontiguousarray(vals, np.float64)),
                         _p(np.ascontiguousarray(x, np.float64)), _p(y))
        return y

    def residual_dd(self, rownnz, colidx, vals, f, u_hi, u_lo):
        """r = f - K (u_hi + u_lo) in double-double, rounded once; returns (r, ||r||)."""
        W, n = colidx.shape
        r = np.zeros(n)
        rr = self.lib.or_residual_dd(n, W, _p(rownnz), _p(np.ascontiguousarray(colidx)),
                                     _p(np.ascontiguousarray(vals, np.float64)),
                                     _p(np.ascontiguousarray(f, np.float64)),
                                     _p(np.ascontiguousarray(u_hi, np.float64)),
                                     _p(np.ascontiguousarray(u_lo, np.float64)), _p(r))
        return r, float(np.sqrt(rr))

    def cg(self, rownnz, colidx, vals, b, maxit=10000, eps=1e-10, precond=True):
        W, n = colidx.shape
        x = np.zeros(n)
        it = self.lib.or_cg(n, W, _p(rownnz), _p(np.ascontiguousarray(colidx)),
                            _p(np.ascontiguousarray(vals, np.float64)),
                            _p(np.ascontiguousarray(b, np.float64)), _p(x), maxit, eps,
                            1 if precond else 0)
        return x, it

    def greedy_color(self, et, nnodes, conn1):
        conn1 = np.ascontiguousarray(conn1, np.int32)
        col = np.zeros(conn1.shape[0], np.int32)
        nc = self.lib.or_greedy_color(et, nnodes, conn1.shape[0], _p(conn1), _p(col))
        return col, nc


class Reference:
    """The reference's CPU code (oracle/_ref/libref_<tag>.so), tag fp32 or fp64."""

    def __init__(self, tag: str = "fp64"):
        path = REF_DIR / f"libref_{tag}.so"
        if not path.exists():
            raise FileNotFoundError(path)
        self.lib = L = C.CDLL(str(path))
        self.tag = tag
        v, i32, d = C.c_void_p, C.c_int, C.c_double
        L.ref_open.restype = v
        L.ref_open.argtypes = [C.c_char_p, i32, d, d, i32]
        L.ref_close.argtypes = [v]
        L.ref_dims.argtypes = [v, v]
        L.ref_get_D.argtypes = [v, v]
        L.ref_get_connect.argtypes = [v, v]
        L.ref_get_coords.argtypes = [v, v]
        L.ref_get_gauss.argtypes = [v, v, v]
        L.ref_assemble.restype = d
        L.ref_assemble.argtypes = [v, i32, i32]
        L.ref_num_colors.argtypes = [v]
        L.ref_num_supports.argtypes = [v]
        L.ref_get_supports.argtypes = [v, v]
        L.ref_ell_width.argtypes = [v]
        L.ref_ell_stored_width.argtypes = [v]
        L.ref_ell_export.argtypes = [v, i32, v, v, v]
        L.ref_apply_penalty.argtypes = [v]
        L.ref_get_force.argtypes = [v, v]
        L.ref_cg.restype = d
        L.ref_cg.argtypes = [v, v, v, i32, d, i32]
        L.ref_axy.argtypes = [v, v, v, i32]
        L.ref_mat_new.restype = v
        L.ref_mat_new.argtypes = [i32]
        L.ref_mat_free.argtypes = [v]
        L.ref_mat_add.argtypes = [v, i32, i32, d]
        L.ref_mat_set.argtypes = [v, i32, i32, d]
        L.ref_mat_get.restype = d
        L.ref_mat_get.argtypes = [v, i32, i32]
        L.ref_mat_cg.argtypes = [v, v, v, i32, d]
        L.ref_mat_axy.argtypes = [v, v, v]
        L.ref_ell_axy_external.argtypes = [i32, i32, v, v, v, v, v, i32]
        L.ref_ell_axy_external.restype = d
        L.ref_binsearch_step.argtypes = [v, i32, i32, i32, i32]
        L.ref_binsearch_step.restype = i32

    def ell_axy(self, rownnz, colidx, vals, x, nthreads: int = 0):
        """The reference's ELLmatrix::Axy on a caller's column-major ELL (colidx, vals of
        shape (width, n)); FP64 build only.  Returns (y, seconds)."""
        if self.tag != "fp64":
            raise ValueError("ell_axy takes FP64 arrays: use the fp64 build")
        W, n = colidx.shape
        rownnz = np.ascontiguousarray(rownnz, np.int32)
        colidx = np.ascontiguousarray(colidx, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(n)
        t = self.lib.ref_ell_axy_external(n, W, _p(rownnz), _p(colidx), _p(vals), _p(x), _p(y),
                                          nthreads)
        return y, t

    @staticmethod
    def available(tag: str = "fp64") -> bool:
        return (REF_DIR / f"libref_{tag}.so").exists()

    def open(self, nf_path: str, ngp: int, E: float, nu: float, plane_stress: bool = True):
        h = self.lib.ref_open(str(nf_path).encode(), ngp, E, nu, 1 if plane_stress else 0)
        if not h:
            raise RuntimeError(f"ReadNF failed for {nf_path}")
        return RefSession(self, h)

    def open_mesh(self, mesh, plane_stress: bool = True):
        """Write `mesh` as a neutral file and open it with the reference's reader."""
        from gpufem_b200.meshgen import write_nf
        fd, path = tempfile.mkstemp(suffix=".nf")
        os.close(fd)
        try:
            write_nf(mesh, path)
            return self.open(path, mesh.ngauss, mesh.E0, mesh.nu, plane_stress)
        finally:
            os.unlink(path)


class RefSession:
    def __init__(self, ref: Reference, h):
        self.ref, self.h, self.L = ref, h, ref.lib
        d = (C.c_int * 5)()
        self.L.ref_dims(h, d)
        self.dim, self.nnodes, self.nelem, self.nen, self.n = list(d)

    def close(self):
        if self.h:
            self.L.ref_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def D(self):
        s = 3 if self.dim == 2 else 6
        out = np.zeros(s * s)
        self.L.ref_get_D(self.h, _p(out))
        return out.reshape(s, s)

    def connect(self):
        out = np.zeros(self.nelem * self.nen, np.int32)
        self.L.ref_get_connect(self.h, _p(out))
        return out.reshape(self.nelem, self.nen)

    def coords(self):
        out = np.zeros(self.nnodes * self.dim)
        self.L.ref_get_coords(self.h, _p(out))
        return out.reshape(self.nnodes, self.dim)

    def supports(self):
        ns = self.L.ref_num_supports(self.h)
        out = np.zeros(ns * (self.dim + 1), np.int32)
        if ns:
            self.L.ref_get_supports(self.h, _p(out))
        return out.reshape(ns, self.dim + 1)

    def assemble(self, coloring: bool = False, nthreads: int = 0) -> float:
        return self.L.ref_assemble(self.h, 1 if coloring else 0, nthreads)

    def num_colors(self) -> int:
        return self.L.ref_num_colors(self.h)

    def ell(self):
        W = self.L.ref_ell_width(self.h)
        rownnz = np.zeros(self.n, np.int32)
        colidx = np.zeros(W * self.n, np.int32)
        vals = np.zeros(W * self.n)
        self.L.ref_ell_export(self.h, W, _p(rownnz), _p(colidx), _p(vals))
        return rownnz, colidx.reshape(W, self.n), vals.reshape(W, self.n)

    def stored_width(self) -> int:
        return self.L.ref_ell_stored_width(self.h)

    def penalty(self):
        self.L.ref_apply_penalty(self.h)

    def force(self):
        f = np.zeros(self.n)
        self.L.ref_get_force(self.h, _p(f))
        return f

    def cg(self, maxit: int, eps: float, b: Optional[np.ndarray] = None, nthreads: int = 0):
        x = np.zeros(self.n)
        b = None if b is None else np.ascontiguousarray(b, np.float64)
        t = self.L.ref_cg(self.h, _p(x), _p(b), maxit, eps, nthreads)
        return x, t

    def axy(self, x, nthreads: int = 0):
        y = np.zeros(self.n)
        self.L.ref_axy(self.h, _p(np.ascontiguousarray(x, np.float64)), _p(y), nthreads)
        return y
