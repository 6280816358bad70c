"""Generate the golden vectors in tests/golden/ from the reference's own CPU code.

Runs the reference (fpaboim/gpufem src/, compiled unmodified by oracle/build_ref.sh
into oracle/_ref/libref_fp32.so and libref_fp64.so) on:
  * small seeded structured meshes of every element type (written as neutral files
    and read back with the reference's FileIO::ReadNF), and
  * the reference's own small test meshes (test_models/_testmodels/*.nf and
    test_models/Q4/placa16_Q4.nf),
and stores what the reference produced: connectivity / coordinates as parsed, the
ELL matrix (rownnz, column indices, values) in FP64 and FP32, the penalty-modified
matrix diagonal, and the CG solution with the reference's solver.

Usage (needs the reference sources, i.e. this runs only where they are mounted):
    python tests/golden/make_golden.py REFERENCE_ROOT   (or GPUFEM_REFERENCE_ROOT set)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from gpufem_b200 import meshgen as mg  # noqa: E402
from oracle.oracle import Reference, build_reference, reference_root  # noqa: E402

OUT = Path(__file__).resolve().parent

SYNTH = [
    # name, element, n, ngauss, jitter, seed
    ("q4_4x3", mg.Q4, (4, 3), 2, 0.2, 11),
    ("q8_3x3", mg.Q8, (3, 3), 3, 0.15, 12),
    ("q8_3x2_g2", mg.Q8, (3, 2), 2, 0.15, 13),
    ("brick8_3", mg.BRICK8, (3, 3, 3), 2, 0.1, 14),
    ("brick8_2_g3", mg.BRICK8, (2, 2, 2), 3, 0.1, 15),
    ("brick20_2", mg.BRICK20, (2, 2, 2), 3, 0.05, 16),
    ("brick20_2x1x1_g2", mg.BRICK20, (2, 1, 1), 2, 0.05, 17),
]
REF_MESHES = [
    ("ref_Q4", "test_models/_testmodels/Q4.nf", 2),
    ("ref_Q8", "test_models/_testmodels/Q8.nf", 3),
    ("ref_brick8", "test_models/_testmodels/brick_brk8.nf", 2),
    ("ref_2bricks20", "test_models/_testmodels/2bricks_brk20.nf", 3),
    ("ref_placa16_Q4", "test_models/Q4/placa16_Q4.nf", 2),
]
E, NU = 100.0, 0.25  # the reference's batch settings (src/interface.cpp:79-80)


def run(open_fn):
    out = {}
    for tag in ("fp64", "fp32"):
        R = Reference(tag)
        s = open_fn(R)
        s.assemble(coloring=False, nthreads=1)
        rn, ci, v = s.ell()
        out[f"rownnz_{tag}"] = rn
        out[f"colidx_{tag}"] = ci
        out[f"vals_{tag}"] = v if tag == "fp64" else v.astype(np.float32)
        if tag == "fp64":
            out["conn"] = s.connect()
            out["coords"] = s.coords()
            out["D"] = s.D()
            out["force"] = s.force()
            out["supports"] = s.supports()
        s.penalty()
        rnp, cip, vp = s.ell()
        diag = np.array([vp[np.nonzero(cip[:rnp[r], r] == r)[0][0], r] if np.any(cip[:rnp[r], r] == r)
                         else 0.0 for r in range(s.n)])
        out[f"diag_pen_{tag}"] = diag
        x, _ = s.cg(maxit=20000, eps=1e-10 if tag == "fp64" else 1e-5, nthreads=1)
        out[f"u_cg_{tag}"] = x
        s.close()
    return out


def main(ref_root: str | None = None) -> None:
    ref_root = reference_root(ref_root)
    if ref_root is None:
        raise SystemExit("give the reference root as an argument or in GPUFEM_REFERENCE_ROOT")
    if not (Reference.available("fp64") and Reference.available("fp32")):
        if not build_reference(ref_root):
            raise SystemExit("reference sources not available")
    for name, et, n, ng, jit, seed in SYNTH:
        m = mg.clamp_and_load(mg.structured(et, n, jitter=jit, seed=seed, ngauss=ng, E0=E, nu=NU))
        data = run(lambda R: R.open_mesh(m))
        assert np.array_equal(data["supports"], m.supports)
        data.update(elem_type=np.int32(et), ngauss=np.int32(ng), E=np.float64(E),
                    nu=np.float64(NU))
        np.savez_compressed(OUT / f"{name}.npz", **data)
        print("wrote", name)
    for name, rel, ng in REF_MESHES:
        path = Path(ref_root) / rel
        data = run(lambda R: R.open(str(path), ng, E, NU, True))
        nen = data["conn"].shape[1]
        dim = data["coords"].shape[1]
        et = {(4, 2): mg.Q4, (8, 2): mg.Q8, (8, 3): mg.BRICK8, (20, 3): mg.BRICK20}[(nen, dim)]
        data.update(elem_type=np.int32(et), ngauss=np.int32(ng), E=np.float64(E),
                    nu=np.float64(NU), source=np.array(rel))
        np.savez_compressed(OUT / f"{name}.npz", **data)
        print("wrote", name)


if __name__ == "__main__":
    main(*sys.argv[1:])
