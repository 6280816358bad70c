"""The reference-side classes (tests/adapter/StiffAlgoCUDA.h, ELLmatrixCUDA.h) compile and
link against the reference's own headers and CPU library (the oracle build of its
sources) and libgpufem_b200, and run: the driver reads a neutral file with the
reference's FileIO, initialises the reference's FemData, calls CalcGlobalStiffness and
uses K through the SPRmatrix interface.  Without a GPU the C-ABI reports GF_ERR_CUDA at
gf_create and every call fails cleanly."""
import os
import subprocess
from pathlib import Path

import pytest

from gpufem_b200 import _lib
from gpufem_b200 import meshgen as mg

ROOT = Path(__file__).resolve().parents[1]
REF = ROOT / "oracle" / "_ref"


def test_strategy_builds_against_reference_and_runs(tmp_path):
    tree = REF / "src_fp32"
    if not (tree / "FEM" / "StiffAlgo.h").exists() or not (REF / "libref_fp32.so").exists():
        pytest.skip("reference oracle build absent")
    exe = tmp_path / "adapter"
    cmd = ["g++", "-std=c++17", "-O1", "-fopenmp", "-fpermissive", "-w", "-include", "cmath",
           "-include", "windows.h", f"-I{ROOT / 'oracle' / 'shims'}", f"-I{tree}",
           f"-I{ROOT / 'include'}", f"-I{ROOT / 'tests' / 'adapter'}",
           str(ROOT / "tests" / "adapter" / "adapter_main.cc"), "-o", str(exe),
           f"-L{REF}", "-lref_fp32", f"-L{_lib.LIB_PATH.parent}", "-lgpufem_b200",
           f"-Wl,-rpath,{REF}", f"-Wl,-rpath,{_lib.LIB_PATH.parent}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-3000:]
    m = mg.clamp_and_load(mg.structured(mg.Q4, (4, 3), jitter=0.1, seed=1))
    nf = tmp_path / "q4.nf"
    mg.write_nf(m, str(nf))
    run = subprocess.run([str(exe), str(nf)], capture_output=True, text=True, timeout=120,
                         env=dict(os.environ))
    assert run.returncode == 0, run.stdout + run.stderr[-2000:]
    lines = dict(ln.split(" ", 1) for ln in run.stdout.splitlines() if " " in ln)
    create = int(lines["create"])
    if create == _lib.GF_OK:      # a GPU: the strategy assembled the reference's mesh
        assert int(lines["assemble"].split()[0]) == _lib.GF_OK
        n, nnz = map(int, lines["ell"].split())
        assert n == m.ndof and nnz > 0
        assert float(lines["k00"]) > 0 and float(lines["rigid"]) < 1e-4
    else:
        assert create == _lib.GF_ERR_CUDA
        assert int(lines["assemble"].split()[0]) == _lib.GF_ERR_INVALID_ARG
        assert lines["ell"].split() == ["0", "0"]
