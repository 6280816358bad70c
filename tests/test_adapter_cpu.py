"""The reference-side classes (tests/adapter/StiffAlgoCUDA.h, ELLmatrixCUDA.h) compile and
link against the reference's own headers and CPU library (the oracle build of its
sources, FP32 as shipped and the FP64 overlay) and libgpufem_b200, and run: the driver
reads a neutral file with the reference's FileIO, initialises the reference's FemData and
calls CalcGlobalStiffness.  On a machine without a GPU the C-ABI reports GF_ERR_CUDA at
gf_create and every later call fails cleanly; the values are compared on a GPU by
tests/test_adapter_gpu.py."""
import pytest

from gpufem_b200 import _lib
from gpufem_b200 import meshgen as mg
from tests.adapter import build_adapter as ba


@pytest.mark.parametrize("kind", ["fp32", "fp64"])
def test_strategy_builds_against_reference_and_runs(tmp_path, kind):
    exe = ba.build(kind)
    if exe is None:
        pytest.skip("reference oracle build absent")
    m = mg.clamp_and_load(mg.structured(mg.Q4, (4, 3), jitter=0.1, seed=1))
    nf = tmp_path / "q4.nf"
    mg.write_nf(m, str(nf))
    lines = ba.run(kind, str(nf), 2, "plane_stress")
    create = int(lines["create"])
    if create == _lib.GF_OK:      # a GPU is present: the values are checked by the GPU test
        assert int(lines["assemble"].split()[0]) == _lib.GF_OK
        assert int(lines["ell"].split()[0]) == m.ndof
    else:
        assert create == _lib.GF_ERR_CUDA
        assert int(lines["assemble"].split()[0]) == _lib.GF_ERR_INVALID_ARG
        assert lines["ell"].split() == ["0", "0"]
        assert "kdiff" not in lines
