"""The C-ABI library loads and exports every symbol include/gpufem_b200.h declares.
CPU only: no compute call is made (without a GPU gf_create reports GF_ERR_CUDA)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def header_symbols():
    txt = (ROOT / "include" / "gpufem_b200.h").read_text()
    return re.findall(r"GF_API\s+[\w\s\*]+?\b(gf_\w+)\s*\(", txt)


def test_header_declares_entry_points():
    syms = header_symbols()
    assert len(syms) >= 25
    assert len(set(syms)) == len(syms)


def test_library_exports_every_declared_symbol():
    from gpufem_b200 import _lib
    for name in header_symbols():
        assert hasattr(_lib.lib, name), f"{name} not exported"
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT\s+(gf_\w+)", out))
    assert set(header_symbols()) <= exported
    # nothing else with the public prefix leaks out
    assert exported <= set(header_symbols())


def test_bindings_cover_header():
    from gpufem_b200 import _lib
    assert set(_lib.SIGNATURES) == set(header_symbols())


def test_build_targets_sm100a_only():
    from gpufem_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_no_gpu_reports_cuda_error_without_crashing():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from gpufem_b200 import _lib
    h = C.c_void_p()
    st = _lib.lib.gf_create(C.byref(h), 0)
    assert st == _lib.GF_ERR_CUDA and not h.value
    assert _lib.lib.gf_version().decode().startswith("gpufem_b200")
    # null-context calls fail cleanly
    assert _lib.lib.gf_assemble(None, 0, 0, 0) == _lib.GF_ERR_INVALID_ARG
    assert _lib.lib.gf_solve(None, None, None) == _lib.GF_ERR_INVALID_ARG


def test_every_context_entry_point_rejects_a_null_context():
    """Each gf_status entry point whose first parameter is the context returns
    GF_ERR_INVALID_ARG for a null context (zero / null for the other arguments)."""
    from gpufem_b200 import _lib
    txt = (ROOT / "include" / "gpufem_b200.h").read_text()
    checked = 0
    for name, args in re.findall(r"GF_API\s+gf_status\s+(gf_\w+)\s*\(([^)]*)\)", txt):
        first = args.split(",")[0].strip()
        if not re.match(r"(const\s+)?gf_ctx\s*\*\s*\w+$", first):
            continue
        _, argtypes = _lib.SIGNATURES[name]
        vals = [t(0) if t in (C.c_double, C.c_float, C.c_int32, C.c_int64, C.c_uint64) else None
                for t in argtypes]
        assert getattr(_lib.lib, name)(*vals) == _lib.GF_ERR_INVALID_ARG, name
        checked += 1
    assert checked >= 35


def test_noalloc_maximum_matches_header():
    """The Python binding's copy of GF_PCG_NOALLOC_MAX_N equals the header's."""
    from gpufem_b200 import _lib
    hdr = (ROOT / "include" / "gpufem_b200.h").read_text()
    m = re.search(r"#define\s+GF_PCG_NOALLOC_MAX_N\s+(\d+)", hdr)
    assert m and int(m.group(1)) == _lib.GF_PCG_NOALLOC_MAX_N


def test_enum_values_match_header():
    """Every GF_SOLVER_* / GF_SCATTER_* / GF_ENGINE_* / GF_BC_* / GF_LP_LOSS_* constant of
    the Python binding equals the header's enumerator of the same name."""
    from gpufem_b200 import _lib
    hdr = (ROOT / "include" / "gpufem_b200.h").read_text()
    found = dict((k, int(v)) for k, v in re.findall(
        r"\b(GF_(?:SOLVER|SCATTER|ENGINE|BC|LP_LOSS)_[A-Z0-9_]+)\s*=\s*(\d+)", hdr))
    assert "GF_SOLVER_TWOLEVEL_PCG32" in found
    for name, value in found.items():
        assert getattr(_lib, name) == value, name
