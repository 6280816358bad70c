"""Compile the reference-side adapter driver (adapter_main.cc with StiffAlgoCUDA.h and
ELLmatrixCUDA.h) against the reference's own headers and CPU library (the oracle build
in oracle/_ref) and libgpufem_b200.  The executables go to oracle/_ref/adapter_fp32 and
adapter_fp64 (fem_float = float as shipped, double in the FP64 overlay), beside the
reference libraries they link, so that they travel with the prebuilt oracle to machines
where the reference sources are absent.  Test infrastructure only."""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF = ROOT / "oracle" / "_ref"


def adapter_path(kind: str) -> Path:
    return REF / f"adapter_{kind}"


def build(kind: str, force: bool = False) -> Path | None:
    """Build adapter_<kind> (kind "fp32" or "fp64") where the reference tree is present;
    return the executable's path, or None when neither it nor the sources exist."""
    exe = adapter_path(kind)
    tree = REF / f"src_{kind}"
    lib = REF / f"libref_{kind}.so"
    srcs = [HERE / "adapter_main.cc", HERE / "StiffAlgoCUDA.h", HERE / "ELLmatrixCUDA.h",
            ROOT / "include" / "gpufem_b200.h"]
    if not (tree / "FEM" / "StiffAlgo.h").exists() or not lib.exists():
        return exe if exe.exists() else None
    if not force and exe.exists() and all(exe.stat().st_mtime >= p.stat().st_mtime for p in srcs):
        return exe
    cmd = ["g++", "-std=c++17", "-O1", "-fopenmp", "-fpermissive", "-w", "-include", "cmath",
           "-include", "windows.h", f"-I{ROOT / 'oracle' / 'shims'}", f"-I{tree}",
           f"-I{ROOT / 'include'}", f"-I{HERE}", str(HERE / "adapter_main.cc"),
           "-o", str(exe), f"-L{REF}", f"-lref_{kind}", f"-L{ROOT / 'gpufem_b200'}",
           "-lgpufem_b200", "-Wl,-rpath,$ORIGIN", "-Wl,-rpath,$ORIGIN/../../gpufem_b200"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"adapter build failed:\n{res.stderr[-3000:]}")
    return exe


def run(kind: str, nf: str, ngauss: int, analysis: str = "-", timeout: int = 300) -> dict:
    """Run the driver on a neutral file; returns its "key value..." lines as a dict."""
    exe = adapter_path(kind)
    res = subprocess.run([str(exe), nf, str(ngauss), analysis], capture_output=True, text=True,
                         timeout=timeout)
    if res.returncode != 0:
        raise RuntimeError(f"adapter exited {res.returncode}:\n{res.stdout}\n{res.stderr[-2000:]}")
    return dict(ln.split(" ", 1) for ln in res.stdout.splitlines() if " " in ln)


if __name__ == "__main__":
    for k in ("fp32", "fp64"):
        print(build(k, force=True))
