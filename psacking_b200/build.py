"""Build the engine in-tree for sm_100a.

    python psacking_b200/build.py          # or __graft_entry__.build()

Produces, next to this file:
  libpsb200.so   the C-ABI library (include/psb200.h), nvcc, sm_100a only
  _core*.so      the pybind11 module bound to that library (rpath $ORIGIN)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libpsb200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def _core_name() -> str:
    return "_core" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so")


def _stale(target: Path, sources) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(s).stat().st_mtime > t for s in sources)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    return r


def build(force: bool = False, verbose: bool = False) -> None:
    nvcc = _nvcc()
    cu_sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "psb200.h"]
    if force or _stale(LIB, cu_sources):
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
               "--expt-relaxed-constexpr",
               "-o", str(LIB), str(CSRC / "psb_engine.cu")]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = _run(cmd)
        if verbose:
            sys.stderr.write(r.stderr)
    core = PKG / _core_name()
    if force or _stale(core, [CSRC / "psb_core.cpp", ROOT / "include" / "psb200.h", LIB]):
        import pybind11
        cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
               f"-I{pybind11.get_include()}", f"-I{sysconfig.get_paths()['include']}",
               "-o", str(core), str(CSRC / "psb_core.cpp"),
               f"-L{PKG}", "-lpsb200", "-Wl,-rpath,$ORIGIN"]
        _run(cmd)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built", LIB, PKG / _core_name())
