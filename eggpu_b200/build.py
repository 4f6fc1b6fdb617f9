"""Builds the native libraries of eggpu_b200 in-tree.

* ``libegpr.so``       the CUDA engine (sm_100a) behind the C ABI in include/egpr.h
* ``libegpr_synth.so`` the seeded synthetic graph generators (host C++/OpenMP)
* ``_graph_walk*.so``  Python graph -> out-edge CSR (CPython extension, host C++)

Run ``python -m eggpu_b200.build`` (or call :func:`build`).  Objects go to
``eggpu_b200/_build/``; a library is rebuilt when any of its sources or headers
is newer than it.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libegpr.so"
SYNTH = PKG / "libegpr_synth.so"

CUDA_SOURCES = ["prep.cu", "sweep.cu", "spmm.cu", "api.cu", "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libegpr.so")


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    res = subprocess.run([str(c) for c in cmd], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"build step failed ({res.returncode}):\n{' '.join(map(str, cmd))}\n{res.stdout}\n{res.stderr}")
    return res


def build_engine(verbose: bool = False, ptxas_info: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    headers = list(CSRC.glob("*.cuh")) + [ROOT / "include" / "egpr.h"]
    objs = []
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if _newer(o, [s, *headers]) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            res = _run([nvcc, *ARCH, *NVCC_FLAGS, *extra, "-I", ROOT / "include", "-c", s, "-o", o], verbose)
            if ptxas_info:
                sys.stderr.write(res.stderr)
    if _newer(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", LIB, *objs], verbose)
    return LIB


def build_synth(verbose: bool = False) -> Path:
    src = CSRC / "synth.cpp"
    if _newer(SYNTH, [src]):
        BUILD.mkdir(exist_ok=True)
        gxx = "g++"
        gomp = subprocess.run([gxx, "-print-file-name=libgomp.so"], capture_output=True, text=True).stdout.strip()
        obj = BUILD / "synth.o"
        _run([gxx, "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-c", src, "-o", obj], verbose)
        _run([gxx, "-shared", "-o", SYNTH, obj, f"-L{Path(gomp).parent}", "-lgomp"], verbose)
    return SYNTH


def build_graph_walk(verbose: bool = False) -> Path:
    """The CPython extension that turns a Python graph's adjacency into the out-edge CSR."""
    import sysconfig

    src = CSRC / "graph_walk.cpp"
    out = PKG / ("_graph_walk" + sysconfig.get_config_var("EXT_SUFFIX"))
    if _newer(out, [src]):
        inc = sysconfig.get_paths()["include"]
        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", f"-I{inc}", src, "-o", out],
             verbose)
    return out


def build(verbose: bool = False) -> None:
    build_engine(verbose)
    build_synth(verbose)
    build_graph_walk(verbose)


if __name__ == "__main__":
    build(verbose=True)
    if "--ptxas" in sys.argv:
        build_engine(verbose=True, ptxas_info=True)
