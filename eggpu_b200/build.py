"""Builds the native libraries of eggpu_b200 in-tree.

* ``libegpr.so``       the CUDA engine (sm_100a) behind the C ABI in include/egpr.h
* ``libegpr_synth.so`` the seeded synthetic graph generators (host C++/OpenMP)
* ``_graph_walk*.so``  Python graph -> out-edge CSR (CPython extension, host C++)

Run ``python -m eggpu_b200.build`` (or call :func:`build`).  Objects go to
``eggpu_b200/_build/``; a library is rebuilt when any of its sources or headers
is newer than it or when its compiler flags changed (recorded in
``_build/flags.txt``).  ``python -m eggpu_b200.build --force`` (or
``build(force=True)``, or ``EGPR_FORCE_REBUILD=1``) rebuilds everything; every
build prints which targets it compiled and which it reused.
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

CUDA_SOURCES = ["prep.cu", "sweep.cu", "bins.cu", "spmm.cu", "api.cu", "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-Xcompiler", "-fopenmp", "--expt-relaxed-constexpr"]


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


REPORT = []  # (target, "compiled" | "reused") of the last build


def _forced(force: bool) -> bool:
    return force or os.environ.get("EGPR_FORCE_REBUILD", "") not in ("", "0")


def _flags_changed(key: str, flags) -> bool:
    """True (and records the new flags) when `key` was last built with other flags."""
    BUILD.mkdir(exist_ok=True)
    stamp = BUILD / "flags.txt"
    lines = dict(ln.split("=", 1) for ln in stamp.read_text().splitlines() if "=" in ln) if stamp.exists() else {}
    want = " ".join(str(f) for f in flags)
    if lines.get(key) == want:
        return False
    lines[key] = want
    stamp.write_text("".join(f"{k}={v}\n" for k, v in sorted(lines.items())))
    return True


def build_engine(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    headers = list(CSRC.glob("*.cuh")) + [ROOT / "include" / "egpr.h"]
    all_new = _forced(force) | _flags_changed("libegpr", [*ARCH, *NVCC_FLAGS])
    objs = []
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if all_new or _newer(o, [s, *headers]) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            res = _run([nvcc, *ARCH, *NVCC_FLAGS, *extra, "-I", ROOT / "include", "-c", s, "-o", o], verbose)
            REPORT.append((o.name, "compiled"))
            if ptxas_info:
                sys.stderr.write(res.stderr)
        else:
            REPORT.append((o.name, "reused"))
    if all_new or _newer(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", LIB, *objs, f"-L{_gomp_dir()}", "-lgomp"], verbose)
        REPORT.append((LIB.name, "compiled"))
    else:
        REPORT.append((LIB.name, "reused"))
    return LIB


def _gomp_dir() -> str:
    """Directory of the host compiler's libgomp (host threads of the staged upload)."""
    out = subprocess.run(["g++", "-print-file-name=libgomp.so"], capture_output=True, text=True).stdout.strip()
    return str(Path(out).parent)


def build_synth(verbose: bool = False, force: bool = False) -> Path:
    src = CSRC / "synth.cpp"
    if _forced(force) or _newer(SYNTH, [src]):
        REPORT.append((SYNTH.name, "compiled"))
        BUILD.mkdir(exist_ok=True)
        gxx = "g++"
        gomp = subprocess.run([gxx, "-print-file-name=libgomp.so"], capture_output=True, text=True).stdout.strip()
        obj = BUILD / "synth.o"
        _run([gxx, "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-c", src, "-o", obj], verbose)
        _run([gxx, "-shared", "-o", SYNTH, obj, f"-L{Path(gomp).parent}", "-lgomp"], verbose)
    else:
        REPORT.append((SYNTH.name, "reused"))
    return SYNTH


def build_graph_walk(verbose: bool = False, force: bool = False) -> Path:
    """The CPython extension that turns a Python graph's adjacency into the out-edge CSR."""
    import sysconfig

    src = CSRC / "graph_walk.cpp"
    out = PKG / ("_graph_walk" + sysconfig.get_config_var("EXT_SUFFIX"))
    if _forced(force) or _newer(out, [src]):
        REPORT.append((out.name, "compiled"))
        inc = sysconfig.get_paths()["include"]
        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", f"-I{inc}", src, "-o", out],
             verbose)
    else:
        REPORT.append((out.name, "reused"))
    return out


def build(verbose: bool = False, force: bool = False) -> None:
    REPORT.clear()
    build_engine(verbose, force=force)
    build_synth(verbose, force=force)
    build_graph_walk(verbose, force=force)
    print("eggpu_b200 build: " + ", ".join(f"{t} {how}" for t, how in REPORT), flush=True)


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
    if "--ptxas" in sys.argv:
        build_engine(verbose=True, ptxas_info=True)
