"""Seeded synthetic graphs for the PageRank workloads (R-MAT and Erdos-Renyi).

The generators run in ``libegpr_synth.so`` (host C++/OpenMP, counter-based
SplitMix64 randomness: a graph depends only on its parameters).  They return
an out-edge CSR shaped like the reference's ``gen_CSR`` output
(cpp_easygraph/classes/graph.cpp:719-886): int32 offsets, int32 destinations
sorted inside each row, no duplicate pairs, no self-loops, all ``n`` vertices
kept (dangling and isolated ones included).

R-MAT: ``edgefactor * 2**scale`` sampled pairs, each bit level picks a quadrant
with probabilities a/b/c/d (default 0.57/0.19/0.19/0.05), no noise, no
permutation.  ``keep_n`` < 2**scale keeps vertices [0, keep_n) and drops every
sampled pair with an endpoint >= keep_n (how non-power-of-two sizes are made).
Weights (``weighted=True``): i.i.d. ``1 - U``, U uniform in [0, 1) rounded to
FP32, one per final CSR entry, stored as float64.
"""

from __future__ import annotations

import ctypes
from ctypes import c_double, c_int32, c_int64, c_uint64, c_void_p
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "libegpr_synth.so"
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            from . import build as _build

            _build.build_synth()
        lib = ctypes.CDLL(str(_LIB_PATH))
        lib.egpr_synth_rmat.restype = c_int64
        lib.egpr_synth_rmat.argtypes = [c_int32, c_int32, c_double, c_double, c_double, c_uint64, c_int32,
                                        c_void_p, c_void_p, c_void_p]
        lib.egpr_synth_er.restype = c_int64
        lib.egpr_synth_er.argtypes = [c_int32, c_int64, c_uint64, c_void_p, c_void_p, c_void_p]
        _lib = lib
    return _lib


@dataclass
class CSR:
    """Out-edge CSR of a directed graph with vertices 0..n-1."""

    V: np.ndarray  # int32[n+1]
    E: np.ndarray  # int32[m]
    W: np.ndarray | None = None  # float64[m]
    params: dict | None = None

    @property
    def n(self) -> int:
        return int(self.V.shape[0]) - 1

    @property
    def m(self) -> int:
        return int(self.E.shape[0])


def rmat(scale, edgefactor=16, a=0.57, b=0.19, c=0.19, seed=0, keep_n=0, weighted=False) -> CSR:
    lib = _load()
    n_full = 1 << int(scale)
    n = min(int(keep_n), n_full) if keep_n else n_full
    cap = int(edgefactor) << int(scale)
    V = np.empty(n + 1, np.int32)
    E = np.empty(max(cap, 1), np.int32)
    W = np.empty(max(cap, 1), np.float64) if weighted else None
    m = lib.egpr_synth_rmat(int(scale), int(edgefactor), float(a), float(b), float(c), int(seed) & (2**64 - 1),
                            int(keep_n), V.ctypes.data, E.ctypes.data, W.ctypes.data if weighted else None)
    if m < 0:
        raise ValueError("invalid R-MAT parameters")
    E = E[:m].copy()
    W = W[:m].copy() if weighted else None
    params = dict(kind="rmat", scale=int(scale), edgefactor=int(edgefactor), a=a, b=b, c=c, seed=int(seed),
                  keep_n=int(keep_n), weighted=bool(weighted))
    return CSR(V, E, W, params)


def erdos_renyi(n, mean_degree, seed=0, weighted=False) -> CSR:
    lib = _load()
    msamp = int(round(n * float(mean_degree)))
    V = np.empty(int(n) + 1, np.int32)
    E = np.empty(max(msamp, 1), np.int32)
    W = np.empty(max(msamp, 1), np.float64) if weighted else None
    m = lib.egpr_synth_er(int(n), msamp, int(seed) & (2**64 - 1), V.ctypes.data, E.ctypes.data,
                          W.ctypes.data if weighted else None)
    if m < 0:
        raise ValueError("invalid Erdos-Renyi parameters")
    E = E[:m].copy()
    W = W[:m].copy() if weighted else None
    return CSR(V, E, W, dict(kind="er", n=int(n), mean_degree=float(mean_degree), seed=int(seed),
                             weighted=bool(weighted)))


def seed_sets(n, k, min_size, max_size, seed) -> list[np.ndarray]:
    """k seed sets: sizes uniform in [min_size, max_size], members drawn
    uniformly without replacement from [0, n)."""
    rng = np.random.Generator(np.random.PCG64(int(seed)))
    sizes = rng.integers(min_size, max_size + 1, size=k)
    return [np.sort(rng.choice(n, size=int(s), replace=False)).astype(np.int32) for s in sizes]
