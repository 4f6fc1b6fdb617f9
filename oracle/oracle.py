"""ORACLE — test infrastructure only.

Python access to the CPU restatement of the reference's PageRank
(oracle/pagerank_oracle.c, built into oracle/_build/liboracle.so) and, where it
was built, to the reference's own compiled PageRank translation unit
(oracle/_ref/libref_pagerank.so, recipe oracle/Makefile.ref).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs use this module, always to check results or as the timed CPU baseline.  The
engine in eggpu_b200/ never imports it.

Reference functions restated (paths relative to the reference project root):
  build_inbound     gpu_easygraph/functions/centrality/pagerank.cu:286-347
  inbound_values    pagerank.cu:343
  pagerank_push     easygraph/functions/centrality/pagerank.py:75-139
  pagerank_pull     same maths as pagerank_push, pulled over the inbound CSR
  cpu_pagerank_omp  cpp_easygraph/functions/pagerank/pagerank.cpp:21-122
  graph_to_csr      cpp_easygraph/classes/graph_convert.cpp:72-134 (build_graph /
                    build_digraph) followed by cpp_easygraph/classes/graph.cpp:719-886
                    (Graph::gen_CSR): rows in node-insertion order, each row
                    sorted by destination index
Parity pins: tests/golden/ (vectors produced by the reference itself, script
tests/golden/make_golden.py).
"""

from __future__ import annotations

import ctypes
import subprocess
from ctypes import POINTER, c_double, c_int32, c_int64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref_pagerank.so"

_lib = None
_ref = None


def build() -> Path:
    subprocess.run(["make", "-s", "-f", str(HERE / "Makefile")], check=True, cwd=str(HERE.parent))
    return LIB


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = ctypes.CDLL(str(LIB))
        lib.orc_build_inbound.restype = ctypes.c_int
        lib.orc_build_inbound.argtypes = [c_void_p, c_void_p, c_void_p, c_int32, c_int64, c_void_p, c_void_p,
                                          c_void_p, c_void_p, c_void_p, POINTER(c_int64)]
        lib.orc_inbound_values.restype = None
        lib.orc_inbound_values.argtypes = [c_void_p, c_void_p, c_void_p, c_int64, c_double, c_void_p]
        lib.orc_pagerank_push.restype = ctypes.c_int
        lib.orc_pagerank_push.argtypes = [c_void_p, c_void_p, c_void_p, c_int32, c_int64, c_int32, c_double,
                                          c_double, c_int32, c_double, c_void_p, c_void_p, POINTER(c_int32),
                                          POINTER(c_double)]
        lib.orc_pagerank_pull.restype = ctypes.c_int
        lib.orc_pagerank_pull.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_double, c_double,
                                          c_int32, c_double, c_void_p, c_void_p, POINTER(c_int32),
                                          POINTER(c_double), c_int32]
        lib.orc_cpu_pagerank_omp.restype = ctypes.c_int
        lib.orc_cpu_pagerank_omp.argtypes = [c_void_p, c_void_p, c_void_p, c_int32, c_double, c_int32, c_double,
                                             c_void_p, POINTER(c_int32), c_int32]
        lib.orc_max_threads.restype = ctypes.c_int
        lib.orc_max_threads.argtypes = []
        _lib = lib
    return _lib


def ref_available() -> bool:
    return REF_LIB.exists()


def _load_ref():
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(str(REF_LIB))
        lib.ref_build_inbound.restype = ctypes.c_int
        lib.ref_build_inbound.argtypes = [c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_double, c_void_p,
                                          c_void_p, c_void_p, c_void_p, POINTER(ctypes.c_int)]
        lib.ref_cuda_pagerank.restype = ctypes.c_int
        lib.ref_cuda_pagerank.argtypes = [c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_double, c_int32,
                                          c_double, c_void_p, POINTER(c_double)]
        _ref = lib
    return _ref


def _p(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


def _prep(V, E, W):
    V = np.ascontiguousarray(V, np.int32)
    E = np.ascontiguousarray(E, np.int32)
    W = None if W is None else np.ascontiguousarray(W, np.float64)
    return V, E, W


def max_threads() -> int:
    return int(_load().orc_max_threads())


def build_inbound(V, E, W=None):
    """Restated build_inbound_from_csr: (in_row, in_col, in_w f64, dangling01, out_weight_sum)."""
    V, E, W = _prep(V, E, W)
    n = V.shape[0] - 1
    m = E.shape[0]
    in_row = np.empty(n + 1, np.int32)
    in_col = np.empty(max(m, 1), np.int32)
    in_w = np.empty(max(m, 1), np.float64)
    dang = np.empty(max(n, 1), np.int32)
    outw = np.empty(max(n, 1), np.float64)
    nnz = c_int64(0)
    rc = _load().orc_build_inbound(_p(V), _p(E), _p(W), n, m, _p(in_row), _p(in_col), _p(in_w), _p(dang), _p(outw),
                                   ctypes.byref(nnz))
    if rc != 0:
        raise RuntimeError(f"orc_build_inbound failed ({rc})")
    k = nnz.value
    return in_row, in_col[:k].copy(), in_w[:k].copy(), dang[:n].copy(), outw[:n].copy()


def inbound_values(in_col, in_w, outw, alpha):
    """pagerank.cu:343 in_val (FP32, alpha-scaled)."""
    in_col = np.ascontiguousarray(in_col, np.int32)
    in_w = np.ascontiguousarray(in_w, np.float64)
    outw = np.ascontiguousarray(outw, np.float64)
    out = np.empty(max(in_col.shape[0], 1), np.float32)
    _load().orc_inbound_values(_p(in_col), _p(in_w), _p(outw), in_col.shape[0], float(alpha), _p(out))
    return out[: in_col.shape[0]]


def pagerank_push(V, E, W=None, alpha=0.85, max_iter=100, tol=1e-6, teleport=None, sanitize=False,
                  dangling_eps=1e-15):
    """Restated _pagerank_power_iteration. Returns (ranks, iterations, last residual)."""
    V, E, W = _prep(V, E, W)
    n = V.shape[0] - 1
    out = np.empty(max(n, 1), np.float64)
    tp = None if teleport is None else np.ascontiguousarray(teleport, np.float64)
    it = c_int32(0)
    res = c_double(0.0)
    rc = _load().orc_pagerank_push(_p(V), _p(E), _p(W), n, E.shape[0], 1 if sanitize else 0, float(dangling_eps),
                                   float(alpha), int(max_iter), float(tol), _p(tp), _p(out), ctypes.byref(it),
                                   ctypes.byref(res))
    if rc != 0:
        raise RuntimeError(f"orc_pagerank_push failed ({rc})")
    return out[:n], it.value, res.value


def pagerank_pull(V, E, W=None, alpha=0.85, max_iter=100, tol=1e-6, teleport=None, dangling_eps=1e-15,
                  threads=0, inbound=None):
    """Same maths as pagerank_push over the inbound CSR (OpenMP). (ranks, iterations, residual)."""
    if inbound is None:
        inbound = build_inbound(V, E, W)
    in_row, in_col, in_w, _, outw = inbound
    n = in_row.shape[0] - 1
    out = np.empty(max(n, 1), np.float64)
    tp = None if teleport is None else np.ascontiguousarray(teleport, np.float64)
    it = c_int32(0)
    res = c_double(0.0)
    rc = _load().orc_pagerank_pull(_p(in_row), _p(in_col), _p(in_w) if W is not None else None, _p(outw), n,
                                   float(dangling_eps), float(alpha), int(max_iter), float(tol), _p(tp), _p(out),
                                   ctypes.byref(it), ctypes.byref(res), int(threads))
    if rc != 0:
        raise RuntimeError(f"orc_pagerank_pull failed ({rc})")
    return out[:n], it.value, res.value


def cpu_pagerank_omp(V, E, W=None, alpha=0.85, max_iter=100, threshold=1e-6, threads=0):
    """Port of the reference's OpenMP _pagerank. (unnormalised ranks, sweeps)."""
    V, E, W = _prep(V, E, W)
    n = V.shape[0] - 1
    out = np.empty(max(n, 1), np.float64)
    sw = c_int32(0)
    rc = _load().orc_cpu_pagerank_omp(_p(V), _p(E), _p(W), n, float(alpha), int(max_iter), float(threshold), _p(out),
                                      ctypes.byref(sw), int(threads))
    if rc != 0:
        raise RuntimeError(f"orc_cpu_pagerank_omp failed ({rc})")
    return out[:n], sw.value


def ref_build_inbound(V, E, W=None, alpha=0.85):
    """The reference's own build_inbound_from_csr (compiled from its sources).
    Returns (in_row, in_col, in_val f32, dangling01)."""
    V, E, W = _prep(V, E, W)
    n = V.shape[0] - 1
    m = E.shape[0]
    in_row = np.empty(n + 1, np.int32)
    in_col = np.empty(max(m, 1), np.int32)
    in_val = np.empty(max(m, 1), np.float32)
    dang = np.empty(max(n, 1), np.int32)
    nnz = ctypes.c_int(0)
    _load_ref().ref_build_inbound(_p(V), _p(E), _p(W), n, m, float(alpha), _p(in_row), _p(in_col), _p(in_val),
                                  _p(dang), ctypes.byref(nnz))
    k = nnz.value
    return in_row, in_col[:k].copy(), in_val[:k].copy(), dang[:n].copy()


def ref_cuda_pagerank(V, E, W, alpha, max_iter, threshold):
    """The reference's own cuSPARSE GPU solve (needs a GPU). (ranks, kernel_seconds)."""
    V, E, W = _prep(V, E, W)
    n = V.shape[0] - 1
    out = np.empty(max(n, 1), np.float64)
    ks = c_double(0.0)
    rc = _load_ref().ref_cuda_pagerank(_p(V), _p(E), _p(W), n, E.shape[0], float(alpha), int(max_iter),
                                       float(threshold), _p(out), ctypes.byref(ks))
    if rc != 0:
        raise RuntimeError(f"reference cuda_pagerank failed ({rc})")
    return out[:n], ks.value


def graph_to_csr(nodes, adj, directed, weight=None):
    """Restates build_digraph / build_graph + gen_CSR on plain Python data.

    nodes: node labels in insertion order; adj: {u: {v: attr_dict}}.
    Returns (V int32, E int32, W float64 or None).
    """
    index = {}
    for u in nodes:
        if u not in index:
            index[u] = len(index)
    for u, nbrs in adj.items():
        if u not in index:
            index[u] = len(index)
        for v in nbrs:
            if v not in index:
                index[v] = len(index)
    n = len(index)
    rows = [dict() for _ in range(n)]
    if directed:
        for u, nbrs in adj.items():
            for v, attr in nbrs.items():
                rows[index[u]][index[v]] = attr
    else:
        seen = set()
        for u, nbrs in adj.items():
            for v, attr in nbrs.items():
                iu, iv = index[u], index[v]
                if iu == iv:
                    continue
                key = (min(iu, iv), max(iu, iv))
                if key in seen:
                    continue
                seen.add(key)
                rows[iu][iv] = attr
                rows[iv][iu] = attr
    V = [0]
    E = []
    W = []
    for r in rows:
        for dst in sorted(r):
            E.append(dst)
            attr = r[dst] or {}
            W.append(float(attr.get(weight, 1.0)) if weight is not None else 1.0)
        V.append(len(E))
    return (np.asarray(V, np.int32), np.asarray(E, np.int32),
            np.asarray(W, np.float64) if weight is not None else None)
