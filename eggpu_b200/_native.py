"""ctypes binding of libegpr.so (the C ABI declared in include/egpr.h).

This module is the only place Python touches the native engine.  Importing it
loads ``eggpu_b200/libegpr.so``; if the library is missing the import fails
with instructions to build it — there is no CPU fallback.  Every pointer handed
to the library is a host pointer to a contiguous numpy array.
"""

from __future__ import annotations

import ctypes
import threading
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_uint32, c_uint64, c_void_p
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libegpr.so"

# Status codes (include/egpr.h); 0..6 keep gpu_easygraph's EG_GPU_STATUS_CODE numbering.
EGPR_SUCC = 0
EGPR_FAILED_TO_ALLOCATE_HOST_MEM = 1
EGPR_FAILED_TO_ALLOCATE_DEVICE_MEM = 2
EGPR_DEVICE_ERR = 3
EGPR_UNKNOWN_ERROR = 4
EGPR_UNSUPPORTED_GRAPH = 5
EGPR_NEGATIVE_CYCLE = 6
EGPR_TIMEOUT = 7
EGPR_INVALID_ARGUMENT = 8

EGPR_FLAG_NO_CORRECTION = 1


class EgprStats(ctypes.Structure):
    _fields_ = [
        ("iterations", c_int32),
        ("converged", c_int32),
        ("residual", c_double),
        ("kernel_seconds", c_double),
        ("total_seconds", c_double),
        ("bytes_per_iter", c_int64),
        ("launches", c_int32),
        ("reserved", c_int32),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class EgprGraphInfo(ctypes.Structure):
    _fields_ = [
        ("n", c_int32),
        ("device", c_int32),
        ("m_input", c_int64),
        ("nnz", c_int64),
        ("weighted", c_int32),
        ("n_dangling", c_int32),
        ("device_bytes", c_int64),
        ("prep_seconds", c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class EgprCacheStats(ctypes.Structure):
    _fields_ = [
        ("graphs", c_int64),
        ("device_bytes", c_int64),
        ("hits", c_int64),
        ("misses", c_int64),
        ("evictions", c_int64),
        ("budget_bytes", c_int64),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class EgprTuning(ctypes.Structure):
    _fields_ = [
        ("chunks_per_warp", c_int32),
        ("row_cost", c_int32),
        ("spmm_chunk", c_int32),
        ("configs_tried", c_int32),
        ("sweep_ms", c_double),
        ("spmm_sweep_ms", c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


EGPR_TUNE_SWEEP = 1
EGPR_TUNE_SPMM = 2


# (name, restype, argtypes) for every entry point of include/egpr.h.
_SIGNATURES = [
    ("egpr_status_string", c_char_p, [c_int]),
    ("egpr_last_error", c_char_p, []),
    ("egpr_graph_create", c_int, [c_void_p, c_void_p, c_void_p, c_int32, c_int64, POINTER(c_void_p)]),
    ("egpr_graph_destroy", c_int, [c_void_p]),
    ("egpr_graph_info_get", c_int, [c_void_p, POINTER(EgprGraphInfo)]),
    ("egpr_graph_export_inbound", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("egpr_graph_set_stream", c_int, [c_void_p, c_void_p]),
    ("egpr_graph_autotune", c_int, [c_void_p, c_uint32, POINTER(EgprTuning)]),
    ("egpr_graph_get_tuning", c_int, [c_void_p, POINTER(EgprTuning)]),
    ("egpr_graph_set_tuning", c_int, [c_void_p, POINTER(EgprTuning)]),
    ("egpr_pagerank", c_int, [c_void_p, c_double, c_int32, c_double, c_void_p, c_uint32, c_void_p, POINTER(EgprStats)]),
    ("egpr_pagerank_enqueue", c_int, [c_void_p, c_double, c_int32, c_double, c_uint32]),
    ("egpr_pagerank_collect", c_int, [c_void_p, c_void_p, POINTER(EgprStats)]),
    ("egpr_pagerank_batch", c_int,
     [c_void_p, c_double, c_int32, c_double, c_int32, c_void_p, c_uint32, c_void_p, c_void_p]),
    ("egpr_pagerank_seeds", c_int,
     [c_void_p, c_double, c_int32, c_double, c_int32, c_void_p, c_void_p, c_uint32, c_void_p, c_void_p]),
    ("egpr_pagerank_multi", c_int,
     [c_int32, c_void_p, c_double, c_int32, c_double, c_uint32, c_void_p, c_void_p]),
    ("egpr_pagerank_csr", c_int,
     [c_void_p, c_int32, c_void_p, c_int64, c_void_p, c_uint64, c_double, c_int32, c_double, c_void_p,
      POINTER(c_double)]),
    ("egpr_pagerank_device_noalloc", c_int,
     [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_int32, c_double, c_uint32, c_void_p,
      c_void_p, POINTER(EgprStats)]),
    ("egpr_session_create", c_int, [c_void_p, c_double, c_double, c_int32, POINTER(c_void_p)]),
    ("egpr_session_admit", c_int, [c_void_p, c_int32, c_void_p, c_void_p, c_int32, c_void_p]),
    ("egpr_session_step", c_int, [c_void_p, c_int32, c_void_p, POINTER(c_int32)]),
    ("egpr_session_collect", c_int, [c_void_p, c_int32, c_void_p, c_uint32, c_void_p, c_void_p]),
    ("egpr_session_info", c_int, [c_void_p, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32)]),
    ("egpr_session_destroy", c_int, [c_void_p]),
    ("egpr_cache_stats_get", c_int, [POINTER(EgprCacheStats)]),
    ("egpr_cache_reset", c_int, []),
    ("egpr_cache_set_budget", c_int, [c_int64]),
]

EXPORTED_SYMBOLS = tuple(name for name, _, _ in _SIGNATURES)


def _load():
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is not built; run `python -m eggpu_b200.build` (needs nvcc). "
            "eggpu_b200 has no CPU fallback."
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, restype, argtypes in _SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    return lib


lib = _load()


class EgprError(RuntimeError):
    """A non-zero status from libegpr (message = egpr_status_string + detail)."""

    def __init__(self, status: int, where: str = ""):
        self.status = int(status)
        detail = lib.egpr_last_error().decode(errors="replace")
        msg = lib.egpr_status_string(self.status).decode(errors="replace")
        if detail:
            msg = f"{msg} ({detail})"
        if where:
            msg = f"{where}: {msg}"
        super().__init__(msg)


def check(status: int, where: str = "") -> None:
    if status != EGPR_SUCC:
        raise EgprError(status, where)


def status_string(status: int) -> str:
    return lib.egpr_status_string(int(status)).decode()


def _ptr(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class PreparedGraph:
    """A graph prepared on the current CUDA device (owns an ``egpr_graph``).

    ``V``/``E``/``W`` form an out-edge CSR: ``V`` int32[n+1], ``E`` int32[m],
    ``W`` float64[m] or None for unit weights.
    """

    def __init__(self, V, E, W=None):
        V = _i32(V)
        E = _i32(E)
        W = None if W is None else _f64(W)
        n = int(V.shape[0]) - 1
        m = int(E.shape[0])
        if W is not None and W.shape[0] != m:
            raise ValueError("W must have one weight per CSR entry")
        h = c_void_p()
        check(lib.egpr_graph_create(_ptr(V), _ptr(E), _ptr(W), n, m, ctypes.byref(h)), "egpr_graph_create")
        self._h = h
        self._lock = threading.Lock()
        info = self.info()
        self.n = info["n"]
        self.nnz = info["nnz"]
        self.m_input = info["m_input"]
        self.weighted = bool(info["weighted"])
        self.device = info["device"]

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("PreparedGraph is closed")
        return self._h

    def info(self) -> dict:
        inf = EgprGraphInfo()
        check(lib.egpr_graph_info_get(self.handle, ctypes.byref(inf)), "egpr_graph_info_get")
        return inf.as_dict()

    def export_inbound(self):
        """(in_row, in_col, in_w float32, dangling01, out_weight_sum) copied to the host."""
        n, nnz = self.n, self.nnz
        in_row = np.empty(n + 1, np.int32)
        in_col = np.empty(max(nnz, 1), np.int32)
        in_w = np.empty(max(nnz, 1), np.float32)
        dang = np.empty(n, np.int32)
        outw = np.empty(n, np.float64)
        check(lib.egpr_graph_export_inbound(self.handle, _ptr(in_row), _ptr(in_col), _ptr(in_w), _ptr(dang), _ptr(outw)),
              "egpr_graph_export_inbound")
        return in_row, in_col[:nnz], in_w[:nnz], dang, outw

    def autotune(self, sweep=True, spmm=True) -> dict:
        """Times candidate work layouts on this graph and keeps the fastest
        (egpr_graph_autotune); returns the chosen parameters and timings."""
        what = (EGPR_TUNE_SWEEP if sweep else 0) | (EGPR_TUNE_SPMM if spmm else 0)
        if what == 0:
            return self.tuning()
        t = EgprTuning()
        check(lib.egpr_graph_autotune(self.handle, what, ctypes.byref(t)), "egpr_graph_autotune")
        return t.as_dict()

    def tuning(self) -> dict:
        t = EgprTuning()
        check(lib.egpr_graph_get_tuning(self.handle, ctypes.byref(t)), "egpr_graph_get_tuning")
        return {k: v for k, v in t.as_dict().items() if k in ("chunks_per_warp", "row_cost", "spmm_chunk")}

    def set_tuning(self, chunks_per_warp=None, row_cost=None, spmm_chunk=None) -> None:
        cur = self.tuning()
        t = EgprTuning()
        t.chunks_per_warp = cur["chunks_per_warp"] if chunks_per_warp is None else int(chunks_per_warp)
        t.row_cost = cur["row_cost"] if row_cost is None else int(row_cost)
        t.spmm_chunk = cur["spmm_chunk"] if spmm_chunk is None else int(spmm_chunk)
        check(lib.egpr_graph_set_tuning(self.handle, ctypes.byref(t)), "egpr_graph_set_tuning")

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib.egpr_graph_set_stream(self.handle, None if not stream_ptr else c_void_p(int(stream_ptr))),
              "egpr_graph_set_stream")

    def pagerank(self, alpha=0.85, max_iter=100, tol=1e-6, personalization=None, correction=True, out=None):
        """Returns (ranks float64[n], stats dict).  out: optional float64[n]
        result array (page-locked memory makes the copy back faster)."""
        res = self._vec_out(out)
        pers = None if personalization is None else _f64(personalization)
        if pers is not None and pers.shape[0] != self.n:
            raise ValueError("personalization must have n entries")
        st = EgprStats()
        flags = 0 if correction else EGPR_FLAG_NO_CORRECTION
        check(lib.egpr_pagerank(self.handle, float(alpha), int(max_iter), float(tol), _ptr(pers), flags, _ptr(res),
                                ctypes.byref(st)), "egpr_pagerank")
        return res, st.as_dict()

    def enqueue(self, alpha=0.85, max_iter=100, tol=1e-6, correction=True) -> None:
        flags = 0 if correction else EGPR_FLAG_NO_CORRECTION
        check(lib.egpr_pagerank_enqueue(self.handle, float(alpha), int(max_iter), float(tol), flags),
              "egpr_pagerank_enqueue")

    def collect(self, out=None, copy=True):
        res = self._vec_out(out) if copy else None
        st = EgprStats()
        check(lib.egpr_pagerank_collect(self.handle, _ptr(res), ctypes.byref(st)), "egpr_pagerank_collect")
        return res, st.as_dict()

    def _vec_out(self, out):
        if out is None:
            return np.empty(self.n, np.float64)
        if (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.shape != (self.n,)
                or not out.flags.c_contiguous or not out.flags.writeable):
            raise ValueError(f"out must be a writeable C-contiguous float64 array of shape ({self.n},)")
        return out

    def _batch_out(self, k, out):
        if out is None:
            return np.empty((k, self.n), np.float64)
        if (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.shape != (k, self.n)
                or not out.flags.c_contiguous or not out.flags.writeable):
            raise ValueError(f"out must be a writeable C-contiguous float64 array of shape ({k}, {self.n})")
        return out

    def pagerank_batch(self, teleport, alpha=0.85, max_iter=100, tol=1e-6, correction=True, out=None):
        """teleport: (k, n) array of non-negative vectors. Returns ((k, n) ranks, [stats]).
        out: optional (k, n) float64 result array (page-locked memory makes the copy back faster)."""
        T = _f64(teleport)
        if T.ndim != 2 or T.shape[1] != self.n:
            raise ValueError("teleport must have shape (k, n)")
        k = T.shape[0]
        res = self._batch_out(k, out)
        sts = (EgprStats * k)()
        flags = 0 if correction else EGPR_FLAG_NO_CORRECTION
        check(lib.egpr_pagerank_batch(self.handle, float(alpha), int(max_iter), float(tol), k, _ptr(T), flags,
                                      _ptr(res), ctypes.cast(sts, c_void_p)), "egpr_pagerank_batch")
        return res, [s.as_dict() for s in sts]

    def pagerank_seeds(self, seed_sets, alpha=0.85, max_iter=100, tol=1e-6, correction=True, out=None):
        """seed_sets: list of vertex-id sequences (uniform teleport over each).
        out: optional (k, n) float64 result array, as for pagerank_batch."""
        k = len(seed_sets)
        ptr = np.zeros(k + 1, np.int32)
        for j, s in enumerate(seed_sets):
            ptr[j + 1] = ptr[j] + len(s)
        seeds = np.concatenate([np.asarray(s, np.int32) for s in seed_sets]) if k else np.zeros(0, np.int32)
        seeds = _i32(seeds)
        res = self._batch_out(k, out)
        sts = (EgprStats * k)()
        flags = 0 if correction else EGPR_FLAG_NO_CORRECTION
        check(lib.egpr_pagerank_seeds(self.handle, float(alpha), int(max_iter), float(tol), k, _ptr(ptr),
                                      _ptr(seeds) if seeds.size else None, flags, _ptr(res),
                                      ctypes.cast(sts, c_void_p)), "egpr_pagerank_seeds")
        return res, [s.as_dict() for s in sts]

    def close(self) -> None:
        """Frees the device graph; refused (EgprError, the handle kept) while a
        Session on it is alive."""
        if getattr(self, "_h", None) is not None:
            check(lib.egpr_graph_destroy(self._h), "egpr_graph_destroy")
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Session:
    """A running batched personalised-PageRank solve that requests join and
    leave column by column (owns an ``egpr_session``; see include/egpr.h).

    ``admit`` places seed-set requests in free slots, ``step`` runs a few
    sweeps of every running column and returns the finished slots, ``collect``
    hands back their ranks (FP64 correction sweep, normalisation) and frees
    the slots.  The session keeps its PreparedGraph alive.
    """

    def __init__(self, graph: "PreparedGraph", alpha=0.85, tol=1e-6, slots=32):
        h = c_void_p()
        check(lib.egpr_session_create(graph.handle, float(alpha), float(tol), int(slots), ctypes.byref(h)),
              "egpr_session_create")
        self._h = h
        self.graph = graph
        self.alpha = float(alpha)
        self.tol = float(tol)
        self.n = graph.n
        self.slots = self.info()["slots"]
        self._done = np.zeros(self.slots, np.int32)

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("Session is closed")
        return self._h

    def info(self) -> dict:
        a, b, c = c_int32(), c_int32(), c_int32()
        check(lib.egpr_session_info(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
              "egpr_session_info")
        return {"slots": a.value, "running": b.value, "done": c.value, "free": a.value - b.value - c.value}

    def admit(self, seed_sets, max_iter=100) -> list:
        k = len(seed_sets)
        if k == 0:
            return []
        ptr = np.zeros(k + 1, np.int32)
        for j, s in enumerate(seed_sets):
            ptr[j + 1] = ptr[j] + len(s)
        seeds = _i32(np.concatenate([np.asarray(s, np.int32) for s in seed_sets]))
        out = np.zeros(k, np.int32)
        check(lib.egpr_session_admit(self.handle, k, _ptr(ptr), _ptr(seeds), int(max_iter), _ptr(out)),
              "egpr_session_admit")
        return [int(x) for x in out]

    def step(self, sweeps=4) -> list:
        nd = c_int32()
        check(lib.egpr_session_step(self.handle, int(sweeps), _ptr(self._done), ctypes.byref(nd)),
              "egpr_session_step")
        return [int(x) for x in self._done[: nd.value]]

    def collect(self, slots, correction=True, out=None):
        k = len(slots)
        if out is None:
            out = np.empty((k, self.n), np.float64)
        elif (not isinstance(out, np.ndarray) or out.shape != (k, self.n) or out.dtype != np.float64
              or not out.flags["C_CONTIGUOUS"] or not out.flags.writeable):
            raise ValueError(f"out must be a writeable C-contiguous float64 array of shape {(k, self.n)}")
        sl = np.asarray(slots, np.int32)
        sts = (EgprStats * max(k, 1))()
        flags = 0 if correction else EGPR_FLAG_NO_CORRECTION
        check(lib.egpr_session_collect(self.handle, k, _ptr(sl), flags, _ptr(out), ctypes.cast(sts, c_void_p)),
              "egpr_session_collect")
        return out, [sts[i].as_dict() for i in range(k)]

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            lib.egpr_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pinned_empty(shape, dtype=np.float64):
    """A page-locked host array (CUDA copies into it run at full link speed);
    a plain array where page-locked memory cannot be had.  Keep the array
    alive for as long as its data is used (it keeps the memory)."""
    try:
        import torch

        if torch.cuda.is_available():
            t = torch.empty(tuple(int(x) for x in np.atleast_1d(shape)), dtype=_TORCH_DTYPES[np.dtype(dtype)],
                            pin_memory=True)
            return t.numpy()  # the array's base holds the page-locked storage
    except Exception:
        pass
    return np.empty(shape, dtype)


_TORCH_DTYPES = {}
try:
    import torch as _torch

    _TORCH_DTYPES = {np.dtype(np.float64): _torch.float64, np.dtype(np.float32): _torch.float32,
                     np.dtype(np.int32): _torch.int32, np.dtype(np.int64): _torch.int64}
except Exception:  # torch is optional here
    pass


def pagerank_multi(graphs, alpha=0.85, max_iter=100, tol=1e-6, correction=True, out=None):
    """Solves many prepared graphs in one persistent launch per sweep.
    out: optional list of caller-owned float64[n_i] result arrays; by default
    the results are views of one page-locked block (up to 256 MiB)."""
    count = len(graphs)
    handles = (c_void_p * count)(*[g.handle for g in graphs])
    if out is not None:
        outs = list(out)
        if len(outs) != count or any(
                not isinstance(o, np.ndarray) or o.dtype != np.float64 or o.shape != (g.n,)
                or not o.flags.c_contiguous or not o.flags.writeable for o, g in zip(outs, graphs)):
            raise ValueError("out must hold one writeable contiguous float64[n] array per graph")
    else:
        total = sum(g.n for g in graphs)
        block = pinned_empty(total) if 8 * total <= (256 << 20) else np.empty(total, np.float64)
        offs = np.concatenate([[0], np.cumsum([g.n for g in graphs])])
        outs = [block[offs[i]:offs[i + 1]] for i in range(count)]
    out_ptrs = (c_void_p * count)(*[o.ctypes.data for o in outs])
    sts = (EgprStats * count)()
    flags = 0 if correction else EGPR_FLAG_NO_CORRECTION
    check(lib.egpr_pagerank_multi(count, ctypes.cast(handles, c_void_p), float(alpha), int(max_iter), float(tol),
                                  flags, ctypes.cast(out_ptrs, c_void_p), ctypes.cast(sts, c_void_p)),
          "egpr_pagerank_multi")
    return outs, [s.as_dict() for s in sts]


def pagerank_csr(V, E, W, graph_id, alpha, max_iter, threshold, out=None):
    """Drop-in for gpu_easygraph::pagerank: returns (PR float64[n], kernel_seconds).
    out: optional caller-owned float64[n] result (page-locked memory copies back faster)."""
    V = _i32(V)
    E = _i32(E)
    W = None if W is None or len(W) == 0 else _f64(W)
    n = int(V.shape[0]) - 1
    if out is None:
        PR = np.empty(max(n, 0), np.float64)
    else:
        if (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.shape != (max(n, 0),)
                or not out.flags.c_contiguous or not out.flags.writeable):
            raise ValueError(f"out must be a writeable contiguous float64 array of {max(n, 0)} entries")
        PR = out
    ks = c_double(0.0)
    check(lib.egpr_pagerank_csr(_ptr(V), int(V.shape[0]), _ptr(E), int(E.shape[0]), _ptr(W), int(graph_id) & (2**64 - 1),
                                float(alpha), int(max_iter), float(threshold), _ptr(PR), ctypes.byref(ks)),
          "egpr_pagerank_csr")
    return PR, ks.value


def cache_stats() -> dict:
    cs = EgprCacheStats()
    check(lib.egpr_cache_stats_get(ctypes.byref(cs)), "egpr_cache_stats_get")
    return cs.as_dict()


def cache_reset() -> None:
    check(lib.egpr_cache_reset(), "egpr_cache_reset")


def cache_set_budget(nbytes: int) -> None:
    check(lib.egpr_cache_set_budget(int(nbytes)), "egpr_cache_set_budget")
