"""GPU backend of ``pagerank`` — the mirror of the reference's PageRank path in
easygraph/utils/gpu_eggpu_backend.py.

Reference pieces and their counterparts here:

* ``_DenseValueDict`` (gpu_eggpu_backend.py:254-348): :class:`DenseValueDict`,
  a read-only node -> float Mapping over a dense float64 vector; ``dict(r)``
  works, mutation raises.
* ``_normalize_dense_array`` (:1092-1126) and ``_DenseResultShapeError``:
  :func:`normalize_dense_array`, :class:`DenseResultShapeError` (length n, or
  n+1 with a leading sentinel).
* ``_graph_stamp`` / ``_prepared_graph_usable`` / ``_prepare_graph_cache``
  (:1595-1716): :func:`graph_stamp`, :func:`prepared_graph_usable`,
  :func:`prepare_graph_context` — the prepared context lives in
  ``G.cache["__eggpu_prepared_graph__"]`` and is invalidated by
  ``G._mutation_generation`` (easygraph/classes/graph.py:1641-1644), by a node
  count change, and by a full O(|V|) stamp check every
  ``EASYGRAPH_GPU_CTX_VALIDATE_EVERY`` (32) reuses.
* ``_get_cached_cpp_graph`` (:603-633) + ``gen_CSR`` (cpp_easygraph/classes/
  graph.cpp:719-886): :func:`graph_csr` builds the out-edge CSR (rows in node
  order, each row sorted by destination index, undirected graphs without
  self-loops and with both directions) and :func:`prepared_native` keeps the
  device-prepared graph in ``G.cache`` keyed by (context id, weight).
* ``cpp_easygraph.cpp_gpu_pagerank_dense`` (cpp_easygraph/functions/pagerank/
  pagerank.cpp:176-223): :func:`cpp_gpu_pagerank_dense`, same arguments and
  ``{"values_dense", "kernel_seconds"}`` result, calling the C ABI.
* ``pagerank`` (:1782-1821): :func:`pagerank` with the extra
  ``personalization`` argument; ``set_last_kernel_time`` /
  ``get_last_kernel_time`` (:89-97).

There is no CPU fallback: a native failure raises :class:`EgprError`.
"""

from __future__ import annotations

import os
import time
import weakref
from collections.abc import Mapping

import numpy as np

_LAST_KERNEL_SECONDS: dict = {}
_PREPARED_CACHE_KEY = "__eggpu_prepared_graph__"
_NATIVE_CACHE_KEY = "__egpr_native_graph__"
_HASH_MASK = (1 << 64) - 1
_FALLBACK_GRAPH_CACHE = weakref.WeakKeyDictionary()


def _env_int(name, default, lo):
    try:
        return max(lo, int(os.environ.get(name, str(default))))
    except ValueError:
        return default


_GRAPH_CTX_VALIDATE_EVERY = _env_int("EASYGRAPH_GPU_CTX_VALIDATE_EVERY", 32, 1)


def _env_flag(name, default):
    return os.environ.get(name, default).strip().upper() in {"1", "TRUE", "ON", "YES"}


# Opt-in result cache, per prepared graph context (easygraph/utils/
# gpu_eggpu_backend.py:13-30,1723-1779): off unless EASYGRAPH_GPU_RESULT_CACHE
# is set; at most MAX_ITEMS results per graph, none for graphs above MAX_NODES
# nodes (0 = no limit); a hit hands out a copy unless RETURN_COPY is off.
_RESULT_CACHE_ENABLED = _env_flag("EASYGRAPH_GPU_RESULT_CACHE", "FALSE")
_RESULT_CACHE_RETURN_COPY = _env_flag("EASYGRAPH_GPU_RESULT_CACHE_RETURN_COPY", "TRUE")
_RESULT_CACHE_MAX_ITEMS = _env_int("EASYGRAPH_GPU_RESULT_CACHE_MAX_ITEMS", 8, 1)
_RESULT_CACHE_MAX_NODES = _env_int("EASYGRAPH_GPU_RESULT_CACHE_MAX_NODES", 2_000_000, 0)

# The reference's cache and result-format switches (gpu_eggpu_backend.py:40-75):
# no graph context kept in G.cache, no prepared device graph kept in G.cache,
# and PageRank results as plain dicts instead of the dense read-only mapping
# (EASYGRAPH_GPU_PR_PREFER_CPP_DICT, defaulting to EASYGRAPH_GPU_PREFER_CPP_DICT).
_GRAPH_CONTEXT_CACHE_DISABLED = _env_flag("EASYGRAPH_GPU_DISABLE_GRAPH_CONTEXT_CACHE", "")
_NATIVE_GRAPH_CACHE_DISABLED = _env_flag("EASYGRAPH_GPU_DISABLE_CPP_GRAPH_CACHE", "")
_PR_PREFER_DICT = _env_flag("EASYGRAPH_GPU_PR_PREFER_CPP_DICT", os.environ.get("EASYGRAPH_GPU_PREFER_CPP_DICT", ""))


def set_last_kernel_time(key, seconds):
    if seconds is None:
        _LAST_KERNEL_SECONDS.pop(key, None)
    else:
        _LAST_KERNEL_SECONDS[key] = float(seconds)


def get_last_kernel_time(key):
    return _LAST_KERNEL_SECONDS.get(key)


# ---------------------------------------------------------------- results --
class DenseResultShapeError(ValueError):
    """A native dense result does not have the documented length."""


def normalize_dense_array(raw_values, target_len, dtype="float64", *, allow_leading_sentinel=False,
                          result_name="dense vector"):
    try:
        arr = np.asarray(raw_values, dtype=dtype)
    except Exception as exc:  # noqa: BLE001 - reported as a shape error like the reference
        raise DenseResultShapeError(
            f"{result_name} could not be converted to a one-dimensional dense result: {exc}") from exc
    exact = (int(target_len),)
    if arr.ndim == 1 and arr.shape == exact:
        return arr
    if allow_leading_sentinel and arr.ndim == 1 and arr.shape == (int(target_len) + 1,):
        return arr[1:]
    expected = [exact] + ([(int(target_len) + 1,)] if allow_leading_sentinel else [])
    shown = " or ".join(str(s) for s in expected)
    raise DenseResultShapeError(f"{result_name} has shape {arr.shape}; expected {shown}")


class DenseValueDict(Mapping):
    """Read-only node -> float mapping over a dense result vector.

    Not a ``dict`` subclass on purpose (equality and JSON encoding must see the
    values, not an empty dict storage); ``dict(result)`` materialises a copy.
    Iteration order is the graph's node order.
    """

    def __init__(self, nodes, values, node_to_idx=None):
        self._nodes = nodes if isinstance(nodes, range) else list(nodes)
        self._values = normalize_dense_array(values, len(self._nodes), dtype="float64",
                                             result_name="dense node-value mapping")
        self._values.setflags(write=False)
        self._node_to_idx = node_to_idx if isinstance(node_to_idx, dict) else None
        self._range = isinstance(self._nodes, range) and self._nodes.start == 0 and self._nodes.step == 1
        self._index = None

    def _idx(self, key):
        if self._node_to_idx is not None:
            return self._node_to_idx.get(key)
        if self._range:
            if isinstance(key, (int, np.integer)) and not isinstance(key, bool) and 0 <= key < len(self._nodes):
                return int(key)
            return None
        if self._index is None:
            self._index = {node: i for i, node in enumerate(self._nodes)}
        return self._index.get(key)

    def __len__(self):
        return len(self._nodes)

    def __iter__(self):
        return iter(self._nodes)

    def __contains__(self, key):
        try:
            return self._idx(key) is not None
        except TypeError:
            return False

    def __getitem__(self, key):
        idx = self._idx(key)
        if idx is None:
            raise KeyError(key)
        return float(self._values[idx])

    def get(self, key, default=None):
        idx = self._idx(key)
        return default if idx is None else float(self._values[idx])

    def items(self):
        for i, node in enumerate(self._nodes):
            yield node, float(self._values[i])

    def values(self):
        return self._values

    def copy(self):
        return dict(self.items())

    to_dict = copy

    def to_numpy(self, copy=False):
        return self._values.copy() if copy else self._values

    def tolist(self):
        return self._values.tolist()

    def __array__(self, dtype=None, copy=None):
        return np.asarray(self._values, dtype=dtype)

    def __setitem__(self, key, value):
        raise TypeError("PageRank results are read-only; use dict(result) for a mutable copy")

    def __delitem__(self, key):
        raise TypeError("PageRank results are read-only; use dict(result) for a mutable copy")

    def __repr__(self):
        if len(self._nodes) > 1000:
            return f"{type(self).__name__}(nodes={len(self._nodes)}, dtype=float64)"
        return repr(self.copy())


# ---------------------------------------------------------- result cache --
def _cache_key(name, *parts):
    """Cache key of a solve; floats rounded to 12 digits (gpu_eggpu_backend.py:1723-1730)."""
    return (name,) + tuple(round(float(p), 12) if isinstance(p, float) else p for p in parts)


def _allow_result_cache(prepared):
    if not _RESULT_CACHE_ENABLED:
        return False
    nodes = prepared.get("nodes")
    if nodes is None:
        return False
    return not (_RESULT_CACHE_MAX_NODES > 0 and len(nodes) > _RESULT_CACHE_MAX_NODES)


def _copy_for_return(result):
    if not _RESULT_CACHE_RETURN_COPY:
        return result
    if isinstance(result, DenseValueDict):
        return DenseValueDict(result._nodes, result.to_numpy(copy=True), node_to_idx=result._node_to_idx)
    import copy

    return copy.deepcopy(result)


def _result_cache_get(prepared, key):
    cache = prepared.get("result_cache")
    if not isinstance(cache, dict):
        return None
    entry = cache.get(key)
    if entry is None:
        return None
    return _copy_for_return(entry["result"]), entry["kernel"]


def _result_cache_put(prepared, key, result, kernel):
    """Stores a private snapshot of result under key, least recently stored out first."""
    if not _allow_result_cache(prepared):
        return
    cache = prepared.setdefault("result_cache", {})
    order = prepared.setdefault("result_cache_order", [])
    cache[key] = {"result": _copy_for_return(result), "kernel": kernel}
    if key in order:
        order.remove(key)
    order.append(key)
    while len(order) > _RESULT_CACHE_MAX_ITEMS:
        cache.pop(order.pop(0), None)


# ------------------------------------------------------- prepared context --
def _graph_cache_dict(G):
    cache = getattr(G, "cache", None)
    if isinstance(cache, dict):
        return cache
    try:
        cache = _FALLBACK_GRAPH_CACHE.get(G)
        if cache is None:
            cache = {}
            _FALLBACK_GRAPH_CACHE[G] = cache
        return cache
    except TypeError:
        return None


def is_bulk_graph(G):
    return bool(getattr(G, "_eggpu_bulk_csr", False))


def bulk_weight_available(G, weight):
    """Whether a bulk graph carries edge attribute ``weight``: its own answer
    (eggpu_b200.bulk graphs), else the reference's rule for its
    EGGPUBulkGraph, a weights file under that key
    (easygraph/utils/gpu_eggpu_backend.py:120-126)."""
    if weight is None or not is_bulk_graph(G):
        return False
    if hasattr(G, "has_weight"):
        return bool(G.has_weight(weight))
    return getattr(G, "weights_path", None) is not None and getattr(G, "weight_key", None) == str(weight)


def _bulk_csr(G, weight):
    """(V, E, W) of a bulk graph: the arrays of an eggpu_b200.bulk graph, or
    the artifact files of the reference's EGGPUBulkGraph, which keeps them
    in its C++ graph and exposes only their paths."""
    if hasattr(G, "csr_arrays"):
        return G.csr_arrays(weight)
    if weight is not None and not bulk_weight_available(G, weight):
        raise NotImplementedError(
            f"weighted PageRank requires an EGGPU CSR artifact containing the {weight!r} edge attribute")
    n, m = int(G.num_nodes), int(G.num_entries)

    def read(path, dtype, count):
        arr = np.fromfile(path, dtype=dtype)
        if arr.shape[0] != count:
            raise ValueError(f"{path}: expected {count} values of {np.dtype(dtype).name}, found {arr.shape[0]}")
        return arr

    V = read(G.offsets_path, np.int32, n + 1)
    E = read(G.indices_path, np.int32, m)
    W = read(G.weights_path, np.float64, m) if weight is not None else None
    return V, E, W


def _adj_dict(G):
    adj = getattr(G, "_adj", None)
    if adj is None:
        adj = G.adj
    return adj


def _mix64(h, x):
    h ^= (int(x) + 0x9E3779B97F4A7C15 + ((h << 6) & _HASH_MASK) + (h >> 2)) & _HASH_MASK
    return h & _HASH_MASK


def graph_stamp(G):
    """O(|V|) fingerprint: node count, adjacency slots, node hashes and degrees,
    and the first neighbours of the first 32 nodes (native when the graph
    walk extension is built; _graph_stamp_py is its specification)."""
    adj = _adj_dict(G)
    if _graph_walk is not None and isinstance(adj, dict):
        res = _graph_walk.stamp(adj)
        if res is not None:
            nodes, slots, h = res
            return (bool(G.is_directed()), nodes, slots, h)
    return _graph_stamp_py(G, adj)


def _graph_stamp_py(G, adj):
    edge_slots = 0
    h = 1469598103934665603
    for i, (u, nbrs) in enumerate(adj.items()):
        deg = len(nbrs)
        edge_slots += deg
        h = _mix64(h, hash(u))
        h = _mix64(h, deg)
        if i < 32:
            for j, v in enumerate(nbrs):
                if j >= 4:
                    break
                h = _mix64(h, hash(v))
    return (bool(G.is_directed()), len(adj), edge_slots, h)


def prepared_graph_usable(G, prepared):
    if not isinstance(prepared, dict):
        return False
    if bool(G.is_directed()) != bool(prepared.get("directed")):
        return False
    if is_bulk_graph(G):
        return prepared.get("bulk_signature") == getattr(G, "_eggpu_bulk_signature", None)
    gen = getattr(G, "_mutation_generation", None)
    if gen is not None and prepared.get("mutation_generation") != gen:
        return False
    if len(_adj_dict(G)) != int(prepared.get("node_count", -1)):
        return False
    hits = int(prepared.get("reuse_hits", 0)) + 1
    prepared["reuse_hits"] = hits
    if hits % _GRAPH_CTX_VALIDATE_EVERY != 0:
        return True
    return prepared.get("stamp") == graph_stamp(G)


def prepare_graph_context(G):
    cache = None if _GRAPH_CONTEXT_CACHE_DISABLED else _graph_cache_dict(G)
    prepared = cache.get(_PREPARED_CACHE_KEY) if cache is not None else None
    if prepared is not None and prepared_graph_usable(G, prepared):
        return prepared
    if is_bulk_graph(G):
        n = int(G.num_nodes)
        prepared = {
            "ctx_id": time.time_ns(),
            "stamp": (bool(G.is_directed()), n, int(G.num_entries), hash(G._eggpu_bulk_signature) & _HASH_MASK),
            "bulk_csr": True,
            "bulk_signature": G._eggpu_bulk_signature,
            "node_count": n,
            "directed": bool(G.is_directed()),
            "nodes": range(n),
            "node_to_idx": None,
            "reuse_hits": 0,
            "mutation_generation": None,
        }
    else:
        nodes = list(G.nodes.keys()) if hasattr(G.nodes, "keys") else list(G.nodes)
        prepared = {
            "ctx_id": time.time_ns(),
            "stamp": graph_stamp(G),
            "node_count": len(nodes),
            "directed": bool(G.is_directed()),
            "nodes": nodes,
            "node_to_idx": {node: i for i, node in enumerate(nodes)},
            "reuse_hits": 0,
            "mutation_generation": getattr(G, "_mutation_generation", None),
        }
    if cache is not None:
        cache[_PREPARED_CACHE_KEY] = prepared
    return prepared


# -------------------------------------------------------------- CSR build --
def _weight_of(attr, weight):
    if weight is None or not attr:
        return 1.0
    val = attr.get(weight, 1.0)
    try:
        return float(val)
    except (TypeError, ValueError):
        return 1.0


try:  # the native walk (eggpu_b200/csrc/graph_walk.cpp); same arrays as _graph_csr_py
    from . import _graph_walk
except ImportError:  # not built: the Python walk below gives the same result
    _graph_walk = None


def graph_csr(G, prepared, weight=None):
    """Out-edge CSR (V int32, E int32, W float64 or None) of G in prepared["nodes"] order.

    Directed graphs keep every arc (self-loops included); undirected graphs
    drop self-loops and store each pair once per direction, the rules of
    build_digraph / build_graph (cpp_easygraph/classes/graph_convert.cpp:72-134).
    Rows are sorted by destination index as gen_CSR does.  The walk over the
    adjacency dicts runs in native code when the extension is built.
    """
    if is_bulk_graph(G):
        return _bulk_csr(G, weight)
    if _graph_walk is not None:
        adj = _adj_dict(G)
        index = prepared["node_to_idx"]
        if isinstance(adj, dict) and isinstance(index, dict):
            res = _graph_walk.out_csr(adj, index, len(prepared["nodes"]), bool(prepared["directed"]), weight)
            if res is not None:
                V, E, W = res
                return (np.frombuffer(V, dtype=np.int32), np.frombuffer(E, dtype=np.int32),
                        None if W is None else np.frombuffer(W, dtype=np.float64))
    return _graph_csr_py(G, prepared, weight)


def _graph_csr_py(G, prepared, weight=None):
    """graph_csr's walk in Python (the specification of the native walk)."""
    index = prepared["node_to_idx"]
    n = len(prepared["nodes"])
    if n >= 2**31 - 1:
        raise ValueError("node count exceeds the signed 32-bit CSR limit")
    adj = _adj_dict(G)
    directed = bool(prepared["directed"])
    src, dst, wts = [], [], []
    if directed:
        for u, nbrs in adj.items():
            iu = index[u]
            for v, attr in nbrs.items():
                src.append(iu)
                dst.append(index[v])
                if weight is not None:
                    wts.append(_weight_of(attr, weight))
    else:
        seen = set()
        for u, nbrs in adj.items():
            iu = index[u]
            for v, attr in nbrs.items():
                iv = index[v]
                if iu == iv:
                    continue
                key = (iu, iv) if iu < iv else (iv, iu)
                if key in seen:
                    continue
                seen.add(key)
                w = _weight_of(attr, weight) if weight is not None else 1.0
                src.extend((iu, iv))
                dst.extend((iv, iu))
                if weight is not None:
                    wts.extend((w, w))
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    if src.size >= 2**31 - 1:
        raise ValueError("adjacency entry count exceeds the signed 32-bit CSR limit")
    order = np.lexsort((dst, src))
    E = dst[order].astype(np.int32)
    counts = np.bincount(src, minlength=n) if src.size else np.zeros(n, np.int64)
    V = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=V[1:])
    W = None
    if weight is not None:
        W = np.asarray(wts, dtype=np.float64)[order]
    return V.astype(np.int32), E, W


def prepared_native(G, prepared, weight=None):
    """The device-prepared graph for (G, weight), cached in G.cache."""
    from ._native import PreparedGraph

    cache = None if _NATIVE_GRAPH_CACHE_DISABLED else _graph_cache_dict(G)
    key = f"{_NATIVE_CACHE_KEY}:{'directed' if prepared['directed'] else 'undirected'}:{weight!r}"
    if cache is not None:
        hit = cache.get(key)
        if hit is not None and hit[0] == prepared["ctx_id"]:
            return hit[1]
    V, E, W = graph_csr(G, prepared, weight)
    pg = PreparedGraph(V, E, W)
    if cache is not None:
        cache[key] = (prepared["ctx_id"], pg)
    return pg


# ------------------------------------------------------------- solves -------
def cpp_gpu_pagerank_dense(csr, alpha, max_iterator, threshold, weight=None, personalization=None):
    """Mirror of cpp_easygraph.cpp_gpu_pagerank_dense on a (V, E, W) CSR or a
    PreparedGraph: returns {"values_dense": float64[n], "kernel_seconds": s}."""
    from ._native import PreparedGraph

    pg = csr if isinstance(csr, PreparedGraph) else PreparedGraph(*csr)
    ranks, stats = pg.pagerank(alpha=float(alpha), max_iter=int(max_iterator), tol=float(threshold),
                               personalization=personalization, out=_result_vector(pg.n))
    return {"values_dense": ranks, "kernel_seconds": stats["kernel_seconds"], "stats": stats}


_PINNED_RESULT_MAX = 256 << 20


def _result_vector(n):
    """The array the ranks are copied into, which the result Mapping then
    wraps without a copy: page-locked (faster copy; the allocator reuses it
    once the result is dropped) up to 256 MiB."""
    from ._native import pinned_empty

    return pinned_empty(n) if 8 * n <= _PINNED_RESULT_MAX else None


def _personalization_vector(personalization, prepared):
    if personalization is None:
        return None
    n = len(prepared["nodes"])
    if isinstance(personalization, Mapping):
        vec = np.zeros(n, np.float64)
        idx_of = prepared["node_to_idx"]
        for node, val in personalization.items():
            if idx_of is not None:
                i = idx_of.get(node)
            else:  # bulk graphs: the nodes are 0..n-1
                ok = isinstance(node, (int, np.integer)) and not isinstance(node, bool) and 0 <= node < n
                i = int(node) if ok else None
            if i is None:
                raise KeyError(f"personalization node {node!r} is not in the graph")
            vec[i] = float(val)
    else:
        vec = np.asarray(personalization, dtype=np.float64)
        if vec.shape != (n,):
            raise ValueError(f"personalization must have {n} entries")
    if not np.all(np.isfinite(vec)) or np.any(vec < 0) or not vec.sum() > 0:
        raise ValueError("personalization values must be finite, >= 0 and not all zero")
    return vec


def pagerank(G, alpha=0.85, max_iter=200, eps=1e-6, weight=None, personalization=None):
    prepared = prepare_graph_context(G)
    if prepared.get("bulk_csr") and weight is not None and not bulk_weight_available(G, weight):
        raise NotImplementedError(
            f"weighted PageRank requires an EGGPU CSR artifact containing the {weight!r} edge attribute")
    # personalised solves are not cached: their key would be the whole vector
    key = None
    if personalization is None:
        key = _cache_key("pagerank", bool(prepared["directed"]), float(alpha), int(max_iter), float(eps), str(weight))
        cached = _result_cache_get(prepared, key)
        if cached is not None:
            result, kernel_s = cached
            set_last_kernel_time("pagerank", kernel_s)
            return result
    nodes = prepared["nodes"]
    if len(nodes) == 0:
        set_last_kernel_time("pagerank", 0.0)
        return {}
    pg = prepared_native(G, prepared, weight)
    pvec = _personalization_vector(personalization, prepared)
    out = cpp_gpu_pagerank_dense(pg, alpha, max_iter, eps, weight, personalization=pvec)
    vals = normalize_dense_array(out["values_dense"], len(nodes), allow_leading_sentinel=True,
                                 result_name="PageRank values_dense")
    set_last_kernel_time("pagerank", out["kernel_seconds"])
    result = DenseValueDict(nodes, vals, node_to_idx=prepared.get("node_to_idx"))
    if _PR_PREFER_DICT:
        result = dict(result.items())
    if key is not None:
        _result_cache_put(prepared, key, result, out["kernel_seconds"])
    return result


def pagerank_batch(G, personalizations, alpha=0.85, max_iter=200, eps=1e-6, weight=None):
    """Personalised PageRank for several teleport vectors in one batched solve.

    personalizations: a list of dicts (node -> weight), or a (k, n) array in
    node order.  Returns a list of read-only Mappings.
    """
    prepared = prepare_graph_context(G)
    nodes = prepared["nodes"]
    if len(nodes) == 0:
        return [{} for _ in range(len(personalizations))]
    if len(personalizations) == 0:
        return []
    pg = prepared_native(G, prepared, weight)
    if isinstance(personalizations, np.ndarray):
        T = np.asarray(personalizations, np.float64)
    else:
        T = np.stack([_personalization_vector(p, prepared) for p in personalizations])
    ranks, stats = pg.pagerank_batch(T, alpha=alpha, max_iter=max_iter, tol=eps)
    set_last_kernel_time("pagerank_batch", stats[0]["kernel_seconds"] if stats else 0.0)
    return [DenseValueDict(nodes, ranks[j], node_to_idx=prepared.get("node_to_idx")) for j in range(ranks.shape[0])]
