"""``eggpu-csr-v1`` bulk CSR graphs — PageRank on 10^8-edge graphs without
Python adjacency dicts.

Mirrors the reference's bulk path for what PageRank needs:
easygraph/classes/eggpu_bulk_graph.py:191-335 (``EGGPUBulkGraph.__init__``:
manifest validation, node labels 0..n-1) and cpp_easygraph/classes/
graph_convert.cpp:447-526 (``load_csr_files``: exact-size int32 offsets /
indices and optional float64 weights, finite weights, offsets starting at 0
and ending at num_entries, optional full validation of monotone offsets and
in-range indices).  The manifest is a JSON file::

    {"format": "eggpu-csr-v1", "directed": bool, "num_nodes": n,
     "num_entries": m, "offsets_path": ..., "indices_path": ...,
     "offset_dtype": "int32", "index_dtype": "int32",
     ["weights_path": ..., "weight_dtype": "float64", "weight_key": "weight"]}

For an undirected graph the CSR holds both directions of every edge, as the
reference's writer does (tests/test_eggpu_bulk_csr.py:15-61).
"""

from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

import numpy as np

FORMAT = "eggpu-csr-v1"


class BulkCSRGraph:
    """Immutable CSR graph with node labels 0..n-1 (duck-types the graph API PageRank uses)."""

    _eggpu_bulk_csr = True

    def __init__(self, V, E, W=None, weight_key=None, directed=True, name="", validate=True):
        V = np.ascontiguousarray(V, np.int32)
        E = np.ascontiguousarray(E, np.int32)
        n = int(V.shape[0]) - 1
        m = int(E.shape[0])
        if n < 0 or n >= 2**31 - 1 or m >= 2**31 - 1:
            raise ValueError("CSR exceeds the signed 32-bit limits")
        if V.shape[0] == 0 or int(V[0]) != 0 or int(V[-1]) != m:
            raise ValueError("invalid CSR offsets: first offset must be zero and final offset must equal num_entries")
        if W is not None:
            W = np.ascontiguousarray(W, np.float64)
            if W.shape[0] != m:
                raise ValueError("weights must have num_entries values")
            if not np.all(np.isfinite(W)):
                raise ValueError("bulk CSR weights must be finite")
            if not weight_key:
                raise ValueError("weight_key must be non-empty when weights are provided")
        if validate:
            if n > 0 and np.any(np.diff(V) < 0):
                raise ValueError("invalid CSR offsets: offsets must be monotonic and in range")
            if m > 0 and (int(E.min()) < 0 or int(E.max()) >= n):
                raise ValueError("invalid CSR index: endpoint is outside [0, num_nodes)")
        self.V, self.E, self.W = V, E, W
        self.weight_key = weight_key
        self._directed = bool(directed)
        self.name = name
        self.num_nodes = n
        self.num_entries = m
        self.cache = {}
        h = hashlib.blake2b(digest_size=16)
        for a in (V, E) + ((W,) if W is not None else ()):
            h.update(memoryview(a).cast("B"))
        self._eggpu_bulk_signature = (n, m, bool(directed), weight_key, h.hexdigest())

    # graph API used by pagerank
    def __len__(self):
        return self.num_nodes

    @property
    def nodes(self):
        return range(self.num_nodes)

    def is_directed(self):
        return self._directed

    def is_multigraph(self):
        return False

    def has_weight(self, key):
        return self.W is not None and key == self.weight_key

    def csr_arrays(self, weight=None):
        if weight is None:
            return self.V, self.E, None
        if not self.has_weight(weight):
            raise NotImplementedError(
                f"weighted PageRank requires an EGGPU CSR artifact containing the {weight!r} edge attribute")
        return self.V, self.E, self.W


def _read_exact(path, dtype, count):
    arr = np.fromfile(path, dtype=dtype)
    if arr.shape[0] != count:
        raise ValueError(f"{path}: expected {count} values of {np.dtype(dtype).name}, found {arr.shape[0]}")
    return arr


def read_eggpu_csr(manifest_path, validate=None):
    """Loads an ``eggpu-csr-v1`` manifest into a :class:`BulkCSRGraph`.

    ``validate`` defaults to EASYGRAPH_GPU_BULK_VALIDATE (on unless set to 0/false).
    """
    manifest_path = Path(manifest_path)
    meta = json.loads(manifest_path.read_text(encoding="utf-8"))
    if meta.get("format") != FORMAT:
        raise ValueError(f"unsupported CSR artifact format {meta.get('format')!r}; expected {FORMAT!r}")
    for key, want in (("offset_dtype", "int32"), ("index_dtype", "int32")):
        if meta.get(key, want) != want:
            raise ValueError(f"{key} must be {want}")
    if "weights_path" in meta and meta.get("weight_dtype", "float64") != "float64":
        raise ValueError("weight_dtype must be float64")
    if validate is None:
        validate = os.environ.get("EASYGRAPH_GPU_BULK_VALIDATE", "1").strip().upper() not in {"0", "FALSE", "OFF", "NO"}
    n = int(meta["num_nodes"])
    m = int(meta["num_entries"])
    base = manifest_path.parent
    V = _read_exact(base / meta["offsets_path"], np.int32, n + 1)
    E = _read_exact(base / meta["indices_path"], np.int32, m)
    W = None
    key = None
    if "weights_path" in meta:
        W = _read_exact(base / meta["weights_path"], np.float64, m)
        key = meta.get("weight_key", "weight")
    return BulkCSRGraph(V, E, W, weight_key=key, directed=bool(meta.get("directed", True)),
                        name=str(meta.get("name", "")), validate=bool(validate))


def write_eggpu_csr(directory, name, V, E, W=None, directed=True, weight_key="weight"):
    """Writes an ``eggpu-csr-v1`` artifact (offsets, indices, optional weights, manifest)."""
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    V = np.ascontiguousarray(V, np.int32)
    E = np.ascontiguousarray(E, np.int32)
    V.tofile(d / f"{name}.offsets.i32")
    E.tofile(d / f"{name}.indices.i32")
    meta = {
        "format": FORMAT, "generation": 1, "name": name, "directed": bool(directed),
        "num_nodes": int(V.shape[0]) - 1, "num_entries": int(E.shape[0]),
        "node_labels": "zero_based_contiguous", "offset_dtype": "int32", "index_dtype": "int32",
        "offsets_path": f"{name}.offsets.i32", "indices_path": f"{name}.indices.i32",
    }
    if W is not None:
        np.ascontiguousarray(W, np.float64).tofile(d / f"{name}.weights.f64")
        meta.update(weights_path=f"{name}.weights.f64", weight_dtype="float64", weight_key=weight_key)
    path = d / f"{name}.json"
    path.write_text(json.dumps(meta), encoding="utf-8")
    return path
