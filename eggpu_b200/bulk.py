"""``eggpu-csr-v1`` bulk CSR graphs — PageRank on 10^8-edge graphs without
Python adjacency dicts.

Mirrors the reference's bulk path for what PageRank needs:

* ``EGGPUBulkGraph(metadata_path, validate=None)`` and ``read_eggpu_csr``
  follow easygraph/classes/eggpu_bulk_graph.py:191-335,551-562: manifest
  checks (format, int32 dtypes, zero-based contiguous labels, 32-bit limits,
  file sizes, float64 weights, non-empty weight key) in the same order and
  with the same messages, paths resolved against the manifest's folder, the
  EASYGRAPH_GPU_BULK_VALIDATE switch, and the signature built from the
  manifest path and its ``generation``;
* the array checks follow load_csr_files (cpp_easygraph/classes/
  graph_convert.cpp:447-526): exact-size arrays, finite weights, offsets
  starting at 0 and ending at num_entries, and, when validating, monotone
  in-range offsets and endpoints in [0, num_nodes);
* the graph object keeps the reference's read-only API: ``len``, iteration,
  ``nodes``, ``number_of_nodes``, ``number_of_edges`` (from the manifest's
  ``num_edges``), ``has_node``, ``memory_estimate``, ``repr``, no adjacency
  dictionaries, and mutators that raise ``TypeError``.

The manifest is a JSON file::

    {"format": "eggpu-csr-v1", "generation": g, "name": ..., "directed": bool,
     "num_nodes": n, "num_edges": e, "num_entries": m,
     "node_labels": "zero_based_contiguous",
     "offset_dtype": "int32", "index_dtype": "int32",
     "offsets_path": ..., "indices_path": ...,
     ["weights_path": ..., "weight_dtype": "float64", "weight_key": "weight"]}

For an undirected graph the CSR holds both directions of every edge, as the
reference's writer does (tests/test_eggpu_bulk_csr.py:15-61).  A logical
undirected projection named by the manifest serves algorithms other than
PageRank; its path is recorded, and it is not loaded.
"""

from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path

import numpy as np

FORMAT = "eggpu-csr-v1"
_INT32_LIMIT = (1 << 31) - 1


def _check_arrays(V, E, W, weight_key, num_nodes, num_entries, validate):
    """The checks of load_csr_files (graph_convert.cpp:447-526), in its order."""
    if num_nodes < 0 or num_nodes >= _INT32_LIMIT:
        raise ValueError("num_nodes exceeds the signed 32-bit EGGPU CSR limit")
    if num_entries < 0 or num_entries >= _INT32_LIMIT:
        raise ValueError("num_entries exceeds the signed 32-bit EGGPU CSR limit")
    if W is not None:
        if not weight_key:
            raise ValueError("weight_key must be non-empty when weights_path is provided")
        if W.shape[0] != num_entries:
            raise ValueError(f"weights must have num_entries ({num_entries}) values, found {W.shape[0]}")
        if not np.all(np.isfinite(W)):
            raise ValueError("bulk CSR weights must be finite")
    if V.shape[0] == 0 or int(V[0]) != 0 or int(V[-1]) != num_entries:
        raise ValueError("invalid CSR offsets: first offset must be zero and final offset must equal num_entries")
    if validate:
        if np.any(np.diff(V) < 0) or int(V.min()) < 0 or int(V.max()) > num_entries:
            raise ValueError("invalid CSR offsets: offsets must be monotonic and in range")
        if num_entries > 0 and (int(E.min()) < 0 or int(E.max()) >= num_nodes):
            raise ValueError("invalid CSR index: endpoint is outside [0, num_nodes)")


class BulkCSRGraph:
    """Immutable CSR graph with node labels 0..n-1, built from arrays.

    Duck-types the graph API that PageRank uses; :class:`EGGPUBulkGraph`
    builds one from an ``eggpu-csr-v1`` manifest.
    """

    cflag = 0
    _eggpu_bulk_csr = True

    def __init__(self, V, E, W=None, weight_key=None, directed=True, name="", validate=True, num_edges=None,
                 signature=None):
        V = np.ascontiguousarray(V, np.int32)
        E = np.ascontiguousarray(E, np.int32)
        n = int(V.shape[0]) - 1
        m = int(E.shape[0])
        if W is not None:
            W = np.ascontiguousarray(W, np.float64)
        _check_arrays(V, E, W, weight_key, n, m, validate)
        self.V, self.E, self.W = V, E, W
        self.weight_key = weight_key if W is not None else None
        self._directed = bool(directed)
        self.name = name
        self.num_nodes = n
        self.num_entries = m
        self.num_edges = int(num_edges) if num_edges is not None else m
        self.nodes = range(n)
        self.cache = {}
        self.graph = {"name": name, "source": "", "eggpu_bulk_csr": True}
        self.undirected_projection_path = None
        if signature is None:  # arrays without a manifest: identified by their content
            h = hashlib.blake2b(digest_size=16)
            for a in (V, E) + ((W,) if W is not None else ()):
                h.update(memoryview(a).cast("B"))
            signature = (n, m, bool(directed), self.weight_key, h.hexdigest())
        self._eggpu_bulk_signature = signature

    # ---- read-only graph API (eggpu_bulk_graph.py:353-380) ----
    def __len__(self):
        return self.num_nodes

    def __iter__(self):
        return iter(self.nodes)

    def __contains__(self, node):
        return isinstance(node, (int, np.integer)) and 0 <= int(node) < self.num_nodes

    def is_directed(self):
        return self._directed

    def is_multigraph(self):
        return False

    def number_of_nodes(self):
        return self.num_nodes

    def number_of_edges(self, u=None, v=None):
        if u is not None or v is not None:
            raise NotImplementedError("per-pair edge lookup is not available on EGGPUBulkGraph")
        return self.num_edges

    def has_node(self, node):
        return node in self

    def copy(self):
        return self  # immutable

    @property
    def adj(self):
        raise NotImplementedError("EGGPUBulkGraph intentionally does not materialize Python adjacency dictionaries")

    @property
    def pred(self):
        if not self._directed:
            raise AttributeError("undirected EGGPUBulkGraph has no predecessor view")
        raise NotImplementedError("EGGPUBulkGraph intentionally does not materialize Python predecessor dictionaries")

    def _immutable(self, *args, **kwargs):
        raise TypeError("EGGPUBulkGraph is immutable; regenerate its CSR artifact to change it")

    add_node = add_nodes = add_nodes_from = _immutable
    add_edge = add_edges = add_edges_from = _immutable
    remove_node = remove_nodes = remove_edge = remove_edges = _immutable

    def memory_estimate(self):
        """Host bytes of the CSR arrays (eggpu_bulk_graph.py:521-539); no projection is held."""
        weights = self.num_entries * 8 if self.W is not None else 0
        total = (self.num_nodes + 1 + self.num_entries) * 4 + weights
        return {
            "host_offsets_bytes": (self.num_nodes + 1) * 4,
            "host_indices_bytes": self.num_entries * 4,
            "host_weights_bytes": weights,
            "host_total_bytes": total,
            "host_undirected_projection_bytes": 0,
            "host_total_with_projection_bytes": total,
            "implicit_unit_weights": self.W is None,
            "weight_key": self.weight_key,
        }

    def __repr__(self):
        kind = "DiGraph" if self._directed else "Graph"
        return (f"EGGPUBulk{kind}(name={self.name!r}, nodes={self.num_nodes}, edges={self.num_edges}, "
                f"csr_entries={self.num_entries}, undirected_projection=False)")

    # ---- what the PageRank path reads ----
    def has_weight(self, key):
        return self.W is not None and key == self.weight_key

    def csr_arrays(self, weight=None):
        if weight is None:
            return self.V, self.E, None
        if not self.has_weight(weight):
            raise NotImplementedError(
                f"weighted PageRank requires an EGGPU CSR artifact containing the {weight!r} edge attribute")
        return self.V, self.E, self.W


def _resolved_path(metadata_path: Path, value) -> Path:
    """A manifest path: ``~`` expanded, relative paths against the manifest's folder."""
    path = Path(str(value)).expanduser()
    if not path.is_absolute():
        path = metadata_path.parent / path
    return path.resolve()


def _check_size(path: Path, expected: int, what: str):
    found = path.stat().st_size
    if found != expected:
        raise ValueError(f"{what} file size mismatch: expected {expected}, found {found}")


def _validate_default():
    return os.environ.get("EASYGRAPH_GPU_BULK_VALIDATE", "TRUE").strip().upper() in {"1", "TRUE", "ON", "YES"}


class EGGPUBulkGraph(BulkCSRGraph):
    """An ``eggpu-csr-v1`` artifact loaded as an immutable CSR graph.

    Same constructor, manifest checks and messages as the reference's
    EGGPUBulkGraph (easygraph/classes/eggpu_bulk_graph.py:191-335).  The
    arrays are read with numpy instead of the C++ loader, and the optional
    undirected projection is recorded but not loaded (PageRank does not use
    it).
    """

    def __init__(self, metadata_path, validate=None, undirected_projection_path=None):
        metadata_path = Path(metadata_path).expanduser().resolve()
        with metadata_path.open("r", encoding="utf-8") as handle:
            metadata = json.load(handle)
        if metadata.get("format") != FORMAT:
            raise ValueError(f"unsupported EGGPU CSR format {metadata.get('format')!r}; expected {FORMAT!r}")
        if metadata.get("offset_dtype") != "int32" or metadata.get("index_dtype") != "int32":
            raise ValueError("EGGPU bulk CSR requires int32 offsets and int32 indices")
        if metadata.get("node_labels") != "zero_based_contiguous":
            raise ValueError("EGGPU bulk CSR requires zero-based contiguous node labels")
        num_nodes = int(metadata["num_nodes"])
        num_entries = int(metadata["num_entries"])
        if num_nodes < 0 or num_nodes >= _INT32_LIMIT:
            raise ValueError("num_nodes exceeds the signed 32-bit EGGPU CSR limit")
        if num_entries < 0 or num_entries >= _INT32_LIMIT:
            raise ValueError("num_entries exceeds the signed 32-bit EGGPU CSR limit")
        offsets_path = _resolved_path(metadata_path, metadata["offsets_path"])
        indices_path = _resolved_path(metadata_path, metadata["indices_path"])
        weights_value = metadata.get("weights_path")
        weights_path = _resolved_path(metadata_path, weights_value) if weights_value else None
        weight_key = str(metadata.get("weight_key", "weight"))
        _check_size(offsets_path, (num_nodes + 1) * 4, "offset")
        _check_size(indices_path, num_entries * 4, "index")
        if weights_path is not None:
            if metadata.get("weight_dtype") != "float64":
                raise ValueError("EGGPU bulk CSR explicit weights require float64")
            _check_size(weights_path, num_entries * 8, "weight")
            if not weight_key:
                raise ValueError("weight_key must be non-empty")
        if validate is None:
            validate = _validate_default()
        if undirected_projection_path is None:
            undirected_projection_path = metadata.get("undirected_projection_manifest")
        projection = (_resolved_path(metadata_path, undirected_projection_path)
                      if undirected_projection_path is not None else None)

        V = np.fromfile(offsets_path, dtype=np.int32)
        E = np.fromfile(indices_path, dtype=np.int32)
        W = np.fromfile(weights_path, dtype=np.float64) if weights_path is not None else None
        name = str(metadata.get("name", metadata_path.stem))
        directed = bool(metadata["directed"])
        # path + generation, as the reference keys its caches: an artifact is
        # immutable and a rewrite bumps its generation
        signature = (str(metadata_path), int(metadata.get("generation", 0)), num_nodes, num_entries, directed,
                     str(projection) if projection is not None else None)
        super().__init__(V, E, W, weight_key=weight_key if W is not None else None, directed=directed, name=name,
                         validate=bool(validate), num_edges=int(metadata.get("num_edges", num_entries)),
                         signature=signature)
        self.metadata_path = metadata_path
        self.metadata = metadata
        self.offsets_path = offsets_path
        self.indices_path = indices_path
        self.weights_path = weights_path
        self.undirected_projection_path = projection
        self.graph = {"name": name, "source": metadata.get("source", ""), "eggpu_bulk_csr": True}


def read_eggpu_csr(metadata_path, validate=None, undirected_projection_path=None):
    """Loads an ``eggpu-csr-v1`` manifest (eggpu_bulk_graph.py:551-562).

    ``validate`` defaults to EASYGRAPH_GPU_BULK_VALIDATE (on for 1/TRUE/ON/YES,
    the default TRUE).
    """
    return EGGPUBulkGraph(metadata_path, validate=validate, undirected_projection_path=undirected_projection_path)


def write_eggpu_csr(directory, name, V, E, W=None, directed=True, weight_key="weight", num_edges=None,
                    generation=1):
    """Writes an ``eggpu-csr-v1`` artifact (offsets, indices, optional weights, manifest).

    ``num_edges`` defaults to the entry count of a directed graph and to half
    of it for an undirected one, whose CSR stores both directions.
    """
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    V = np.ascontiguousarray(V, np.int32)
    E = np.ascontiguousarray(E, np.int32)
    V.tofile(d / f"{name}.offsets.i32")
    E.tofile(d / f"{name}.indices.i32")
    m = int(E.shape[0])
    meta = {
        "format": FORMAT, "generation": int(generation), "name": name, "directed": bool(directed),
        "num_nodes": int(V.shape[0]) - 1, "num_edges": int(num_edges) if num_edges is not None else (m if directed else m // 2),
        "num_entries": m, "node_labels": "zero_based_contiguous", "offset_dtype": "int32", "index_dtype": "int32",
        "offsets_path": f"{name}.offsets.i32", "indices_path": f"{name}.indices.i32",
    }
    if W is not None:
        np.ascontiguousarray(W, np.float64).tofile(d / f"{name}.weights.f64")
        meta.update(weights_path=f"{name}.weights.f64", weight_dtype="float64", weight_key=weight_key)
    path = d / f"{name}.json"
    path.write_text(json.dumps(meta), encoding="utf-8")
    return path


__all__ = ["BulkCSRGraph", "EGGPUBulkGraph", "read_eggpu_csr", "write_eggpu_csr"]
