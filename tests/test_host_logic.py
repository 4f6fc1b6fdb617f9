"""Host-side contracts of the PageRank path that need no GPU: the dense
read-only result mapping, the dense-shape contract, env defaults, graph ->
CSR conversion, the prepared-graph context and its invalidation, bulk CSR
manifests, and the easygraph install hook (exercised with a fake native
backend, like the reference's test_eggpu_cache_contracts.py:190-221)."""

import json
import types

import numpy as np
import pytest

from eggpu_b200 import backend, bulk
from eggpu_b200 import api as prmod
from oracle import oracle
from tests.graphs import DiGraph, Graph, MultiDiGraph, golden_small_cases


def test_dense_value_dict_is_a_read_only_mapping():
    r = backend.DenseValueDict(["a", "b", "c"], np.array([0.2, 0.3, 0.5]))
    assert dict(r) == {"a": 0.2, "b": 0.3, "c": 0.5}
    assert r == {"a": 0.2, "b": 0.3, "c": 0.5}
    assert list(r) == ["a", "b", "c"] and len(r) == 3 and "b" in r and "z" not in r
    assert r.get("z", 7) == 7
    with pytest.raises(KeyError):
        r["z"]
    with pytest.raises(TypeError):
        r["a"] = 1.0
    with pytest.raises(ValueError):
        r.to_numpy()[0] = 1.0
    assert json.dumps(dict(r))
    rng = backend.DenseValueDict(range(3), np.array([1.0, 2.0, 3.0]))
    assert rng[2] == 3.0 and 3 not in rng and True not in rng


def test_dense_result_wraps_the_result_vector_without_a_copy():
    # the ranks land in one host vector and the Mapping is a read-only view of it
    vec = np.linspace(0.0, 1.0, 5)
    r = backend.DenseValueDict(range(5), vec)
    assert np.shares_memory(r.to_numpy(), vec) and not r.to_numpy().flags.writeable
    with_sentinel = np.concatenate([[-1.0], vec])
    r2 = backend.DenseValueDict(range(5), backend.normalize_dense_array(with_sentinel, 5, allow_leading_sentinel=True))
    assert np.shares_memory(r2.to_numpy(), with_sentinel) and r2[4] == 1.0


def test_dense_shape_contract():
    # gpu_eggpu_backend.py:1092-1126 / test_eggpu_cache_contracts.py:199-221
    with pytest.raises(backend.DenseResultShapeError, match=r"expected \(3,\) or \(4,\)"):
        backend.normalize_dense_array(np.zeros(5), 3, allow_leading_sentinel=True, result_name="PageRank values_dense")
    assert backend.normalize_dense_array(np.arange(4.0), 3, allow_leading_sentinel=True).tolist() == [1.0, 2.0, 3.0]


def test_env_defaults_and_clamping(monkeypatch):
    assert prmod._effective_limits(None, None) == (200, 1e-6)
    monkeypatch.setenv("EASYGRAPH_CPU_PR_MAX_ITER", "0")
    monkeypatch.setenv("EASYGRAPH_CPU_PR_TOL", "-1")
    assert prmod._effective_limits(None, None) == (1, 0.0)
    assert prmod._effective_limits(-5, -2.0) == (1, 0.0)


def test_runtime_switches(monkeypatch):
    # gpu_runtime.py:10-15 / test_eggpu_runtime.py:37-56
    for val, want in (("TRUE", True), ("1", True), ("on", True), ("yes", True), ("false", False), ("", False)):
        monkeypatch.setenv("EASYGRAPH_ENABLE_GPU", val)
        assert prmod.gpu_runtime_enabled() is want


def test_multigraph_and_empty_graph():
    G = MultiDiGraph()
    G.add_edge(0, 1)
    with pytest.raises(prmod.EasyGraphNotImplemented):
        prmod.pagerank(G)
    assert prmod.pagerank(DiGraph()) == {}
    assert prmod.pagerank(Graph()) == {}


@pytest.mark.parametrize("case", golden_small_cases(), ids=lambda c: c[0])
def test_graph_csr_matches_restated_gen_csr(case):
    name, G, kw, _ = case
    prepared = backend.prepare_graph_context(G)
    weight = kw.get("weight")
    V, E, W = backend.graph_csr(G, prepared, weight)
    V2, E2, W2 = oracle.graph_to_csr(list(G.nodes), G._adj, G.is_directed(), weight)
    assert np.array_equal(V, V2) and np.array_equal(E, E2)
    if weight is not None:
        assert np.array_equal(W, W2)


@pytest.mark.skipif(backend._graph_walk is None, reason="native graph walk not built")
@pytest.mark.parametrize("directed", [True, False])
@pytest.mark.parametrize("weighted", [False, True])
def test_native_graph_walk_equals_the_python_walk(directed, weighted):
    rng = np.random.default_rng(7 + 2 * directed + weighted)
    n = 1500
    nodes = [("v", int(i)) for i in rng.permutation(n)]
    adj = {u: {} for u in nodes}
    for _ in range(12000):
        a, b = rng.integers(0, n, 2)
        r = rng.random()
        # odd attributes: missing, None, numeric strings, junk strings, empty dicts
        attr = ({} if r > 0.95 else {"w": None} if r > 0.9 else {"w": str(r)} if r < 0.1 else
                {"w": "x"} if r < 0.12 else {"w": r, "other": 1})
        adj[nodes[a]][nodes[b]] = attr
        if not directed:
            adj[nodes[b]][nodes[a]] = attr
    G = types.SimpleNamespace(_adj=adj)
    prepared = {"node_to_idx": {u: i for i, u in enumerate(nodes)}, "nodes": nodes, "directed": directed}
    w = "w" if weighted else None
    V, E, W = backend.graph_csr(G, prepared, w)
    V2, E2, W2 = backend._graph_csr_py(G, prepared, w)
    assert V.dtype == V2.dtype == np.int32 and E.dtype == E2.dtype == np.int32
    assert np.array_equal(V, V2) and np.array_equal(E, E2)
    assert (W is None and W2 is None) or np.array_equal(W, W2)
    # a neighbour missing from the node index fails the same way
    adj[nodes[0]][("v", -1)] = {}
    with pytest.raises(KeyError):
        backend.graph_csr(G, prepared, w)


@pytest.mark.skipif(backend._graph_walk is None, reason="native graph walk not built")
def test_native_undirected_walk_on_an_asymmetric_adjacency():
    # each unordered pair once per direction, its weight from where it is first met,
    # also when the two directions disagree or only one of them is present
    rng = np.random.default_rng(11)
    n = 800
    adj = {i: {} for i in range(n)}
    for _ in range(6000):
        a, b = (int(x) for x in rng.integers(0, n, 2))
        adj[a][b] = {"w": float(rng.random())}
        r = rng.random()
        if r < 0.6:
            adj[b][a] = {"w": float(rng.random())}  # the other direction, another weight
    G = types.SimpleNamespace(_adj=adj)
    prepared = {"node_to_idx": {i: i for i in range(n)}, "nodes": list(range(n)), "directed": False}
    for w in (None, "w"):
        a, b = backend.graph_csr(G, prepared, w), backend._graph_csr_py(G, prepared, w)
        assert all((x is None and y is None) or np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.skipif(backend._graph_walk is None, reason="native graph walk not built")
def test_native_graph_stamp_equals_the_python_stamp():
    rng = np.random.default_rng(5)
    labels = [("v", i) for i in range(500)] + list(range(-3, 60)) + [f"s{i}" for i in range(40)] + [2.5, None]
    adj = {u: {} for u in labels}
    for _ in range(4000):
        a, b = rng.integers(0, len(labels), 2)
        adj[labels[a]][labels[b]] = {}
    for directed in (True, False):
        G = types.SimpleNamespace(_adj=adj, is_directed=lambda d=directed: d)
        assert backend.graph_stamp(G) == backend._graph_stamp_py(G, adj)
    # a row that is not a plain dict: the Python stamp answers
    odd = dict(adj)
    odd[labels[0]] = types.MappingProxyType(dict(adj[labels[0]]))
    G = types.SimpleNamespace(_adj=odd, is_directed=lambda: True)
    assert backend._graph_walk.stamp(odd) is None
    assert backend.graph_stamp(G) == backend._graph_stamp_py(G, odd)


def test_personalization_keys_of_a_bulk_graph():
    p = {"nodes": range(4), "node_to_idx": None}
    vec = backend._personalization_vector({0: 1.0, np.int64(3): 3.0}, p)
    assert vec.tolist() == [1.0, 0.0, 0.0, 3.0]  # the engine normalises it
    for bad in ("a", 4, -1, True, 1.5):
        with pytest.raises(KeyError, match="is not in the graph"):
            backend._personalization_vector({bad: 1.0}, p)


def test_batch_of_no_teleport_vectors_is_an_empty_list(monkeypatch):
    monkeypatch.setattr(backend, "prepared_native", lambda *a, **k: pytest.fail("no solve for an empty batch"))
    G = DiGraph()
    G.add_edge(0, 1)
    assert backend.pagerank_batch(G, []) == []
    assert backend.pagerank_batch(G, np.zeros((0, 2))) == []


def test_runtime_switches_as_the_reference_reads_them(monkeypatch):
    # easygraph/tests/test_eggpu_runtime.py:43-56
    for name in ("EASYGRAPH_ENABLE_GPU", "EASYGRAPH_GPU_STRICT_ERRORS"):
        monkeypatch.delenv(name, raising=False)
    assert not prmod.gpu_runtime_enabled() and not prmod.gpu_strict_errors()
    for val, on in (("TRUE", True), ("1", True), (" yes ", True), ("on", True), ("FALSE", False), ("2", False)):
        monkeypatch.setenv("EASYGRAPH_ENABLE_GPU", val)
        assert prmod.gpu_runtime_enabled() is on
    monkeypatch.delenv("EASYGRAPH_ENABLE_GPU")
    monkeypatch.setenv("EASYGRAPH_GPU_STRICT_ERRORS", "TRUE")
    assert prmod.gpu_strict_errors() and not prmod.gpu_runtime_enabled()  # independent switches


def test_prepared_context_reuse_and_mutation_invalidation():
    G = DiGraph()
    G.add_edge(0, 1, weight=8.0)
    G.add_edge(1, 0, weight=1.0)
    p1 = backend.prepare_graph_context(G)
    assert backend.prepare_graph_context(G) is p1
    G[0][1]["weight"] = 0.25  # graph.py:17-40: attribute mutation bumps the generation
    p2 = backend.prepare_graph_context(G)
    assert p2 is not p1 and p2["ctx_id"] != p1["ctx_id"]
    V, E, W = backend.graph_csr(G, p2, "weight")
    assert W.tolist() == [0.25, 1.0]


def test_prepared_context_full_stamp_check(monkeypatch):
    G = DiGraph()
    G.add_edges_from([(0, 1), (1, 2)])
    p = backend.prepare_graph_context(G)
    monkeypatch.setattr(backend, "_GRAPH_CTX_VALIDATE_EVERY", 1)
    # change the adjacency behind the generation counter: the stamp catches it
    dict.__setitem__(G._adj[2], 0, {})
    assert backend.prepare_graph_context(G) is not p


def test_fake_native_backend_wrong_length_raises(monkeypatch):
    G = DiGraph()
    G.add_edges_from([(0, 1), (1, 2), (2, 0)])
    monkeypatch.setattr(backend, "prepared_native", lambda G, p, w=None: object())
    monkeypatch.setattr(backend, "cpp_gpu_pagerank_dense",
                        lambda *a, **k: {"values_dense": np.zeros(5), "kernel_seconds": 0.0})
    with pytest.raises(backend.DenseResultShapeError, match=r"expected \(3,\) or \(4,\)"):
        backend.pagerank(G)
    monkeypatch.setattr(backend, "cpp_gpu_pagerank_dense",
                        lambda *a, **k: {"values_dense": np.array([9.0, 0.2, 0.3, 0.5]), "kernel_seconds": 0.5})
    res = backend.pagerank(G)
    assert dict(res) == {0: 0.2, 1: 0.3, 2: 0.5}
    assert backend.get_last_kernel_time("pagerank") == 0.5


def test_personalization_vector_validation():
    G = DiGraph()
    G.add_edges_from([("a", "b"), ("b", "c")])
    p = backend.prepare_graph_context(G)
    assert backend._personalization_vector({"b": 2.0}, p).tolist() == [0.0, 2.0, 0.0]
    with pytest.raises(KeyError):
        backend._personalization_vector({"zz": 1.0}, p)
    with pytest.raises(ValueError):
        backend._personalization_vector({"a": 0.0}, p)
    with pytest.raises(ValueError):
        backend._personalization_vector({"a": -1.0, "b": 2.0}, p)


def test_bulk_manifest_roundtrip_and_validation(tmp_path):
    V = np.array([0, 2, 3, 3], np.int32)
    E = np.array([1, 2, 0], np.int32)
    W = np.array([1.0, 2.0, 3.0])
    path = bulk.write_eggpu_csr(tmp_path, "tiny", V, E, W, directed=True)
    G = bulk.read_eggpu_csr(path)
    assert len(G) == 3 and list(G.nodes) == [0, 1, 2] and G.has_weight("weight")
    assert np.array_equal(G.csr_arrays("weight")[2], W)
    with pytest.raises(NotImplementedError, match="weighted PageRank requires an EGGPU CSR artifact"):
        G.csr_arrays("other")
    meta = json.loads(path.read_text())
    meta["format"] = "bogus"
    bad = tmp_path / "bad.json"
    bad.write_text(json.dumps(meta))
    with pytest.raises(ValueError, match="unsupported EGGPU CSR format"):
        bulk.read_eggpu_csr(bad)
    with pytest.raises(ValueError, match="endpoint is outside"):
        bulk.BulkCSRGraph(V, np.array([1, 5, 0], np.int32))
    with pytest.raises(ValueError, match="final offset"):
        bulk.BulkCSRGraph(np.array([0, 1], np.int32), np.array([0, 0], np.int32))
    with pytest.raises(ValueError, match="finite"):
        bulk.BulkCSRGraph(V, E, np.array([1.0, np.nan, 1.0]), weight_key="weight")
    p = backend.prepare_graph_context(G)
    assert p["bulk_csr"] and p["nodes"] == range(3)
    assert backend.prepare_graph_context(G) is p


# the six-node graph of the reference's bulk tests (tests/test_eggpu_bulk_csr.py:12-61)
_BULK_EDGES = [(0, 1), (1, 2), (2, 0), (2, 3), (3, 4), (4, 5), (5, 3)]


def _write_reference_style_bulk(tmp_path, directed=False, weighted=False):
    """The artifact the reference's test writer produces, written here with the array module as it does."""
    from array import array

    rows = [[] for _ in range(6)]
    for u, v in _BULK_EDGES:
        rows[u].append(v)
        if not directed:
            rows[v].append(u)
    offsets, indices = [0], []
    for row in rows:
        indices.extend(row)
        offsets.append(len(indices))
    with (tmp_path / "tiny.offsets.i32").open("wb") as f:
        array("i", offsets).tofile(f)
    with (tmp_path / "tiny.indices.i32").open("wb") as f:
        array("i", indices).tofile(f)
    meta = {"format": "eggpu-csr-v1", "generation": 1, "name": "tiny", "directed": directed, "num_nodes": 6,
            "num_edges": len(_BULK_EDGES), "num_entries": len(indices), "node_labels": "zero_based_contiguous",
            "offset_dtype": "int32", "index_dtype": "int32", "offsets_path": "tiny.offsets.i32",
            "indices_path": "tiny.indices.i32"}
    if weighted:
        weights = [1.0 + ((src * dst) % 6) for src, row in enumerate(rows) for dst in row]
        with (tmp_path / "tiny.weights.f64").open("wb") as f:
            array("d", weights).tofile(f)
        meta.update(weights_path="tiny.weights.f64", weight_dtype="float64", weight_key="weight")
    path = tmp_path / "tiny.json"
    path.write_text(json.dumps(meta), encoding="utf-8")
    return path, meta


def test_bulk_graph_contract_as_the_reference_pins_it(tmp_path):
    # tests/test_eggpu_bulk_csr.py:188-195 and :256-262
    path, _ = _write_reference_style_bulk(tmp_path)
    G = bulk.read_eggpu_csr(path)
    assert isinstance(G, bulk.EGGPUBulkGraph)
    assert len(G) == 6 and G.number_of_edges() == 7 and list(G.nodes) == list(range(6))
    assert G.memory_estimate()["host_total_bytes"] == (7 + 14) * 4
    assert "materialize" not in repr(G) and repr(G).startswith("EGGPUBulkGraph(name='tiny'")
    assert 5 in G and 6 not in G and "a" not in G and G.has_node(0) and list(G) == list(range(6))
    assert G.copy() is G and not G.is_directed() and G.weight_key is None
    with pytest.raises(TypeError, match="immutable"):
        G.add_edge(0, 5)
    with pytest.raises(NotImplementedError, match="does not materialize"):
        G.adj
    with pytest.raises(NotImplementedError, match="per-pair"):
        G.number_of_edges(0, 1)

    wdir = tmp_path / "w"
    wdir.mkdir()
    Gw = bulk.read_eggpu_csr(_write_reference_style_bulk(wdir, weighted=True)[0])
    est = Gw.memory_estimate()
    assert est["implicit_unit_weights"] is False and est["host_weights_bytes"] == Gw.num_entries * 8
    assert est["host_total_bytes"] == (7 + 14) * 4 + 14 * 8 and Gw.weight_key == "weight"
    assert Gw.has_weight("weight") and not Gw.has_weight("cost")
    # the signature follows the manifest path and generation, not the array bytes
    assert Gw._eggpu_bulk_signature[:2] == (str(Gw.metadata_path), 1)


def test_bulk_graph_records_an_undirected_projection_without_loading_it(tmp_path):
    path, meta = _write_reference_style_bulk(tmp_path, directed=True)
    meta["undirected_projection_manifest"] = "tiny.projection.json"  # serves other algorithms; need not exist
    path.write_text(json.dumps(meta), encoding="utf-8")
    G = bulk.read_eggpu_csr(path)
    assert G.undirected_projection_path == (tmp_path / "tiny.projection.json").resolve()
    assert G._eggpu_bulk_signature[-1] == str(G.undirected_projection_path)
    other = bulk.read_eggpu_csr(path, undirected_projection_path=str(tmp_path / "elsewhere.json"))
    assert other._eggpu_bulk_signature != G._eggpu_bulk_signature
    assert G.memory_estimate()["host_undirected_projection_bytes"] == 0


def test_bulk_manifest_checks_match_the_reference_messages(tmp_path, monkeypatch):
    # easygraph/classes/eggpu_bulk_graph.py:200-247 and graph_convert.cpp:447-516
    path, meta = _write_reference_style_bulk(tmp_path, weighted=True)

    def load_with(**changes):
        m = dict(meta)
        for k, v in changes.items():
            if v is None:
                m.pop(k, None)
            else:
                m[k] = v
        p = tmp_path / "variant.json"
        p.write_text(json.dumps(m), encoding="utf-8")
        return bulk.read_eggpu_csr(p)

    with pytest.raises(ValueError, match="requires int32 offsets and int32 indices"):
        load_with(offset_dtype=None)
    with pytest.raises(ValueError, match="requires int32 offsets and int32 indices"):
        load_with(index_dtype="int64")
    with pytest.raises(ValueError, match="zero-based contiguous node labels"):
        load_with(node_labels=None)
    with pytest.raises(ValueError, match="num_nodes exceeds the signed 32-bit EGGPU CSR limit"):
        load_with(num_nodes=2**31 - 1)
    with pytest.raises(ValueError, match="num_entries exceeds the signed 32-bit EGGPU CSR limit"):
        load_with(num_entries=-1)
    with pytest.raises(ValueError, match="offset file size mismatch: expected 32, found 28"):
        load_with(num_nodes=7)
    with pytest.raises(ValueError, match="index file size mismatch: expected 60, found 56"):
        load_with(num_entries=15)
    with pytest.raises(ValueError, match="explicit weights require float64"):
        load_with(weight_dtype=None)
    with pytest.raises(ValueError, match="weight_key must be non-empty"):
        load_with(weight_key="")
    # contents: offsets that do not end at num_entries, out-of-range endpoints, non-finite weights
    idx = np.fromfile(tmp_path / "tiny.indices.i32", dtype=np.int32)
    bad = idx.copy()
    bad[3] = 6
    bad.tofile(tmp_path / "bad.indices.i32")
    with pytest.raises(ValueError, match=r"endpoint is outside \[0, num_nodes\)"):
        load_with(indices_path="bad.indices.i32")
    # EASYGRAPH_GPU_BULK_VALIDATE: only 1/TRUE/ON/YES (default TRUE) validate the contents
    monkeypatch.setenv("EASYGRAPH_GPU_BULK_VALIDATE", "FALSE")
    assert len(load_with(indices_path="bad.indices.i32")) == 6
    monkeypatch.setenv("EASYGRAPH_GPU_BULK_VALIDATE", "maybe")
    assert len(load_with(indices_path="bad.indices.i32")) == 6
    monkeypatch.delenv("EASYGRAPH_GPU_BULK_VALIDATE")
    with pytest.raises(ValueError, match="endpoint is outside"):
        load_with(indices_path="bad.indices.i32")
    w = np.fromfile(tmp_path / "tiny.weights.f64", dtype=np.float64)
    w[0] = np.inf
    w.tofile(tmp_path / "bad.weights.f64")
    with pytest.raises(ValueError, match="bulk CSR weights must be finite"):
        load_with(weights_path="bad.weights.f64")
    off = np.fromfile(tmp_path / "tiny.offsets.i32", dtype=np.int32)
    off[-1] = 13
    off.tofile(tmp_path / "bad.offsets.i32")
    with pytest.raises(ValueError, match="final offset must equal num_entries"):
        load_with(offsets_path="bad.offsets.i32")
    # absolute paths are taken as they are
    assert len(load_with(offsets_path=str(tmp_path / "tiny.offsets.i32"))) == 6


class _ReferenceStyleBulk:
    """The attributes the reference's EGGPUBulkGraph exposes after loading
    (easygraph/classes/eggpu_bulk_graph.py:296-333): artifact paths and
    sizes, no arrays (those live in its C++ graph)."""

    _eggpu_bulk_csr = True

    def __init__(self, path, meta):
        base = path.parent
        self.num_nodes, self.num_entries = meta["num_nodes"], meta["num_entries"]
        self.offsets_path = base / meta["offsets_path"]
        self.indices_path = base / meta["indices_path"]
        self.weights_path = base / meta["weights_path"] if "weights_path" in meta else None
        self.weight_key = meta.get("weight_key", "weight") if self.weights_path else None
        self._directed = meta["directed"]
        self._eggpu_bulk_signature = (str(path), meta["generation"], self.num_nodes, self.num_entries,
                                      self._directed, None, 0)
        self.nodes = range(self.num_nodes)
        self.cache = {}

    def is_directed(self):
        return self._directed

    def is_multigraph(self):
        return False

    def __len__(self):
        return self.num_nodes


def test_backend_reads_the_reference_bulk_graph_from_its_artifact(tmp_path):
    path, meta = _write_reference_style_bulk(tmp_path, directed=True, weighted=True)
    ours = bulk.read_eggpu_csr(path)
    theirs = _ReferenceStyleBulk(path, meta)
    p = backend.prepare_graph_context(theirs)
    assert p["bulk_csr"] and p["nodes"] == range(6) and backend.prepare_graph_context(theirs) is p
    for weight in (None, "weight"):
        a, b = backend.graph_csr(theirs, p, weight), ours.csr_arrays(weight)
        assert all((x is None and y is None) or np.array_equal(x, y) for x, y in zip(a, b))
    assert backend.bulk_weight_available(theirs, "weight") and not backend.bulk_weight_available(theirs, "cost")
    assert backend.bulk_weight_available(ours, "weight") and not backend.bulk_weight_available(ours, "cost")
    with pytest.raises(NotImplementedError, match="weighted PageRank requires an EGGPU CSR artifact"):
        backend.graph_csr(theirs, p, "cost")
    udir = tmp_path / "u"
    udir.mkdir()
    upath, umeta = _write_reference_style_bulk(udir)
    with pytest.raises(NotImplementedError, match="weighted PageRank requires an EGGPU CSR artifact"):
        backend.pagerank(_ReferenceStyleBulk(upath, umeta), weight="weight")


def test_opt_in_result_cache_owns_independent_snapshots(monkeypatch):
    # test_eggpu_cache_contracts.py:284-307, on this backend's cache
    monkeypatch.setattr(backend, "_RESULT_CACHE_ENABLED", True)
    monkeypatch.setattr(backend, "_RESULT_CACHE_RETURN_COPY", True)
    prepared = {"nodes": [0], "result_cache": {}, "result_cache_order": []}
    original = {0: [1]}
    key = ("test",)
    backend._result_cache_put(prepared, key, original, 0.25)
    original[0].append(2)
    first, kernel = backend._result_cache_get(prepared, key)
    first[0].append(3)
    second, _ = backend._result_cache_get(prepared, key)
    assert kernel == 0.25 and first == {0: [1, 3]} and second == {0: [1]}
    # a dense result comes back over an array of its own
    dense = backend.DenseValueDict(range(3), np.array([0.2, 0.3, 0.5]))
    backend._result_cache_put(prepared, ("dense",), dense, 0.5)
    a, _ = backend._result_cache_get(prepared, ("dense",))
    b, _ = backend._result_cache_get(prepared, ("dense",))
    assert a == dense and b == dense and a is not b and a.to_numpy() is not b.to_numpy()


def test_result_cache_is_opt_in_bounded_and_keyed_like_the_reference(monkeypatch):
    prepared = {"nodes": list(range(4))}
    backend._result_cache_put(prepared, ("k",), {0: 1}, 0.1)
    assert backend._result_cache_get(prepared, ("k",)) is None  # off by default
    monkeypatch.setattr(backend, "_RESULT_CACHE_ENABLED", True)
    monkeypatch.setattr(backend, "_RESULT_CACHE_MAX_ITEMS", 2)
    for i in range(3):
        backend._result_cache_put(prepared, ("k", i), {0: i}, float(i))
    assert backend._result_cache_get(prepared, ("k", 0)) is None
    assert backend._result_cache_get(prepared, ("k", 2)) == ({0: 2}, 2.0)
    monkeypatch.setattr(backend, "_RESULT_CACHE_MAX_NODES", 3)
    backend._result_cache_put(prepared, ("big",), {0: 1}, 0.1)
    assert backend._result_cache_get(prepared, ("big",)) is None
    # floats rounded to 12 digits, other parts kept (gpu_eggpu_backend.py:1723-1730)
    assert backend._cache_key("pagerank", True, 0.85 + 1e-15, 100, 1e-6, "None") == \
        ("pagerank", True, 0.85, 100, 1e-6, "None")


def test_pagerank_result_cache_hits_skip_the_solve(monkeypatch):
    calls = []

    def fake_dense(pg, alpha, max_iter, eps, weight=None, personalization=None):
        calls.append((alpha, personalization is not None))
        return {"values_dense": np.full(3, 1.0 / 3.0), "kernel_seconds": 0.125}

    monkeypatch.setattr(backend, "prepared_native", lambda G, prepared, weight=None: object())
    monkeypatch.setattr(backend, "cpp_gpu_pagerank_dense", fake_dense)
    monkeypatch.setattr(backend, "_RESULT_CACHE_ENABLED", True)
    G = DiGraph()
    G.add_edges_from([(0, 1), (1, 2), (2, 0)])
    r1 = backend.pagerank(G, alpha=0.85, max_iter=100, eps=1e-6)
    r2 = backend.pagerank(G, alpha=0.85, max_iter=100, eps=1e-6)
    assert len(calls) == 1 and r1 == r2 and r1 is not r2
    assert backend.get_last_kernel_time("pagerank") == 0.125
    backend.pagerank(G, alpha=0.9, max_iter=100, eps=1e-6)  # another alpha: another key
    backend.pagerank(G, alpha=0.85, max_iter=100, eps=1e-6, personalization={0: 1.0})  # never cached
    backend.pagerank(G, alpha=0.85, max_iter=100, eps=1e-6, personalization={0: 1.0})
    assert [c[0] for c in calls] == [0.85, 0.9, 0.85, 0.85]
    G.add_edge(2, 1)  # a mutation drops the graph context and its results
    backend.pagerank(G, alpha=0.85, max_iter=100, eps=1e-6)
    assert len(calls) == 5


def test_reference_cache_and_result_format_switches(monkeypatch):
    # gpu_eggpu_backend.py:40-75: EASYGRAPH_GPU_DISABLE_GRAPH_CONTEXT_CACHE,
    # EASYGRAPH_GPU_DISABLE_CPP_GRAPH_CACHE and EASYGRAPH_GPU_PR_PREFER_CPP_DICT
    from eggpu_b200 import _native

    made = []

    class FakePrepared:
        def __init__(self, V, E, W=None):
            made.append(len(V) - 1)

    monkeypatch.setattr(_native, "PreparedGraph", FakePrepared)
    monkeypatch.setattr(backend, "cpp_gpu_pagerank_dense",
                        lambda pg, a, m, e, w=None, personalization=None: {"values_dense": np.array([0.25, 0.75]),
                                                                           "kernel_seconds": 0.5})
    G = DiGraph()
    G.add_edge("a", "b")
    r = backend.pagerank(G)
    assert isinstance(r, backend.DenseValueDict) and r == {"a": 0.25, "b": 0.75}
    backend.pagerank(G)
    assert made == [2]  # the prepared graph and the context are kept in G.cache
    assert backend.prepare_graph_context(G) is backend.prepare_graph_context(G)

    monkeypatch.setattr(backend, "_PR_PREFER_DICT", True)
    d = backend.pagerank(G)
    assert type(d) is dict and d == {"a": 0.25, "b": 0.75}
    d["a"] = 1.0  # a plain dict belongs to the caller
    assert backend.pagerank(G)["a"] == 0.25

    monkeypatch.setattr(backend, "_NATIVE_GRAPH_CACHE_DISABLED", True)
    backend.pagerank(G)
    backend.pagerank(G)
    assert made == [2, 2, 2]  # prepared again on every call

    H = DiGraph()
    H.add_edge(0, 1)
    monkeypatch.setattr(backend, "_GRAPH_CONTEXT_CACHE_DISABLED", True)
    c1, c2 = backend.prepare_graph_context(H), backend.prepare_graph_context(H)
    assert c1 is not c2 and c1["nodes"] == c2["nodes"] == [0, 1]
    assert backend._PREPARED_CACHE_KEY not in H.cache


def test_install_hook_with_fake_easygraph(monkeypatch):
    import sys

    calls = {}
    fake_backend = types.SimpleNamespace(pagerank=lambda *a, **k: "orig-backend")
    fake_pr = types.SimpleNamespace(pagerank=lambda G, **k: calls.setdefault("cpu", k) or "cpu")
    fake_eg = types.ModuleType("easygraph")
    fake_eg.pagerank = fake_pr.pagerank
    fake_utils = types.ModuleType("easygraph.utils")
    fake_utils.gpu_eggpu_backend = fake_backend
    fake_funcs = types.ModuleType("easygraph.functions")
    fake_cent = types.ModuleType("easygraph.functions.centrality")
    fake_cent.pagerank = fake_pr
    for name, mod in (("easygraph", fake_eg), ("easygraph.utils", fake_utils),
                      ("easygraph.utils.gpu_eggpu_backend", fake_backend), ("easygraph.functions", fake_funcs),
                      ("easygraph.functions.centrality", fake_cent),
                      ("easygraph.functions.centrality.pagerank", fake_pr)):
        monkeypatch.setitem(sys.modules, name, mod)
    monkeypatch.setattr(prmod, "_INSTALLED", {})
    assert prmod.install() is True
    assert fake_eg.pagerank is fake_pr.pagerank
    G = DiGraph()
    G.add_edge(0, 1)
    fake_eg.pagerank(G, alpha=0.5)  # GPU switch off -> easygraph's own CPU code
    assert calls["cpu"]["alpha"] == 0.5
    with pytest.raises(ValueError, match="personalization needs the GPU"):
        fake_eg.pagerank(G, personalization={0: 1.0})
    seen = {}
    monkeypatch.setattr(backend, "pagerank", lambda G, **k: seen.update(k) or {"ok": 1})
    monkeypatch.setenv("EASYGRAPH_ENABLE_GPU", "TRUE")
    assert fake_eg.pagerank(G, alpha=0.6, personalization={0: 1.0}) == {"ok": 1}
    assert seen["alpha"] == 0.6 and seen["personalization"] == {0: 1.0}
    assert fake_backend.pagerank(G, alpha=0.7, max_iter=3, eps=1e-3) == {"ok": 1}
    assert seen["max_iter"] == 3 and seen["eps"] == 1e-3
    # a C++ graph (cflag) keeps easygraph's own routing (hybrid -> cpp_pagerank) unless personalised
    GC = DiGraph()
    GC.add_edge(0, 1)
    GC.cflag = 1
    calls.clear()
    seen.clear()
    fake_eg.pagerank(GC, alpha=0.4, max_iter=7)
    assert calls["cpu"]["alpha"] == 0.4 and calls["cpu"]["max_iter"] == 7 and not seen
    assert fake_eg.pagerank(GC, alpha=0.3, personalization={0: 1.0}) == {"ok": 1} and seen["alpha"] == 0.3
