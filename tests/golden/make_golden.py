"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference tree (read-only) at REF_ROOT:

    python tests/golden/make_golden.py [REF_ROOT] [--only small|rmat|config|inbound|ppr]

What it records:
  pagerank_small.json  eg.pagerank results (GPU runtime off, i.e. the
                       reference's _pagerank_power_iteration,
                       easygraph/functions/centrality/pagerank.py:75-139) on the
                       small graphs the reference's own tests and scripts use
                       (functions/centrality/tests/test_pagerank.py,
                       tests/test_eggpu_bulk_csr.py:296-377,
                       tests/run_eggpu_gpu_contract_regression.py:83-146,
                       scripts/correctness_smoke.py:38-51,137) plus a few edge
                       cases.
  pagerank_rmat.npz    _pagerank_power_iteration on seeded R-MAT graphs built by
                       eggpu_b200.synth (CSR stored alongside).
  pagerank_config.npz  _pagerank_power_iteration on the scale-14 workload (R-MAT
                       scale 14, seed 0, alpha 0.85): its own stop rule (tol
                       1e-6, max_iter 100) and 20 fixed sweeps.  The graph is
                       not stored: the test regenerates it with eggpu_b200.synth
                       and checks it against the SHA-256 recorded here.
  inbound_ref.npz      the reference's compiled build_inbound_from_csr
                       (gpu_easygraph/functions/centrality/pagerank.cu:286-347,
                       via oracle/_ref/libref_pagerank.so) on edge-case CSRs.
  ppr_networkx.npz     networkx.pagerank with personalisation and uniform
                       dangling weights (third-party oracle for the PPR
                       extension, which the reference does not have).

The reference's optional imports fastjsonschema and matplotlib are stubbed in
a temporary directory; nothing from the reference is copied into this repo.
"""

from __future__ import annotations

import json
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

REF_ROOT = Path(sys.argv[1] if len(sys.argv) > 1 and not sys.argv[1].startswith("--")
                else os.environ.get("EGPR_REFERENCE_ROOT", "/root/reference"))


def _import_reference():
    tmp = Path(tempfile.mkdtemp(prefix="egref_"))
    (tmp / "easygraph").symlink_to(REF_ROOT / "Easy-Graph" / "easygraph")
    (tmp / "fastjsonschema.py").write_text(
        "def compile(*a, **k):\n    return lambda x: x\nclass JsonSchemaException(Exception):\n    pass\n"
    )
    mp = tmp / "matplotlib"
    mp.mkdir()
    (mp / "__init__.py").write_text(
        "import sys, types\n"
        "class _Any(types.ModuleType):\n"
        "    def __getattr__(self, name):\n"
        "        if name.startswith('__'):\n"
        "            raise AttributeError(name)\n"
        "        return type(name, (), {})\n"
        "for _n in ['axes', 'pyplot', 'patches', 'collections', 'colors', 'lines', 'figure', 'cm', 'path',\n"
        "           'transforms', 'animation']:\n"
        "    sys.modules['matplotlib.' + _n] = _Any('matplotlib.' + _n)\n"
    )
    sys.path.insert(0, str(tmp))
    os.environ.pop("EASYGRAPH_ENABLE_GPU", None)
    import easygraph as eg
    from easygraph.functions.centrality.pagerank import _pagerank_power_iteration

    return eg, _pagerank_power_iteration


def _encode_node(x):
    if isinstance(x, tuple):
        return {"tuple": [_encode_node(v) for v in x]}
    return x


def small_cases(eg):
    cases = []

    def add(name, G, directed, kwargs):
        nodes = list(G.nodes)
        edges = []
        for u, v, data in G.edges:
            edges.append([_encode_node(u), _encode_node(v), {k: float(val) for k, val in data.items()
                                                             if isinstance(val, (int, float))}])
        res = eg.pagerank(G, **kwargs)
        cases.append({
            "name": name,
            "directed": directed,
            "nodes": [_encode_node(x) for x in nodes],
            "edges": edges,
            "kwargs": kwargs,
            "expected": [[_encode_node(k), float(v)] for k, v in res.items()],
        })

    # test_pagerank.py:10-38
    g = eg.DiGraph()
    g.add_edges_from([(0, 1), (1, 2), (2, 0)])
    add("directed_triangle", g, True, {})
    g = eg.Graph()
    g.add_edges_from([(0, 1), (1, 2), (2, 0)])
    add("undirected_triangle", g, False, {})
    g = eg.DiGraph()
    g.add_edges_from([(0, 1), (2, 3)])
    add("disconnected", g, True, {})
    g = eg.DiGraph()
    g.add_edges_from([(0, 0), (0, 1), (1, 2)])
    add("self_loop", g, True, {})
    g = eg.DiGraph()
    g.add_edges_from([("A", "B"), ("B", "C"), ("C", (1, 2))])
    add("mixed_labels", g, True, {})
    g = eg.DiGraph()
    g.add_node("solo")
    add("single_node", g, True, {})
    g = eg.DiGraph()
    g.add_edges_from([(1, 2), (2, 3), ("String", "Bool"), (2, 1), (0, 0)])
    add("test_pagerank_g", g, True, {})
    # test_eggpu_bulk_csr.py:296-311 (undirected 6-node graph, alpha 0.75)
    g = eg.Graph()
    g.add_nodes(range(6))
    g.add_edges([(0, 1), (1, 2), (2, 0), (2, 3), (3, 4), (4, 5), (5, 3)])
    add("bulk_regular_undirected", g, False, {"alpha": 0.75, "max_iter": 200, "tol": 1.0e-6})
    # test_eggpu_bulk_csr.py:339-377 (7-node digraph, alpha 0.75 then 0.90, tol 1e-7)
    g = eg.DiGraph()
    g.add_nodes(range(7))
    g.add_edges([(0, 1), (0, 2), (1, 2), (2, 0), (2, 3), (3, 2), (3, 4), (4, 5), (5, 4), (5, 6)])
    add("alpha_075", g, True, {"alpha": 0.75, "max_iter": 200, "tol": 1.0e-7})
    add("alpha_090", g, True, {"alpha": 0.90, "max_iter": 200, "tol": 1.0e-7})
    # run_eggpu_gpu_contract_regression.py:83-118 (weighted, after mutation)
    g = eg.DiGraph()
    g.add_edge(0, 1, weight=0.25)
    g.add_edge(0, 2, weight=1.0)
    g.add_edge(1, 2, weight=2.0)
    g.add_edge(2, 0, weight=1.0)
    add("weight_mutation", g, True, {"weight": "weight"})
    g = eg.DiGraph()
    g.add_edge(0, 1, weight=8.0)
    g.add_edge(0, 2, weight=1.0)
    g.add_edge(1, 2, weight=2.0)
    g.add_edge(2, 0, weight=1.0)
    add("weight_before_mutation", g, True, {"weight": "weight"})
    # run_eggpu_gpu_contract_regression.py:138-146
    g = eg.DiGraph()
    g.add_edges_from([(0, 1), (1, 2), (2, 0), (2, 3)])
    add("identity_a", g, True, {})
    g = eg.DiGraph()
    g.add_edges_from([(0, 1), (1, 0), (1, 2), (3, 2)])
    add("identity_b", g, True, {})
    # scripts/correctness_smoke.py:38-51,137
    g = eg.DiGraph()
    g.add_weighted_edges_from([(0, 1, 1.0), (1, 2, 2.0), (2, 0, 0.5), (2, 3, 1.5), (3, 4, 1.0), (4, 3, 0.75),
                               (1, 4, 4.0)])
    add("smoke_weighted", g, True, {"alpha": 0.75, "weight": "weight", "max_iter": 200, "tol": 1e-6})
    # extra edge cases
    g = eg.DiGraph()
    g.add_nodes(range(4))
    add("no_edges", g, True, {})
    g = eg.DiGraph()
    g.add_edges_from([(0, 1), (0, 2), (0, 3)])
    add("star_all_dangling_leaves", g, True, {"alpha": 0.85, "max_iter": 50, "tol": 0.0})
    g = eg.Graph()
    g.add_weighted_edges_from([(0, 1, 1.0), (1, 2, 2.0), (2, 0, 0.5), (2, 3, 1.5), (3, 4, 1.0), (4, 5, 2.5),
                               (5, 3, 0.75), (1, 5, 4.0)])
    add("undirected_weighted", g, False, {"weight": "weight", "max_iter": 30, "tol": 0.0})
    return cases


def rmat_cases(eg, pr_iter):
    from eggpu_b200 import synth

    specs = [
        ("rmat10_s0", dict(scale=10, edgefactor=16, seed=0), None, {"alpha": 0.85, "max_iter": 100, "tol": 1e-6}),
        ("rmat10_s0_fixed20", dict(scale=10, edgefactor=16, seed=0), None, {"alpha": 0.85, "max_iter": 20, "tol": 0.0}),
        ("rmat10_w5", dict(scale=10, edgefactor=8, seed=5, weighted=True), "weight",
         {"alpha": 0.85, "max_iter": 100, "tol": 1e-7}),
        ("rmat12_s0", dict(scale=12, edgefactor=16, seed=0), None, {"alpha": 0.85, "max_iter": 100, "tol": 1e-6}),
        ("rmat12_s0_a05", dict(scale=12, edgefactor=16, seed=0), None, {"alpha": 0.5, "max_iter": 100, "tol": 1e-8}),
    ]
    out = {}
    names = []
    for name, params, weight, kw in specs:
        csr = synth.rmat(**params)
        G = eg.DiGraph()
        G.add_nodes(range(csr.n))
        edges = []
        for u in range(csr.n):
            for p in range(csr.V[u], csr.V[u + 1]):
                v = int(csr.E[p])
                if weight is None:
                    edges.append((u, v))
                else:
                    edges.append((u, v, {"weight": float(csr.W[p])}))
        if weight is None:
            G.add_edges(edges)
        else:
            for u, v, d in edges:
                G.add_edge(u, v, **d)
        res = pr_iter(G, weight=weight, **kw)
        vec = np.array([res[i] for i in range(csr.n)], np.float64)
        names.append(name)
        out[f"{name}/V"] = csr.V
        out[f"{name}/E"] = csr.E
        if csr.W is not None:
            out[f"{name}/W"] = csr.W
        out[f"{name}/expected"] = vec
        out[f"{name}/kwargs"] = np.frombuffer(json.dumps(kw).encode(), np.uint8)
    out["names"] = np.frombuffer(json.dumps(names).encode(), np.uint8)
    return out


def graph_digest(V, E, W=None):
    """SHA-256 over the CSR arrays (int32 V, int32 E, float64 W if any)."""
    import hashlib

    h = hashlib.sha256()
    for a in (np.ascontiguousarray(V, np.int32), np.ascontiguousarray(E, np.int32)) + (
            () if W is None else (np.ascontiguousarray(W, np.float64),)):
        h.update(a.tobytes())
    return h.hexdigest()


def config_cases(eg, pr_iter):
    from eggpu_b200 import synth

    params = dict(scale=14, edgefactor=16, seed=0)
    csr = synth.rmat(**params)
    G = eg.DiGraph()
    G.add_nodes(range(csr.n))
    G.add_edges([(u, int(csr.E[p])) for u in range(csr.n) for p in range(csr.V[u], csr.V[u + 1])])
    out, names = {}, []
    for name, kw in (("rmat14_s0", {"alpha": 0.85, "max_iter": 100, "tol": 1e-6}),
                     ("rmat14_s0_fixed20", {"alpha": 0.85, "max_iter": 20, "tol": 0.0})):
        res = pr_iter(G, **kw)
        names.append(name)
        out[f"{name}/params"] = np.frombuffer(json.dumps(params).encode(), np.uint8)
        out[f"{name}/kwargs"] = np.frombuffer(json.dumps(kw).encode(), np.uint8)
        out[f"{name}/sha256"] = np.frombuffer(graph_digest(csr.V, csr.E).encode(), np.uint8)
        out[f"{name}/expected"] = np.array([res[i] for i in range(csr.n)], np.float64)
    out["names"] = np.frombuffer(json.dumps(names).encode(), np.uint8)
    return out


def inbound_cases():
    sys.path.insert(0, str(ROOT))
    from oracle import oracle

    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libref_pagerank.so missing: run make -f oracle/Makefile.ref")
    from eggpu_b200 import synth

    rng = np.random.default_rng(7)
    cases = []
    # 1. plain R-MAT, unweighted and weighted
    c = synth.rmat(scale=9, edgefactor=8, seed=11)
    cases.append(("rmat9", c.V, c.E, None))
    c = synth.rmat(scale=9, edgefactor=8, seed=12, weighted=True)
    cases.append(("rmat9_w", c.V, c.E, c.W))
    # 2. duplicates, self-loops, invalid endpoints, odd weights, empty rows
    n = 12
    rows = []
    for u in range(n):
        deg = int(rng.integers(0, 6))
        rows.append(sorted(int(x) for x in rng.integers(-2, n + 2, size=deg)))
    rows[3] = []
    rows[4] = [4, 4, 5, 5, 5]
    V = np.zeros(n + 1, np.int32)
    for u in range(n):
        V[u + 1] = V[u] + len(rows[u])
    E = np.array([x for r in rows for x in r], np.int32)
    W = rng.uniform(0.0, 3.0, size=E.shape[0])
    W[::5] = -1.0
    W[1::7] = np.nan
    W[2::9] = np.inf
    W[3::11] = 0.0
    cases.append(("messy", V, E, W))
    cases.append(("messy_unweighted", V, E, None))
    # 3. a row whose only weights are zero -> dangling under the reference mask
    V = np.array([0, 2, 3, 3], np.int32)
    E = np.array([1, 2, 0], np.int32)
    W = np.array([0.0, 0.0, 1.0])
    cases.append(("zero_weight_row", V, E, W))
    # 4. single vertex with a self-loop; single vertex without edges
    cases.append(("one_selfloop", np.array([0, 1], np.int32), np.array([0], np.int32), None))
    cases.append(("one_bare", np.array([0, 0], np.int32), np.zeros(0, np.int32), None))
    out = {"names": np.frombuffer(json.dumps([c[0] for c in cases]).encode(), np.uint8)}
    for name, V, E, W in cases:
        in_row, in_col, in_val, dang = oracle.ref_build_inbound(V, E, W, alpha=0.85)
        out[f"{name}/V"] = V
        out[f"{name}/E"] = E
        if W is not None:
            out[f"{name}/W"] = W
        out[f"{name}/in_row"] = in_row
        out[f"{name}/in_col"] = in_col
        out[f"{name}/in_val"] = in_val
        out[f"{name}/dangling"] = dang
    return out


def ppr_cases():
    import networkx as nx
    from eggpu_b200 import synth

    c = synth.rmat(scale=10, edgefactor=8, seed=21)
    G = nx.DiGraph()
    G.add_nodes_from(range(c.n))
    for u in range(c.n):
        for p in range(c.V[u], c.V[u + 1]):
            G.add_edge(u, int(c.E[p]))
    sets = synth.seed_sets(c.n, 6, 1, 16, seed=5)
    out = {"V": c.V, "E": c.E}
    res = []
    for j, s in enumerate(sets):
        pers = {int(v): 1.0 for v in s}
        r = nx.pagerank(G, alpha=0.85, personalization=pers, dangling={v: 1.0 for v in range(c.n)}, tol=1e-10,
                        max_iter=500)
        res.append([r[i] for i in range(c.n)])
        out[f"seeds/{j}"] = s
    out["expected"] = np.array(res, np.float64)
    out["k"] = np.array([len(sets)], np.int32)
    return out


def main():
    # --only NAME writes one fixture: small, rmat, config, inbound or ppr
    only = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None
    eg, pr_iter = _import_reference()
    if only in (None, "small"):
        (HERE / "pagerank_small.json").write_text(json.dumps(small_cases(eg), indent=1))
    if only in (None, "rmat"):
        np.savez_compressed(HERE / "pagerank_rmat.npz", **rmat_cases(eg, pr_iter))
    if only in (None, "config"):
        np.savez_compressed(HERE / "pagerank_config.npz", **config_cases(eg, pr_iter))
    if only in (None, "inbound"):
        np.savez_compressed(HERE / "inbound_ref.npz", **inbound_cases())
    if only in (None, "ppr"):
        np.savez_compressed(HERE / "ppr_networkx.npz", **ppr_cases())
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
