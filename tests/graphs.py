"""Small dict-of-dicts graphs with the attributes the PageRank path reads from
an easygraph Graph/DiGraph (_node, _adj, nodes, edges, cache,
_mutation_generation, is_directed, is_multigraph), so the tests run where
easygraph is not installed.  Mutation through G[u][v][key] = value bumps the
generation and clears the cache like easygraph/classes/graph.py:17-40,1641-1644.
"""

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


class _AttrDict(dict):
    def __init__(self, graph, *a, **k):
        super().__init__(*a, **k)
        self._graph = graph

    def __setitem__(self, key, value):
        super().__setitem__(key, value)
        self._graph._touch()


class DiGraph:
    directed = True

    def __init__(self):
        self._node = {}
        self._adj = {}
        self.cache = {}
        self._mutation_generation = 0

    def _touch(self):
        self._mutation_generation += 1
        self.cache = {}

    def add_node(self, u):
        if u not in self._node:
            self._node[u] = {}
            self._adj[u] = {}
            self._touch()

    def add_nodes(self, nodes):
        for u in nodes:
            self.add_node(u)

    def add_edge(self, u, v, **attr):
        self.add_node(u)
        self.add_node(v)
        d = self._adj[u].get(v)
        if d is None:
            d = _AttrDict(self)
            self._adj[u][v] = d
            if not self.directed:
                self._adj[v][u] = d
        dict.update(d, attr)
        self._touch()

    def add_edges_from(self, edges):
        for e in edges:
            if len(e) == 3 and isinstance(e[2], dict):
                self.add_edge(e[0], e[1], **e[2])
            elif len(e) == 3:
                self.add_edge(e[0], e[1], weight=e[2])
            else:
                self.add_edge(e[0], e[1])

    def __getitem__(self, u):
        return self._adj[u]

    def __len__(self):
        return len(self._node)

    @property
    def nodes(self):
        return self._node

    @property
    def edges(self):
        seen = set()
        for u, nbrs in self._adj.items():
            for v, d in nbrs.items():
                if not self.directed:
                    key = frozenset((u, v)) if u != v else (u,)
                    if key in seen:
                        continue
                    seen.add(key)
                yield u, v, d

    def is_directed(self):
        return self.directed

    def is_multigraph(self):
        return False


class Graph(DiGraph):
    directed = False


class MultiDiGraph(DiGraph):
    def is_multigraph(self):
        return True


def decode_node(x):
    if isinstance(x, dict) and "tuple" in x:
        return tuple(decode_node(v) for v in x["tuple"])
    if isinstance(x, list):
        return tuple(decode_node(v) for v in x)
    return x


def golden_small_cases():
    cases = json.loads((GOLDEN / "pagerank_small.json").read_text())
    out = []
    for c in cases:
        G = DiGraph() if c["directed"] else Graph()
        for u in c["nodes"]:
            G.add_node(decode_node(u))
        for u, v, d in c["edges"]:
            G.add_edge(decode_node(u), decode_node(v), **d)
        expected = {decode_node(k): v for k, v in c["expected"]}
        out.append((c["name"], G, c["kwargs"], expected))
    return out


def golden_rmat_cases():
    d = np.load(GOLDEN / "pagerank_rmat.npz")
    names = json.loads(bytes(d["names"]).decode())
    out = []
    for nm in names:
        W = d[nm + "/W"] if nm + "/W" in d else None
        kw = json.loads(bytes(d[nm + "/kwargs"]).decode())
        out.append((nm, d[nm + "/V"], d[nm + "/E"], W, kw, d[nm + "/expected"]))
    return out


def golden_config_cases():
    """The scale-14 workload's reference vectors; the graph is regenerated
    here and checked against the digest the fixture recorded."""
    import hashlib

    from eggpu_b200 import synth

    d = np.load(GOLDEN / "pagerank_config.npz")
    names = json.loads(bytes(d["names"]).decode())
    out = []
    graphs = {}
    for nm in names:
        params = json.loads(bytes(d[nm + "/params"]).decode())
        key = json.dumps(params, sort_keys=True)
        if key not in graphs:
            csr = synth.rmat(**params)
            h = hashlib.sha256()
            h.update(np.ascontiguousarray(csr.V, np.int32).tobytes())
            h.update(np.ascontiguousarray(csr.E, np.int32).tobytes())
            graphs[key] = (csr, h.hexdigest())
        csr, digest = graphs[key]
        assert digest == bytes(d[nm + "/sha256"]).decode(), f"{nm}: the generator no longer makes the recorded graph"
        kw = json.loads(bytes(d[nm + "/kwargs"]).decode())
        out.append((nm, csr.V, csr.E, None, kw, d[nm + "/expected"]))
    return out


def golden_inbound_cases():
    d = np.load(GOLDEN / "inbound_ref.npz")
    names = json.loads(bytes(d["names"]).decode())
    out = []
    for nm in names:
        W = d[nm + "/W"] if nm + "/W" in d else None
        out.append((nm, d[nm + "/V"], d[nm + "/E"], W, d[nm + "/in_row"], d[nm + "/in_col"], d[nm + "/in_val"],
                    d[nm + "/dangling"]))
    return out


def golden_ppr():
    d = np.load(GOLDEN / "ppr_networkx.npz")
    k = int(d["k"][0])
    return d["V"], d["E"], [d[f"seeds/{j}"] for j in range(k)], d["expected"]
