"""The engine's Python-graph -> out-edge CSR walk against the reference's own
C++ code, array for array.

tests/golden/gencsr_ref.npz holds CSRs that the reference's build_digraph /
build_graph (cpp_easygraph/classes/graph_convert.cpp:72-134) and
Graph::gen_CSR (cpp_easygraph/classes/graph.cpp:719-886) produced for graphs
built by the reference's Python package (script tests/golden/make_gencsr.py;
shuffled node and edge insertion orders, undirected duplicates and
self-loops, weights on part of the edges, nodes that are only endpoints).
The same graphs are rebuilt here from the recorded insertion orders and walked
by backend.graph_csr (native walk) and its Python specification.
"""

from pathlib import Path

import numpy as np
import pytest

from eggpu_b200 import backend
from tests.graphs import DiGraph, Graph

FIXTURE = Path(__file__).resolve().parent / "golden" / "gencsr_ref.npz"
_DATA = np.load(FIXTURE)
NAMES = sorted({k.split("/")[0] for k in _DATA.files})


def _graph(name):
    d = {k.split("/", 1)[1]: _DATA[k] for k in _DATA.files if k.startswith(name + "/")}
    G = DiGraph() if bool(d["directed"][0]) else Graph()
    G.add_nodes([int(v) for v in d["nodes"]])
    key = "weight" if "w" in d else None
    for i, (a, b) in enumerate(d["edges"]):
        if key is not None and not np.isnan(d["w"][i]):
            G.add_edge(int(a), int(b), **{key: float(d["w"][i])})
        else:
            G.add_edge(int(a), int(b))
    return G, key, d


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("walk", ["native", "python"])
def test_out_edge_csr_equals_reference_gen_csr(name, walk):
    G, key, d = _graph(name)
    prepared = backend.prepare_graph_context(G)
    if walk == "native":
        V, E, W = backend.graph_csr(G, prepared, key)
    else:
        V, E, W = backend._graph_csr_py(G, prepared, key)
    assert np.array_equal(V, d["V"]) and V.dtype == np.int32
    assert np.array_equal(E, d["E"]) and E.dtype == np.int32
    if key is None:
        assert W is None
    else:
        assert np.array_equal(W.view(np.uint64), d["W"].view(np.uint64))


def test_fixture_covers_the_conversion_rules():
    """The cases exercise what the rules decide: undirected duplicates and
    self-loops, and nodes that appear only as edge endpoints."""
    assert {"rmat12_digraph", "rmat12_graph", "rmat12_digraph_weighted", "rmat12_graph_weighted",
            "endpoints_only"} <= set(NAMES)
    G, _, d = _graph("rmat12_graph")
    e = d["edges"]
    assert (e[:, 0] == e[:, 1]).any()  # self-loops were added
    assert len(d["E"]) < 2 * len(e)    # and duplicates dropped
    _, _, d2 = _graph("endpoints_only")
    assert len(d2["V"]) - 1 == 4       # 7, 3 listed; 9 and 11 only as endpoints
