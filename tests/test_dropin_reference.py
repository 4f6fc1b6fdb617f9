"""The engine installed into the reference's own easygraph package.

``eggpu_b200.api.install()`` is run against the real easygraph Python package
of the reference checkout (imported as tests/golden/make_golden.py imports it:
the optional fastjsonschema / matplotlib dependencies stubbed), and the
reference's own contract assertions are replayed on real ``eg.DiGraph`` /
``eg.Graph`` objects through ``eg.pagerank`` with EASYGRAPH_ENABLE_GPU on:

* easygraph/tests/test_eggpu_cache_contracts.py:16-49 — edge-attribute
  mutation clears ``G.cache`` (the prepared context and the prepared device
  graph go with it) and the next call prepares again;
* :190-221 — the dense result: a read-only Mapping in node order, length n;
* easygraph/tests/test_eggpu_bulk_csr.py:339-377 — a new alpha does not reuse
  values computed for the previous one;
* scripts/correctness_smoke.py:38-51,137 — the weighted 5-node digraph at
  alpha 0.75 against easygraph's own CPU power iteration.

The native solve is replaced by a stand-in computed with the oracle (the
reference's contract tests fake their native module the same way), so this
runs without a GPU; the GPU numerics of the same calls are pinned by
tests/test_gpu_parity.py.  The reference checkout is found through
EGPR_REFERENCE_ROOT; without it the test is skipped.  It runs in a child
process, so the real easygraph never shadows the fake one other tests use.
"""

import os
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = Path(os.environ.get("EGPR_REFERENCE_ROOT", "/root/reference")) / "Easy-Graph" / "easygraph"

SCRIPT = textwrap.dedent(r'''
    import os, sys
    root = os.environ["EGPR_DROPIN_REPO"]
    sys.argv = ["dropin"]  # make_golden reads an optional reference root from argv
    sys.path.insert(0, root)
    sys.path.insert(0, root + "/tests/golden")
    import numpy as np
    from collections.abc import Mapping
    import make_golden
    eg, power_iteration = make_golden._import_reference()
    assert eg.__file__.startswith(make_golden.REF_ROOT.as_posix()) or "egref_" in eg.__file__
    from eggpu_b200 import _native, api, backend
    from oracle import oracle

    class OracleGraph:
        """Stand-in for the native prepared graph: the oracle's FP64 solve."""
        created = 0
        def __init__(self, V, E, W=None):
            OracleGraph.created += 1
            self.V, self.E, self.W = V, E, W
            self.n = V.shape[0] - 1
            self.inbound = oracle.build_inbound(V, E, W)
        def pagerank(self, alpha=0.85, max_iter=100, tol=1e-6, personalization=None, correction=True, out=None):
            # the C ABI normalises a personalisation vector to sum 1 (egpr_pagerank)
            tele = None if personalization is None else personalization / personalization.sum()
            r, it, res = oracle.pagerank_pull(self.V, self.E, self.W, alpha=alpha, max_iter=max_iter, tol=tol,
                                              teleport=tele, inbound=self.inbound)
            return r, {"iterations": it, "converged": 1, "residual": res, "kernel_seconds": 0.0}

    _native.PreparedGraph = OracleGraph
    backend._result_vector = lambda n: None
    assert api.install() is True
    os.environ["EASYGRAPH_ENABLE_GPU"] = "TRUE"
    os.environ["EASYGRAPH_GPU_STRICT_ERRORS"] = "TRUE"

    def close(a, b, nodes, rtol=2e-5, atol=1e-7):
        return np.allclose([a[v] for v in nodes], [b[v] for v in nodes], rtol=rtol, atol=atol)

    # correctness_smoke.py:38-51,137: weighted 5-node digraph, alpha 0.75
    G = eg.DiGraph()
    G.add_edges([(0, 1), (1, 2), (2, 0), (2, 3), (3, 4), (4, 2)],
                edges_attr=[{"weight": w} for w in (1.0, 2.0, 0.5, 1.5, 3.0, 1.0)])
    got = eg.pagerank(G, alpha=0.75, weight="weight")
    want = power_iteration(G, alpha=0.75, weight="weight", max_iter=200, tol=1e-6)
    assert close(got, want, range(5)), (dict(got), want)

    # test_eggpu_cache_contracts.py:190-221: the dense result Mapping
    assert isinstance(got, Mapping) and not isinstance(got, dict)
    assert list(got) == list(G.nodes) and len(got) == len(G)
    try:
        got[0] = 1.0
        raise AssertionError("the result must be read-only")
    except TypeError:
        pass
    assert dict(got) == {v: got[v] for v in G.nodes}

    # test_eggpu_cache_contracts.py:16-49: prepared state lives in G.cache and
    # an edge-attribute mutation clears it
    assert "__eggpu_prepared_graph__" in G.cache
    made = OracleGraph.created
    eg.pagerank(G, alpha=0.75, weight="weight")
    assert OracleGraph.created == made, "a second call reuses the prepared graph"
    gen = G._mutation_generation
    G[2][3]["weight"] = 7.0  # vertex 2 has two out-edges, so its split changes
    assert G.cache == {} and G._mutation_generation == gen + 1
    got2 = eg.pagerank(G, alpha=0.75, weight="weight")
    assert OracleGraph.created == made + 1, "the mutated graph is prepared again"
    want2 = power_iteration(G, alpha=0.75, weight="weight", max_iter=200, tol=1e-6)
    assert close(got2, want2, range(5)) and not close(got2, got, range(5), rtol=1e-9, atol=0.0)

    # test_eggpu_bulk_csr.py:339-377: a new alpha is not served from the old one
    H = eg.DiGraph()
    H.add_nodes(range(7))
    H.add_edges([(0, 1), (0, 2), (1, 2), (2, 0), (2, 3), (3, 2), (3, 4), (4, 5), (5, 4), (5, 6)])
    eg.pagerank(H, alpha=0.75, max_iter=200, tol=1.0e-7)
    got3 = eg.pagerank(H, alpha=0.90, max_iter=200, tol=1.0e-7)
    want3 = power_iteration(H, alpha=0.90, max_iter=200, tol=1.0e-7)
    assert close(got3, want3, range(7))

    # undirected graph, string labels, and easygraph's own CPU path with the switch off
    U = eg.Graph()
    U.add_edges([("a", "b"), ("b", "c"), ("c", "a"), ("c", "d"), ("d", "d")])
    got4 = eg.pagerank(U)
    os.environ["EASYGRAPH_ENABLE_GPU"] = "FALSE"
    cpu4 = eg.pagerank(U)
    os.environ["EASYGRAPH_ENABLE_GPU"] = "TRUE"
    assert close(got4, cpu4, ["a", "b", "c", "d"])

    # test_pagerank.py:75-82 edge cases; a personalised solve through eg.pagerank
    assert eg.pagerank(eg.DiGraph()) == {}
    S = eg.DiGraph()
    S.add_node("solo")
    assert dict(eg.pagerank(S)) == {"solo": 1.0}
    P = eg.pagerank(H, personalization={0: 1.0, 4: 1.0})
    tele = np.zeros(7); tele[[0, 4]] = 0.5
    ref = oracle.pagerank_pull(*backend.graph_csr(H, backend.prepare_graph_context(H)), alpha=0.85, max_iter=200,
                               tol=1e-6, teleport=tele)[0]
    assert np.allclose([P[v] for v in range(7)], ref, rtol=1e-12, atol=1e-15)
    M = eg.MultiDiGraph()
    M.add_edge(0, 1)
    try:
        eg.pagerank(M)
        raise AssertionError("a multigraph must be refused")
    except Exception as exc:
        assert type(exc).__name__ == "EasyGraphNotImplemented", type(exc)
    print("DROPIN_OK")
''')


@pytest.mark.skipif(not REF.is_dir(), reason="the reference checkout is not present (EGPR_REFERENCE_ROOT)")
def test_engine_installed_into_the_reference_easygraph():
    env = dict(os.environ)
    env.pop("EASYGRAPH_ENABLE_GPU", None)
    env["EGPR_DROPIN_REPO"] = str(ROOT)
    res = subprocess.run([sys.executable, "-c", SCRIPT], capture_output=True, text=True, timeout=600, env=env,
                         cwd=str(ROOT))
    assert res.returncode == 0 and "DROPIN_OK" in res.stdout, res.stdout[-3000:] + res.stderr[-3000:]
