"""The oracle is pinned before it is trusted: every function of the CPU
restatement is checked against vectors produced by the reference itself
(tests/golden/, made by tests/golden/make_golden.py) and, where the reference's
own compiled translation unit is present (oracle/_ref), against it live."""

import numpy as np
import pytest

from oracle import oracle
from tests.graphs import golden_config_cases, golden_inbound_cases, golden_ppr, golden_rmat_cases, golden_small_cases

# R-MAT scales 10-12 with the CSR stored, and the scale-14 workload regenerated
_RMAT_CASES = golden_rmat_cases() + golden_config_cases()


@pytest.mark.parametrize("case", _RMAT_CASES, ids=lambda c: c[0])
def test_push_oracle_bit_exact_vs_reference_python(case):
    name, V, E, W, kw, expected = case
    ranks, iters, _ = oracle.pagerank_push(V, E, W, **kw)
    assert np.array_equal(ranks, expected), np.abs(ranks - expected).max()
    assert iters >= 1


@pytest.mark.parametrize("case", _RMAT_CASES, ids=lambda c: c[0])
def test_pull_oracle_bit_exact_vs_reference_python(case):
    name, V, E, W, kw, expected = case
    ranks, iters, _ = oracle.pagerank_pull(V, E, W, **kw)
    assert np.array_equal(ranks, expected)
    ranks_push, iters_push, _ = oracle.pagerank_push(V, E, W, **kw)
    assert iters == iters_push


@pytest.mark.parametrize("case", golden_inbound_cases(), ids=lambda c: c[0])
def test_build_inbound_bit_exact_vs_reference(case):
    name, V, E, W, in_row, in_col, in_val, dangling = case
    r, c, w, d, outw = oracle.build_inbound(V, E, W)
    assert np.array_equal(r, in_row)
    assert np.array_equal(c, in_col)
    assert np.array_equal(d, dangling)
    vals = oracle.inbound_values(c, w, outw, 0.85)
    assert np.array_equal(vals.view(np.uint32), in_val.view(np.uint32))


@pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (needs the reference tree)")
def test_build_inbound_matches_compiled_reference_on_random_csr():
    from eggpu_b200 import synth

    for seed in range(3):
        c = synth.rmat(scale=11, edgefactor=8, seed=100 + seed, weighted=bool(seed % 2))
        r, col, w, d, outw = oracle.build_inbound(c.V, c.E, c.W)
        rr, rc, rv, rd = oracle.ref_build_inbound(c.V, c.E, c.W, alpha=0.85)
        assert np.array_equal(r, rr) and np.array_equal(col, rc) and np.array_equal(d, rd)
        assert np.array_equal(oracle.inbound_values(col, w, outw, 0.85).view(np.uint32), rv.view(np.uint32))


def _csr_of(G, weight):
    nodes = list(G.nodes)
    return oracle.graph_to_csr(nodes, G._adj, G.is_directed(), weight)


@pytest.mark.parametrize("case", golden_small_cases(), ids=lambda c: c[0])
def test_small_reference_cases_through_csr_restatement(case):
    name, G, kw, expected = case
    V, E, W = _csr_of(G, kw.get("weight"))
    args = dict(alpha=kw.get("alpha", 0.85), max_iter=kw.get("max_iter", 200), tol=kw.get("tol", 1e-6))
    ranks, _, _ = oracle.pagerank_push(V, E, W, **args)
    nodes = list(G.nodes)
    got = {nodes[i]: ranks[i] for i in range(len(nodes))}
    assert set(got) == set(expected)
    for k, v in expected.items():
        assert got[k] == pytest.approx(v, rel=1e-12, abs=1e-15)


def test_ppr_oracle_matches_networkx():
    V, E, sets, expected = golden_ppr()
    n = V.shape[0] - 1
    for j, s in enumerate(sets):
        p = np.zeros(n)
        p[s] = 1.0 / len(s)
        ranks, _, _ = oracle.pagerank_push(V, E, None, alpha=0.85, max_iter=500, tol=1e-10, teleport=p)
        assert np.abs(ranks - expected[j]).sum() < 1e-9


def test_uniform_teleport_reproduces_plain_pagerank():
    V, E, W, kw, expected = golden_rmat_cases()[0][1:]
    n = V.shape[0] - 1
    ranks, _, _ = oracle.pagerank_push(V, E, W, teleport=np.full(n, 1.0 / n), **kw)
    assert np.abs(ranks - expected).sum() < 1e-12


def test_openmp_cpu_port_agrees_with_power_iteration():
    name, V, E, W, kw, expected = golden_rmat_cases()[0]
    raw, sweeps = oracle.cpu_pagerank_omp(V, E, W, alpha=kw["alpha"], max_iter=kw["max_iter"],
                                          threshold=kw["tol"], threads=4)
    assert np.abs(raw / raw.sum() - expected).sum() < 1e-12
    _, iters, _ = oracle.pagerank_push(V, E, W, **kw)
    assert sweeps == iters


def test_push_oracle_edge_cases():
    # no edges -> uniform (pagerank.py:96-98)
    r, it, _ = oracle.pagerank_push(np.zeros(5, np.int32), np.zeros(0, np.int32))
    assert np.allclose(r, 0.25) and it == 0
    # single vertex with a self-loop
    r, it, _ = oracle.pagerank_push(np.array([0, 1], np.int32), np.array([0], np.int32))
    assert r[0] == 1.0
