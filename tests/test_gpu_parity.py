"""Parity of the CUDA engine with the oracle and the reference's golden vectors.

Bars: preparation (inbound CSR, dangling mask, FP64 out-weight sums) bit-exact;
ranks within L1 <= 1e-6 of the FP64 oracle with the iteration count within
+-1 of the oracle's (when the counts differ, ranks are compared with the oracle
run for the engine's count); per entry also within the reference's own GPU test
tolerance rtol 2e-5 / atol 1e-7 (tests/test_eggpu_bulk_csr.py:339-377).
Every call goes through the C ABI (libegpr.so).
"""

import numpy as np
import pytest

from eggpu_b200 import _native, backend, synth
from eggpu_b200 import api as prmod
from oracle import oracle
from tests.graphs import (DiGraph, Graph, golden_config_cases, golden_inbound_cases, golden_ppr,
                          golden_rmat_cases, golden_small_cases)

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


def _check_against_oracle(V, E, W, ranks, stats, alpha, max_iter, tol, teleport=None):
    ref, it_ref, _ = oracle.pagerank_pull(V, E, W, alpha=alpha, max_iter=max_iter, tol=tol, teleport=teleport)
    it = stats["iterations"]
    assert abs(it - it_ref) <= 1, (it, it_ref)
    if it != it_ref:
        ref, _, _ = oracle.pagerank_pull(V, E, W, alpha=alpha, max_iter=it, tol=0.0, teleport=teleport)
    l1 = np.abs(ranks - ref).sum()
    assert l1 <= L1_TOL, l1
    assert np.allclose(ranks, ref, rtol=2e-5, atol=1e-7)
    return l1


@pytest.mark.parametrize("case", golden_inbound_cases(), ids=lambda c: c[0])
def test_preparation_bit_exact_vs_reference(case):
    name, V, E, W, in_row, in_col, in_val, dangling = case
    pg = _native.PreparedGraph(V, E, W)
    r, c, w, d, outw = pg.export_inbound()
    assert np.array_equal(r, in_row)
    assert np.array_equal(c, in_col)
    assert np.array_equal(d, dangling)
    _, _, ow, _, o_outw = oracle.build_inbound(V, E, W)
    assert np.array_equal(outw.view(np.uint64), o_outw.view(np.uint64))
    assert np.array_equal(w, ow.astype(np.float32))
    # the reference's alpha-scaled in_val follows bit for bit from what is stored
    vals = oracle.inbound_values(c, ow, outw, 0.85)
    assert np.array_equal(vals.view(np.uint32), in_val.view(np.uint32))


@pytest.mark.parametrize("scale,weighted", [(14, False), (16, True), (18, False)])
def test_preparation_bit_exact_rmat(scale, weighted):
    g = synth.rmat(scale=scale, edgefactor=16, seed=scale, weighted=weighted)
    pg = _native.PreparedGraph(g.V, g.E, g.W)
    r, c, w, d, outw = pg.export_inbound()
    orow, ocol, ow, od, oout = oracle.build_inbound(g.V, g.E, g.W)
    assert np.array_equal(r, orow) and np.array_equal(c, ocol) and np.array_equal(d, od)
    assert np.array_equal(outw.view(np.uint64), oout.view(np.uint64))
    assert np.array_equal(w, ow.astype(np.float32))
    assert pg.info()["n_dangling"] == int(od.sum())


@pytest.mark.parametrize("kind", ["fp32_values", "full_doubles", "mixed_scales"])
def test_out_weight_sums_bit_exact_with_the_sequential_sum(kind):
    """The out-weight sums are taken in parallel where that is provably the
    sequential sum and sequentially elsewhere: bit-identical to the
    reference's sequential FP64 loop (pagerank.cu:301-316) either way, on
    long rows (R-MAT hubs) and for weights that force the sequential path."""
    g = synth.rmat(scale=15, edgefactor=16, seed=41)
    rng = np.random.Generator(np.random.PCG64(41))
    if kind == "fp32_values":  # the synthetic workloads' weights: always order-free
        W = (1.0 - rng.random(g.m, dtype=np.float32)).astype(np.float64)
    elif kind == "full_doubles":  # 53-bit mantissas: long rows need the sequential path
        W = rng.random(g.m)
    else:  # several rows mix weights 2^100 apart, plus zeros, NaN and negatives
        W = rng.random(g.m) * np.where(rng.random(g.m) < 0.5, 2.0**60, 2.0**-40)
        W[rng.random(g.m) < 0.01] = 0.0
        W[rng.random(g.m) < 0.001] = np.nan
        W[rng.random(g.m) < 0.001] = -1.0
    pg = _native.PreparedGraph(g.V, g.E, W)
    _, _, _, _, outw = pg.export_inbound()
    _, _, _, _, oout = oracle.build_inbound(g.V, g.E, W)
    assert np.array_equal(outw.view(np.uint64), oout.view(np.uint64))


@pytest.mark.parametrize("kind", ["unweighted", "fp32_values", "full_doubles", "mixed_scales"])
def test_out_weight_sums_of_huge_rows_bit_exact(kind):
    """Sources of more than 16384 entries are summed in segments by several
    warps: the sums (and unit-weight counts) stay bit-identical to the
    sequential sum, including rows that need the sequential path."""
    rng = np.random.Generator(np.random.PCG64(42))
    n = 1 << 17
    rows = {0: 60000, 1: 20000, 7: 16385, 9: 16384}  # over, at and just past the segment threshold
    V = np.zeros(n + 1, np.int64)
    cols = []
    for u in range(n):
        k = rows.get(u, int(rng.integers(0, 8)))
        cols.append(np.sort(rng.choice(n, k, replace=False)) if k else np.zeros(0, np.int64))
        V[u + 1] = V[u] + k
    E = np.concatenate(cols).astype(np.int32)
    V = V.astype(np.int32)
    m = len(E)
    if kind == "unweighted":
        W = None
    elif kind == "fp32_values":
        W = (1.0 - rng.random(m, dtype=np.float32)).astype(np.float64)
    elif kind == "full_doubles":
        W = rng.random(m)
    else:
        W = rng.random(m) * np.where(rng.random(m) < 0.5, 2.0**60, 2.0**-40)
        W[rng.random(m) < 0.01] = 0.0
        W[rng.random(m) < 0.001] = np.nan
    pg = _native.PreparedGraph(V, E, W)
    r, c, _, _, outw = pg.export_inbound()
    orow, ocol, _, _, oout = oracle.build_inbound(V, E, W)
    assert np.array_equal(outw.view(np.uint64), oout.view(np.uint64))
    assert np.array_equal(r, orow) and np.array_equal(c, ocol)
    ranks, st = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
    _check_against_oracle(V, E, W, ranks, st, 0.85, 100, 1e-6)


@pytest.mark.parametrize("case", golden_small_cases(), ids=lambda c: c[0])
def test_reference_small_cases_through_the_api(case, monkeypatch):
    monkeypatch.setenv("EASYGRAPH_ENABLE_GPU", "TRUE")
    name, G, kw, expected = case
    res = prmod.pagerank(G, **kw)
    assert set(res) == set(expected)
    assert list(res) == list(G.nodes)
    for k, v in expected.items():
        assert res[k] == pytest.approx(v, rel=2e-5, abs=1e-7), (k, res[k], v)
    got = np.array([res[k] for k in expected])
    want = np.array(list(expected.values()))
    assert np.abs(got - want).sum() <= L1_TOL


@pytest.mark.parametrize("case", golden_rmat_cases(), ids=lambda c: c[0])
def test_reference_rmat_vectors(case):
    name, V, E, W, kw, expected = case
    pg = _native.PreparedGraph(V, E, W)
    ranks, stats = pg.pagerank(**kw)
    _check_against_oracle(V, E, W, ranks, stats, kw["alpha"], kw["max_iter"], kw["tol"])


@pytest.mark.parametrize("case", golden_config_cases(), ids=lambda c: c[0])
def test_reference_vectors_of_the_scale14_workload(case):
    # the reference's own ranks on the scale-14 workload (its stop rule, and 20 fixed sweeps)
    name, V, E, W, kw, expected = case
    pg = _native.PreparedGraph(V, E, W)
    ranks, stats = pg.pagerank(**kw)
    _check_against_oracle(V, E, W, ranks, stats, kw["alpha"], kw["max_iter"], kw["tol"])
    _, it_ref, _ = oracle.pagerank_pull(V, E, W, **kw)
    if stats["iterations"] == it_ref:  # the same sweep count as the reference: compare with it directly
        assert np.abs(ranks - expected).sum() <= L1_TOL
        assert np.allclose(ranks, expected, rtol=2e-5, atol=1e-7)


def test_config_scale14_parity():
    # R-MAT scale 14, edgefactor 16, seed 0, alpha 0.85, tol 1e-6, max_iter 100
    g = synth.rmat(scale=14, edgefactor=16, seed=0)
    pg = _native.PreparedGraph(g.V, g.E)
    ranks, stats = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
    _check_against_oracle(g.V, g.E, None, ranks, stats, 0.85, 100, 1e-6)
    assert stats["iterations"] >= 3 and stats["converged"] == 1


@pytest.mark.parametrize("correction", [True, False])
def test_fixed_iterations_scale16(correction):
    g = synth.rmat(scale=16, edgefactor=16, seed=3)
    pg = _native.PreparedGraph(g.V, g.E)
    ranks, stats = pg.pagerank(alpha=0.85, max_iter=20, tol=0.0, correction=correction)
    assert stats["iterations"] == 20 and stats["converged"] == 0
    _check_against_oracle(g.V, g.E, None, ranks, stats, 0.85, 20, 0.0)


def test_weighted_scale14_tight_tol():
    g = synth.rmat(scale=14, edgefactor=16, seed=2, weighted=True)
    pg = _native.PreparedGraph(g.V, g.E, g.W)
    ranks, stats = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-7)
    _check_against_oracle(g.V, g.E, g.W, ranks, stats, 0.85, 100, 1e-7)


def test_deterministic_bit_identical_runs():
    g = synth.rmat(scale=15, edgefactor=16, seed=9)
    pg = _native.PreparedGraph(g.V, g.E)
    a, sa = pg.pagerank(alpha=0.85, max_iter=30, tol=0.0)
    b, sb = pg.pagerank(alpha=0.85, max_iter=30, tol=0.0)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    assert sa["residual"] == sb["residual"]


def test_alpha_is_not_baked_into_the_prepared_graph():
    # tests/test_eggpu_bulk_csr.py:339-377: a new alpha must not reuse old values
    G = DiGraph()
    G.add_nodes(range(7))
    G.add_edges_from([(0, 1), (0, 2), (1, 2), (2, 0), (2, 3), (3, 2), (3, 4), (4, 5), (5, 4), (5, 6)])
    r75 = prmod.pagerank(G, alpha=0.75, max_iter=200, tol=1e-7)
    r90 = prmod.pagerank(G, alpha=0.90, max_iter=200, tol=1e-7)
    V, E, _ = oracle.graph_to_csr(list(G.nodes), G._adj, True)
    for alpha, r in ((0.75, r75), (0.90, r90)):
        ref, _, _ = oracle.pagerank_push(V, E, None, alpha=alpha, max_iter=200, tol=1e-7)
        assert np.allclose(r.to_numpy(), ref, rtol=2e-5, atol=1e-7)


def test_weight_mutation_rebuilds():
    # run_eggpu_gpu_contract_regression.py:83-118
    G = DiGraph()
    for u, v, w in ((0, 1, 8.0), (0, 2, 1.0), (1, 2, 2.0), (2, 0, 1.0)):
        G.add_edge(u, v, weight=w)
    first = dict(prmod.pagerank(G, weight="weight"))
    G[0][1]["weight"] = 0.25
    second = dict(prmod.pagerank(G, weight="weight"))
    V, E, W = oracle.graph_to_csr(list(G.nodes), G._adj, True, "weight")
    ref, _, _ = oracle.pagerank_push(V, E, W)
    assert np.allclose([second[i] for i in range(3)], ref, rtol=5e-5, atol=5e-5)
    assert any(abs(first[i] - second[i]) > 1e-4 for i in range(3))


def test_graphs_isolated_by_identity():
    # run_eggpu_gpu_contract_regression.py:138-146
    a = DiGraph()
    a.add_edges_from([(0, 1), (1, 2), (2, 0), (2, 3)])
    b = DiGraph()
    b.add_edges_from([(0, 1), (1, 0), (1, 2), (3, 2)])
    for G in (a, b, a):
        V, E, _ = oracle.graph_to_csr(list(G.nodes), G._adj, True)
        ref, _, _ = oracle.pagerank_push(V, E)
        assert np.allclose(prmod.pagerank(G).to_numpy(), ref, rtol=5e-5, atol=5e-5)


def test_personalization_matches_oracle_and_networkx():
    V, E, sets, expected = golden_ppr()
    n = V.shape[0] - 1
    pg = _native.PreparedGraph(V, E)
    for j, s in enumerate(sets[:3]):
        p = np.zeros(n)
        p[s] = 1.0
        ranks, stats = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6, personalization=p)
        _check_against_oracle(V, E, None, ranks, stats, 0.85, 100, 1e-6, teleport=p / p.sum())
        conv, _ = pg.pagerank(alpha=0.85, max_iter=300, tol=0.0, personalization=p)
        assert np.abs(conv - expected[j]).sum() <= L1_TOL


def test_personalization_through_the_api():
    G = DiGraph()
    G.add_edges_from([("a", "b"), ("b", "c"), ("c", "a"), ("c", "d")])
    r = prmod.pagerank(G, personalization={"a": 1.0, "d": 3.0})
    V, E, _ = oracle.graph_to_csr(list(G.nodes), G._adj, True)
    ref, _, _ = oracle.pagerank_push(V, E, None, teleport=np.array([0.25, 0, 0, 0.75]))
    assert np.allclose(r.to_numpy(), ref, rtol=2e-5, atol=1e-7)


def test_multi_graph_persistent_launch_matches_single_solves():
    graphs, csrs = [], []
    for i, (n, d) in enumerate(((1000, 8.0), (5000, 20.0), (20000, 12.0), (3000, 32.0), (70000, 9.0))):
        c = synth.erdos_renyi(n, d, seed=1000 + i)
        csrs.append(c)
        graphs.append(_native.PreparedGraph(c.V, c.E))
    outs, stats = _native.pagerank_multi(graphs, alpha=0.85, max_iter=100, tol=1e-6)
    for c, r, st in zip(csrs, outs, stats):
        _check_against_oracle(c.V, c.E, None, r, st, 0.85, 100, 1e-6)
    outs2, _ = _native.pagerank_multi(graphs, alpha=0.85, max_iter=100, tol=1e-6)
    for a, b in zip(outs, outs2):
        assert np.array_equal(a, b)


def test_drop_in_csr_entry_and_its_cache():
    _native.cache_reset()
    g = synth.rmat(scale=12, edgefactor=16, seed=4)
    PR, ks = _native.pagerank_csr(g.V, g.E, None, 77, 0.85, 100, 1e-6)
    st = _native.cache_stats()
    assert st["misses"] == 1 and ks > 0
    PR2, _ = _native.pagerank_csr(g.V, g.E, None, 77, 0.85, 100, 1e-6)
    assert _native.cache_stats()["hits"] == 1
    assert np.array_equal(PR, PR2)
    ref, _, _ = oracle.pagerank_pull(g.V, g.E, None, alpha=0.85, max_iter=100, tol=1e-6)
    assert np.abs(PR - ref).sum() <= L1_TOL
    _native.cache_reset()


def test_enqueue_collect_and_user_stream():
    import torch

    g = synth.rmat(scale=13, edgefactor=16, seed=5)
    pg = _native.PreparedGraph(g.V, g.E)
    want, _ = pg.pagerank(alpha=0.85, max_iter=25, tol=0.0)
    s = torch.cuda.Stream()
    pg.set_stream(s.cuda_stream)
    pg.enqueue(alpha=0.85, max_iter=25, tol=0.0)
    got, st = pg.collect()
    pg.set_stream(None)
    assert np.array_equal(got, want) and st["iterations"] == 25


@pytest.mark.parametrize("name,V,E,W", [
    ("one_selfloop", [0, 1], [0], None),
    ("one_bare", [0, 0], [], None),
    ("no_edges", [0, 0, 0, 0, 0, 0], [], None),
    ("star_dangling", [0, 3, 3, 3, 3], [1, 2, 3], None),
    ("invalid_endpoints", [0, 3, 4, 6], [1, -1, 7, 2, 0, 3], None),
    ("zero_weight_row", [0, 2, 3, 3], [1, 2, 0], [0.0, 0.0, 1.0]),
    ("neg_nan_weights", [0, 2, 4, 5], [1, 2, 0, 2, 0], [-1.0, 2.0, float("nan"), 1.0, 3.0]),
])
def test_edge_cases(name, V, E, W):
    V = np.array(V, np.int32)
    E = np.array(E, np.int32)
    W = None if W is None else np.array(W, np.float64)
    pg = _native.PreparedGraph(V, E, W)
    ranks, stats = pg.pagerank(alpha=0.85, max_iter=50, tol=1e-6)
    n = V.shape[0] - 1
    inb = oracle.build_inbound(V, E, W)
    if inb[0][-1] == 0:
        assert np.allclose(ranks, 1.0 / n) and stats["iterations"] == 0
        return
    ref, it, _ = oracle.pagerank_pull(V, E, W, alpha=0.85, max_iter=50, tol=1e-6, inbound=inb)
    assert abs(stats["iterations"] - it) <= 1
    assert np.abs(ranks - ref).sum() <= L1_TOL
    assert ranks.sum() == pytest.approx(1.0, abs=1e-12)


def test_undirected_and_bulk_paths_agree(tmp_path):
    from eggpu_b200 import bulk

    edges = [(0, 1), (1, 2), (2, 0), (2, 3), (3, 4), (4, 5), (5, 3)]
    G = Graph()
    G.add_nodes(range(6))
    G.add_edges_from(edges)
    rows = [[] for _ in range(6)]
    for u, v in edges:
        rows[u].append(v)
        rows[v].append(u)
    V = np.cumsum([0] + [len(r) for r in rows]).astype(np.int32)
    E = np.array([x for r in rows for x in sorted(r)], np.int32)
    B = bulk.read_eggpu_csr(bulk.write_eggpu_csr(tmp_path, "tiny", V, E, directed=False))
    a = prmod.pagerank(G, alpha=0.75, max_iter=200, tol=1e-6)
    b = prmod.pagerank(B, alpha=0.75, max_iter=200, tol=1e-6)
    assert np.allclose([a[i] for i in range(6)], [b[i] for i in range(6)], rtol=1e-6, atol=1e-8)
    with pytest.raises(NotImplementedError, match="weighted PageRank requires an EGGPU CSR artifact"):
        prmod.pagerank(B, weight="weight")


def test_scale22_full_size_properties_and_parity():
    # the scale-22 workload: R-MAT scale 22, seed 1, reference stop rule -> one sweep at this size
    g = synth.rmat(scale=22, edgefactor=16, seed=1)
    pg = _native.PreparedGraph(g.V, g.E)
    ranks, stats = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
    assert stats["iterations"] == 1 and stats["converged"] == 1
    assert ranks.min() >= 0 and ranks.sum() == pytest.approx(1.0, abs=1e-12)
    ref, it, _ = oracle.pagerank_pull(g.V, g.E, None, alpha=0.85, max_iter=100, tol=1e-6)
    assert it == 1
    assert np.abs(ranks - ref).sum() <= L1_TOL
    fixed, st = pg.pagerank(alpha=0.85, max_iter=5, tol=0.0)
    again, _ = pg.pagerank(alpha=0.85, max_iter=5, tol=0.0)
    assert np.array_equal(fixed, again) and st["iterations"] == 5
    ref5, _, _ = oracle.pagerank_pull(g.V, g.E, None, alpha=0.85, max_iter=5, tol=0.0)
    assert np.abs(fixed - ref5).sum() <= L1_TOL


def test_config_scale25_weighted_precision_full_size():
    """The precision config: R-MAT scale 25 (seed 2, edgefactor 16), weights
    i.i.d. U(0,1] FP32, weighted out-degree normalisation, alpha 0.85, tol
    1e-7.  The stop rule (one sweep at this size, N*tol = 3.36 > 2) and ten
    fixed sweeps with and without the FP64 correction sweep, each against the
    FP64 oracle: iterations within +-1, L1 <= 1e-6 and the reference's
    per-entry tolerance; max-abs and L1 are printed."""
    g = synth.rmat(scale=25, edgefactor=16, seed=2, weighted=True)
    pg = _native.PreparedGraph(g.V, g.E, g.W)
    inbound = oracle.build_inbound(g.V, g.E, g.W)
    for label, max_iter, tol, corr in (("rule_tol1e-7", 100, 1e-7, True), ("fixed10", 10, 0.0, True),
                                       ("fixed10_no_correction", 10, 0.0, False)):
        ranks, st = pg.pagerank(alpha=0.85, max_iter=max_iter, tol=tol, correction=corr)
        ref, it, _ = oracle.pagerank_pull(g.V, g.E, g.W, alpha=0.85, max_iter=max_iter, tol=tol, inbound=inbound)
        assert abs(st["iterations"] - it) <= 1, (label, st["iterations"], it)
        if st["iterations"] != it:
            ref, _, _ = oracle.pagerank_pull(g.V, g.E, g.W, alpha=0.85, max_iter=st["iterations"], tol=0.0,
                                             inbound=inbound)
        l1 = float(np.abs(ranks - ref).sum())
        mx = float(np.abs(ranks - ref).max())
        print(f"scale-25 weighted {label}: iterations {st['iterations']} (oracle {it}), L1 {l1:.3e}, max-abs {mx:.3e}")
        assert l1 <= L1_TOL, (label, l1)
        assert np.allclose(ranks, ref, rtol=2e-5, atol=1e-7), label
        if label == "rule_tol1e-7":
            assert st["converged"] == 1


@pytest.mark.parametrize("case", ["scale14", "scale16w_fixed", "scale15_personalised"])
def test_binned_layout_opt_in_matches_oracle(case, monkeypatch):
    """The degree-binned layout (EGPR_BINS=1: vertices renumbered by hub block
    and in-degree, rows served by length class) gives the oracle's ranks."""
    monkeypatch.setenv("EGPR_BINS", "1")
    if case == "scale14":
        g = synth.rmat(scale=14, edgefactor=16, seed=0)
        pg = _native.PreparedGraph(g.V, g.E)
        ranks, st = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
        _check_against_oracle(g.V, g.E, None, ranks, st, 0.85, 100, 1e-6)
    elif case == "scale16w_fixed":
        g = synth.rmat(scale=16, edgefactor=16, seed=5, weighted=True)
        pg = _native.PreparedGraph(g.V, g.E, g.W)
        for corr in (True, False):
            ranks, st = pg.pagerank(alpha=0.85, max_iter=12, tol=0.0, correction=corr)
            assert st["iterations"] == 12
            _check_against_oracle(g.V, g.E, g.W, ranks, st, 0.85, 12, 0.0)
    else:
        g = synth.rmat(scale=15, edgefactor=16, seed=6)
        pg = _native.PreparedGraph(g.V, g.E)
        tele = _seed_teleport(g.n, np.array([3, 17, 400, 9000]))
        ranks, st = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6, personalization=tele)
        _check_against_oracle(g.V, g.E, None, ranks, st, 0.85, 100, 1e-6, teleport=tele)


def _seed_teleport(n, s):
    p = np.zeros(n)
    p[np.unique(s)] = 1.0
    return p / p.sum()


@pytest.mark.parametrize("weighted", [False, True])
def test_ppr_batch_seed_sets_match_oracle(weighted):
    g = synth.rmat(scale=12, edgefactor=16, seed=31, weighted=weighted)
    sets = synth.seed_sets(g.n, 40, 1, 64, seed=3)  # 40 columns: one full panel and a partial one
    pg = _native.PreparedGraph(g.V, g.E, g.W)
    ranks, stats = pg.pagerank_seeds(sets, alpha=0.85, max_iter=100, tol=1e-6)
    assert ranks.shape == (40, g.n)
    for j in range(0, 40, 3):
        _check_against_oracle(g.V, g.E, g.W, ranks[j], stats[j], 0.85, 100, 1e-6, teleport=_seed_teleport(g.n, sets[j]))
    # the same columns solved one at a time through the plain path
    for j in (0, 33):
        single, st = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6, personalization=_seed_teleport(g.n, sets[j]))
        assert st["iterations"] == stats[j]["iterations"]
        assert np.abs(single - ranks[j]).sum() <= L1_TOL


def test_ppr_batch_fixed_iterations_and_dense_teleport():
    g = synth.rmat(scale=13, edgefactor=16, seed=32)
    rng = np.random.default_rng(0)
    T = rng.random((5, g.n))
    T[1] = 0.0
    T[1, 7] = 2.0
    pg = _native.PreparedGraph(g.V, g.E)
    ranks, stats = pg.pagerank_batch(T, alpha=0.85, max_iter=15, tol=0.0)
    for j in range(5):
        assert stats[j]["iterations"] == 15
        _check_against_oracle(g.V, g.E, None, ranks[j], stats[j], 0.85, 15, 0.0, teleport=T[j] / T[j].sum())


def test_ppr_batch_uniform_column_reproduces_plain_pagerank():
    g = synth.rmat(scale=12, edgefactor=16, seed=33)
    pg = _native.PreparedGraph(g.V, g.E)
    plain, st = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
    ranks, stats = pg.pagerank_batch(np.full((1, g.n), 1.0), alpha=0.85, max_iter=100, tol=1e-6)
    assert stats[0]["iterations"] == st["iterations"]
    assert np.abs(ranks[0] - plain).sum() <= L1_TOL


def test_ppr_batch_is_deterministic_and_columns_independent():
    g = synth.rmat(scale=12, edgefactor=16, seed=34)
    sets = synth.seed_sets(g.n, 64, 1, 16, seed=9)
    pg = _native.PreparedGraph(g.V, g.E)
    a, _ = pg.pagerank_seeds(sets, alpha=0.85, max_iter=30, tol=1e-6)
    b, _ = pg.pagerank_seeds(sets, alpha=0.85, max_iter=30, tol=1e-6)
    assert np.array_equal(a, b)
    held = _native.pinned_empty(a.shape)  # a caller's reused (page-locked) result array
    c, _ = pg.pagerank_seeds(sets, alpha=0.85, max_iter=30, tol=1e-6, out=held)
    assert c is held and np.array_equal(a, c)
    with pytest.raises(ValueError):
        pg.pagerank_seeds(sets, alpha=0.85, max_iter=30, tol=1e-6, out=np.empty((3, g.n)))
    sub, _ = pg.pagerank_seeds(sets[5:9], alpha=0.85, max_iter=30, tol=1e-6)
    assert np.abs(sub - a[5:9]).sum(axis=1).max() <= L1_TOL


def test_ppr_batch_rows_across_many_chunks_and_several_device_groups():
    # vertex 0 has an inbound entry from every other vertex (a row cut into
    # several chunks), and 520 columns need two device solves of 16 panels
    rng = np.random.default_rng(5)
    n = 4000
    src = np.concatenate([np.arange(1, n), rng.integers(0, n, 6000)])
    dst = np.concatenate([np.zeros(n - 1, np.int64), rng.integers(0, n, 6000)])
    keep = src != dst
    pairs = np.unique(np.stack([src[keep], dst[keep]], 1).astype(np.int32), axis=0)  # sorted by source
    V = np.zeros(n + 1, np.int32)
    V[1:] = np.cumsum(np.bincount(pairs[:, 0], minlength=n))
    E = np.ascontiguousarray(pairs[:, 1])
    sets = synth.seed_sets(n, 520, 1, 8, seed=4)
    pg = _native.PreparedGraph(V, E)
    ranks, stats = pg.pagerank_seeds(sets, alpha=0.85, max_iter=100, tol=1e-9)
    assert ranks.shape == (520, n)
    for j in (0, 31, 255, 511, 512, 519):
        _check_against_oracle(V, E, None, ranks[j], stats[j], 0.85, 100, 1e-9, teleport=_seed_teleport(n, sets[j]))


def test_ppr_through_the_api_batch():
    G = DiGraph()
    G.add_edges_from([("a", "b"), ("b", "c"), ("c", "a"), ("c", "d"), ("d", "a")])
    res = prmod.pagerank_batch(G, [{"a": 1.0}, {"d": 1.0, "b": 1.0}])
    V, E, _ = oracle.graph_to_csr(list(G.nodes), G._adj, True)
    for r, p in zip(res, ([1, 0, 0, 0], [0, 0.5, 0, 0.5])):
        ref, _, _ = oracle.pagerank_push(V, E, None, teleport=np.array(p, float))
        assert np.allclose(r.to_numpy(), ref, rtol=2e-5, atol=1e-7)


def test_ppr_config_full_size_k256_rmat20():
    # the batched PPR workload: R-MAT scale 20, seed 3, k = 256 seed sets of 1-64 vertices, at full size
    g = synth.rmat(scale=20, edgefactor=16, seed=3)
    sets = synth.seed_sets(g.n, 256, 1, 64, seed=3)
    pg = _native.PreparedGraph(g.V, g.E)
    for max_iter, tol in ((100, 1e-6), (20, 0.0)):
        ranks, stats = pg.pagerank_seeds(sets, alpha=0.85, max_iter=max_iter, tol=tol)
        assert ranks.shape == (256, g.n) and ranks.min() >= 0.0
        assert np.abs(ranks.sum(axis=1) - 1.0).max() <= 1e-12
        again, _ = pg.pagerank_seeds(sets, alpha=0.85, max_iter=max_iter, tol=tol)
        assert np.array_equal(ranks, again)
        for j in (0, 127, 255):
            _check_against_oracle(g.V, g.E, None, ranks[j], stats[j], 0.85, max_iter, tol,
                                  teleport=_seed_teleport(g.n, sets[j]))


def test_many_graphs_config_full_size_512_er():
    # the many-graphs workload: 512 directed Erdos-Renyi graphs (n log-uniform in [1e3, 2e5], mean
    # out-degree U[8, 32])
    rng = np.random.Generator(np.random.PCG64(1000))
    ns = np.exp(rng.uniform(np.log(1e3), np.log(2e5), size=512)).astype(np.int64)
    ds = rng.uniform(8.0, 32.0, size=512)
    csrs = [synth.erdos_renyi(int(ns[i]), float(ds[i]), seed=1000 + i) for i in range(512)]
    graphs = [_native.PreparedGraph(c.V, c.E) for c in csrs]
    outs, sts = _native.pagerank_multi(graphs, alpha=0.85, max_iter=100, tol=1e-6)
    for o in outs:
        assert o.min() >= 0.0 and abs(o.sum() - 1.0) <= 1e-12
    for i in (0, 1, 255, 510, 511):
        c = csrs[i]
        _check_against_oracle(c.V, c.E, None, outs[i], sts[i], 0.85, 100, 1e-6)
        single, st = graphs[i].pagerank(alpha=0.85, max_iter=100, tol=1e-6)
        assert st["iterations"] == sts[i]["iterations"] and np.abs(single - outs[i]).sum() <= L1_TOL


def test_ppr_few_columns_are_single_vector_solves():
    # fewer than six columns: egpr_pagerank_seeds / _batch run single-vector solves (seed sets uploaded sparse)
    g = synth.rmat(scale=13, edgefactor=16, seed=35)
    sets = synth.seed_sets(g.n, 3, 1, 16, seed=8)
    pg = _native.PreparedGraph(g.V, g.E)
    ranks, stats = pg.pagerank_seeds(sets, alpha=0.85, max_iter=100, tol=1e-6)
    dense, dstats = pg.pagerank_batch(np.stack([_seed_teleport(g.n, s) for s in sets]), alpha=0.85, max_iter=100,
                                      tol=1e-6)
    for j in range(3):
        single, st = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6, personalization=_seed_teleport(g.n, sets[j]))
        assert np.array_equal(ranks[j], single) and np.array_equal(dense[j], single)
        assert stats[j]["iterations"] == st["iterations"] == dstats[j]["iterations"]
        _check_against_oracle(g.V, g.E, None, ranks[j], stats[j], 0.85, 100, 1e-6,
                              teleport=_seed_teleport(g.n, sets[j]))
