"""Per-graph work-layout tuning (egpr_graph_autotune / egpr_graph_set_tuning):
the chosen layout is one of the candidates, and results under any layout stay
within the engine's parity bar against the FP64 oracle."""

import numpy as np
import pytest

from eggpu_b200 import _native, synth
from oracle import oracle

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


def _seed_teleport(n, s):
    p = np.zeros(n)
    p[np.unique(s)] = 1.0
    return p / p.sum()


def test_autotune_picks_a_candidate_and_keeps_results():
    g = synth.rmat(scale=14, edgefactor=16, seed=41)
    pg = _native.PreparedGraph(g.V, g.E)
    before, st0 = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
    t = pg.autotune()
    assert t["chunks_per_warp"] in (4, 8, 16) and t["row_cost"] in (2, 4, 8)
    assert t["spmm_chunk"] in (512, 1024, 2048)
    assert t["configs_tried"] == 12 and t["sweep_ms"] > 0 and t["spmm_sweep_ms"] > 0
    assert pg.tuning() == {k: t[k] for k in ("chunks_per_warp", "row_cost", "spmm_chunk")}
    after, st1 = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
    ref, it, _ = oracle.pagerank_pull(g.V, g.E, None, alpha=0.85, max_iter=100, tol=1e-6)
    assert abs(st1["iterations"] - it) <= 1
    assert np.abs(after - ref).sum() <= L1_TOL
    assert np.abs(after - before).sum() <= L1_TOL
    sets = synth.seed_sets(g.n, 40, 1, 16, seed=5)
    ranks, sts = pg.pagerank_seeds(sets, alpha=0.85, max_iter=100, tol=1e-6)
    for j in (0, 39):
        ref, it, _ = oracle.pagerank_pull(g.V, g.E, None, alpha=0.85, max_iter=100, tol=1e-6,
                                          teleport=_seed_teleport(g.n, sets[j]))
        assert abs(sts[j]["iterations"] - it) <= 1
        assert np.abs(ranks[j] - ref).sum() <= L1_TOL


@pytest.mark.parametrize("cpw,rc,chunk", [(1, 0, 64), (64, 64, 4096), (3, 7, 96)])
def test_any_valid_layout_gives_the_same_answer(cpw, rc, chunk):
    g = synth.rmat(scale=13, edgefactor=12, seed=42, weighted=True)
    pg = _native.PreparedGraph(g.V, g.E, g.W)
    pg.set_tuning(chunks_per_warp=cpw, row_cost=rc, spmm_chunk=chunk)
    assert pg.tuning() == {"chunks_per_warp": cpw, "row_cost": rc, "spmm_chunk": chunk}
    ranks, st = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
    ref, it, _ = oracle.pagerank_pull(g.V, g.E, g.W, alpha=0.85, max_iter=100, tol=1e-6)
    assert abs(st["iterations"] - it) <= 1 and np.abs(ranks - ref).sum() <= L1_TOL
    sets = synth.seed_sets(g.n, 33, 1, 8, seed=6)
    b, sts = pg.pagerank_seeds(sets, alpha=0.85, max_iter=100, tol=1e-6)
    for j in (0, 32):
        ref, it, _ = oracle.pagerank_pull(g.V, g.E, g.W, alpha=0.85, max_iter=100, tol=1e-6,
                                          teleport=_seed_teleport(g.n, sets[j]))
        assert abs(sts[j]["iterations"] - it) <= 1 and np.abs(b[j] - ref).sum() <= L1_TOL


def test_out_of_range_tuning_is_refused():
    g = synth.rmat(scale=10, edgefactor=8, seed=43)
    pg = _native.PreparedGraph(g.V, g.E)
    for kw in ({"chunks_per_warp": 0}, {"row_cost": 65}, {"spmm_chunk": 100}, {"spmm_chunk": 32}):
        with pytest.raises(_native.EgprError):
            pg.set_tuning(**kw)
    assert pg.tuning()["spmm_chunk"] in (512, 1024, 2048) or pg.tuning()["spmm_chunk"] % 32 == 0


def test_autotune_choice_is_recorded_and_applied_to_new_graphs(tmp_path, monkeypatch):
    """egpr_graph_autotune records its choice per GPU model and graph-shape
    bucket; a graph of the same bucket prepared later starts with it."""
    store = tmp_path / "tuning.txt"
    monkeypatch.setenv("EGPR_TUNE_CACHE", str(store))
    for name in ("EGPR_CHUNKS_PER_WARP", "EGPR_ROW_COST", "EGPR_SPMM_CHUNK"):
        monkeypatch.delenv(name, raising=False)
    g = synth.rmat(scale=14, edgefactor=16, seed=44)
    pg = _native.PreparedGraph(g.V, g.E)
    pg.autotune(sweep=True, spmm=False)
    lines = store.read_text().splitlines()
    assert len(lines) == 1 and "|n2^14|" in lines[0] and lines[0].split()[0].endswith("|w0")
    # a recorded choice unlike the defaults, to see it applied
    key = lines[0].split()[0]
    store.write_text(f"{key} 16 2 512 0.01\n")
    h = synth.rmat(scale=14, edgefactor=16, seed=45)  # another graph of the same shape bucket
    ph = _native.PreparedGraph(h.V, h.E)
    assert ph.tuning() == {"chunks_per_warp": 16, "row_cost": 2, "spmm_chunk": 512}
    ranks, st = ph.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
    ref, it, _ = oracle.pagerank_pull(h.V, h.E, None, alpha=0.85, max_iter=100, tol=1e-6)
    assert abs(st["iterations"] - it) <= 1 and np.abs(ranks - ref).sum() <= L1_TOL
    # a weighted graph is another bucket; the store switched off gives the defaults
    w = synth.rmat(scale=14, edgefactor=16, seed=45, weighted=True)
    assert _native.PreparedGraph(w.V, w.E, w.W).tuning() != {"chunks_per_warp": 16, "row_cost": 2,
                                                            "spmm_chunk": 512}
    monkeypatch.setenv("EGPR_TUNE_CACHE", "0")
    assert _native.PreparedGraph(h.V, h.E).tuning() != {"chunks_per_warp": 16, "row_cost": 2, "spmm_chunk": 512}
