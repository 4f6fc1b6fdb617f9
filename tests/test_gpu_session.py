"""Continuous batching of personalised PageRank (egpr_session_*): requests
join a running batched solve in free column slots between steps, leave it
when their own stop rule fires, and their slots are reused.

Bars: every request's ranks equal the same request solved in a one-shot
batched solve (egpr_pagerank_seeds with six or more columns, the same column
arithmetic) to 1e-12 in L1 with the same sweep count, and the FP64 oracle to
the engine's parity bar (L1 <= 1e-6, iterations within +-1); admission in
the middle of a solve, into a panel whose other columns are at another sweep
count, and into reused slots changes none of that."""

import numpy as np
import pytest

from eggpu_b200 import _native, synth
from oracle import oracle

pytestmark = pytest.mark.gpu

L1_TOL = 1e-6


def _tele(n, s):
    p = np.zeros(n)
    p[np.unique(s)] = 1.0
    return p / p.sum()


@pytest.fixture(scope="module")
def graph():
    g = synth.rmat(scale=14, edgefactor=16, seed=51)
    return g, _native.PreparedGraph(g.V, g.E)


def _alone(pg, sets, max_iter, tol):
    """The same requests in one-shot batched solves (at least six columns, so
    the batched path serves them)."""
    pad = list(sets) + [sets[0]] * max(0, 6 - len(sets))
    r, st = pg.pagerank_seeds(pad, alpha=0.85, max_iter=max_iter, tol=tol)
    return r[: len(sets)], st[: len(sets)]


def test_requests_joining_mid_solve_match_their_alone_solves(graph):
    g, pg = graph
    tol = 1e-7
    sets = synth.seed_sets(g.n, 12, 1, 16, seed=52)
    ref, ref_st = _alone(pg, sets, 100, tol)
    S = _native.Session(pg, alpha=0.85, tol=tol, slots=64)
    assert S.slots == 64 and S.info()["free"] == 64
    first = S.admit(sets[:5], max_iter=100)
    got = {}
    stats = {}
    S.step(3)  # the first five are three sweeps in
    second = S.admit(sets[5:], max_iter=100)  # join mid-solve, some in the first requests' panel
    slot_of = dict(zip(first + second, range(12)))
    steps = 0
    while len(got) < 12:
        done = S.step(2)
        steps += 1
        assert steps < 200
        if done:
            out, sts = S.collect(done)
            for i, sl in enumerate(done):
                got[slot_of[sl]] = out[i].copy()
                stats[slot_of[sl]] = sts[i]
    assert S.info()["free"] == 64
    for j in range(12):
        assert stats[j]["iterations"] == ref_st[j]["iterations"], (j, stats[j], ref_st[j])
        assert np.abs(got[j] - ref[j]).sum() <= 1e-12, (j, np.abs(got[j] - ref[j]).sum())
    for j in (0, 7):
        o, it, _ = oracle.pagerank_pull(g.V, g.E, None, alpha=0.85, max_iter=100, tol=tol, teleport=_tele(g.n, sets[j]))
        assert abs(stats[j]["iterations"] - it) <= 1
        assert np.abs(got[j] - o).sum() <= L1_TOL
    S.close()


def test_slots_are_reused_and_columns_keep_their_own_sweep_limits(graph):
    g, pg = graph
    sets = synth.seed_sets(g.n, 40, 1, 8, seed=53)
    S = _native.Session(pg, alpha=0.85, tol=0.0, slots=32)  # tol 0: each column runs to its own limit
    limits = [3 + (j % 9) for j in range(40)]
    pending = list(range(40))
    slot_of, got, stats = {}, {}, {}
    while pending or S.info()["running"] or S.info()["done"]:
        free = S.info()["free"]
        take, pending = pending[:free], pending[free:]
        for j in take:  # one admission per request: each with its own sweep limit
            (sl,) = S.admit([sets[j]], max_iter=limits[j])
            slot_of[sl] = j
        done = S.step(2)
        if done:
            out, sts = S.collect(done, correction=False)
            for i, sl in enumerate(done):
                j = slot_of.pop(sl)
                got[j], stats[j] = out[i].copy(), sts[i]
    assert len(got) == 40 and S.info()["free"] == 32
    for j in (0, 5, 17, 33, 39):
        assert stats[j]["iterations"] == limits[j]
        o, _, _ = oracle.pagerank_pull(g.V, g.E, None, alpha=0.85, max_iter=limits[j], tol=0.0,
                                       teleport=_tele(g.n, sets[j]))
        assert np.abs(got[j] - o).sum() <= L1_TOL, (j, np.abs(got[j] - o).sum())
    S.close()


@pytest.mark.parametrize("sweeps", [2, 3])
def test_waves_admitted_after_columns_stop_inside_a_step(graph, sweeps):
    """Requests arrive three at a time while earlier ones stop part-way
    through a multi-sweep step; each new request joins a panel whose
    remaining columns are at a later sweep than the ones that just stopped,
    in slots freed by collected requests."""
    g, pg = graph
    tol = 1e-6
    sets = synth.seed_sets(g.n, 30, 1, 16, seed=54)
    ref, ref_st = _alone(pg, sets, 100, tol)
    S = _native.Session(pg, alpha=0.85, tol=tol, slots=32)
    pending = list(range(30))
    slot_of, got, stats = {}, {}, {}
    steps = 0
    while pending or S.info()["running"] or S.info()["done"]:
        take, pending = pending[: min(3, S.info()["free"])], pending[min(3, S.info()["free"]):]
        if take:
            for j, sl in zip(take, S.admit([sets[j] for j in take], max_iter=100)):
                slot_of[sl] = j
        done = S.step(sweeps)
        steps += 1
        assert steps < 500
        if done:
            out, sts = S.collect(done)
            for i, sl in enumerate(done):
                j = slot_of.pop(sl)
                got[j], stats[j] = out[i].copy(), sts[i]
    assert len(got) == 30 and S.info()["free"] == 32
    for j in range(30):
        assert stats[j]["iterations"] == ref_st[j]["iterations"], (j, stats[j], ref_st[j])
        assert np.abs(got[j] - ref[j]).sum() <= 1e-12, (j, np.abs(got[j] - ref[j]).sum())
    S.close()


def test_session_refusals(graph):
    g, pg = graph
    S = _native.Session(pg, alpha=0.85, tol=1e-6, slots=32)
    with pytest.raises(_native.EgprError):
        S.admit([[0]] * 33)  # more requests than slots: none admitted
    assert S.info()["free"] == 32
    with pytest.raises(_native.EgprError):
        S.admit([[g.n]])  # a seed outside the graph
    (sl,) = S.admit([[1, 2]])
    with pytest.raises(_native.EgprError):
        S.collect([sl])  # not finished yet
    with pytest.raises(_native.EgprError):
        pg.close()  # a graph with a live session is not destroyed
    assert pg._h is not None
    S.close()
