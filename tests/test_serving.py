"""Serving loop: scheduling and admission on CPU with a fake native engine,
and on the GPU that every request's answer in the mix equals its answer alone."""

import threading
import time

import numpy as np
import pytest

from eggpu_b200 import _native, serving, synth
from oracle import oracle


class FakePrepared:
    """Stands in for _native.PreparedGraph: answers with the oracle, records calls."""

    calls = []
    live = 0
    lock = threading.Lock()

    def __init__(self, V, E, W=None):
        self.V, self.E, self.W = V, E, W
        self.n = len(V) - 1
        self.nnz = len(E)
        with FakePrepared.lock:
            FakePrepared.live += 1

    def info(self):
        return {"device_bytes": serving.GraphRegistry.estimate_bytes(self.V, self.E, self.W)}

    def pagerank(self, alpha, max_iter, tol, personalization=None, out=None):
        FakePrepared.calls.append(("pr", self.n))
        time.sleep(0.002)
        r, it, res = oracle.pagerank_push(self.V, self.E, self.W, alpha=alpha, max_iter=max_iter, tol=tol,
                                          teleport=personalization)
        if out is not None:
            out[:] = r
            r = out
        return r, {"iterations": it}

    def pagerank_seeds(self, seed_sets, alpha, max_iter, tol, out=None):
        FakePrepared.calls.append(("ppr", self.n, len(seed_sets)))
        time.sleep(0.002)
        outs, sts = [], []
        for s in seed_sets:
            p = np.zeros(self.n)
            p[np.unique(s)] = 1.0
            r, it, _ = oracle.pagerank_push(self.V, self.E, self.W, alpha=alpha, max_iter=max_iter, tol=tol,
                                            teleport=p / p.sum())
            outs.append(r)
            sts.append({"iterations": it})
        if out is not None:
            out[:] = np.array(outs)
            return out, sts
        return np.array(outs), sts

    def close(self):
        with FakePrepared.lock:
            FakePrepared.live -= 1


class FakeSession:
    """Stands in for _native.Session: a request's answer comes from the oracle
    when it is admitted and it finishes after ceil(iterations / sweeps) steps;
    admissions and steps are recorded in order."""

    def __init__(self, graph, alpha=0.85, tol=1e-6, slots=32):
        self.g, self.alpha, self.tol, self.slots, self.n = graph, alpha, tol, slots, graph.n
        self.cols = {}  # slot -> [ranks, stats, steps left]
        FakePrepared.calls.append(("session", self.n))

    def info(self):
        running = sum(1 for c in self.cols.values() if c[2] > 0)
        done = len(self.cols) - running
        return {"slots": self.slots, "running": running, "done": done, "free": self.slots - len(self.cols)}

    def admit(self, seed_sets, max_iter=100):
        free = [j for j in range(self.slots) if j not in self.cols][: len(seed_sets)]
        assert len(free) == len(seed_sets)
        for j, s in zip(free, seed_sets):
            p = np.zeros(self.n)
            p[np.unique(s)] = 1.0
            r, it, _ = oracle.pagerank_push(self.g.V, self.g.E, self.g.W, alpha=self.alpha, max_iter=max_iter,
                                            tol=self.tol, teleport=p / p.sum())
            self.cols[j] = [r, {"iterations": it}, it]
        FakePrepared.calls.append(("admit", self.n, len(seed_sets)))
        return free

    def step(self, sweeps=4):
        FakePrepared.calls.append(("step", self.n))
        time.sleep(0.002)
        for c in self.cols.values():
            c[2] = max(0, c[2] - sweeps)
        return [j for j, c in self.cols.items() if c[2] == 0]

    def collect(self, slots, out=None):
        rows = np.array([self.cols[j][0] for j in slots])
        sts = [self.cols.pop(j)[1] for j in slots]
        if out is not None:
            out[:] = rows
            return out, sts
        return rows, sts

    def close(self):
        pass


def fake_multi(graphs, alpha, max_iter, tol):
    FakePrepared.calls.append(("multi", len(graphs)))
    outs, sts = [], []
    for g in graphs:
        r, st = g.pagerank(alpha, max_iter, tol)
        outs.append(r)
        sts.append(st)
    return outs, sts


@pytest.fixture
def fake_engine(monkeypatch):
    FakePrepared.calls = []
    FakePrepared.live = 0
    monkeypatch.setattr(_native, "PreparedGraph", FakePrepared)
    monkeypatch.setattr(_native, "pagerank_multi", fake_multi)
    monkeypatch.setattr(_native, "Session", FakeSession)
    yield


def _sources(k=5):
    out = {}
    for i in range(k):
        c = synth.erdos_renyi(200 + 150 * i, 6.0, seed=2000 + i)
        out[i] = (c.V, c.E, None)
    return out


def test_requests_are_folded_and_answers_match_standalone(fake_engine):
    src = _sources()
    reg = serving.GraphRegistry(src, budget_bytes=1 << 40)
    srv = serving.Server(reg, workers=2, ppr_min_batch=2, sessions=True, session_min=2, session_min_sweeps=0,
                         session_min_nnz=0)
    rng = np.random.default_rng(0)
    reqs = []
    for i in range(60):
        gid = int(rng.integers(0, len(src)))
        if i % 2:
            reqs.append(serving.Request(gid, "ppr", seeds=rng.choice(src[gid][0].shape[0] - 1, 3, replace=False)))
        else:
            reqs.append(serving.Request(gid, "pr"))
    for r in reqs:  # a burst: everything arrives at once
        srv.submit(r)
    for r in reqs:
        ranks, st = r.future.result(timeout=60)
        V, E, W = src[r.graph]
        tele = None
        if r.kind == "ppr":
            p = np.zeros(V.shape[0] - 1)
            p[np.unique(r.seeds)] = 1.0
            tele = p / p.sum()
        alone, it, _ = oracle.pagerank_push(V, E, W, teleport=tele)
        assert np.array_equal(ranks, alone) and st["iterations"] == it
    srv.close()
    solves = [c for c in FakePrepared.calls if c[0] in ("pr", "ppr", "admit")]
    assert len(solves) < len(reqs)  # folding happened
    assert any(c[0] == "admit" and c[2] > 1 for c in solves)  # several PPR requests joined one batched solve
    lat = serving.latency_summary(reqs)
    assert lat["count"] == 60 and lat["p99_ms"] >= lat["p50_ms"]


@pytest.mark.parametrize("multi_min,expect_multi", [(2, True), (100, False)])
def test_plain_requests_of_small_graphs_share_a_launch_past_a_threshold(fake_engine, multi_min, expect_multi):
    src = _sources()
    reg = serving.GraphRegistry(src, budget_bytes=1 << 40)
    srv = serving.Server(reg, workers=1, multi_min=multi_min)
    gate = threading.Event()
    first = serving.Request(0, "pr")
    orig = srv._run

    def held(work):  # the first solve waits until the others have queued up
        gate.wait(10)
        orig(work)

    srv._run = held
    srv.submit(first)
    time.sleep(0.05)
    reqs = [serving.Request(gid, "pr") for gid in (1, 2, 3, 4)]
    for r in reqs:
        srv.submit(r)
    gate.set()
    for r in [first] + reqs:
        ranks, st = r.future.result(timeout=60)
        alone, it, _ = oracle.pagerank_push(*src[r.graph])
        assert np.array_equal(ranks, alone) and st["iterations"] == it
    srv.close()
    assert any(c[0] == "multi" for c in FakePrepared.calls) == expect_multi
    reg.close()


def test_a_few_ppr_requests_are_solved_one_by_one(fake_engine):
    src = _sources()
    reg = serving.GraphRegistry(src, budget_bytes=1 << 40)
    srv = serving.Server(reg, workers=1, ppr_min_batch=4, sessions=False)
    rng = np.random.default_rng(1)
    reqs = [serving.Request(2, "ppr", seeds=rng.choice(src[2][0].shape[0] - 1, 3, replace=False)) for _ in range(3)]
    for r in reqs:
        srv.submit(r)
    for r in reqs:
        ranks, st = r.future.result(timeout=60)
        V, E, W = src[2]
        p = np.zeros(V.shape[0] - 1)
        p[np.unique(r.seeds)] = 1.0
        alone, it, _ = oracle.pagerank_push(V, E, W, teleport=p / p.sum())
        assert np.array_equal(ranks, alone) and st["iterations"] == it
    srv.close()
    assert not any(c[0] == "ppr" for c in FakePrepared.calls)
    assert srv.stats["ppr_single"] == 3
    reg.close()


def test_requests_arriving_mid_solve_join_the_running_batched_solve(fake_engine):
    """Continuous batching: PPR requests that arrive while a graph's batched
    solve is running are admitted into it between steps (no waiting for the
    running requests to finish), and every answer is its answer alone."""
    src = _sources()
    reg = serving.GraphRegistry(src, budget_bytes=1 << 40)
    srv = serving.Server(reg, workers=1, session_sweeps=2, sessions=True, session_min=2, session_min_sweeps=0,
                         session_min_nnz=0)
    rng = np.random.default_rng(4)
    n = src[3][0].shape[0] - 1
    early = [serving.Request(3, "ppr", seeds=rng.choice(n, 3, replace=False), max_iter=200, tol=1e-9)
             for _ in range(3)]
    late = [serving.Request(3, "ppr", seeds=rng.choice(n, 2, replace=False), max_iter=200, tol=1e-9)
            for _ in range(4)]
    for r in early:
        srv.submit(r)
    while not any(c[0] == "step" for c in FakePrepared.calls):
        time.sleep(0.001)
    for r in late:  # the early requests are on the device now
        srv.submit(r)
    for r in early + late:
        ranks, st = r.future.result(timeout=60)
        p = np.zeros(n)
        p[np.unique(r.seeds)] = 1.0
        alone, it, _ = oracle.pagerank_push(*src[3], teleport=p / p.sum(), max_iter=200, tol=1e-9)
        assert np.array_equal(ranks, alone) and st["iterations"] == it
    srv.close()
    events = [c[0] for c in FakePrepared.calls if c[0] in ("session", "admit", "step")]
    assert events.count("session") == 1  # one running solve served both waves
    first_admit, second_admit = [i for i, e in enumerate(events) if e == "admit"][:2]
    assert "step" in events[first_admit:second_admit]  # the second wave joined after the solve had started
    assert max(r.done_at for r in early) > min(r.arrival for r in late)  # ... while the first wave was running
    reg.close()


def test_sessions_open_only_for_long_solves(fake_engine):
    """A burst of short solves (a stop rule whose sweep count is not known yet,
    or is known to be short) takes one-shot batched solves; fixed-sweep
    requests of at least session_min_sweeps sweeps open a session, unless the
    graph has fewer than session_min_nnz inbound entries."""
    src = _sources()
    reg = serving.GraphRegistry(src, budget_bytes=1 << 40)
    srv = serving.Server(reg, workers=1, sessions=True, session_min=2, session_min_sweeps=32, session_min_nnz=0)
    rng = np.random.default_rng(5)
    n = src[1][0].shape[0] - 1

    def burst(**kw):
        FakePrepared.calls = []
        reqs = [serving.Request(1, "ppr", seeds=rng.choice(n, 2, replace=False), **kw) for _ in range(8)]
        for r in reqs:
            srv.submit(r)
        for r in reqs:
            r.future.result(timeout=60)
        return [c[0] for c in FakePrepared.calls]

    assert "session" not in burst(tol=1e-6)  # nothing known yet
    assert srv.sweeps_seen[(1, 0.85, 1e-6)] < 32
    assert "session" not in burst(tol=1e-6)  # known to be short
    assert "session" not in burst(tol=0.0, max_iter=8)  # fixed and short
    assert "session" in burst(tol=0.0, max_iter=40)  # fixed and long
    srv.close()
    srv = serving.Server(reg, workers=1, sessions=True, session_min=2, session_min_sweeps=32,
                         session_min_nnz=10**9)
    assert "session" not in burst(tol=0.0, max_iter=40)  # long, but on a graph too small for a session
    srv.close()
    reg.close()


def test_admission_by_bytes_evicts_idle_graphs(fake_engine):
    src = _sources()
    sizes = [serving.GraphRegistry.estimate_bytes(*src[i]) for i in src]
    reg = serving.GraphRegistry(src, budget_bytes=max(sizes) * 2 + 1)
    for gid in list(src) * 2:
        pg = reg.acquire(gid)
        assert pg is reg.resident[gid]
        assert sum(g.info()["device_bytes"] for g in reg.resident.values()) <= reg.budget
        reg.release(gid)
    assert reg.evictions > 0 and FakePrepared.live == len(reg.resident) <= 2
    reg.close()


def test_poisson_arrivals_are_seeded():
    a = serving.poisson_arrivals(1000.0, 500, seed=1)
    assert np.array_equal(a, serving.poisson_arrivals(1000.0, 500, seed=1))
    assert 0.3 < a[-1] < 0.7 and np.all(np.diff(a) > 0)


@pytest.mark.gpu
def test_served_results_equal_standalone_results_on_gpu():
    src = {}
    for i, (scale, ef) in enumerate(((10, 8), (12, 16), (13, 12), (11, 32))):
        c = synth.rmat(scale=scale, edgefactor=ef, seed=2000 + i)
        src[i] = (c.V, c.E, None)
    reg = serving.GraphRegistry(src, budget_bytes=1 << 34)
    # batched, session and single PPR solves all occur
    srv = serving.Server(reg, workers=3, ppr_min_batch=2, sessions=True, session_min=2, session_min_sweeps=0,
                         session_min_nnz=0)
    rng = np.random.default_rng(1)
    reqs = []
    for i in range(300):
        gid = int(rng.integers(0, len(src)))
        n = src[gid][0].shape[0] - 1
        if i % 2:
            reqs.append(serving.Request(gid, "ppr", seeds=rng.choice(n, int(rng.integers(1, 17)), replace=False)))
        else:
            reqs.append(serving.Request(gid, "pr"))
    times = serving.poisson_arrivals(2000.0, len(reqs), seed=2)
    serving.replay(srv, reqs, times)
    srv.close()
    alone = {gid: _native.PreparedGraph(*src[gid]) for gid in src}
    for r in reqs:
        ranks, st = r.future.result()
        pg = alone[r.graph]
        if r.kind == "pr":
            ref, rst = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
        else:
            p = np.zeros(pg.n)
            p[np.unique(r.seeds)] = 1.0
            ref, rst = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6, personalization=p)
        assert abs(st["iterations"] - rst["iterations"]) <= 1
        assert np.abs(ranks - ref).sum() <= 1e-6
    assert srv.stats["ppr_columns"] >= srv.stats["ppr_batches"]
    reg.close()


def test_dropped_results_reuse_the_worker_buffer(fake_engine):
    """Results nobody keeps land in the worker thread's own reusable buffer;
    a kept result always gets an array of its own."""
    src = _sources()
    reg = serving.GraphRegistry(src, budget_bytes=1 << 40)
    srv = serving.Server(reg, workers=1)
    dropped = [serving.Request(0, "pr", keep_result=False) for _ in range(2)]
    kept = [serving.Request(0, "pr") for _ in range(2)]
    a = srv._out((3, 100), dropped)
    b = srv._out(100, dropped[:1])
    assert np.shares_memory(a, b)  # the same buffer, reshaped
    c = srv._out(100, kept)
    d = srv._out(100, dropped + kept[:1])
    assert not np.shares_memory(c, a) and not np.shares_memory(d, a) and not np.shares_memory(c, d)
    for r in dropped + kept:
        srv.submit(r)
    for r in dropped:
        ranks, st = r.future.result(timeout=60)
        assert ranks is None and st["iterations"] > 0
    for r in kept:
        ranks, _ = r.future.result(timeout=60)
        assert ranks is not None and np.isclose(ranks.sum(), 1.0)
    srv.close()
    reg.close()
