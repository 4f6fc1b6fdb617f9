"""Continuous-batching request loop for PageRank and personalised PageRank.

Requests (plain PageRank or PPR over a seed set) arrive for graphs held in a
registry.  The server keeps prepared graphs (inbound CSR and rank state) on
the device, admits graphs by HBM bytes with least-recently-used eviction of
idle graphs, and serves requests as they arrive:

* PPR requests waiting for a graph share one one-shot batched solve
  (``egpr_pagerank_seeds``; fewer than six go as single-vector solves), so
  the batch grows with the queue;
* slot-level continuous batching of PPR for long solves on large graphs: a
  graph of at least ``session_min_nnz`` inbound entries with several PPR
  requests waiting whose solves are expected to take many sweeps keeps one
  batched SpMM solve running (``egpr_session``); requests that arrive while it
  runs join it in free column slots between steps of a few sweeps, each
  leaves it (FP64 correction, normalisation, copy out) as soon as its own stop
  rule fires, and its slot is reused.  On B200 this beat one-shot batches for
  60-100-sweep requests on an R-MAT scale-20 graph (p50 -14%, p99 -10% at
  200 req/s) and lost on scale-16/18 graphs, where a step's host round trips
  and each collection's FP64 correction pass outweigh the sweeps;
* queued plain requests for a graph share one solve (their answer is
  identical);
* solves on different graphs run concurrently from a pool of worker threads,
  each prepared graph on its own CUDA stream, so their kernels overlap on the
  device;
* plain requests for several small graphs that are all waiting are folded into
  one persistent multi-graph launch (``egpr_pagerank_multi``).

Every result is the answer the same request gets alone (the batched solve
keeps per-column stop rules and iteration counts); tests/test_serving.py
checks that within the engine's stated tolerance.  Latency is measured from a
request's arrival to the moment its result is on the host.
"""

from __future__ import annotations

import collections
import heapq
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from . import _native


@dataclass
class Request:
    graph: object
    kind: str  # "pr" or "ppr"
    seeds: np.ndarray | None = None
    alpha: float = 0.85
    max_iter: int = 100
    tol: float = 1e-6
    arrival: float = 0.0
    future: Future = field(default_factory=Future)
    done_at: float = 0.0
    iterations: int = 0
    keep_result: bool = True  # False: the future gets (None, stats) once the ranks are on the host


class GraphRegistry:
    """Device-resident prepared graphs, admitted by HBM bytes (LRU eviction of idle graphs)."""

    def __init__(self, sources, budget_bytes, priority_max_n=1_000_000):
        self.sources = dict(sources)  # graph id -> (V, E, W)
        self.budget = int(budget_bytes)
        self.resident = collections.OrderedDict()  # id -> PreparedGraph
        self.busy = collections.Counter()
        self.lock = threading.Condition()
        self.evictions = 0
        self.admissions = 0
        self.loading = {}  # id -> bytes reserved while its graph is prepared (outside the lock)
        # graphs of at most priority_max_n vertices solve on high-priority
        # streams: their kernels take the SMs first whenever a long launch of
        # a large graph ends
        self.priority_max_n = int(priority_max_n)
        self.streams = {}

    def _bytes(self):
        return sum(pg.info()["device_bytes"] for pg in self.resident.values()) + sum(self.loading.values())

    @staticmethod
    def estimate_bytes(V, E, W):
        n = len(V) - 1
        m = len(E)
        return 4 * (n + 1) + 4 * m * (2 if W is not None else 1) + 8 * n + 4 * n + 24 * n + 16 * n + 64 * 1024

    def _prioritize(self, gid, pg):
        if pg.n > self.priority_max_n:
            return
        try:
            import torch

            if not torch.cuda.is_available():
                return
            lo, hi = torch.cuda.Stream.priority_range()
            st = torch.cuda.Stream(priority=min(lo, hi))  # the numerically lowest value is the highest priority
            pg.set_stream(st.cuda_stream)
            self.streams[gid] = st
        except Exception:  # priorities are an optimisation only
            pass

    def _evict(self, gid):
        self.resident.pop(gid).close()
        self.streams.pop(gid, None)
        self.evictions += 1

    def acquire(self, gid):
        """The prepared graph for gid, marked busy; waits for HBM room if needed.
        A graph is prepared outside the lock, so requests for resident graphs
        go on meanwhile."""
        with self.lock:
            while True:
                pg = self.resident.get(gid)
                if pg is not None:
                    self.resident.move_to_end(gid)
                    self.busy[gid] += 1
                    return pg
                if gid in self.loading:  # another thread prepares it
                    self.lock.wait(0.01)
                    continue
                V, E, W = self.sources[gid]
                need = self.estimate_bytes(V, E, W)
                used = self._bytes()
                for victim in list(self.resident):
                    if used + need <= self.budget:
                        break
                    if self.busy[victim] == 0:
                        used -= self.resident[victim].info()["device_bytes"]
                        self._evict(victim)
                if used + need <= self.budget or not (any(self.busy.values()) or self.loading):
                    self.loading[gid] = need
                    break
                self.lock.wait(0.01)
        try:
            pg = _native.PreparedGraph(V, E, W)
        except BaseException:
            with self.lock:
                self.loading.pop(gid, None)
                self.lock.notify_all()
            raise
        with self.lock:
            self._prioritize(gid, pg)
            self.loading.pop(gid, None)
            self.resident[gid] = pg
            self.admissions += 1
            self.busy[gid] += 1
            self.lock.notify_all()
        return pg

    def warm(self, gids):
        """Prepares the given graphs ahead of traffic (as a server loads its
        graphs before it takes requests); returns the seconds it took."""
        t0 = time.perf_counter()
        for gid in gids:
            self.acquire(gid)
            self.release(gid)
        return time.perf_counter() - t0

    def release(self, gid):
        with self.lock:
            self.busy[gid] -= 1
            self.lock.notify_all()

    def close(self):
        with self.lock:
            for pg in self.resident.values():
                pg.close()
            self.resident.clear()
            self.streams.clear()


class Server:
    """Serves Request objects; submit() returns a Future resolving to (ranks, stats)."""

    def __init__(self, registry, workers=4, max_columns=256, multi_max_n=200_000, fold_multi=True, pinned=True,
                 multi_min=8, ppr_min_batch=1, sessions=True, session_slots=256, session_sweeps=4, session_min=6,
                 session_min_sweeps=48, session_min_nnz=8_000_000, session_max_bytes=2 << 30):
        self.registry = registry
        # continuous batching: a graph with at least session_min PPR requests
        # waiting gets a running batched solve (egpr_session) of session_slots
        # column slots; requests join it between steps of session_sweeps sweeps.
        # A sweep of a 32-column panel costs about as much as four or five
        # single-vector sweeps, so fewer waiting requests take one-shot solves
        # (the batched entry's own threshold is six columns as well).
        self.sessions = bool(sessions)
        self.session_slots = int(session_slots)
        self.session_sweeps = int(session_sweeps)
        self.session_min = int(session_min)
        # a session's iterates and results take 16 bytes per slot and vertex:
        # its slots are cut (in panels of 32, at least one) to session_max_bytes
        self.session_max_bytes = int(session_max_bytes)
        # ... and only for requests whose solves are long: a session pays when
        # requests arriving during a solve would otherwise wait for many
        # sweeps.  The expected sweep count is max_iter for fixed-sweep
        # requests (tol 0), else a running mean of the counts seen for the same
        # graph and parameters (unknown: one-shot solves, which record it).
        # session_min_sweeps <= 0 drops the condition.  Graphs of fewer than
        # session_min_nnz inbound entries take one-shot solves: there a step's
        # host round trips and the FP64 correction pass of each collection
        # outweigh the sweeps, and one-shot batches measured faster.
        self.session_min_sweeps = int(session_min_sweeps)
        self.session_min_nnz = int(session_min_nnz)
        self.sweeps_seen = {}  # (graph, alpha, tol) -> running mean of PPR sweep counts
        # PPR groups smaller than this go through the dense single-vector
        # entry one request at a time; otherwise through egpr_pagerank_seeds,
        # which itself solves fewer than six columns as single-vector solves
        # with the seed sets uploaded sparse
        self.ppr_min_batch = int(ppr_min_batch)
        # plain requests of small graphs share one multi-graph launch once at
        # least multi_min such graphs wait (a launch plan over a new set of
        # graphs costs more than a few single solves)
        self.multi_min = int(multi_min)
        # results land in page-locked host arrays (copied at full link speed;
        # the allocator reuses the memory once a result is dropped)
        self.pinned = bool(pinned)
        self.pinned_max_bytes = 64 << 20
        self.max_columns = int(max_columns)
        self.multi_max_n = int(multi_max_n)
        self.fold_multi = fold_multi
        self.queues = collections.defaultdict(collections.deque)  # graph id -> pending requests
        self.running = set()  # graph ids with a solve in flight
        self.cv = threading.Condition()
        self._tls = threading.local()  # per worker thread: a reusable page-locked result buffer
        self.stop = False
        self.stats = collections.Counter()
        self.threads = [threading.Thread(target=self._worker, daemon=True) for _ in range(int(workers))]
        for t in self.threads:
            t.start()

    def submit(self, req: Request) -> Future:
        if not req.arrival:
            req.arrival = time.perf_counter()
        with self.cv:
            self.queues[req.graph].append(req)
            self.cv.notify()
        return req.future

    def close(self):
        with self.cv:
            self.stop = True
            self.cv.notify_all()
        for t in self.threads:
            t.join()

    # -- scheduling ------------------------------------------------------
    def _take_work(self):
        """Picks the graph whose oldest waiting request arrived first; may add small PR-only graphs."""
        best, best_t = None, None
        for gid, q in self.queues.items():
            if q and gid not in self.running:
                t = q[0].arrival
                if best_t is None or t < best_t:
                    best, best_t = gid, t
        if best is None:
            return None
        self.running.add(best)
        reqs = list(self.queues.pop(best))
        work = [(best, reqs)]
        if self.fold_multi and all(r.kind == "pr" for r in reqs) and self._small(best):
            more = [gid for gid, q in self.queues.items()
                    if q and gid not in self.running and all(r.kind == "pr" for r in q) and self._small(gid)]
            if len(more) + 1 >= self.multi_min:
                for gid in more[:63]:
                    self.running.add(gid)
                    work.append((gid, list(self.queues.pop(gid))))
        return work

    def _small(self, gid):
        V = self.registry.sources[gid][0]
        return len(V) - 1 <= self.multi_max_n

    def _worker(self):
        while True:
            with self.cv:
                work = None
                while not self.stop:
                    work = self._take_work()
                    if work is not None:
                        break
                    self.cv.wait(0.005)
                if work is None:
                    return
            try:
                self._run(work)
            except BaseException as exc:  # noqa: BLE001 - delivered to every waiting request
                for _, reqs in work:
                    for r in reqs:
                        if not r.future.done():
                            r.future.set_exception(exc)
            finally:
                with self.cv:
                    for gid, _ in work:
                        self.running.discard(gid)
                    self.cv.notify_all()

    def _finish(self, req, ranks, stats):
        req.done_at = time.perf_counter()
        req.iterations = int(stats["iterations"])
        if req.kind == "ppr":
            key = (req.graph, req.alpha, req.tol)
            old = self.sweeps_seen.get(key)
            self.sweeps_seen[key] = req.iterations if old is None else 0.8 * old + 0.2 * req.iterations
        req.future.set_result((ranks if req.keep_result else None, stats))

    def _session_slots(self, n):
        fit = self.session_max_bytes // (16 * max(int(n), 1)) // 32 * 32
        return max(32, min(self.session_slots, fit))

    def _long_solves(self, gid, r, pg):
        """Whether PPR requests like r on graph gid (prepared as pg) are expected to take at least
        session_min_sweeps sweeps, on a graph large enough for a session to pay."""
        if getattr(pg, "nnz", self.session_min_nnz) < self.session_min_nnz:
            return False
        if self.session_min_sweeps <= 0:
            return True
        expected = r.max_iter if r.tol <= 0 else self.sweeps_seen.get((gid, r.alpha, r.tol))
        return expected is not None and expected >= self.session_min_sweeps

    def _out(self, shape, reqs=()):
        # page-locked up to pinned_max_bytes: pinning a fresh multi-GB block
        # costs more than the faster copy saves.  When none of the requests
        # keeps its result, the worker thread's own page-locked buffer is
        # reused (no allocation, no page-locking on the request's path).
        count = int(np.prod(shape))
        if not (self.pinned and 8 * count <= self.pinned_max_bytes):
            return None
        if any(r.keep_result for r in reqs) or not reqs:
            return _native.pinned_empty(shape)
        buf = getattr(self._tls, "scratch", None)
        if buf is None or buf.size < count:
            buf = _native.pinned_empty(self.pinned_max_bytes // 8)
            self._tls.scratch = buf
        return buf[:count].reshape(shape)

    def _run(self, work):
        if len(work) > 1:
            self._run_multi(work)
            return
        gid, reqs = work[0]
        pg = self.registry.acquire(gid)
        session = None
        try:
            if not self.sessions:
                self._serve_groups(pg, reqs)
                return
            # Continuous batching: while this graph has PPR work, one batched
            # solve stays running; requests that arrive meanwhile join it in free
            # column slots between steps of a few sweeps, and each leaves it as
            # soon as its own stop rule fires.
            running = {}  # slot -> request
            waiting = []  # PPR requests of the session's parameters without a free slot yet
            pending = list(reqs)
            while True:
                with self.cv:  # requests that arrived while this graph was being served
                    more = self.queues.pop(gid, None)
                if more:
                    pending.extend(more)
                ppr = [r for r in pending if r.kind == "ppr"]
                others = [r for r in pending if r.kind != "ppr"]
                pending = []
                if session is None and len(ppr) >= self.session_min and self._long_solves(gid, ppr[0], pg):
                    r0 = ppr[0]
                    session = _native.Session(pg, alpha=r0.alpha, tol=r0.tol, slots=self._session_slots(pg.n))
                    self.stats["sessions"] += 1
                if session is not None:
                    fits = [r for r in ppr if r.alpha == session.alpha and r.tol == session.tol]
                    others += [r for r in ppr if not (r.alpha == session.alpha and r.tol == session.tol)]
                    waiting += fits
                else:
                    others += ppr
                if others:
                    self._serve_groups(pg, others)
                if session is not None:
                    free = session.info()["free"]
                    take, waiting = waiting[:free], waiting[free:]
                    by_iter = collections.defaultdict(list)
                    for r in take:
                        by_iter[r.max_iter].append(r)
                    for max_iter, group in by_iter.items():
                        for sl, r in zip(session.admit([r.seeds for r in group], max_iter=max_iter), group):
                            running[sl] = r
                        self.stats["session_admitted"] += len(group)
                    if running:
                        done = session.step(self.session_sweeps)
                        self.stats["session_steps"] += 1
                        if done:
                            out, sts = session.collect(done, out=self._out((len(done), pg.n), [running[sl] for sl in done]))
                            for i, sl in enumerate(done):
                                self._finish(running.pop(sl), out[i], sts[i])
                if session is None:
                    break  # no running solve: the worker goes back to the scheduler, as the one-shot path does
                if not running and not waiting:
                    with self.cv:
                        if not self.queues.get(gid):
                            break  # nothing left for this graph; later requests start a new round
        finally:
            if session is not None:
                session.close()
            self.registry.release(gid)

    def _serve_groups(self, pg, reqs):
        """Requests served by one-shot solves: plain PageRank (one solve per
        parameter set, shared by its requests), and PPR as single-vector solves
        (small groups) or one batched solve per group."""
        by_params = collections.defaultdict(list)
        for r in reqs:
            by_params[(r.kind, r.alpha, r.max_iter, r.tol)].append(r)
        for (kind, alpha, max_iter, tol), group in by_params.items():
            if kind == "pr":
                ranks, st = pg.pagerank(alpha=alpha, max_iter=max_iter, tol=tol, out=self._out(pg.n, group))
                self.stats["pr_solves"] += 1
                for r in group:
                    self._finish(r, ranks, st)
            elif len(group) < self.ppr_min_batch:
                for r in group:
                    ranks, st = pg.pagerank(alpha=alpha, max_iter=max_iter, tol=tol,
                                            personalization=_teleport(pg.n, r.seeds), out=self._out(pg.n, [r]))
                    self.stats["ppr_single"] += 1
                    self._finish(r, ranks, st)
            else:
                for s in range(0, len(group), self.max_columns):
                    part = group[s:s + self.max_columns]
                    ranks, sts = pg.pagerank_seeds([r.seeds for r in part], alpha=alpha, max_iter=max_iter,
                                                   tol=tol, out=self._out((len(part), pg.n), part))
                    self.stats["ppr_batches"] += 1
                    self.stats["ppr_columns"] += len(part)
                    for j, r in enumerate(part):
                        self._finish(r, ranks[j], sts[j])

    def _run_multi(self, work):
        gids = [gid for gid, _ in work]
        pgs = []
        try:
            for gid in gids:
                pgs.append(self.registry.acquire(gid))
            by_params = collections.defaultdict(list)
            for (gid, reqs), pg in zip(work, pgs):
                for r in reqs:
                    by_params[(r.alpha, r.max_iter, r.tol)].append((pg, r))
            for (alpha, max_iter, tol), items in by_params.items():
                uniq = list(dict.fromkeys(pg for pg, _ in items))
                outs, sts = _native.pagerank_multi(uniq, alpha=alpha, max_iter=max_iter, tol=tol)
                self.stats["multi_launches"] += 1
                self.stats["multi_graphs"] += len(uniq)
                res = {id(pg): (o, s) for pg, o, s in zip(uniq, outs, sts)}
                for pg, r in items:
                    o, s = res[id(pg)]
                    self._finish(r, o, s)
        finally:
            for gid in gids[:len(pgs)]:
                self.registry.release(gid)


def _teleport(n, seeds):
    """Uniform teleport vector over a seed set (the batched solve's column)."""
    p = np.zeros(n)
    p[np.unique(np.asarray(seeds, np.int64))] = 1.0
    return p / p.sum()


def poisson_arrivals(rate, count, seed):
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=count))


def replay(server, requests, times):
    """Submits requests at the given offsets (seconds from now); returns when all are done."""
    t0 = time.perf_counter()
    for req, t in zip(requests, times):
        delay = t0 + t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        req.arrival = time.perf_counter()
        server.submit(req)
    for req in requests:
        req.future.result()
    return time.perf_counter() - t0


def latency_summary(requests):
    lat = np.array([r.done_at - r.arrival for r in requests])
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "max_ms": float(lat.max() * 1e3), "count": int(lat.size)}
