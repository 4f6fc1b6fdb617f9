"""Result read-back into pageable host memory: copies of 1 MiB and more go
through the page-locked staging buffers (32 MiB chunks, several in flight);
the bytes must equal a direct copy into page-locked memory, for a single
solve, a batched solve spanning several chunks with a ragged last one, a
session's collected columns, and a destination that is not 16-byte
aligned."""

import numpy as np
import pytest

from eggpu_b200 import _native, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graph():
    g = synth.rmat(scale=20, edgefactor=8, seed=61)
    return g, _native.PreparedGraph(g.V, g.E)


def test_single_solve_pageable_equals_page_locked(graph):
    g, pg = graph
    a, sa = pg.pagerank(alpha=0.85, max_iter=30, tol=0.0, out=_native.pinned_empty(pg.n))
    b, sb = pg.pagerank(alpha=0.85, max_iter=30, tol=0.0, out=np.empty(pg.n))
    assert sa["iterations"] == sb["iterations"] == 30
    assert np.array_equal(a, b)
    raw = np.empty(pg.n + 1)  # an 8-byte offset: not 16-byte aligned
    c, _ = pg.pagerank(alpha=0.85, max_iter=30, tol=0.0, out=raw[1:])
    assert np.array_equal(a, c)


def test_batched_solve_over_several_staging_chunks(graph):
    g, pg = graph
    sets = synth.seed_sets(g.n, 13, 1, 16, seed=62)  # 13 x n x 8 B: four chunks and a ragged tail
    assert 13 * pg.n * 8 > 3 * (32 << 20)
    a, _ = pg.pagerank_seeds(sets, alpha=0.85, max_iter=20, tol=0.0, out=_native.pinned_empty((13, pg.n)))
    b, _ = pg.pagerank_seeds(sets, alpha=0.85, max_iter=20, tol=0.0, out=np.empty((13, pg.n)))
    assert np.array_equal(a, b)
    assert np.all(np.abs(b.sum(axis=1) - 1.0) < 1e-9)


def test_session_collect_pageable_equals_page_locked(graph):
    g, pg = graph
    sets = synth.seed_sets(g.n, 6, 1, 8, seed=63)
    outs = []
    for out in (_native.pinned_empty((6, pg.n)), np.empty((6, pg.n))):
        S = _native.Session(pg, alpha=0.85, tol=0.0, slots=32)
        slots = S.admit(sets, max_iter=12)
        done = []
        while len(done) < 6:
            done += S.step(4)
        order = np.argsort([slots.index(sl) for sl in done])
        r, _ = S.collect([done[i] for i in order], out=out)
        outs.append(r.copy())
        S.close()
    assert np.array_equal(outs[0], outs[1])


def test_result_arrays_of_the_wrong_shape_are_refused(graph):
    g, pg = graph
    for bad in (np.empty(pg.n - 1), np.empty(pg.n, np.float32), np.empty((2, pg.n))[:, 0]):
        with pytest.raises(ValueError):
            pg.pagerank(alpha=0.85, max_iter=5, tol=0.0, out=bad)
    with pytest.raises(ValueError):
        pg.pagerank_seeds([[1, 2]] * 6, alpha=0.85, max_iter=5, tol=0.0, out=np.empty((5, pg.n)))
