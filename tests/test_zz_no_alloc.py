"""egpr_pagerank_device_noalloc: PageRank for callers that may not call
cudaMalloc (a framework that owns device memory through its own pool, a
serving thread with a fixed memory budget, a plug-in whose host forbids
allocations during a request).  The caller hands over device pointers to the
inbound CSR, the out-weights and the result; the solve's own buffers live in a
fixed array compiled into the library, which limits n to 262144.

The entry point is called through the C ABI with torch-owned device memory and
compared with the prepared-graph solve egpr_pagerank on the same graph and
with the FP64 oracle, twice in a row (the second call runs on the scratch the
first one left behind); also without the FP64 correction sweep, on a side
stream, and without a stats struct.  This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 262144
L1_TOL = 1e-6  # the parity bar of the prepared-graph solve against the oracle


def _noalloc(lib, n, nnz, in_row, in_col, in_w, outw, out, alpha, max_iter, tol, flags, stats, stream=None):
    ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    return lib.egpr_pagerank_device_noalloc(n, nnz, ptr(in_row), ptr(in_col), ptr(in_w), ptr(outw), alpha,
                                            max_iter, tol, flags, ptr(out),
                                            ctypes.c_void_p(stream) if stream else None,
                                            ctypes.byref(stats) if stats is not None else None)


def _device_inputs(pg, weighted):
    import torch

    in_row, in_col, in_w, _dang, outw = pg.export_inbound()
    dev = torch.device("cuda", 0)
    d_row = torch.from_numpy(np.ascontiguousarray(in_row, np.int32)).to(dev)
    d_col = torch.from_numpy(np.ascontiguousarray(in_col, np.int32)).to(dev)
    d_w = torch.from_numpy(np.ascontiguousarray(in_w, np.float32)).to(dev) if weighted else None
    d_outw = torch.from_numpy(np.ascontiguousarray(outw, np.float64)).to(dev)
    return int(in_row[-1]), d_row, d_col, d_w, d_outw


@pytest.mark.parametrize("weighted", [False, True])
def test_noalloc_matches_prepared_solve_on_two_calls_in_a_row(weighted):
    import torch

    from eggpu_b200 import _native, synth
    from oracle import oracle

    g = synth.rmat(scale=14, edgefactor=16, seed=11, weighted=weighted)
    pg = _native.PreparedGraph(g.V, g.E, g.W)
    ref, ref_stats = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
    orc, orc_it, _ = oracle.pagerank_pull(g.V, g.E, g.W, alpha=0.85, max_iter=100, tol=1e-6)
    n = g.n
    nnz, d_row, d_col, d_w, d_outw = _device_inputs(pg, weighted)
    out = torch.empty(n, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    for call in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        st = _native.EgprStats()
        rc = _noalloc(_native.lib, n, nnz, d_row, d_col, d_w, d_outw, out, 0.85, 100, 1e-6, 0, st)
        assert rc == _native.EGPR_SUCC, (call, _native.lib.egpr_last_error())
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), call
        assert np.abs(got - ref).sum() <= L1_TOL, (call, np.abs(got - ref).sum())
        assert np.allclose(got, ref, rtol=2e-5, atol=1e-7), call
        assert abs(st.iterations - ref_stats["iterations"]) <= 1, (call, st.iterations, ref_stats["iterations"])
        assert abs(st.iterations - orc_it) <= 1, (call, st.iterations, orc_it)
        assert np.abs(got - orc).sum() <= L1_TOL, (call, np.abs(got - orc).sum())
        assert st.converged == 1
        # device time from the GPU's global timer: positive and below the host wall time
        assert 0.0 < st.kernel_seconds <= st.total_seconds + 1e-3, (st.kernel_seconds, st.total_seconds)


def test_noalloc_without_correction_on_a_side_stream_and_without_stats():
    import torch

    from eggpu_b200 import _native, synth
    from oracle import oracle

    g = synth.rmat(scale=13, edgefactor=16, seed=12)
    pg = _native.PreparedGraph(g.V, g.E)
    n = g.n
    nnz, d_row, d_col, d_w, d_outw = _device_inputs(pg, False)
    side = torch.cuda.Stream()
    # 1. no FP64 correction sweep: the normalised last FP32 iterate, as egpr_pagerank gives it
    ref_nc, st_nc = pg.pagerank(alpha=0.85, max_iter=12, tol=0.0, correction=False)
    orc12, _, _ = oracle.pagerank_pull(g.V, g.E, None, alpha=0.85, max_iter=12, tol=0.0)
    out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    st = _native.EgprStats()
    rc = _noalloc(_native.lib, n, nnz, d_row, d_col, d_w, d_outw, out, 0.85, 12, 0.0,
                  _native.EGPR_FLAG_NO_CORRECTION, st, stream=side.cuda_stream)
    assert rc == _native.EGPR_SUCC, _native.lib.egpr_last_error()
    got = out.cpu().numpy()
    assert st.iterations == 12 and st_nc["iterations"] == 12
    assert np.abs(got - ref_nc).sum() <= L1_TOL, np.abs(got - ref_nc).sum()
    assert np.abs(got - orc12).sum() <= L1_TOL, np.abs(got - orc12).sum()
    # 2. no stats struct: the call only enqueues; the side stream orders the read
    out2 = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    rc = _noalloc(_native.lib, n, nnz, d_row, d_col, d_w, d_outw, out2, 0.85, 100, 1e-6, 0, None,
                  stream=side.cuda_stream)
    assert rc == _native.EGPR_SUCC, _native.lib.egpr_last_error()
    side.synchronize()
    ref, _ = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
    got2 = out2.cpu().numpy()
    assert np.all(np.isfinite(got2))
    assert np.abs(got2 - ref).sum() <= L1_TOL, np.abs(got2 - ref).sum()


def test_noalloc_rejects_graphs_beyond_its_scratch():
    from eggpu_b200 import _native

    st = _native.EgprStats()
    rc = _native.lib.egpr_pagerank_device_noalloc(LIMIT + 1, 0, None, None, None, None, 0.85, 10, 1e-6, 0, None,
                                                  None, ctypes.byref(st))
    assert rc == _native.EGPR_INVALID_ARGUMENT
    assert b"262144" in _native.lib.egpr_last_error()
