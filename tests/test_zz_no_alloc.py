"""egpr_pagerank_device_noalloc: PageRank for callers that may not call
cudaMalloc (a framework that owns device memory through its own pool, a
serving thread with a fixed memory budget, a plug-in whose host forbids
allocations during a request).  The caller hands over device pointers to the
inbound CSR, the out-weights and the result; the solve's own buffers live in a
fixed array compiled into the library, which limits n to 262144.

The entry point is called through the C ABI with torch-owned device memory and
compared with the prepared-graph solve egpr_pagerank on the same graph, twice
in a row (the second call runs on the scratch the first one left behind).
This file is collected last on purpose.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 262144
L1_TOL = 1e-6  # the parity bar of the prepared-graph solve against the oracle


def _noalloc(lib, n, nnz, in_row, in_col, in_w, outw, out, alpha, max_iter, tol, flags, stats):
    from eggpu_b200 import _native

    ptr = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    return lib.egpr_pagerank_device_noalloc(n, nnz, ptr(in_row), ptr(in_col), ptr(in_w), ptr(outw), alpha,
                                            max_iter, tol, flags, ptr(out), None,
                                            ctypes.byref(stats) if stats is not None else None)


@pytest.mark.parametrize("weighted", [False, True])
def test_noalloc_matches_prepared_solve_on_two_calls_in_a_row(weighted):
    import torch

    from eggpu_b200 import _native, synth

    g = synth.rmat(scale=14, edgefactor=16, seed=11, weighted=weighted)
    pg = _native.PreparedGraph(g.V, g.E, g.W)
    ref, ref_stats = pg.pagerank(alpha=0.85, max_iter=100, tol=1e-6)
    in_row, in_col, in_w, _dang, outw = pg.export_inbound()
    n, nnz = g.n, int(in_row[-1])
    dev = torch.device("cuda", 0)
    d_row = torch.from_numpy(np.ascontiguousarray(in_row, np.int32)).to(dev)
    d_col = torch.from_numpy(np.ascontiguousarray(in_col, np.int32)).to(dev)
    d_w = torch.from_numpy(np.ascontiguousarray(in_w, np.float32)).to(dev) if weighted else None
    d_outw = torch.from_numpy(np.ascontiguousarray(outw, np.float64)).to(dev)
    out = torch.empty(n, dtype=torch.float64, device=dev)
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
        assert st.converged == 1


def test_noalloc_rejects_graphs_beyond_its_scratch():
    from eggpu_b200 import _native

    st = _native.EgprStats()
    rc = _native.lib.egpr_pagerank_device_noalloc(LIMIT + 1, 0, None, None, None, None, 0.85, 10, 1e-6, 0, None,
                                                  None, ctypes.byref(st))
    assert rc == _native.EGPR_INVALID_ARGUMENT
    assert b"262144" in _native.lib.egpr_last_error()
