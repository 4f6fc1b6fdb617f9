"""The C ABI library loads on a machine without a GPU and exports exactly the
entry points include/egpr.h declares (no compute call is made here)."""

import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    text = (ROOT / "include" / "egpr.h").read_text()
    return set(re.findall(r"EGPR_API\s+[\w\s\*]+?\b(egpr_\w+)\s*\(", text))


def test_library_loads_and_exports_every_declared_symbol():
    from eggpu_b200 import _native

    declared = _declared()
    assert declared, "no declarations parsed"
    assert declared == set(_native.EXPORTED_SYMBOLS)
    for name in declared:
        assert hasattr(_native.lib, name)


def test_status_strings_keep_reference_numbering():
    from eggpu_b200 import _native

    # gpu_easygraph/common/err.cpp:9-31
    assert _native.status_string(0) == "EasyGraph GPU: success"
    assert _native.status_string(2) == "EasyGraph GPU: failed to allocate gpu mem"
    assert _native.status_string(3) == "EasyGraph GPU: gpu error occurred"
    assert _native.status_string(5) == "EasyGraph GPU: unsupported graph type"
    assert _native.status_string(8) == "EasyGraph GPU: invalid argument"
    assert _native.status_string(99) == "EasyGraph GPU: not a valid err_code"


def test_invalid_csr_is_rejected_before_any_device_work():
    import numpy as np
    import pytest

    from eggpu_b200 import _native

    with pytest.raises(_native.EgprError) as ei:
        _native.PreparedGraph(np.array([0, 3, 2], np.int32), np.array([0, 1, 1], np.int32))
    assert ei.value.status == _native.EGPR_INVALID_ARGUMENT
    with pytest.raises(_native.EgprError) as ei:
        _native.PreparedGraph(np.array([1, 2], np.int32), np.array([0, 0], np.int32))
    assert ei.value.status == _native.EGPR_INVALID_ARGUMENT


def test_empty_csr_call_is_a_no_op_like_the_reference():
    # centrality.cpp:160-165: n <= 0 returns success with nothing written
    import numpy as np

    from eggpu_b200 import _native

    PR, ks = _native.pagerank_csr(np.array([0], np.int32), np.zeros(0, np.int32), None, 1, 0.85, 10, 1e-6)
    assert PR.shape == (0,) and ks == 0.0


def test_bad_arguments_are_refused_through_the_abi_before_any_device_work():
    """Host-side failure injection: every entry point refuses NULL handles and
    missing buffers with EGPR_INVALID_ARGUMENT (status 8) and a message in
    egpr_last_error, without touching a device."""
    import ctypes

    import numpy as np

    from eggpu_b200 import _native

    lib, BAD = _native.lib, _native.EGPR_INVALID_ARGUMENT
    buf = np.zeros(8)
    p = buf.ctypes.data_as(ctypes.c_void_p)
    V = np.array([0, 1, 2], np.int32)
    E = np.array([1, 0], np.int32)
    vp, ep = V.ctypes.data_as(ctypes.c_void_p), E.ctypes.data_as(ctypes.c_void_p)
    handle = ctypes.c_void_p()
    cases = [
        ("egpr_graph_create", (vp, ep, None, 2, 2, None), b"out is NULL"),
        ("egpr_graph_create", (vp, ep, None, 0, 2, ctypes.byref(handle)), b"n must be in"),
        ("egpr_graph_create", (vp, ep, None, 2, -1, ctypes.byref(handle)), b"m must be in"),
        ("egpr_graph_create", (None, ep, None, 2, 2, ctypes.byref(handle)), b"V is NULL"),
        ("egpr_graph_create", (vp, None, None, 2, 2, ctypes.byref(handle)), b"E is NULL"),
        ("egpr_graph_create", (vp, ep, None, 2, 1, ctypes.byref(handle)), b"start at 0 and end at m"),
        ("egpr_graph_info_get", (None, None), b"NULL argument"),
        ("egpr_graph_export_inbound", (None, p, p, p, p, p), b"NULL argument"),
        ("egpr_graph_set_stream", (None, None), b"NULL graph"),
        ("egpr_graph_autotune", (None, 0, None), b"NULL graph"),
        ("egpr_graph_get_tuning", (None, None), b"NULL argument"),
        ("egpr_graph_set_tuning", (None, None), b"NULL argument"),
        ("egpr_pagerank", (None, 0.85, 10, 1e-6, None, 0, p, None), b"NULL graph"),
        ("egpr_pagerank_enqueue", (None, 0.85, 10, 1e-6, 0), b"NULL graph"),
        ("egpr_pagerank_collect", (None, p, None), b"NULL graph"),
        ("egpr_pagerank_batch", (None, 0.85, 10, 1e-6, 8, p, 0, p, None), b"NULL graph"),
        ("egpr_pagerank_seeds", (None, 0.85, 10, 1e-6, 8, p, p, 0, p, None), b"NULL graph"),
        ("egpr_pagerank_multi", (0, None, 0.85, 10, 1e-6, 0, None, None), b"count >= 1"),
        ("egpr_pagerank_csr", (None, 3, ep, 2, None, 1, 0.85, 10, 1e-6, p, None), b"NULL argument"),
        ("egpr_pagerank_csr", (vp, 3, ep, 2, None, 1, 0.85, 10, 1e-6, None, None), b"NULL argument"),
        ("egpr_cache_stats_get", (None,), b"NULL argument"),
        ("egpr_session_create", (None, 0.85, 1e-6, 32, ctypes.byref(handle)), b"NULL argument"),
        ("egpr_session_admit", (None, 1, p, p, 10, p), b"NULL session"),
        ("egpr_session_step", (None, 4, p, ctypes.byref(ctypes.c_int32())), b"NULL session"),
        ("egpr_session_collect", (None, 1, p, 0, p, None), b"NULL session"),
        ("egpr_session_info", (None, None, None, None), b"NULL argument"),
    ]
    for name, args, msg in cases:
        rc = getattr(lib, name)(*args)
        assert rc == BAD, (name, args, rc)
        assert msg in lib.egpr_last_error(), (name, lib.egpr_last_error())
    assert handle.value is None  # nothing was created
    assert lib.egpr_graph_destroy(None) == _native.EGPR_SUCC  # destroying nothing is allowed
    assert lib.egpr_session_destroy(None) == _native.EGPR_SUCC


def test_a_missing_device_is_an_error_status_not_a_crash():
    """Without a usable GPU the engine reports EGPR_DEVICE_ERR with the CUDA
    error text; it never falls back to a CPU path."""
    import numpy as np
    import pytest

    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the device path is covered by the gpu tests")
    from eggpu_b200 import _native

    V = np.array([0, 1, 2], np.int32)
    E = np.array([1, 0], np.int32)
    with pytest.raises(_native.EgprError) as ei:
        _native.PreparedGraph(V, E)
    assert ei.value.status == _native.EGPR_DEVICE_ERR
    assert "cudaGetDevice" in str(ei.value)
    with pytest.raises(_native.EgprError) as ei:
        _native.pagerank_csr(V, E, None, 7, 0.85, 10, 1e-6)
    assert ei.value.status == _native.EGPR_DEVICE_ERR
