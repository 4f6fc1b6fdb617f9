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
