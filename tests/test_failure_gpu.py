"""Failure detection on the GPU without a fault: a bounded wait that nothing
releases must give up, report DRTOPK_ETIMEOUT through the device error word,
and leave the context usable for the next select."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import expected, run_topk

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives():
    import ctypes

    import drtopksc_b200 as D
    ms = ctypes.c_double(0)
    st = D.lib().drtopk_selftest_wait_timeout(0, ctypes.byref(ms))
    assert st == D.ETIMEOUT
    assert 10.0 < ms.value < 10000.0
    x = O.gen("u32", 1 << 16, 5)
    kth, vals, idx, s = run_topk(x, 77, sorted=True)
    ek, ev, ei = expected(x, 77)
    assert kth == ek and np.array_equal(idx, ei)


def test_host_side_errors_leave_handle_usable():
    import drtopksc_b200 as D
    h = D.Handle()
    x = O.gen("u32", 1 << 14, 6)
    from tests.helpers import to_dev
    t = to_dev(x)
    for bad in ({"nbits": 3}, {"beta": 4, "alpha": 3, "path": 2}, {"algo": "bucket", "num_bucket": 1}):
        with pytest.raises(D.DrTopKError):
            h.topk(t, 10, **bad)
    with pytest.raises(D.DrTopKError):
        h.topk(t, x.size + 1)
    kth, _, _ = h.topk(t, 10)
    assert int(kth.cpu().numpy().view(np.uint32)[0]) == O.topk_exact(x, 10, False)[0]
