"""The select that allocates no device memory (drtopk_select_noalloc).

It exists for callers that cannot allocate device memory when they need a
top-k: a framework whose caching allocator already holds all of the GPU's
memory, a latency-critical loop that cannot pay for cudaMalloc's implicit
device synchronisation, or a plugin whose host program forbids allocation.
Its scratch is one fixed 32 MiB array inside the library.  These tests call
it through the C ABI twice in a row per input and check every output
against the oracle and against the regular drtopk_select, bit for bit; they
check that drtopk_noalloc_sync_check reports a clean run, that repeated
calls take no device memory once the first call has loaded the array, and
that a request needing more scratch than the array holds is refused.  The
file is named to be collected last."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import expected, same_bits

pytestmark = pytest.mark.gpu


def _lib():
    import drtopksc_b200 as D
    L = D.lib()
    L.drtopk_select_noalloc.restype = ctypes.c_int
    L.drtopk_select_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                        ctypes.POINTER(D.Params), ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]
    L.drtopk_noalloc_sync_check.restype = ctypes.c_int
    L.drtopk_noalloc_sync_check.argtypes = [ctypes.c_void_p]
    return L


def _noalloc(L, t, dt, n, k, p, kth, vals, idx):
    import drtopksc_b200 as D
    st = L.drtopk_select_noalloc(t.data_ptr(), dt, n, k, ctypes.byref(p), kth.data_ptr(), vals.data_ptr(),
                                 idx.data_ptr(), None)
    assert st == D.OK, st
    assert L.drtopk_noalloc_sync_check(None) == D.OK


CASES = [("u32", 1 << 20, 128, {}), ("f32n", 1 << 18, 1000, {"sorted": True}),
         ("fewdigits", 1 << 19, 4096, {"sorted": True}), ("normal", 300001, 77, {"alpha": 3, "path": 2}),
         ("u32", 1 << 16, 1 << 12, {"algo": "bucket"})]


def test_noalloc_select_matches_oracle_and_select_on_two_calls_in_a_row():
    import torch

    import drtopksc_b200 as D
    L = _lib()
    h = D.Handle()
    for dist, n, k, kw in CASES:
        x = O.gen(dist, n, n + k)
        t = torch.from_numpy(x).cuda() if x.dtype == np.float32 else torch.from_numpy(x.view(np.int32)).cuda()
        dt = D.F32 if x.dtype == np.float32 else D.U32
        p = D.params(**kw)
        # the existing entry point (handle-owned workspace)
        rk = torch.empty(1, dtype=torch.int32, device="cuda")
        rv = torch.empty(k, dtype=torch.int32, device="cuda")
        ri = torch.empty(k, dtype=torch.int64, device="cuda")
        h.select_raw(t.data_ptr(), dt, n, k, p, rk.data_ptr(), rv.data_ptr(), ri.data_ptr(), None)
        h.sync_check()
        want = (rk.cpu().numpy(), rv.cpu().numpy(), ri.cpu().numpy())
        ek, ev, ei = expected(x, k)
        for _ in range(2):
            kth = torch.full((1,), -1, dtype=torch.int32, device="cuda")
            vals = torch.full((k,), -1, dtype=torch.int32, device="cuda")
            idx = torch.full((k,), -1, dtype=torch.int64, device="cuda")
            _noalloc(L, t, dt, n, k, p, kth, vals, idx)
            kth, vals, idx = kth.cpu().numpy(), vals.cpu().numpy(), idx.cpu().numpy()
            assert np.array_equal(kth, want[0]), (dist, n, k)
            vv = vals.view(np.float32) if x.dtype == np.float32 else vals.view(np.uint32)
            kk = kth.view(np.float32) if x.dtype == np.float32 else kth.view(np.uint32)
            assert same_bits(kk[0], ek), (dist, n, k)
            if not kw.get("sorted"):  # unsorted output: order by value desc, index asc
                keys = O.as_keys(vv)
                order = np.lexsort((idx, -keys.astype(np.int64)))
                vv, idx, vals = vv[order], idx[order], vals[order]
                a = sorted(zip(vals.tolist(), idx.tolist()))
                b = sorted(zip(want[1].tolist(), want[2].tolist()))
                assert a == b, (dist, n, k)
            else:
                assert np.array_equal(vals, want[1]) and np.array_equal(idx, want[2]), (dist, n, k)
            assert same_bits(vv, ev) and np.array_equal(idx, ei), (dist, n, k)


def test_noalloc_select_takes_no_device_memory_after_the_first_call():
    import torch

    import drtopksc_b200 as D
    L = _lib()
    x = O.gen("u32", 1 << 20, 9)
    t = torch.from_numpy(x.view(np.int32)).cuda()
    k = 1000
    kth = torch.empty(1, dtype=torch.int32, device="cuda")
    vals = torch.empty(k, dtype=torch.int32, device="cuda")
    idx = torch.empty(k, dtype=torch.int64, device="cuda")
    p = D.params(sorted=True)
    _noalloc(L, t, D.U32, x.size, k, p, kth, vals, idx)  # loads the array on this device
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        _noalloc(L, t, D.U32, x.size, k, p, kth, vals, idx)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    ek, ev, ei = expected(x, k)
    assert np.array_equal(vals.cpu().numpy().view(np.uint32), ev) and np.array_equal(idx.cpu().numpy(), ei)


def test_noalloc_select_refuses_requests_beyond_its_scratch():
    import torch

    import drtopksc_b200 as D
    L = _lib()
    n = 1 << 24  # plain radix on 2^24 keys needs far more than 32 MiB of scratch
    t = torch.zeros(n, dtype=torch.int32, device="cuda")
    p = D.params(algo="plain")
    kth = torch.empty(1, dtype=torch.int32, device="cuda")
    st = L.drtopk_select_noalloc(t.data_ptr(), D.U32, n, 10, ctypes.byref(p), kth.data_ptr(), None, None, None)
    assert st == D.EUNSUPPORTED
    assert L.drtopk_noalloc_sync_check(None) == D.OK
