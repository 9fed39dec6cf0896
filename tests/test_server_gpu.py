"""GPU tests of the served form: requests of different sizes submitted while
others are in flight are all answered exactly, identically to the plain call
(alone vs in the mix); budget, cancel and drain behave."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import expected

pytestmark = pytest.mark.gpu


def _check(res, x, k, sorted_):
    assert res["status"] == 0, res
    ek, ev, ei = expected(x, k)
    kth = res["kth"]
    if x.dtype == np.float32:
        assert np.float32(kth).view(np.uint32) == np.float32(ek).view(np.uint32)
    else:
        assert int(kth) == int(ek)
    v, i = res["values"], res["indices"]
    if not sorted_:
        order = np.lexsort((i, -O.as_keys(np.asarray(v, dtype=x.dtype)).astype(np.int64)))
        v, i = v[order], i[order]
    assert np.array_equal(np.asarray(v).view(np.uint32), np.asarray(ev).view(np.uint32))
    assert np.array_equal(i, ei)


def test_server_mixed_requests_exact():
    import torch

    import drtopksc_b200 as D
    rng = np.random.default_rng(7)
    srv = D.Server(hbm_budget_bytes=8 << 30, max_inflight=16)
    reqs = {}
    dev_keep = []
    for r in range(40):
        n = int(np.exp2(rng.uniform(10, 23)))
        k = int(np.exp2(rng.uniform(0, np.log2(min(n, 1 << 16)))))
        dist = ["u32", "normal", "f32n"][r % 3]
        x = O.gen(dist, n, 100 + r)
        sorted_ = bool(r % 2)
        if r % 4 == 0:
            t = torch.from_numpy(x).cuda() if x.dtype == np.float32 else torch.from_numpy(x.view(np.int32)).cuda()
            dev_keep.append(t)
            rid = srv.submit(t, k, sorted=sorted_)
        else:
            rid = srv.submit(x, k, sorted=sorted_)
        reqs[rid] = (x, k, sorted_)
    srv.drain(60000)
    got = {}
    while True:
        out = srv.poll()
        if not out:
            break
        for res in out:
            got[res["id"]] = res
    assert set(got) == set(reqs)
    for rid, (x, k, s) in reqs.items():
        _check(got[rid], x, k, s)
        assert got[rid]["t_submit"] <= got[rid]["t_start"] <= got[rid]["t_done"]
    assert srv.usage()[0] == 0
    srv.close()


def test_server_same_alone_and_in_mix():
    import drtopksc_b200 as D
    x = O.gen("f32n", 1 << 20, 11)
    alone = D.Server()
    alone.submit(x, 500, sorted=True)
    alone.drain(30000)
    a = alone.poll()[0]
    mix = D.Server(max_inflight=8)
    ids = [mix.submit(O.gen("u32", 1 << 18, i), 100) for i in range(10)]
    rid = mix.submit(x, 500, sorted=True)
    ids += [mix.submit(O.gen("u32", 1 << 16, 50 + i), 7) for i in range(10)]
    mix.drain(30000)
    res = {r["id"]: r for r in mix.poll()}
    b = res[rid]
    assert a["status"] == b["status"] == 0
    assert np.array_equal(a["values"].view(np.uint32), b["values"].view(np.uint32))
    assert np.array_equal(a["indices"], b["indices"])


def test_server_budget_and_cancel():
    import drtopksc_b200 as D
    srv = D.Server(hbm_budget_bytes=1 << 20, max_inflight=1)
    with pytest.raises(D.DrTopKError) as e:
        srv.submit(O.gen("u32", 1 << 20, 1), 10)  # keys alone exceed the budget
    assert e.value.status == D.EBUDGET
    srv2 = D.Server(max_inflight=1)
    ids = [srv2.submit(O.gen("u32", 1 << 22, i), 1000) for i in range(6)]
    cancelled = [i for i in ids[2:] if srv2.cancel(i)]
    srv2.drain(60000)
    res = {r["id"]: r for r in srv2.poll()}
    assert set(res) == set(ids)
    for i in cancelled:
        assert res[i]["status"] == D.ECANCELLED
    for i in ids:
        if i not in cancelled:
            assert res[i]["status"] == 0


def _sampled_chunks(n, stride=64):
    ns = (n >> 9) // stride
    i = np.arange(ns, dtype=np.int64)
    return i * stride + ((i * 37) & (stride - 1))


def test_server_retries_selects_the_sample_misjudges():
    """The served form sizes the candidate buffers of its sampled-threshold
    selects by the sample's estimate.  Inputs that break the estimate --
    heavy ties around the threshold (every key in one 16-bit bin), or
    sampled chunks holding the largest keys -- make the select report that it
    must run again, and the server reruns it with the general plan: the
    results stay exact."""
    import drtopksc_b200 as D
    rng = np.random.default_rng(11)
    n = 1 << 20
    ties = O.gen("fewdigits", n, 5)
    skew = rng.integers(0, 1 << 31, size=n, dtype=np.uint64).astype(np.uint32)
    for c in _sampled_chunks(n):
        skew[c * 512:(c + 1) * 512] = 0xFFFFFFF0 + rng.integers(0, 16, 512).astype(np.uint32)
    nhigh = int((skew >= 0xFFFF0000).sum())
    srv = D.Server(hbm_budget_bytes=8 << 30, max_inflight=16)
    reqs = {}
    for x, k, s in ((ties, 5000, False), (ties, 77, True), (skew, 3 * nhigh, False), (skew, nhigh + 1, True),
                    (O.gen("u32", n, 6), 1000, False)):
        reqs[srv.submit(x, k, sorted=s)] = (x, k, s)
    srv.drain(60000)
    got = {}
    while True:
        out = srv.poll()
        if not out:
            break
        for res in out:
            got[res["id"]] = res
    srv.close()
    assert set(got) == set(reqs)
    for rid, (x, k, s) in reqs.items():
        _check(got[rid], x, k, s)
