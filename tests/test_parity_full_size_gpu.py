"""Parity at the headline sizes, pinned to the reference itself.

tests/golden/ref_radix_big.json holds what the reference's own
sample_radix_select (baseline+filter+beta+shuffle/radixselect.cuh:1782-1894,
built from its sources for sm_100a by `make -C oracle ref`, run on a B200 by
tests/golden/make_golden.py --big) returned on the seeded inputs regenerated
here: the k-th value and its three counters for N = 2^30 uint32 uniform and
normal(2^31, 2^28) keys at k = 2^0..2^24, and for N = 2^28 float32 uniform,
float32 normal and few-digits keys at k in {16, 256, 4096, 65536}.

At those sizes these tests check, through the C ABI:
  * the reference-shaped entry point with the reference's parameters: the
    k-th value, CountSelectedSubrange, CountLonelyElements and write_pos;
  * the autotuned select (the bench's parameters): the k-th value for every
    k, and the whole sorted top-k with lowest-index ties for several k, the
    expected list being every key above the reference's k-th plus the
    lowest-index copies of it (and, at N = 2^28, the oracle's exact top-k);
  * the bucket and bitonic variants on the N = 2^28 inputs.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import expected, reference_counters_match, same_bits

pytestmark = pytest.mark.gpu

BIG = os.path.join(os.path.dirname(__file__), "golden", "ref_radix_big.json")


def _fixtures():
    if not os.path.exists(BIG):
        pytest.skip("reference fixtures at the headline sizes have not been generated")
    return [c for c in json.load(open(BIG))["cases"] if "kth" in c]


_inputs = {}


def _input(dist, log2n, seed):
    """Seeded input (host array as the oracle makes it, device copy as int32/float32 bits)."""
    import torch
    key = (dist, log2n, seed)
    if key not in _inputs:
        _inputs.clear()  # one headline input resident at a time
        x = O.gen(dist, 1 << log2n, seed)
        t = torch.from_numpy(x).cuda() if x.dtype == np.float32 else torch.from_numpy(x.view(np.int32)).cuda()
        _inputs[key] = (x, t)
    return _inputs[key]


def _expected_from_kth(keys, k, kth):
    """Top-k implied by the k-th value: every key above it, then the
    lowest-index copies of it; ordered by key descending, index ascending."""
    gt = np.flatnonzero(keys > kth)
    assert gt.size < k
    eq = np.flatnonzero(keys == kth)[: k - gt.size]
    assert gt.size + eq.size == k
    idx = np.concatenate([gt, eq])
    v = keys[idx]
    order = np.lexsort((idx, -v.astype(np.int64)))
    return v[order], idx[order].astype(np.int64)


def _reference_shaped(t, n, k, alpha):
    import torch

    import drtopksc_b200 as D
    S = 1 << alpha
    nsub = n // S
    dflt = alpha > 5
    Max_d = torch.zeros(nsub * 2, dtype=torch.int32, device="cuda")
    ids = torch.full((nsub * 2,), -1, dtype=torch.int32, device="cuda")
    counters = torch.zeros(3, dtype=torch.int32, device="cuda")
    kth, _ = D.sample_radix_select(t, n, k, 256, 8, 3, nsub, S, alpha, Max_d, 2, dflt, counters, SubrangeId_d=ids)
    st = D.default_handle().stats()
    c = counters.cpu().numpy()
    per = 1 if dflt else 2
    want_ids = torch.arange(nsub * per, dtype=torch.int32, device="cuda") // per
    assert torch.equal(ids[: nsub * per], want_ids)
    del Max_d, ids
    return kth, c, st, dflt


def _check_reference_counters(keys, c, cnt, k, alpha):
    bad = reference_counters_match(keys, c, [int(v) for v in cnt], alpha, k)
    assert not bad, (c, bad)


@pytest.mark.parametrize("dist", ["u32", "normal"])
def test_n30_kth_and_counters_match_the_reference(dist):
    import drtopksc_b200 as D
    cases = [c for c in _fixtures() if c["dist"] == dist and c["log2n"] == 30]
    assert len(cases) == 25
    x, t = _input(dist, 30, cases[0]["seed"])
    n = x.size
    h = D.default_handle()
    for c in cases:
        k = c["k"]
        alpha = D.ref_alpha(30, k)
        assert alpha == c["alpha"]
        kth, cnt, st, dflt = _reference_shaped(t, n, k, alpha)
        assert kth == c["kth"], c
        _check_reference_counters(x, c, cnt, k, alpha)
        # the autotuned select (the bench's parameters)
        kt, _, _ = h.topk(t, k, want_values=False, want_indices=False, alpha=-2)
        assert int(kt.cpu().numpy().view(np.uint32)[0]) == c["kth"], c


@pytest.mark.parametrize("dist", ["u32", "normal"])
def test_n30_sorted_topk_with_indices_exact(dist):
    import drtopksc_b200 as D
    cases = {c["k"]: c for c in _fixtures() if c["dist"] == dist and c["log2n"] == 30}
    x, t = _input(dist, 30, cases[1]["seed"])
    h = D.default_handle()
    for k in (1, 1 << 10, 1 << 20, 1 << 24):
        kth, vals, idx = h.topk(t, k, sorted=True, alpha=-2)
        ref = cases[k]["kth"]
        assert int(kth.cpu().numpy().view(np.uint32)[0]) == ref
        ev, ei = _expected_from_kth(x, k, np.uint32(ref))
        assert np.array_equal(vals.cpu().numpy().view(np.uint32), ev), k
        assert np.array_equal(idx.cpu().numpy(), ei), k
        del kth, vals, idx
        # unsorted output: the same (value, index) set
        kth, vals, idx = h.topk(t, k, sorted=False, alpha=-2)
        v = vals.cpu().numpy().view(np.uint32)
        i = idx.cpu().numpy()
        order = np.lexsort((i, -v.astype(np.int64)))
        assert np.array_equal(v[order], ev) and np.array_equal(i[order], ei), k
    # the oracle's own multi-threaded top-k agrees with the reference's k-th
    _, okth, ovals = O.topk_mt(x, 1 << 20, os.cpu_count() or 1)
    assert okth == cases[1 << 20]["kth"]


@pytest.mark.parametrize("dist", ["f32u", "f32n", "fewdigits"])
def test_n28_variant_inputs_all_algorithms(dist):
    import drtopksc_b200 as D
    cases = [c for c in _fixtures() if c["dist"] == dist and c["log2n"] == 28]
    assert len(cases) == 4
    x, t = _input(dist, 28, cases[0]["seed"])
    n = x.size
    keys = O.as_keys(x)
    h = D.default_handle()
    for c in cases:
        k = c["k"]
        alpha = D.ref_alpha(28, k)
        # the reference-shaped entry point runs on mapped keys, as the reference does
        if x.dtype == np.float32:
            tk = _input_keys(keys)
        else:
            tk = t
        kth, cnt, st, dflt = _reference_shaped(tk, n, k, alpha)
        assert kth == c["kth"], c
        _check_reference_counters(keys, c, cnt, k, alpha)
        del tk
        ek, ev, ei = expected(x, k)
        assert int(O.as_keys(np.array([ek], dtype=x.dtype))[0]) == c["kth"]
        for kw in ({"alpha": -2}, {}, {"algo": "bucket"}, {"algo": "bitonic"}):
            if kw.get("algo") == "bitonic" and k > 2048:
                continue
            kt, vals, idx = h.topk(t, k, sorted=True, **kw)
            kt = kt.cpu().numpy()
            vv = vals.cpu().numpy()
            if x.dtype != np.float32:
                kt, vv = kt.view(np.uint32), vv.view(np.uint32)
            assert same_bits(kt[0], ek), (dist, k, kw)
            assert same_bits(vv, ev), (dist, k, kw)
            assert np.array_equal(idx.cpu().numpy(), ei), (dist, k, kw)
            del vals, idx


def _input_keys(keys):
    import torch
    return torch.from_numpy(keys.view(np.int32)).cuda()
