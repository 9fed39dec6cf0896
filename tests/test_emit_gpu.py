"""The sampled-threshold path (params.path = 4): a strided key sample
predicts a threshold, the streaming pass appends every key at or above it,
and the second select runs on those candidates -- or, when fewer than k
keys reach the prediction, over all keys.  Results must be bit-exact with
the oracle whatever the input, including inputs built to fool the sample."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import expected, run_topk, same_bits

pytestmark = pytest.mark.gpu

PRE_STRIDE = 64  # the planner's sampling stride for n <= 2^27 (one 512-key chunk in 64)


def check(x, k, largest=True, offset=0, **kw):
    kw.setdefault("sorted", True)
    kth, vals, idx, st = run_topk(x, k, offset=offset, largest=largest, path=4, **kw)
    ek, ev, ei = expected(x, k, largest)
    if not kw["sorted"]:
        keys = O.as_keys(vals)
        if not largest:
            keys = ~keys
        order = np.lexsort((idx, -keys.astype(np.int64)))
        vals, idx = vals[order], idx[order]
    assert same_bits(kth, ek), (k, kw, st)
    assert same_bits(vals, ev), (k, kw, st)
    assert np.array_equal(idx, ei), (k, kw, st)
    assert st["device_error"] == 0
    return st


@pytest.mark.parametrize("dist", ["u32", "normal", "f32u", "f32n", "fewdigits"])
def test_sampled_threshold_all_distributions(dist):
    x = O.gen(dist, 1 << 22, 4242)
    for k in (1, 100, 4096, 1 << 16, 1 << 19, 1 << 21):
        for sorted_ in (True, False):
            check(x, k, sorted=sorted_)


def test_sampled_threshold_candidates_close_to_k():
    n = 1 << 23
    x = O.gen("u32", n, 7)
    ns_keys = ((n >> 9) // PRE_STRIDE) * 512
    for k in (1 << 16, 1 << 20):
        st = check(x, k, sorted=False)
        assert st["beta"] == 0 and st["levels_first"] == 2 and st["sample_stride"] == PRE_STRIDE
        # sample passes (4), the appending pass, k_cand_hist, k_split0, k_fused
        assert st["kernel_launches"] == 8, st
        # k scaled to the sample plus the six-sigma margin, plus the sample's
        # own error in the other direction (another six sigma), plus one
        # 16-bit prefix bin of uniform keys
        ks = k * ns_keys / n
        bound = (ks + 12 * ks ** 0.5 + 32) * n / ns_keys + 2 * n / 65536
        assert k <= st["n_candidates"] <= bound, (st, bound)


@pytest.mark.parametrize("dist,levels", [("fewdigits", 4), ("range16", 3)])
def test_narrow_inputs_refine_the_threshold(dist, levels):
    # keys sharing their top 24 (few digits) or 16 bits: a 16-bit threshold
    # would admit every key; the sample passes refine it byte by byte until
    # the picked bin is small
    n = 1 << 22
    if dist == "range16":
        x = (0x12340000 | (O.gen("u32", n, 5) & 0xFFFF)).astype(np.uint32)
    else:
        x = O.gen(dist, n, 5)
    ns_keys = ((n >> 9) // PRE_STRIDE) * 512
    for k in (16, 4096, 1 << 16):
        st = check(x, k, sorted=False)
        assert st["beta"] == 0 and st["levels_first"] == levels, st
        ks = k * ns_keys / n
        # the margin as above, plus one bin of the last refined level
        bound = (ks + 12 * ks ** 0.5 + 32) * n / ns_keys + 2 * n / (1 << (8 * (levels - 2)))
        bound = max(bound, 2 * n / 256)  # few digits: one value's copies
        assert k <= st["n_candidates"] <= bound, (st, bound)


@pytest.mark.parametrize("n", [(1 << 20) + 12345, 1000003, 40000, 5000])
def test_sampled_threshold_ragged_sizes(n):
    x = O.gen("normal", n, n)
    for k in (1, 77, n // 3, n):
        check(x, k)


@pytest.mark.parametrize("offset", [1, 3])
def test_sampled_threshold_unaligned_and_smallest(offset):
    x = O.gen("f32n", (1 << 20) + 3, 13)
    for k in (5, 3000, 1 << 17):
        check(x, k, offset=offset)
        check(x, k, largest=False)


def _sampled_chunks(n):
    ns = (n >> 9) // PRE_STRIDE
    i = np.arange(ns, dtype=np.int64)
    return i * PRE_STRIDE + ((i * 37) & (PRE_STRIDE - 1))


def test_prediction_that_overshoots_falls_back_to_an_exact_select():
    # every sampled 512-key chunk holds the largest keys, the rest is small:
    # the sample predicts a threshold that fewer than k keys reach
    n = 1 << 22
    rng = np.random.default_rng(3)
    x = rng.integers(0, 1 << 31, size=n, dtype=np.uint64).astype(np.uint32)
    for c in _sampled_chunks(n):
        x[c * 512:(c + 1) * 512] = 0xFFFFFFF0 + (rng.integers(0, 16, 512)).astype(np.uint32)
    nhigh = int((x >= 0xFFFF0000).sum())
    for k in (nhigh + 1, 3 * nhigh, n // 2):
        st = check(x, k, sorted=True)
        assert st["n_candidates"] == n  # the select ran over all keys
    # the sample sees only the largest keys, so it refines the threshold to
    # their top value: the prediction holds for k up to that value's copies
    st = check(x, nhigh // 64)
    assert st["n_candidates"] < n


def test_heavy_ties_and_constant_input():
    # every key ties: the threshold refines to the tied value itself
    for x in (np.full(1 << 20, 9, dtype=np.uint32), np.repeat(np.arange(64, dtype=np.uint32), 1 << 14)):
        for k in (1, 1000, x.size // 2, x.size):
            check(x, k)
            check(x, k, sorted=False)


def test_last_levels_team_follows_k():
    # unsorted selects with k <= n/2048 finish their last levels in one CTA,
    # larger ones and sorted outputs on the cooperative grid
    x = O.gen("u32", 1 << 22, 99)
    assert check(x, 1 << 11, sorted=False)["team_cluster"] == 5
    assert check(x, 1 << 11, largest=False, sorted=False)["team_cluster"] == 5
    assert check(x, (1 << 11) + 1, sorted=False)["team_cluster"] == 0
    assert check(x, 1 << 11, sorted=True)["team_cluster"] == 0
