"""CPU tests of the oracle: self-consistency of the restated Dr.Top-k path and
agreement with the k-th values the reference itself produced (golden
fixtures made by tests/golden/make_golden.py on a B200)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import reference_counters_match

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_radix_kth.json")


def _load_golden():
    if not os.path.exists(GOLDEN):
        return []
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("dist", ["u32", "normal", "fewdigits", "f32u", "f32n"])
@pytest.mark.parametrize("log2n", [10, 14, 18])
def test_restatement_is_exact(dist, log2n):
    x = O.gen(dist, 1 << log2n, 77 + log2n)
    keys = O.as_keys(x)
    n = keys.size
    for k in sorted({1, 2, 5, 16, 128, 1000, n // 4, n // 2, n}):
        if k > n:
            continue
        want, vals, idx = O.topk_exact(keys, k)
        got, st = O.radix_final_kth(keys, k, 8)
        assert got == want, (dist, log2n, k, st)
        got_b, _ = O.bucket_kth(keys, k, 256)
        assert got_b == want
        # exact top-k semantics: every key above kth, lowest-index ties
        assert vals[-1] == want and (vals[:-1] >= vals[1:]).all()
        gt = np.flatnonzero(keys > want)
        eq = np.flatnonzero(keys == want)[: k - gt.size]
        assert set(idx.tolist()) == set(gt.tolist()) | set(eq.tolist())


@pytest.mark.parametrize("nbits", [1, 2, 4, 8])
def test_digit_widths(nbits):
    x = O.gen("u32", 1 << 12, 5)
    for k in (1, 3, 64, 1000, 4096):
        assert O.radix_final_kth(x, k, nbits)[0] == O.topk_exact(x, k, False)[0]


def test_delegate_definitions():
    x = O.gen("u32", 1 << 12, 9)
    m = O.sample_max(x, 5)
    assert np.array_equal(m, x.reshape(-1, 32).max(axis=1))
    t2 = O.sample_top2(x, 4).reshape(-1, 2)
    s = np.sort(x.reshape(-1, 16), axis=1)
    assert np.array_equal(t2[:, 0], s[:, -1]) and np.array_equal(t2[:, 1], s[:, -2])
    # one-key trailing subrange: Second stays 0 (the reference's Second=0 start)
    y = O.gen("u32", 33, 1)
    t = O.sample_top2(y, 5).reshape(-1, 2)
    assert t[1, 0] == y[32] and t[1, 1] == 0


def test_float_key_map_is_order_preserving():
    f = np.array([-np.inf, -3.5, -1e-30, -0.0, 0.0, 1e-30, 2.0, np.inf], dtype=np.float32)
    k = O.f32_to_key(f)
    assert (np.diff(k.astype(np.int64)) > 0).all()
    assert np.array_equal(O.key_to_f32(k).view(np.uint32), f.view(np.uint32))


def test_generators_are_seeded():
    a = O.gen("normal", 1000, 3)
    b = O.gen("normal", 1000, 3)
    c = O.gen("normal", 1000, 4)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    f = O.gen("fewdigits", 1 << 12, 1)
    assert (f >> 8 == 0xABCDEF).all()


def test_oracle_matches_reference_golden_kth():
    cases = _load_golden()
    if not cases:
        pytest.skip("golden fixtures from the reference have not been generated yet")
    checked = 0
    for c in cases:
        if "kth" not in c or c["log2n"] > 22:
            continue
        x = O.gen(c["dist"], 1 << c["log2n"], c["seed"])
        kth, st = O.radix_final_kth(x, c["k"], c["nbits"])
        assert kth == c["kth"], c
        assert st["alpha"] == c["alpha"]
        assert ("B" if st["beta_path"] else "D") == c["path"]
        # the reference's stage counters (radixselect.cuh:585, 1870-1880)
        if "write_pos" in c:
            got = (st["n_selected"], st["n_lonely"] if st["beta_path"] else 0, st["n_candidates"])
            assert not reference_counters_match(O.as_keys(x), c, got, c["alpha"], c["k"]), (c, got)
        checked += 1
    assert checked >= 20


def test_bmw_scan_is_exact_and_skips():
    # the BMW heap scan (threshold active once the heap holds k keys) gives
    # the exact k-th; on uniform keys most subranges are skipped
    for dist in ("u32", "normal", "fewdigits"):
        x = O.gen(dist, 1 << 16, 3)
        for k in (1, 10, 700):
            for alpha in (4, 8):
                kth, sk = O.bmw_kth(x, k, alpha)
                ek = O.topk_exact(x, k, want_topk=False)[0]
                assert kth == ek, (dist, k, alpha)
                assert 0 <= sk < x.size
    kth, sk = O.bmw_kth(O.gen("u32", 1 << 16, 4), 5, 8)
    assert sk > (1 << 15)
