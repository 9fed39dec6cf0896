"""GPU parity tests: the CUDA select (through the C ABI) against the CPU
oracle on the same seeded inputs -- bit-exact k-th value, top-k values and
lowest-index tie-broken indices -- plus per-stage parity with the restated
reference path and size-independent properties at full size."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import expected, run_topk, same_bits, sort_pairs, tie_fill_ambiguous, to_dev

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_radix_kth.json")


def check_exact(x, k, largest=True, offset=0, **kw):
    kth, vals, idx, st = run_topk(x, k, offset=offset, largest=largest, sorted=True, **kw)
    ek, ev, ei = expected(x, k, largest)
    assert same_bits(kth, ek), (k, kw, kth, ek, st)
    assert same_bits(vals, ev), (k, kw, st)
    assert np.array_equal(idx, ei), (k, kw, st)
    assert st["device_error"] == 0
    return st


def test_c1_reference_config():
    # N=2^20 uint32 uniform (seeded mt19937), k=128, 8-bit digits, beta=2, alpha auto
    x = O.gen("u32", 1 << 20, 1)
    st = check_exact(x, 128)
    ref_kth, ost = O.radix_final_kth(x, 128, 8)
    assert st["alpha"] == ost["alpha"] == 8 and st["beta"] == 1
    assert st["first_threshold"] == ost["first_flag"]
    assert st["n_selected"] == ost["n_selected"] == 128


@pytest.mark.parametrize("dist", ["u32", "normal", "fewdigits", "f32u", "f32n"])
@pytest.mark.parametrize("log2n", [10, 16, 20])
def test_reference_alpha_all_k(dist, log2n):
    x = O.gen(dist, 1 << log2n, 1000 + log2n)
    n = x.size
    for k in sorted({1, 2, 3, 16, 128, 1000, 4096, n // 2, n}):
        if k <= n:
            check_exact(x, k)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 31, 1000, 12345, (1 << 20) + 7])
def test_non_power_of_two_sizes(n):
    x = O.gen("u32", n, n)
    for k in sorted({1, 2, max(1, n // 3), n}):
        if k <= n:
            check_exact(x, k)


@pytest.mark.parametrize("nbits", [1, 2, 4, 8])
def test_digit_widths(nbits):
    x = O.gen("u32", 1 << 16, 11)
    for k in (1, 7, 300, 5000, 1 << 15):
        st = check_exact(x, k, nbits=nbits)
        _, ost = O.radix_final_kth(x, k, nbits)
        assert st["first_threshold"] == ost["first_flag"], (nbits, k)


@pytest.mark.parametrize("alpha,path", [(6, 1), (8, 1), (12, 1), (1, 2), (2, 2), (3, 2), (4, 2), (5, 2), (8, 2)])
def test_forced_alpha_and_path_stage_parity(alpha, path):
    x = O.gen("normal", 1 << 18, 3)
    for k in (1, 64, 999, 4096):
        if path == 1 and (x.size >> alpha) < k:
            continue
        st = check_exact(x, k, alpha=alpha, path=path)
        _, ost = O.radix_final_kth(x, k, 8, alpha=alpha, path=path)
        assert st["first_threshold"] == ost["first_flag"]
        assert st["n_selected"] == ost["n_selected"]
        if path == 2:  # the reference appends (Max, Second) per lonely subrange; we append Max only
            assert 2 * st["n_lonely"] == ost["n_lonely"]


@pytest.mark.parametrize("fd", [1, 2, 3, 4])
def test_beta_first_digits(fd):
    x = O.gen("u32", 1 << 18, 4)
    for k in (100, 20000):
        check_exact(x, k, alpha=4, path=2, first_digits=fd)


@pytest.mark.parametrize("dist", ["fewdigits", "f32u"])
def test_tuned_beta_threshold_refines_crowded_bins(dist):
    # first_digits < 0 (the autotuner's form): at least that many digits,
    # more while the chosen bin holds more than max(2k, 4096) delegates --
    # few-digit keys share 24 bits and float keys their exponent, so a
    # 16-bit threshold would make every subrange qualify
    n = 1 << 22
    x = O.gen(dist, n, 11)
    for k in (16, 3000):
        st = check_exact(x, k, alpha=8, path=2, first_digits=-2)
        assert st["levels_first"] >= 3, st
        assert st["n_candidates"] <= max(4 * k, n // 128), st
        if dist == "fewdigits":  # the threshold is one value: only k tied subranges are read
            assert st["n_selected"] + st["n_lonely"] <= k, st
    # explicit digit counts keep exactly their digits
    st = check_exact(x, 16, alpha=8, path=2, first_digits=2)
    assert st["levels_first"] == 2, st


def test_tied_subranges_cut_keeps_the_lowest_index_copies():
    # few-digit keys with larger keys planted: the threshold collapses to the
    # top few-digit value t; subranges with a planted Max and Second >= t are
    # read whole, of those with Max == t only the k lowest-id ones -- the top
    # k (planted keys, then the lowest-index copies of t) must be exact
    n = 1 << 20
    x = O.gen("fewdigits", n, 21)
    rng = np.random.default_rng(5)
    for planted in (1, 100, 2000):
        y = x.copy()
        y[rng.choice(n, planted, replace=False)] = 0xABCE0000 + rng.integers(0, 64, planted).astype(np.uint32)
        for k in (planted, planted + 1, planted + 300, 5000):
            for alpha in (6, 8, 10):
                check_exact(y, k, alpha=alpha, path=2, first_digits=-1)


@pytest.mark.parametrize("nb", [2, 16, 256, 1000, 4096])
def test_bucket_variant_exact(nb):
    for dist in ("u32", "normal", "fewdigits", "f32n"):
        x = O.gen(dist, 1 << 17, nb)
        for k in (1, 16, 256, 4096, 65536):
            st = check_exact(x, k, algo="bucket", num_bucket=nb)
            assert st["algo"] == 1


def test_bucket_reference_alpha_rule():
    x = O.gen("u32", 1 << 20, 8)
    for k in (1, 1024, 1 << 18):
        alpha = O.ref_alpha_bucket(20, k)
        st = check_exact(x, k, algo="bucket", num_bucket=256, alpha=alpha)
        ok, ost = O.bucket_kth(x, k, 256, alpha=alpha)
        assert st["alpha"] == ost["alpha"]
        assert st["first_threshold"] == ost["first_flag"]


@pytest.mark.parametrize("dist", ["u32", "fewdigits", "f32n"])
def test_plain_radix(dist):
    x = O.gen(dist, 1 << 18, 21)
    for k in (1, 100, 1 << 17, 1 << 18):
        check_exact(x, k, algo="plain")


@pytest.mark.parametrize("dist", ["u32", "f32n", "fewdigits"])
def test_smallest(dist):
    x = O.gen(dist, 1 << 16, 31)
    for k in (1, 50, 3000):
        check_exact(x, k, largest=False)


def test_large_sorted_k_uses_grid_sort():
    x = O.gen("u32", 1 << 20, 41)
    for k in (4097, 10000, 1 << 16, 1 << 19):
        check_exact(x, k)
    f = O.gen("fewdigits", 1 << 20, 42)
    check_exact(f, 70000)


@pytest.mark.parametrize("copies", [2, 9, 32, 33, 3000])
def test_large_sorted_k_runs_of_equal_keys(copies):
    # the large-k sort orders the keys first, then each run of equal keys by
    # index; runs longer than 32 send it through every digit instead
    rng = np.random.default_rng(copies)
    n = 1 << 19
    vals = rng.integers(0, 1 << 32, size=n // copies + 1, dtype=np.uint64).astype(np.uint32)
    x = np.repeat(vals, copies)[:n]
    rng.shuffle(x)
    for k in (5000, 1 << 17):
        check_exact(x, k)
        check_exact(x, k, alpha=-2)


def test_heavy_ties():
    for x in (np.full(1 << 16, 7, dtype=np.uint32), np.zeros(5000, dtype=np.uint32),
              np.full(4096, 0xFFFFFFFF, dtype=np.uint32),
              np.repeat(np.arange(16, dtype=np.uint32), 4096)):
        for k in (1, 17, x.size // 2, x.size):
            check_exact(x, k)
            check_exact(x, k, algo="bucket")


def test_float_specials():
    f = np.array([np.nan, -np.nan, np.inf, -np.inf, 0.0, -0.0, 1e-45, -1e-45, 3.0, -3.0] * 300, dtype=np.float32)
    for k in (1, 2, 10, 1000, f.size):
        check_exact(f, k)
        check_exact(f, k, largest=False)


@pytest.mark.parametrize("offset", [1, 2, 3])
def test_unaligned_input(offset):
    x = O.gen("u32", (1 << 16) + 5, 51)
    for k in (1, 99, 5000):
        check_exact(x, k, offset=offset)
        check_exact(x, k, offset=offset, alpha=3, path=2)


def test_unsorted_output_is_the_same_multiset():
    x = O.gen("fewdigits", 1 << 18, 61)
    k = 30000
    kth, vals, idx, _ = run_topk(x, k, sorted=False)
    ek, ev, ei = expected(x, k)
    v, i = sort_pairs(vals, idx, x.dtype)
    assert kth == ek and np.array_equal(v, ev) and np.array_equal(i, ei)


def test_values_only_and_kth_only():
    import drtopksc_b200 as D
    x = O.gen("u32", 1 << 18, 71)
    t = to_dev(x)
    h = D.default_handle()
    for k in (5, 5000):
        ek, ev, _ = expected(x, k)
        kth, vals, idx = h.topk(t, k, want_indices=False, sorted=True)
        assert idx is None and kth.cpu().numpy().view(np.uint32)[0] == ek
        assert np.array_equal(vals.cpu().numpy().view(np.uint32), ev)
        kth, vals, idx = h.topk(t, k, want_values=False, want_indices=False, alpha=3, path=2)
        assert kth.cpu().numpy().view(np.uint32)[0] == ek


def test_deterministic_across_runs():
    x = O.gen("fewdigits", 1 << 20, 81)
    a = run_topk(x, 4000, sorted=True)
    b = run_topk(x, 4000, sorted=True)
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])
    assert a[3]["n_candidates"] == b[3]["n_candidates"]


def test_caller_workspace():
    import ctypes

    import torch

    import drtopksc_b200 as D
    x = O.gen("u32", 1 << 18, 91)
    t = to_dev(x)
    k = 321
    p = D.params(sorted=True)
    need = D.workspace_size(x.size, k, D.U32, p)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    kth = torch.empty(1, dtype=torch.int32, device="cuda")
    vals = torch.empty(k, dtype=torch.int32, device="cuda")
    idx = torch.empty(k, dtype=torch.int64, device="cuda")
    h = D.Handle()
    st = D.lib().drtopk_select_ws(h.ptr, t.data_ptr(), D.U32, x.size, k, ctypes.byref(p), kth.data_ptr(),
                                  vals.data_ptr(), idx.data_ptr(), ws.data_ptr(), need, None)
    assert st == D.OK
    h.sync_check()
    ek, ev, ei = expected(x, k)
    assert kth.cpu().numpy().view(np.uint32)[0] == ek and np.array_equal(idx.cpu().numpy(), ei)
    st = D.lib().drtopk_select_ws(h.ptr, t.data_ptr(), D.U32, x.size, k, ctypes.byref(p), kth.data_ptr(),
                                  None, None, ws.data_ptr(), need // 2, None)
    assert st == D.ENOMEM


def test_budget_is_enforced():
    import drtopksc_b200 as D
    h = D.Handle(hbm_budget_bytes=1 << 20)
    x = to_dev(O.gen("u32", 1 << 20, 1))
    with pytest.raises(D.DrTopKError) as e:
        h.topk(x, 1000)
    assert e.value.status == D.EBUDGET


def test_reference_shaped_wrappers():
    import torch

    import drtopksc_b200 as D
    for log2n, k in ((20, 128), (20, 1 << 16), (18, 1 << 17)):
        x = O.gen("u32", 1 << log2n, log2n + k)
        t = to_dev(x)
        alpha = D.ref_alpha(log2n, k)
        beta = 2
        S = 1 << alpha
        nsub = x.size // S
        dflt = alpha > 5
        Max_d = torch.zeros(nsub * beta, dtype=torch.int32, device="cuda")
        counters = torch.zeros(3, dtype=torch.int32, device="cuda")
        kth, times = D.sample_radix_select(t, x.size, k, 256, 8, 3, nsub, S, alpha, Max_d, beta, dflt, counters)
        want, ost = O.radix_final_kth(x, k, 8)
        assert kth == want
        c = counters.cpu().numpy()
        # the reference's counters, as the restated reference path counts them
        assert c[0] == ost["n_selected"]
        assert c[1] == (0 if dflt else ost["n_lonely"])
        assert c[2] == ost["n_candidates"] or (dflt and tie_fill_ambiguous(x, alpha, k))
        dl = Max_d.cpu().numpy().view(np.uint32)
        if dflt:
            assert np.array_equal(dl[:nsub], O.sample_max(x, alpha))
        else:
            assert np.array_equal(dl, O.sample_top2(x, alpha))
        assert all(v >= 0 for v in times)
        assert D.radix_select(t, x.size, k) == want
        kb, _ = D.sample_bucket_select(t, x.size, k, 256, nsub, S, alpha, 2, dflt)
        assert kb == want


def test_golden_reference_kth_on_gpu():
    if not os.path.exists(GOLDEN):
        pytest.skip("golden fixtures from the reference have not been generated yet")
    cases = json.load(open(GOLDEN))["cases"]
    n = 0
    for c in cases:
        if "kth" not in c:
            continue
        x = O.gen(c["dist"], 1 << c["log2n"], c["seed"])
        kth, _, _, st = run_topk(x, c["k"], nbits=c["nbits"], want_values=False, want_indices=False)
        ref = c["kth"]  # the reference ran on mapped keys for float inputs
        if x.dtype == np.float32:
            got = int(O.f32_to_key(np.array([kth], dtype=np.float32))[0])
        else:
            got = int(kth)
        assert got == ref, c
        assert st["alpha"] == c["alpha"]
        n += 1
    assert n >= 20


@pytest.mark.parametrize("dist", ["u32", "normal"])
def test_full_size_properties(dist):
    """N=2^28 (1 GiB): kth rank property, sortedness and index validity,
    checked with independent torch reductions on the device."""
    import torch

    import drtopksc_b200 as D
    n = 1 << 28
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    if dist == "u32":
        t = torch.randint(-(1 << 31), 1 << 31, (n,), dtype=torch.int64, device="cuda", generator=g).to(torch.int32)
    else:
        z = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
        t = (z * 2.0 ** 28 + 2.0 ** 31).round().clamp(0, 2 ** 32 - 1).to(torch.int64).to(torch.int32)
        del z
    u = t.to(torch.int64) & 0xFFFFFFFF
    h = D.default_handle()
    for k in (1, 1024, 1 << 16, 1 << 20):
        kth, vals, idx = h.topk(t, k, sorted=True)
        K = int(kth.to(torch.int64).item()) & 0xFFFFFFFF
        gt = int((u > K).sum().item())
        ge = int((u >= K).sum().item())
        assert gt < k <= ge, (k, gt, ge)
        v = vals.to(torch.int64) & 0xFFFFFFFF
        assert bool((v[:-1] >= v[1:]).all())
        assert int(v[-1].item()) == K
        assert bool((u[idx] == v).all())
        assert int(torch.unique(idx).numel()) == k
        # ties at K take the lowest indices
        eq_idx = idx[v == K]
        first_eq = torch.nonzero(u == K).flatten()[: eq_idx.numel()]
        assert bool((torch.sort(eq_idx).values == first_eq).all())


@pytest.mark.parametrize("dist", ["u32", "normal", "fewdigits", "f32n"])
def test_bitonic_variant(dist):
    x = O.gen(dist, 1 << 20, 101)
    for k in (1, 2, 16, 128, 1024, 2048):
        st = check_exact(x, k, algo="bitonic")
        alpha = O.ref_alpha(20, k)
        bv, bi = O.bitonic_topk(O.as_keys(x), k, st["alpha"])
        ev, ei = expected(x, k)[1:]
        assert np.array_equal(bi, ei)


def test_bitonic_reference_shape_and_normal():
    import drtopksc_b200 as D
    x = O.gen("u32", 1 << 20, 103)
    t = to_dev(x)
    for k, alpha in ((128, 10), (1024, 8), (16, 12)):
        kth, vals, idx = D.bitonic_topk(t, x.size, k, alpha)
        ek, ev, ei = expected(x, k)
        assert kth == ek
        assert np.array_equal(vals.cpu().numpy().view(np.uint32), ev)
        assert np.array_equal(idx.cpu().numpy(), ei)
        kth2, vals2, _ = D.bitonic_topk(t, x.size, k, alpha, NormalBitonic=1)
        assert kth2 == ek and np.array_equal(vals2.cpu().numpy().view(np.uint32), ev)
    with pytest.raises(D.DrTopKError):
        D.bitonic_topk(t, x.size, 100, 8)  # k not a power of two (sampleBitonic.cu:198-202)
    with pytest.raises(D.DrTopKError):
        D.bitonic_topk(t, x.size, 4096, 8)  # beyond the shared-memory network


@pytest.mark.parametrize("alpha", list(range(1, 17)))
def test_sampler_delegates_every_alpha(alpha):
    """Delegates written by the sampler equal sampleMax / the top-2 sampler of
    the reference (restated by the oracle) for every subrange size."""
    import torch

    import drtopksc_b200 as D
    log2n = 18
    x = O.gen("normal", 1 << log2n, alpha)
    t = to_dev(x)
    S = 1 << alpha
    nsub = x.size // S
    for dflt in ((True, False) if alpha >= 2 else (False,)):
        k = 1 if dflt else 2
        beta = 2
        Max_d = torch.zeros(nsub * beta, dtype=torch.int32, device="cuda")
        kth, _ = D.sample_radix_select(t, x.size, k, 256, 8, 3, nsub, S, alpha, Max_d, beta, dflt)
        dl = Max_d.cpu().numpy().view(np.uint32)
        if dflt:
            assert np.array_equal(dl[:nsub], O.sample_max(x, alpha)), alpha
        else:
            assert np.array_equal(dl, O.sample_top2(x, alpha)), alpha
        assert kth == O.topk_exact(x, k, False)[0]


@pytest.mark.parametrize("dist,n,k,alpha,path", [
    ("u32", 1 << 23, 1 << 14, 2, 2), ("normal", 1 << 23, 1 << 16, 6, 1), ("f32n", 1 << 23, 5000, 1, 2),
    ("fewdigits", 1 << 22, 3000, 1, 2)])
def test_split_mode_large_concatenation(dist, n, k, alpha, path):
    """Concatenations of >= 16 MB run as separate filter/gather kernels between
    two launches of the fused kernel; results must not change."""
    x = O.gen(dist, n, n + k)
    st = check_exact(x, k, alpha=alpha, path=path)
    _, ost = O.radix_final_kth(x, k, 8, alpha=alpha, path=path)
    assert st["first_threshold"] == ost["first_flag"]
    assert st["n_selected"] == ost["n_selected"]


@pytest.mark.parametrize("dist,n,k,alpha,digits,sorted_", [
    ("u32", 1 << 23, 1 << 15, 3, 2, False), ("u32", 1 << 23, 1 << 15, 3, 2, True),
    ("f32n", 1 << 23, 1 << 14, 3, 2, False), ("normal", 1 << 23, 1 << 17, 2, 1, False),
    ("fewdigits", 1 << 22, 1 << 12, 1, 2, False)])
def test_split_mode_unsorted_and_two_digit_threshold(dist, n, k, alpha, digits, sorted_):
    """Split mode with the level-1 delegate histogram as its own kernel (two
    threshold digits), and with unsorted output written by the level-0 split
    straight into the caller's arrays: same multiset, same lowest-index ties."""
    x = O.gen(dist, n, 7 * n + k)
    kth, vals, idx, st = run_topk(x, k, sorted=sorted_, alpha=alpha, path=2, first_digits=digits)
    ek, ev, ei = expected(x, k, True)
    if not sorted_:
        keys = O.as_keys(vals)
        order = np.lexsort((idx, -keys.astype(np.int64)))
        vals, idx = vals[order], idx[order]
    assert same_bits(kth, ek), (dist, k, st)
    assert same_bits(vals, ev), (dist, k, st)
    assert np.array_equal(idx, ei), (dist, k, st)
    assert st["device_error"] == 0
    assert st["levels_first"] == digits
