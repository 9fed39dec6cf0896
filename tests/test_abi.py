"""CPU tests of the C ABI boundary: the library loads, exports every symbol
the header declares, and validates arguments without touching a GPU."""
import ctypes
import os
import subprocess

import pytest

import drtopksc_b200 as D


def test_library_exports_every_declared_symbol():
    L = D.lib()
    declared = D.exported_symbols()
    assert len(declared) >= 25
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", D.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert set(declared) <= exported, set(declared) - exported


def test_no_oracle_linked_into_product():
    out = subprocess.run(["nm", "-D", D.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle_" not in out
    ldd = subprocess.run(["ldd", D.LIB_PATH], capture_output=True, text=True).stdout
    assert "liboracle" not in ldd


def test_params_default_and_status_strings():
    p = D.params()
    assert (p.nbits, p.alpha, p.beta, p.path, p.algo, p.num_bucket, p.largest, p.sorted) == (8, -1, 2, 0, 0, 256, 1, 0)
    assert D.lib().drtopk_status_str(D.OK) == b"ok"
    assert b"invalid" in D.lib().drtopk_status_str(D.EINVAL)


@pytest.mark.parametrize("n,k", [(1 << 20, 128), (1 << 30, 1), (1 << 30, 1 << 24), (1000, 7), (1, 1)])
def test_workspace_size_plans_without_gpu(n, k):
    b = D.workspace_size(n, k)
    assert b > 0
    # keys are not part of the workspace; scratch stays a bounded multiple of n
    assert b < 32 * n + (64 << 20)


@pytest.mark.parametrize("n,k,kw", [
    (0, 1, {}), (10, 0, {}), (10, 11, {}), (1 << 20, 5, {"nbits": 3}), (1 << 20, 5, {"nbits": 16}),
    (1 << 20, 5, {"beta": 3, "alpha": 4}), (1 << 20, 5, {"algo": "bucket", "num_bucket": 1}),
    (1 << 20, 5, {"algo": "bucket", "num_bucket": 5000}), (1 << 20, 1 << 19, {"alpha": 10, "path": 1}),
])
def test_invalid_arguments_rejected(n, k, kw):
    with pytest.raises(D.DrTopKError) as e:
        D.workspace_size(n, k, D.U32, D.params(**kw))
    assert e.value.status == D.EINVAL


def test_too_large_n_unsupported():
    with pytest.raises(D.DrTopKError) as e:
        D.workspace_size(1 << 33, 5)
    assert e.value.status == D.EUNSUPPORTED


def test_ref_alpha_matches_reference_formula():
    # main.cu:83 evaluated in double, truncated
    assert [D.ref_alpha(30, 2 ** i) for i in range(25)] == \
        [16, 16, 15, 15, 14, 14, 13, 13, 12, 12, 11, 11, 10, 10, 9, 9, 8, 8, 7, 7, 6, 6, 5, 5, 4]
    from oracle import oracle as O
    for log2n in (10, 20, 26, 30):
        for k in (1, 3, 100, 1000, 1 << 10, 1 << 17):
            if k <= (1 << log2n):
                assert D.ref_alpha(log2n, k) == O.ref_alpha(log2n, k)


def test_autotune_choices_are_valid():
    for n, k in [(1 << 30, 1), (1 << 30, 128), (1 << 30, 1 << 20), (1 << 30, 1 << 24), (1 << 12, 5), (5000, 4999)]:
        p = D.autotune(n, k)
        if p.algo == D.ALGO_PLAIN_RADIX:
            continue
        s = 1 << p.alpha
        m = (n + s - 1) // s
        if p.path == 1:
            assert m >= k
        elif p.path == 4:  # sampled threshold: large k only, no delegate vector
            assert k >= 1 << 16
        else:
            assert p.path == 2 and p.alpha <= 16 and 2 * m >= 1


def test_cli_binary_built():
    assert os.path.exists(os.path.join(os.path.dirname(D.LIB_PATH), "topk.bin"))


def test_autotune_small_problem_and_float_rules():
    # up to 2^13 keys the plain select fits one CTA; up to 2^16 keys it stays
    # the choice above k = 64
    assert D.autotune(1 << 13, 5).algo == D.ALGO_PLAIN_RADIX
    assert D.autotune(1 << 16, 128).algo == D.ALGO_PLAIN_RADIX
    p = D.autotune(1 << 16, 16)
    assert p.algo != D.ALGO_PLAIN_RADIX and p.path in (1, 2)
    # small k: the delegate vector is kept small enough for the one-CTA tail
    for log2n, k in [(20, 1), (20, 128), (22, 1), (22, 16)]:
        p = D.autotune(1 << log2n, k)
        m = (1 << log2n) >> p.alpha
        assert p.path in (1, 2) and (m if p.path == 1 else 2 * m) <= 8192, (log2n, k, p.path, p.alpha)
    # float keys from 2^22: delegate paths below k = 2^13, the sampled threshold from there
    for k in (1, 16, 256, 4096):
        assert D.autotune(1 << 28, k, D.F32).path in (1, 2), k
    for k in (1 << 13, 1 << 16, 1 << 20):
        assert D.autotune(1 << 28, k, D.F32).path == 4, k
    # the N = 2^30 uint32 choices: beta path (alpha 11, 10 from k = 2^15), sampled threshold from 2^17
    for k, alpha in ((1, 11), (1 << 10, 11), (1 << 16, 10)):
        p = D.autotune(1 << 30, k)
        assert (p.path, p.alpha) == (2, alpha), (k, p.path, p.alpha)
    for k in (1 << 17, 1 << 24):
        assert D.autotune(1 << 30, k).path == 4
