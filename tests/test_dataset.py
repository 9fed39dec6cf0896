"""The reference's real-dataset readers (RealDatasets/BinaryDataset/
main.cu:109-148) through drtopk_load_dataset, on small synthetic files: the
keys must equal a numpy restatement of each format, tiling and short-file
rule included.  Host only; the GPU half (selecting on the loaded keys with
topk.bin) is in test_cli_gpu.py."""
import numpy as np
import pytest

import drtopksc_b200 as D


def _text(path, scores):
    with open(path, "w") as f:
        for i, s in enumerate(scores):
            f.write("%.9g%s" % (s, "\n" if i % 7 == 6 else " "))


def _ref_arith(scores):
    """(1 - u) * 10^9 mod 2^32 on the float's bit pattern u (main.cu:134-138)."""
    u = np.asarray(scores, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return (((1 - u) & 0xFFFFFFFF) * 1000000000 & 0xFFFFFFFF).astype(np.uint32)


def _score_map(scores):
    v = (np.float32(1.0) - np.asarray(scores, dtype=np.float32)) * np.float32(1e9)
    d = np.trunc(v.astype(np.float64))
    d = np.where(d >= 0, d, 0)
    return np.minimum(d, 4294967295.0).astype(np.uint32)


def test_binary_int32_keeps_bit_patterns(tmp_path):
    rng = np.random.default_rng(1)
    vals = rng.integers(-(1 << 31), 1 << 31, size=5000, dtype=np.int64).astype("<i4")
    p = tmp_path / "scores.dat"
    vals.tofile(p)
    keys, got = D.load_dataset(str(p), 4096, "bin")
    assert got == 4096
    assert np.array_equal(keys, vals[:4096].view(np.uint32))


def test_binary_short_file_repeats_last_value(tmp_path):
    vals = np.array([7, -1, 123456, -2147483648, 42], dtype="<i4")
    p = tmp_path / "short.dat"
    vals.tofile(p)
    keys, got = D.load_dataset(str(p), 16, "bin")
    assert got == 5
    assert np.array_equal(keys[:5], vals.view(np.uint32)) and np.all(keys[5:] == np.uint32(42))


def test_text_reference_arithmetic_and_tiling(tmp_path):
    rng = np.random.default_rng(2)
    scores = rng.random(1000, dtype=np.float32)
    p = tmp_path / "scores.txt"
    _text(p, scores)
    keys, got = D.load_dataset(str(p), 2500, "txt")
    assert got == 1000
    want = _ref_arith(scores)
    assert np.array_equal(keys[:1000], want)
    assert np.array_equal(keys, want[np.arange(2500) % 1000])


def test_text_intended_score_map(tmp_path):
    scores = np.array([0.0, 0.25, 0.5, 0.999999, 1.0, 1.5, -3.0, 0.1234567], dtype=np.float32)
    p = tmp_path / "s.txt"
    _text(p, scores)
    keys, got = D.load_dataset(str(p), 8, "score")
    assert got == 8
    assert np.array_equal(keys, _score_map(scores))
    assert keys[0] == 1000000000 and keys[4] == 0 and keys[5] == 0 and keys[6] == 4000000000


def test_missing_or_empty_file_is_rejected(tmp_path):
    with pytest.raises(D.DrTopKError) as e:
        D.load_dataset(str(tmp_path / "nope.txt"), 8, "txt")
    assert e.value.status == D.EINVAL
    p = tmp_path / "empty.txt"
    p.write_text("")
    with pytest.raises(D.DrTopKError):
        D.load_dataset(str(p), 8, "bin")
