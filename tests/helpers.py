"""Shared helpers for the parity tests: run the CUDA path through the C ABI
and compare with the CPU oracle (oracle/ is test infrastructure)."""
import numpy as np

from oracle import oracle as O


def to_dev(x: np.ndarray, offset: int = 0):
    """Copy a uint32/float32 array to the GPU (optionally at an element offset
    inside a larger allocation, to exercise unaligned inputs)."""
    import torch
    if x.dtype == np.float32:
        t = torch.empty(x.size + offset, dtype=torch.float32, device="cuda")
        t[offset:] = torch.from_numpy(x).cuda()
    else:
        t = torch.empty(x.size + offset, dtype=torch.int32, device="cuda")
        t[offset:] = torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint32).view(np.int32)).cuda()
    return t[offset:]


def run_topk(x: np.ndarray, k: int, offset: int = 0, handle=None, **kw):
    """GPU top-k; returns (kth, values, indices, stats) with values as the
    input's numpy dtype."""
    import drtopksc_b200 as D
    h = handle or D.default_handle()
    t = to_dev(x, offset)
    kth, vals, idx = h.topk(t, k, **kw)
    st = h.stats()
    kt = kth.cpu().numpy()
    v = vals.cpu().numpy() if vals is not None else None
    i = idx.cpu().numpy() if idx is not None else None
    if x.dtype != np.float32:
        kt = kt.view(np.uint32)
        v = v.view(np.uint32) if v is not None else None
    return kt[0], v, i, st


def expected(x: np.ndarray, k: int, largest: bool = True):
    """Oracle top-k in the input's value space: (kth, sorted values, indices)."""
    keys = O.as_keys(x)
    if not largest:
        keys = ~keys
    kth, vals, idx = O.topk_exact(keys, k)
    if not largest:
        kth, vals = ~np.uint32(kth), ~vals
    if x.dtype == np.float32:
        return O.key_to_f32(np.array([kth], dtype=np.uint32))[0], O.key_to_f32(vals), idx
    return np.uint32(kth), vals, idx


def same_bits(a, b) -> bool:
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype == np.float32 or b.dtype == np.float32:
        return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))
    return np.array_equal(a.astype(np.uint32), b.astype(np.uint32))


def sort_pairs(vals, idx, x_dtype, largest=True):
    """Sort (value, index) pairs best-first then by index (host side)."""
    keys = O.as_keys(np.asarray(vals, dtype=x_dtype))
    if not largest:
        keys = ~keys
    order = np.lexsort((idx, -keys.astype(np.int64)))
    return np.asarray(vals)[order], np.asarray(idx)[order]


def tie_fill_ambiguous(keys: np.ndarray, alpha: int, k: int) -> bool:
    """Default path: whether the reference's race-ordered tie fill
    (FillWithKElementsID, radixselect.cuh:602-618) could keep other subranges
    than the lowest-id ones kept here.  Its first select stops at a digit
    whose bin holds one delegate (then one subrange ties) or runs every digit
    (then the flag is the exact k-th delegate): the fill is ambiguous only
    when more subranges share that k-th delegate than the fill needs."""
    d = O.sample_max(keys, alpha)
    kd = np.partition(d, d.size - k)[d.size - k]
    return int((d == kd).sum()) > k - int((d > kd).sum())


def reference_counters_match(keys, case, got, alpha, k):
    """Compare (CountSelectedSubrange, CountLonelyElements, write_pos) with a
    reference fixture; returns the list of mismatches (empty when equal)."""
    dflt = case["path"] == "D"
    bad = []
    if not (got[0] == case["count_selected"] or (dflt and case["count_selected"] > k and got[0] == k)):
        bad.append(("count_selected", got[0], case["count_selected"]))
    if got[1] != case["count_lonely"]:
        bad.append(("count_lonely", got[1], case["count_lonely"]))
    if got[2] != case["write_pos"] and not (dflt and tie_fill_ambiguous(keys, alpha, k)):
        bad.append(("write_pos", got[2], case["write_pos"]))
    return bad
