"""drtopksc_b200 -- B200-native Dr.Top-k selection (delegate-centric top-k).

Python front-end of ``libdrtopk.so`` (the C ABI in ``include/drtopk.h``).
The compute path is the CUDA library only: if ``libdrtopk.so`` is missing
this module raises on first use; there is no CPU fallback.

Device buffers are torch CUDA tensors (torch is used for device memory and
streams only).  Keys are uint32 (torch.uint32 or int32 bit patterns) or
float32.

Reference operator interface mirrored here (paths inside the reference
project):
  * ``sample_radix_select``  -- baseline+filter+beta+shuffle/radixselect.cuh:1782
  * ``radix_select``         -- baseline+filter+beta+shuffle/radixselect.cuh:1472
  * ``sample_bucket_select`` -- bucket_select/bucketselect_combined.cuh:1279
  * ``bitonic_topk``         -- bitonic/bitonic_com.cuh:609-728 (+ sampleBitonic.cu:192)
  * ``ref_alpha``            -- baseline+filter+beta+shuffle/main.cu:83
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdrtopk.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "drtopk.h")

OK, EINVAL, ENOMEM, ECUDA, EDEVICE, EBUDGET, EUNSUPPORTED, ETIMEOUT, EAGAIN, ECANCELLED = range(10)
U32, F32 = 0, 1
ALGO_RADIX, ALGO_BUCKET, ALGO_BITONIC, ALGO_PLAIN_RADIX, ALGO_AUTO = range(5)
_ALGOS = {"radix": ALGO_RADIX, "bucket": ALGO_BUCKET, "bitonic": ALGO_BITONIC, "plain": ALGO_PLAIN_RADIX,
          "auto": ALGO_AUTO}


class DrTopKError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = _lib_status_str(status)
        super().__init__(f"{what}: {msg} (status {status})" if what else f"{msg} (status {status})")


class Params(ctypes.Structure):
    _fields_ = [("nbits", ctypes.c_int), ("alpha", ctypes.c_int), ("beta", ctypes.c_int), ("path", ctypes.c_int),
                ("algo", ctypes.c_int), ("num_bucket", ctypes.c_int), ("largest", ctypes.c_int),
                ("sorted", ctypes.c_int), ("first_digits", ctypes.c_int), ("team", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("alpha", ctypes.c_int), ("beta", ctypes.c_int), ("algo", ctypes.c_int),
                ("first_threshold", ctypes.c_uint32), ("n_subranges", ctypes.c_uint64),
                ("n_selected", ctypes.c_uint64), ("n_lonely", ctypes.c_uint64), ("n_candidates", ctypes.c_uint64),
                ("levels_first", ctypes.c_int), ("levels_second", ctypes.c_int), ("device_error", ctypes.c_uint32),
                ("ms_sample", ctypes.c_double), ("ms_first", ctypes.c_double), ("ms_concat", ctypes.c_double),
                ("ms_second", ctypes.c_double), ("ms_total", ctypes.c_double), ("team_ctas", ctypes.c_int),
                ("team_cluster", ctypes.c_int), ("kernel_launches", ctypes.c_int),
                ("sample_stride", ctypes.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class SegParams(ctypes.Structure):
    _fields_ = [("algo", ctypes.c_int), ("alpha", ctypes.c_int), ("beta", ctypes.c_int), ("nbits", ctypes.c_int),
                ("bucket", ctypes.c_int), ("chunk_log2", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("singles", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("batched", ctypes.c_uint64),
                ("pinned_allocs", ctypes.c_uint64), ("worker_ticks", ctypes.c_uint64),
                ("host_ms_pinned", ctypes.c_double), ("host_ms_launch", ctypes.c_double),
                ("host_ms_complete", ctypes.c_double), ("retries", ctypes.c_uint64), ("host_ms_retry", ctypes.c_double),
                ("host_ms_alloc", ctypes.c_double)]


class Result(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("status", ctypes.c_int), ("kth", ctypes.c_uint32),
                ("t_submit_ms", ctypes.c_double), ("t_start_ms", ctypes.c_double), ("t_done_ms", ctypes.c_double)]


_lib = None


def build(force: bool = False) -> str:
    """Compile libdrtopk.so and topk.bin in-tree with nvcc (sm_100a)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-j8", "-C", _HERE], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    """The loaded CUDA library.  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} not found: build it with `make -C {_HERE}` "
                               "(or __graft_entry__.build()); there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        vp, u64, i32, sz = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_size_t
        st = ctypes.c_int
        P = ctypes.POINTER
        sig = {
            "drtopk_params_default": (None, [P(Params)]),
            "drtopk_status_str": (ctypes.c_char_p, [st]),
            "drtopk_create": (st, [P(vp), i32, sz]),
            "drtopk_destroy": (st, [vp]),
            "drtopk_workspace_size": (st, [u64, u64, i32, P(Params), P(sz)]),
            "drtopk_select": (st, [vp, vp, i32, u64, u64, P(Params), vp, vp, vp, vp]),
            "drtopk_select_ws": (st, [vp, vp, i32, u64, u64, P(Params), vp, vp, vp, vp, sz, vp]),
            "drtopk_select_noalloc": (st, [vp, i32, u64, u64, P(Params), vp, vp, vp, vp]),
            "drtopk_noalloc_sync_check": (st, [vp]),
            "drtopk_load_dataset": (st, [ctypes.c_char_p, i32, u64, P(ctypes.c_uint32), P(ctypes.c_uint64)]),
            "drtopk_bmw_select": (st, [vp, vp, P(ctypes.c_uint32), u64, u64, i32, P(ctypes.c_uint32),
                                       P(ctypes.c_uint64), P(ctypes.c_double), P(ctypes.c_double)]),
            "drtopk_sync_check": (st, [vp, vp]),
            "drtopk_last_stats": (st, [vp, P(Stats)]),
            "drtopk_autotune": (st, [u64, u64, i32, P(Params)]),
            "drtopk_profile_begin": (st, [vp, i32]),
            "drtopk_selftest_wait_timeout": (st, [i32, P(ctypes.c_double)]),
            "drtopk_profile_end": (st, [vp, P(ctypes.c_double), P(ctypes.c_double), P(ctypes.c_int)]),
            "drtopk_radix_select": (st, [vp, i32, i32, i32, P(ctypes.c_uint32), i32, i32]),
            "drtopk_bitonic_topk": (st, [vp, i32, i32, i32, i32, vp, vp, P(ctypes.c_uint32)]),
            "drtopk_batch_create": (st, [P(vp), i32]),
            "drtopk_batch_destroy": (st, [vp]),
            "drtopk_batch_plan": (st, [vp, i32, P(ctypes.c_uint64), P(ctypes.c_uint32), P(ctypes.c_int), i32]),
            "drtopk_batch_run": (st, [vp, vp, vp, vp, vp, vp]),
            "drtopk_batch_run_graph": (st, [vp, vp, vp, vp, vp, vp]),
            "drtopk_batch_sync_check": (st, [vp, vp]),
            "drtopk_batch_describe": (st, [vp, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int)]),
            "drtopk_batch_plan_params": (st, [vp, i32, P(ctypes.c_uint64), P(ctypes.c_uint32), P(ctypes.c_int), i32,
                                              P(SegParams)]),
            "drtopk_batch_describe_params": (st, [vp, P(SegParams)]),
            "drtopk_server_create": (st, [P(vp), i32, sz, i32]),
            "drtopk_server_destroy": (st, [vp]),
            "drtopk_server_submit": (st, [vp, vp, i32, u64, u64, i32, vp, vp, P(ctypes.c_uint64)]),
            "drtopk_server_submit_device": (st, [vp, vp, i32, u64, u64, i32, vp, vp, P(ctypes.c_uint64)]),
            "drtopk_server_poll": (st, [vp, P(Result), i32, P(ctypes.c_int)]),
            "drtopk_server_cancel": (st, [vp, u64]),
            "drtopk_server_drain": (st, [vp, i32]),
            "drtopk_server_usage": (st, [vp, P(sz), P(ctypes.c_int), P(ctypes.c_int)]),
            "drtopk_server_stats": (st, [vp, P(ServerStats)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        # the reference-shaped entry points take many ints/pointers; declare them fully
        dp = P(ctypes.c_double)
        L.drtopk_sample_radix_select.restype = st
        L.drtopk_sample_radix_select.argtypes = (
            [vp, i32, i32, i32, P(ctypes.c_uint32), i32, i32, i32, i32, i32, dp, dp, dp, dp, vp, vp]
            + [i32] * 12 + [vp, vp, vp, vp, vp])
        L.drtopk_sample_bucket_select.restype = st
        L.drtopk_sample_bucket_select.argtypes = (
            [vp, i32, i32, i32, P(ctypes.c_uint32), i32, i32, i32, dp, dp, dp, dp, vp, vp] + [i32] * 6
            + [vp, vp, vp, vp, vp])
        _lib = L
    return _lib


def _lib_status_str(s: int) -> str:
    try:
        return lib().drtopk_status_str(s).decode()
    except Exception:  # noqa: BLE001 - message formatting must not raise
        return f"status {s}"


def check(status: int, what: str = ""):
    if status != OK:
        raise DrTopKError(status, what)


def exported_symbols() -> list[str]:
    """Function names the public header declares."""
    import re
    txt = open(HEADER_PATH).read()
    return sorted(set(re.findall(r"DRTOPK_API\s+[\w\s\*]+?\b(drtopk_\w+)\s*\(", txt)))


# ----------------------------------------------------------------- params
def params(nbits: int = 8, alpha: int = -1, beta: int = 2, path: int = 0, algo="radix", num_bucket: int = 256,
           largest: bool = True, sorted: bool = False, first_digits: int = 0, team: int = 0) -> Params:
    """team: 0 auto, 1 whole-GPU cooperative grid, 2 one thread-block cluster,
    3 one CTA with the sets in shared memory, 4 shared GPU (auto, with one cluster
    of at most 8 CTAs instead of the whole GPU), for the phases after the sampler."""
    p = Params()
    lib().drtopk_params_default(ctypes.byref(p))
    p.nbits, p.alpha, p.beta, p.path, p.team = nbits, alpha, beta, path, team
    p.algo = _ALGOS[algo] if isinstance(algo, str) else int(algo)
    p.num_bucket, p.largest, p.sorted, p.first_digits = num_bucket, int(bool(largest)), int(bool(sorted)), first_digits
    return p


def ref_alpha(log2n: float, k: int) -> int:
    """alpha = (int)(0.5*(log2N - log(k)/log(2) + 3)) -- baseline+filter+beta+shuffle/main.cu:83."""
    return int(0.5 * (log2n - math.log(k) / math.log(2) + 3))


def workspace_size(n: int, k: int, dtype: int = U32, p: Params | None = None) -> int:
    b = ctypes.c_size_t(0)
    check(lib().drtopk_workspace_size(n, k, dtype, ctypes.byref(p) if p is not None else None, ctypes.byref(b)),
          "drtopk_workspace_size")
    return b.value


def autotune(n: int, k: int, dtype: int = U32, p: Params | None = None) -> Params:
    p = p if p is not None else params(alpha=-2)
    check(lib().drtopk_autotune(n, k, dtype, ctypes.byref(p)), "drtopk_autotune")
    return p


# ----------------------------------------------------------------- torch helpers
def _torch():
    import torch
    return torch


def _dtype_code(t) -> int:
    torch = _torch()
    if t.dtype == torch.float32:
        return F32
    if t.dtype in (torch.int32, getattr(torch, "uint32", torch.int32)):
        return U32
    raise TypeError(f"keys must be uint32/int32 bit patterns or float32, got {t.dtype}")


def _stream_ptr(stream) -> int | None:
    if stream is None:
        torch = _torch()
        return torch.cuda.current_stream().cuda_stream or None
    return getattr(stream, "cuda_stream", stream) or None


class Handle:
    """A drtopk handle: resident workspace + timers on one device."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self._h = ctypes.c_void_p()
        self.device = device
        check(lib().drtopk_create(ctypes.byref(self._h), device, hbm_budget_bytes), "drtopk_create")

    def close(self):
        if self._h:
            lib().drtopk_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    @property
    def ptr(self):
        return self._h

    def select_raw(self, keys_ptr: int, dtype: int, n: int, k: int, p: Params, kth_ptr=None, vals_ptr=None,
                   idx_ptr=None, stream=None):
        check(lib().drtopk_select(self._h, keys_ptr, dtype, n, k, ctypes.byref(p), kth_ptr, vals_ptr, idx_ptr,
                                  stream), "drtopk_select")

    def bmw_select(self, d_keys, h_keys, k: int, alpha: int):
        """BMW experiment (drtopk_bmw_select): device delegates, host heap scan
        with delegate skipping over h_keys (numpy uint32, the same keys as the
        CUDA tensor d_keys).  Returns (kth, keys skipped, ms sample, ms scan)."""
        import numpy as np
        hk = np.ascontiguousarray(h_keys, dtype=np.uint32)
        kth, sk = ctypes.c_uint32(0), ctypes.c_uint64(0)
        m1, m2 = ctypes.c_double(0), ctypes.c_double(0)
        check(lib().drtopk_bmw_select(self._h, d_keys.data_ptr(), hk.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                      hk.size, k, alpha, ctypes.byref(kth), ctypes.byref(sk), ctypes.byref(m1),
                                      ctypes.byref(m2)), "drtopk_bmw_select")
        return kth.value, sk.value, m1.value, m2.value

    def sync_check(self, stream=None):
        check(lib().drtopk_sync_check(self._h, _stream_ptr(stream)), "drtopk_sync_check")

    def profile_begin(self, max_calls: int):
        check(lib().drtopk_profile_begin(self._h, max_calls), "drtopk_profile_begin")

    def profile_end(self):
        """(summed sampler ms, summed fused-kernel ms, calls) since profile_begin."""
        a, b, c = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_int(0)
        check(lib().drtopk_profile_end(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
              "drtopk_profile_end")
        return a.value, b.value, c.value

    def stats(self) -> dict:
        s = Stats()
        check(lib().drtopk_last_stats(self._h, ctypes.byref(s)), "drtopk_last_stats")
        return s.as_dict()

    def topk(self, keys, k: int, *, want_values: bool = True, want_indices: bool = True, stream=None, sync=True,
             out=None, **pkw):
        """Exact top-k of a 1-D CUDA tensor.  Returns (kth, values, indices) tensors
        (kth has shape [1] and the input's dtype)."""
        torch = _torch()
        if keys.dim() != 1 or not keys.is_cuda or not keys.is_contiguous():
            raise ValueError("keys must be a contiguous 1-D CUDA tensor")
        dt = _dtype_code(keys)
        n = keys.numel()
        p = params(**pkw)
        if out is None:
            kth = torch.empty(1, dtype=keys.dtype, device=keys.device)
            vals = torch.empty(k, dtype=keys.dtype, device=keys.device) if want_values else None
            idx = torch.empty(k, dtype=torch.int64, device=keys.device) if want_indices else None
        else:
            kth, vals, idx = out
        sp = _stream_ptr(stream)
        self.select_raw(keys.data_ptr(), dt, n, k, p, kth.data_ptr(), vals.data_ptr() if vals is not None else None,
                        idx.data_ptr() if idx is not None else None, sp)
        if sync:
            check(lib().drtopk_sync_check(self._h, sp), "drtopk_sync_check")
        return kth, vals, idx


_default_handles: dict[int, Handle] = {}


def default_handle(device: int = 0) -> Handle:
    h = _default_handles.get(device)
    if h is None:
        h = _default_handles[device] = Handle(device)
    return h


def topk(keys, k: int, **kw):
    """Exact top-k (k-th value, values, indices) of a 1-D CUDA tensor via the default handle."""
    return default_handle(keys.device.index or 0).topk(keys, k, **kw)


# ----------------------------------------------------------------- real-dataset readers
DATASET_BIN_I32, DATASET_TXT_REF, DATASET_TXT_SCORE = 0, 1, 2
_FORMATS = {"bin": DATASET_BIN_I32, "txt": DATASET_TXT_REF, "score": DATASET_TXT_SCORE}


def load_dataset(path: str, n: int, fmt="txt"):
    """Keys of a score file as the reference's real-dataset build reads them
    (RealDatasets/BinaryDataset/main.cu:109-148; drtopk_load_dataset):
    returns (uint32 numpy array of n keys, values read from the file)."""
    import numpy as np
    code = _FORMATS[fmt] if isinstance(fmt, str) else int(fmt)
    out = np.empty(n, dtype=np.uint32)
    got = ctypes.c_uint64(0)
    check(lib().drtopk_load_dataset(os.fsencode(path), code, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                    ctypes.byref(got)), "drtopk_load_dataset")
    return out, got.value


# ----------------------------------------------------------------- reference-shaped wrappers
def sample_radix_select(vec_d, num_element: int, k: int, num_bucket: int, NBitsperDigit: int, CurrentDigit: int,
                        NSubranges: int, SubRangesize: int, alpha: int, Max_d, beta: int = 2,
                        defaultContribution: bool | None = None, counters=None, SubrangeId_d=None):
    """Mirror of sample_radix_select (radixselect.cuh:1782): returns
    (TopKElement, (sample, first, second, concat) seconds).  Max_d receives
    the delegates and SubrangeId_d (int32 CUDA tensor, optional) their
    subrange ids; counters, if given, is an int32 CUDA tensor of 3 that
    receives the reference's (CountSelectedSubrange, CountLonelyElements,
    write_pos) -- zero it before the call, as the reference's caller does."""
    if defaultContribution is None:
        defaultContribution = alpha > 5
    kth = ctypes.c_uint32(0)
    t = [ctypes.c_double(0) for _ in range(4)]
    c = [None, None, None]
    if counters is not None:
        base = counters.data_ptr()
        c = [base, base + 4, base + 8]
    st = lib().drtopk_sample_radix_select(
        vec_d.data_ptr(), num_element, k, num_bucket, ctypes.byref(kth), NBitsperDigit, CurrentDigit, NSubranges,
        SubRangesize, alpha, ctypes.byref(t[0]), ctypes.byref(t[1]), ctypes.byref(t[2]), ctypes.byref(t[3]),
        Max_d.data_ptr() if Max_d is not None else None,
        SubrangeId_d.data_ptr() if SubrangeId_d is not None else None, 256 << 5, 8, 3, 32, (256 << 5) // 8,
        ((256 << 5) // 8) * SubRangesize, 1, (256 << 5) + (256 << 5 >> 5), 256, beta, int(bool(defaultContribution)),
        min(32, SubRangesize), None, c[1], c[2], None, c[0])
    check(st, "drtopk_sample_radix_select")
    return kth.value, tuple(x.value for x in t)


def radix_select(vec_d, num_element: int, k: int, num_bucket: int = 256, NBitsperDigit: int = 8,
                 CurrentDigit: int | None = None) -> int:
    """Mirror of radix_select (radixselect.cuh:1472): plain radix select, returns TopKElement."""
    if CurrentDigit is None:
        CurrentDigit = 32 // NBitsperDigit - 1
    kth = ctypes.c_uint32(0)
    check(lib().drtopk_radix_select(vec_d.data_ptr(), num_element, k, num_bucket, ctypes.byref(kth), NBitsperDigit,
                                    CurrentDigit), "drtopk_radix_select")
    return kth.value


def sample_bucket_select(vec_d, num_element: int, k: int, num_bucket: int, NSubranges: int, SubRangesize: int,
                         alpha: int, beta: int = 2, defaultContribution: bool | None = None, counters=None,
                         SubrangeId_d=None):
    """Mirror of sample_bucket_select (bucketselect_combined.cuh:1279) with exact integer buckets;
    counters and SubrangeId_d as for sample_radix_select."""
    if defaultContribution is None:
        defaultContribution = alpha > 5
    kth = ctypes.c_uint32(0)
    t = [ctypes.c_double(0) for _ in range(4)]
    c = [None, None, None]
    if counters is not None:
        base = counters.data_ptr()
        c = [base, base + 4, base + 8]
    st = lib().drtopk_sample_bucket_select(
        vec_d.data_ptr(), num_element, k, num_bucket, ctypes.byref(kth), NSubranges, SubRangesize, alpha,
        ctypes.byref(t[0]), ctypes.byref(t[1]), ctypes.byref(t[2]), ctypes.byref(t[3]), None,
        SubrangeId_d.data_ptr() if SubrangeId_d is not None else None, beta,
        int(bool(defaultContribution)), min(32, SubRangesize), 256, (256 << 5) + 256, 256 << 5, None, c[0], c[1],
        c[2], None)
    check(st, "drtopk_sample_bucket_select")
    return kth.value, tuple(x.value for x in t)


def bitonic_topk(A_d, N: int, k: int, alpha: int, NormalBitonic: int = 0, want_indices: bool = True):
    """Dr.Top-k bitonic top-k (bitonic_com.cuh:609-728): returns (kth, sorted-desc values, indices)."""
    torch = _torch()
    out = torch.empty(k, dtype=A_d.dtype, device=A_d.device)
    idx = torch.empty(k, dtype=torch.int64, device=A_d.device) if want_indices else None
    kth = ctypes.c_uint32(0)
    check(lib().drtopk_bitonic_topk(A_d.data_ptr(), N, k, alpha, NormalBitonic, out.data_ptr(),
                                    idx.data_ptr() if idx is not None else None, ctypes.byref(kth)),
          "drtopk_bitonic_topk")
    return kth.value, out, idx


@dataclass
class SegmentResult:
    kth: object
    values: object
    indices: object


class Batch:
    """Batched top-k: many segments of one key buffer in one persistent launch
    (drtopk_batch_*).  Keys of all segments live in one 32-bit buffer (float
    segments as their bit patterns); outputs are packed per segment."""

    def __init__(self, device: int = 0):
        self._b = ctypes.c_void_p()
        self.device = device
        check(lib().drtopk_batch_create(ctypes.byref(self._b), device), "drtopk_batch_create")
        self.nseg = 0
        self.out_offsets = None

    def close(self):
        if self._b:
            lib().drtopk_batch_destroy(self._b)
            self._b = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def plan(self, offsets, ks, dtypes=None, sorted: bool = False, params=None):
        """params: None (every knob tuned) or one dict per segment with any of
        algo ("plain", "radix", "bitonic"), alpha, beta, nbits, bucket,
        chunk_log2 -- the ones left out are tuned (drtopk_seg_params_t)."""
        import numpy as np
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        kk = np.ascontiguousarray(ks, dtype=np.uint32)
        nseg = kk.size
        dt = np.ascontiguousarray(dtypes if dtypes is not None else np.zeros(nseg), dtype=np.int32)
        arr = None
        if params is not None:
            arr = (SegParams * nseg)()
            for s, q in enumerate(params):
                algo = q.get("algo", -1)
                if isinstance(algo, str):
                    algo = _ALGOS[algo]
                arr[s] = SegParams(algo, q.get("alpha", -1), q.get("beta", -1), q.get("nbits", -1),
                                   int(q.get("bucket", -1)), q.get("chunk_log2", -1))
        check(lib().drtopk_batch_plan_params(self._b, nseg, off.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                             kk.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                             dt.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), int(bool(sorted)),
                                             arr),
              "drtopk_batch_plan_params")
        self.nseg = nseg
        self.out_offsets = np.concatenate([[0], np.cumsum(kk.astype(np.int64))])
        return self

    def run(self, keys, kth, vals=None, idx=None, graph: bool = False, stream=None):
        fn = lib().drtopk_batch_run_graph if graph else lib().drtopk_batch_run
        check(fn(self._b, keys.data_ptr(), kth.data_ptr(), vals.data_ptr() if vals is not None else None,
                 idx.data_ptr() if idx is not None else None, _stream_ptr(stream)), "drtopk_batch_run")

    def sync_check(self, stream=None):
        check(lib().drtopk_batch_sync_check(self._b, _stream_ptr(stream)), "drtopk_batch_sync_check")

    def describe(self):
        import numpy as np
        a = np.zeros(self.nseg, dtype=np.int32)
        al = np.zeros(self.nseg, dtype=np.int32)
        be = np.zeros(self.nseg, dtype=np.int32)
        P = ctypes.POINTER(ctypes.c_int)
        check(lib().drtopk_batch_describe(self._b, a.ctypes.data_as(P), al.ctypes.data_as(P), be.ctypes.data_as(P)),
              "drtopk_batch_describe")
        return a, al, be

    def describe_params(self):
        """The tuned knobs of every segment, as dicts (drtopk_seg_params_t)."""
        arr = (SegParams * self.nseg)()
        check(lib().drtopk_batch_describe_params(self._b, arr), "drtopk_batch_describe_params")
        return [{f: getattr(q, f) for f, _ in SegParams._fields_} for q in arr]


class Server:
    """Served form (drtopk_server_*): continuous batching of top-k requests
    under an HBM byte budget.  submit() takes a host numpy array (copied) or
    a CUDA tensor (kept resident, caller-owned until the request finishes)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 120 << 30, max_inflight: int = 64):
        self._s = ctypes.c_void_p()
        check(lib().drtopk_server_create(ctypes.byref(self._s), device, hbm_budget_bytes, max_inflight),
              "drtopk_server_create")
        self._bufs = {}

    def close(self):
        if self._s:
            lib().drtopk_server_destroy(self._s)
            self._s = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def submit(self, keys, k: int, sorted: bool = False, want_values: bool = True, want_indices: bool = True) -> int:
        """Returns the request id; results (kth, values, indices) come from poll()."""
        import numpy as np
        rid = ctypes.c_uint64(0)
        if hasattr(keys, "is_cuda"):
            n = keys.numel()
            dt = _dtype_code(keys)
            vdtype = np.float32 if dt == F32 else np.uint32
        else:
            keys = np.ascontiguousarray(keys)
            n = keys.size
            dt = F32 if keys.dtype == np.float32 else U32
            vdtype = keys.dtype if dt == F32 else np.uint32
        vals = np.empty(k, dtype=vdtype) if want_values else None
        idx = np.empty(k, dtype=np.int64) if want_indices else None
        vp = vals.ctypes.data if vals is not None else None
        ip = idx.ctypes.data if idx is not None else None
        if hasattr(keys, "is_cuda"):
            st = lib().drtopk_server_submit_device(self._s, keys.data_ptr(), dt, n, k, int(bool(sorted)), vp, ip,
                                                   ctypes.byref(rid))
        else:
            st = lib().drtopk_server_submit(self._s, keys.ctypes.data, dt, n, k, int(bool(sorted)), vp, ip,
                                            ctypes.byref(rid))
        check(st, "drtopk_server_submit")
        self._bufs[rid.value] = (keys, vals, idx, dt)
        return rid.value

    def poll(self, max_results: int = 1024):
        """List of dicts: id, status, kth, values, indices, t_submit/t_start/t_done (ms)."""
        import numpy as np
        arr = (Result * max_results)()
        cnt = ctypes.c_int(0)
        st = lib().drtopk_server_poll(self._s, arr, max_results, ctypes.byref(cnt))
        if st not in (OK, EAGAIN):
            check(st, "drtopk_server_poll")
        out = []
        for i in range(cnt.value):
            r = arr[i]
            keys, vals, idx, dt = self._bufs.pop(r.id, (None, None, None, U32))
            kth = np.array([r.kth], dtype=np.uint32)
            if dt == F32:
                kth = kth.view(np.float32)
            out.append({"id": r.id, "status": r.status, "kth": kth[0], "values": vals, "indices": idx,
                        "t_submit": r.t_submit_ms, "t_start": r.t_start_ms, "t_done": r.t_done_ms})
        return out

    def cancel(self, rid: int) -> bool:
        return lib().drtopk_server_cancel(self._s, rid) == OK

    def drain(self, timeout_ms: int = -1):
        check(lib().drtopk_server_drain(self._s, timeout_ms), "drtopk_server_drain")

    def usage(self):
        b, i, q = ctypes.c_size_t(0), ctypes.c_int(0), ctypes.c_int(0)
        check(lib().drtopk_server_usage(self._s, ctypes.byref(b), ctypes.byref(i), ctypes.byref(q)), "usage")
        return b.value, i.value, q.value

    def stats(self) -> dict:
        """Worker counters since creation (drtopk_server_stats)."""
        st = ServerStats()
        check(lib().drtopk_server_stats(self._s, ctypes.byref(st)), "drtopk_server_stats")
        return {f: getattr(st, f) for f, _ in ServerStats._fields_}
