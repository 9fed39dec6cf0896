"""ctypes front-end of the CPU oracle (oracle/liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Used by tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
as the checker.  The product library (drtopksc_b200) never imports this module.
Every function restates part of the reference's Dr.Top-k path; the C source
(oracle/drtopk_oracle.cpp) cites the reference file:line each one follows.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


class OracleStats(ctypes.Structure):
    _fields_ = [
        ("alpha", ctypes.c_int),
        ("beta_path", ctypes.c_int),
        ("n_subranges", ctypes.c_uint64),
        ("first_flag", ctypes.c_uint32),
        ("first_digits", ctypes.c_int),
        ("n_selected", ctypes.c_uint64),
        ("n_lonely", ctypes.c_uint64),
        ("n_candidates", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def build() -> str:
    """Compile liboracle.so with g++ (seconds)."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        f32p = ctypes.POINTER(ctypes.c_float)
        i64p = ctypes.POINTER(ctypes.c_int64)
        u64, i64, i32, u32 = ctypes.c_uint64, ctypes.c_int64, ctypes.c_int, ctypes.c_uint32
        sig = {
            "oracle_gen_uniform_u32": (None, [u32, u64, u32p]),
            "oracle_gen_normal_u32": (None, [u32, u64, ctypes.c_double, ctypes.c_double, u32p]),
            "oracle_gen_uniform_f32": (None, [u32, u64, f32p]),
            "oracle_gen_normal_f32": (None, [u32, u64, f32p]),
            "oracle_gen_fewdigits_u32": (None, [u32, u64, u32, u32p]),
            "oracle_f32_to_key": (None, [f32p, u64, u32p]),
            "oracle_key_to_f32": (None, [u32p, u64, f32p]),
            "oracle_ref_alpha": (i32, [i32, ctypes.c_double]),
            "oracle_ref_alpha_bucket": (i32, [i32, ctypes.c_double]),
            "oracle_sample_max": (None, [u32p, u64, i32, u32p]),
            "oracle_sample_top2": (None, [u32p, u64, i32, u32p]),
            "oracle_digit_select": (u32, [u32p, u64, i64, i32, i32, i32, i32, ctypes.POINTER(i32)]),
            "oracle_radix_final_kth": (i32, [u32p, u64, i64, i32, i32, i32, u32p, ctypes.POINTER(OracleStats)]),
            "oracle_topk_exact": (None, [u32p, u64, i64, u32p, u32p, i64p]),
            "oracle_topk_mt": (ctypes.c_double, [u32p, u64, i64, i32, u32p, u32p]),
            "oracle_bucket_select": (u32, [u32p, u64, i64, i32]),
            "oracle_bucket_kth": (i32, [u32p, u64, i64, i32, i32, i32, u32p, ctypes.POINTER(OracleStats)]),
            "oracle_bitonic_topk": (i32, [u32p, u64, i64, i32, u32p, i64p]),
            "oracle_digest": (ctypes.c_uint64, [u32p, i64p, i64]),
            "oracle_bmw_kth": (u32, [u32p, u64, i64, i32, ctypes.POINTER(ctypes.c_uint64)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


# ----------------------------------------------------------------- generators
def gen(dist: str, n: int, seed: int) -> np.ndarray:
    """Seeded inputs.  u32/normal/fewdigits give uint32 keys; f32u/f32n give float32."""
    L = lib()
    if dist in ("f32u", "f32n"):
        out = np.empty(n, dtype=np.float32)
        (L.oracle_gen_uniform_f32 if dist == "f32u" else L.oracle_gen_normal_f32)(seed, n, _p(out, ctypes.c_float))
        return out
    out = np.empty(n, dtype=np.uint32)
    if dist == "u32":
        L.oracle_gen_uniform_u32(seed, n, _p(out, ctypes.c_uint32))
    elif dist == "normal":
        L.oracle_gen_normal_u32(seed, n, 2.0 ** 31, 2.0 ** 28, _p(out, ctypes.c_uint32))
    elif dist == "fewdigits":
        L.oracle_gen_fewdigits_u32(seed, n, 0xABCDEF, _p(out, ctypes.c_uint32))
    else:
        raise ValueError(dist)
    return out


def f32_to_key(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.size, dtype=np.uint32)
    lib().oracle_f32_to_key(_p(x, ctypes.c_float), x.size, _p(out, ctypes.c_uint32))
    return out


def key_to_f32(k: np.ndarray) -> np.ndarray:
    k = np.ascontiguousarray(k, dtype=np.uint32)
    out = np.empty(k.size, dtype=np.float32)
    lib().oracle_key_to_f32(_p(k, ctypes.c_uint32), k.size, _p(out, ctypes.c_float))
    return out


def as_keys(x: np.ndarray) -> np.ndarray:
    return f32_to_key(x) if x.dtype == np.float32 else np.ascontiguousarray(x, dtype=np.uint32)


# ----------------------------------------------------------------- algorithm
def ref_alpha(log2n: int, k: int) -> int:
    return lib().oracle_ref_alpha(log2n, float(k))


def ref_alpha_bucket(log2n: int, k: int) -> int:
    return lib().oracle_ref_alpha_bucket(log2n, float(k))


def sample_max(x: np.ndarray, alpha: int) -> np.ndarray:
    x = as_keys(x)
    m = (x.size + (1 << alpha) - 1) >> alpha
    out = np.empty(m, dtype=np.uint32)
    lib().oracle_sample_max(_p(x, ctypes.c_uint32), x.size, alpha, _p(out, ctypes.c_uint32))
    return out


def sample_top2(x: np.ndarray, alpha: int) -> np.ndarray:
    x = as_keys(x)
    m = (x.size + (1 << alpha) - 1) >> alpha
    out = np.empty(2 * m, dtype=np.uint32)
    lib().oracle_sample_top2(_p(x, ctypes.c_uint32), x.size, alpha, _p(out, ctypes.c_uint32))
    return out


def radix_final_kth(x: np.ndarray, k: int, nbits: int = 8, alpha: int | None = None, path: int = 0):
    """The reference FINAL path (sample_radix_select) restated; returns (kth, stats dict)."""
    x = as_keys(x)
    if alpha is None:
        alpha = ref_alpha(int(np.log2(x.size)), k)
    kth = ctypes.c_uint32(0)
    st = OracleStats()
    rc = lib().oracle_radix_final_kth(_p(x, ctypes.c_uint32), x.size, k, nbits, alpha, path,
                                      ctypes.byref(kth), ctypes.byref(st))
    if rc != 0:
        raise ValueError("oracle_radix_final_kth rejected the input")
    return kth.value, st.as_dict()


def bucket_kth(x: np.ndarray, k: int, nb: int = 256, alpha: int | None = None, path: int = 0):
    x = as_keys(x)
    if alpha is None:
        alpha = ref_alpha_bucket(int(np.log2(x.size)), k)
    kth = ctypes.c_uint32(0)
    st = OracleStats()
    rc = lib().oracle_bucket_kth(_p(x, ctypes.c_uint32), x.size, k, nb, alpha, path,
                                 ctypes.byref(kth), ctypes.byref(st))
    if rc != 0:
        raise ValueError("oracle_bucket_kth rejected the input")
    return kth.value, st.as_dict()


def bitonic_topk(x: np.ndarray, k: int, alpha: int):
    x = as_keys(x)
    vals = np.empty(k, dtype=np.uint32)
    idx = np.empty(k, dtype=np.int64)
    rc = lib().oracle_bitonic_topk(_p(x, ctypes.c_uint32), x.size, k, alpha, _p(vals, ctypes.c_uint32),
                                   _p(idx, ctypes.c_int64))
    if rc != 0:
        raise ValueError("oracle_bitonic_topk rejected the input")
    return vals, idx


def topk_exact(x: np.ndarray, k: int, want_topk: bool = True):
    """Exact k-th largest key plus the top-k sorted (value desc, index asc); keys are uint32."""
    x = as_keys(x)
    kth = ctypes.c_uint32(0)
    if not want_topk:
        lib().oracle_topk_exact(_p(x, ctypes.c_uint32), x.size, k, ctypes.byref(kth), None, None)
        return kth.value, None, None
    vals = np.empty(k, dtype=np.uint32)
    idx = np.empty(k, dtype=np.int64)
    lib().oracle_topk_exact(_p(x, ctypes.c_uint32), x.size, k, ctypes.byref(kth), _p(vals, ctypes.c_uint32),
                            _p(idx, ctypes.c_int64))
    return kth.value, vals, idx


def topk_mt(x: np.ndarray, k: int, threads: int):
    """Multi-threaded host top-k (CPU baseline).  Returns (seconds, kth, sorted values)."""
    x = as_keys(x)
    kth = ctypes.c_uint32(0)
    vals = np.empty(k, dtype=np.uint32)
    sec = lib().oracle_topk_mt(_p(x, ctypes.c_uint32), x.size, k, threads, ctypes.byref(kth),
                               _p(vals, ctypes.c_uint32))
    return sec, kth.value, vals


def bmw_kth(x: np.ndarray, k: int, alpha: int):
    """The BMW experiment's heap scan with delegate skipping
    (BMW/radixselect.cuh:1746-1832): (k-th largest key, keys skipped)."""
    x = np.ascontiguousarray(x, dtype=np.uint32)
    sk = ctypes.c_uint64(0)
    kth = lib().oracle_bmw_kth(_p(x, ctypes.c_uint32), x.size, k, alpha, ctypes.byref(sk))
    return int(kth), int(sk.value)


def digest(vals: np.ndarray, idx: np.ndarray | None = None) -> int:
    vals = np.ascontiguousarray(vals, dtype=np.uint32)
    ip = None
    if idx is not None:
        idx = np.ascontiguousarray(idx, dtype=np.int64)
        ip = _p(idx, ctypes.c_int64)
    return int(lib().oracle_digest(_p(vals, ctypes.c_uint32), ip, vals.size))
