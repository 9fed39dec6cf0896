#!/usr/bin/env python3
"""bench.py -- Dr.Top-k selection throughput on B200.

Workload (the reference's headline configuration): N = 2^30
uint32 keys (4 GiB) drawn uniform over [0, 2^32-1] (seeded Philox on the
device -- synthetic data standing in for the reference's unseeded
random_device draws), 8-bit digits, beta = 2, alpha (and path) per k from
the autotuner (--alpha-mode ref: the reference's formula), k swept over
2^0..2^24.  One step = one pass of the sweep: 25
exact top-k calls (k-th value + the k largest values) over the resident
keys.  metric: keys/s = 25 * N * steps / device time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own implementation of the path --
sample_radix_select from baseline+filter+beta+shuffle/radixselect.cuh, a
CUDA program, built from its sources for sm_100a by `make -C oracle ref`
(oracle/_ref/ref_harness) -- on the same workload with its stock parameters,
and prints the same metric.  Both arms carry the same cpu_baseline: the
multi-threaded host top-k (oracle port) on one bounded 2^26-key sample.
Under torchrun (N > 1) every rank runs an independent replica on its own
GPU (the select does not shard; value = sum over ranks, time = max over
ranks).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SWEEP = [1 << i for i in range(25)]
# the reference's own published V100S totals (ms) at N=2^30 for some k (its optimum_FICO results)
REF_V100S_MS = {1: 7.157, 128: 6.331, 1024: 6.408, 1 << 16: 7.665, 1 << 20: 12.703, 1 << 22: 18.649, 1 << 24: 33.691}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    """DRAM bytes per sampler launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "sampler_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = f"/tmp/drtopk_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in open(self.path):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names[1:], parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_topk_rate(sample, ks, budget_s: float):
    """Multi-threaded host top-k (oracle port) on a host sample; keys/s."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    done = 0
    t0 = time.perf_counter()
    calls = 0
    while True:
        for k in ks:
            O.topk_mt(sample, min(k, sample.size), threads)
            done += sample.size
            calls += 1
        if time.perf_counter() - t0 > budget_s or calls >= 60:
            break
    dt = time.perf_counter() - t0
    return done / dt, threads, calls, dt


def bench_batched(D, torch, dev, stream, args):
    """C4: 4096 segments, lengths log-uniform 2^10..2^22, 80% float32 N(0,1)
    and 20% uint32 uniform, k log-uniform 1..min(len, 1024); one persistent
    graph-replayed launch vs a loop of plain calls on the same GPU."""
    import numpy as np
    rng = np.random.default_rng(2024)
    nseg = args.batch_segments
    lens = np.exp2(rng.uniform(10, 22, nseg)).astype(np.int64)
    f32 = rng.random(nseg) < 0.8
    ks = np.array([int(np.exp2(rng.uniform(0, np.log2(min(L, 1024))))) for L in lens], dtype=np.uint32)
    offsets = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    total = int(offsets[-1])
    g = torch.Generator(device=dev)
    g.manual_seed(77)
    keys = torch.randint(-(1 << 31), 1 << 31, (total,), dtype=torch.int32, device=dev, generator=g)
    fv = keys.view(torch.float32)
    for s_ in np.flatnonzero(f32):
        a, b = int(offsets[s_]), int(offsets[s_ + 1])
        fv[a:b] = torch.randn(b - a, dtype=torch.float32, device=dev, generator=g)
    dtypes = f32.astype(np.int32)
    bt = D.Batch(dev.index or 0).plan(offsets, ks, dtypes, sorted=False)
    ktot = int(ks.astype(np.int64).sum())
    kth = torch.zeros(nseg, dtype=torch.int32, device=dev)
    vals = torch.zeros(ktot, dtype=torch.int32, device=dev)
    for _ in range(2):
        bt.run(keys, kth, vals, None, graph=True, stream=stream)
    bt.sync_check(stream)
    reps = 5
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        bt.run(keys, kth, vals, None, graph=True, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    bms = e0.elapsed_time(e1) / reps
    bt.sync_check(stream)
    # loop of plain calls (autotuned parameters), same outputs
    h = D.Handle(dev.index or 0)
    sp = stream.cuda_stream or None
    kth2 = torch.zeros(nseg, dtype=torch.int32, device=dev)
    vals2 = torch.zeros(int(ks.max()), dtype=torch.int32, device=dev)
    plist = [D.autotune(int(lens[i]), int(ks[i]), int(dtypes[i]), D.params(alpha=-2)) for i in range(nseg)]

    def loop():
        for i in range(nseg):
            h.select_raw(keys.data_ptr() + 4 * int(offsets[i]), int(dtypes[i]), int(lens[i]), int(ks[i]), plist[i],
                         kth2.data_ptr() + 4 * i, vals2.data_ptr(), None, sp)

    loop()
    h.sync_check(stream)
    e0.record(stream)
    t0 = time.perf_counter()
    loop()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    lwall = (time.perf_counter() - t0) * 1e3
    lms = max(e0.elapsed_time(e1), lwall)
    exact = bool(torch.equal(kth, kth2))
    h.close()
    algo, alpha, _ = bt.describe()
    bt.close()
    return {"config": "4096 segments, len log-uniform 2^10..2^22, 80% f32 N(0,1) / 20% u32, k log-uniform "
                      "1..min(len,1024); one persistent launch (CUDA graph)",
            "segments": nseg, "total_keys": total, "ms_batch": bms, "req_per_s": nseg / (bms * 1e-3),
            "keys_per_s": total / (bms * 1e-3), "ms_loop_of_plain_calls": lms,
            "loop_req_per_s": nseg / (lms * 1e-3), "speedup_vs_loop": lms / bms, "exact_vs_loop": exact,
            "segments_delegate": int((algo == 0).sum()), "segments_plain": int((algo == 3).sum())}


def bench_served(D, torch, dev, stream, args):
    """C5: Poisson arrivals of requests with N log-uniform 2^12..2^28 keys
    (u32 uniform, u32 normal or f32 normal, evenly), k log-uniform
    1..min(N, 2^20); keys resident on the device; 120 GB budget.  The server
    is first driven at saturation (every request offered at once) for its
    capacity, then at 0.5x and 0.9x of that rate, where p50/p99 are service
    latencies rather than queue growth.  Every result (k-th value and the
    k values, compared as a sorted digest) must equal the loop's."""
    import hashlib

    import numpy as np
    rng = np.random.default_rng(31)
    npool = args.serve_pool
    g = torch.Generator(device=dev)
    g.manual_seed(91)
    pool = []
    for i in range(npool):
        n = int(np.exp2(rng.uniform(12, 28)))
        kind = i % 3
        if kind == 0:
            t = torch.randint(-(1 << 31), 1 << 31, (n,), dtype=torch.int32, device=dev, generator=g)
            dt = D.U32
        elif kind == 1:
            z = torch.randn(n, dtype=torch.float64, device=dev, generator=g)
            t = (z * 2.0 ** 28 + 2.0 ** 31).round().clamp(0, 2 ** 32 - 1).to(torch.int64).to(torch.int32)
            dt = D.U32
        else:
            t = torch.randn(n, dtype=torch.float32, device=dev, generator=g)
            dt = D.F32
        pool.append((t, n, dt))
    R = args.serve_requests
    reqs = []
    for r in range(R):
        t, n, dt = pool[int(rng.integers(npool))]
        k = int(np.exp2(rng.uniform(0, np.log2(min(n, 1 << 20)))))
        reqs.append((t, n, dt, k))

    def digest(v):
        return hashlib.sha1(np.sort(np.asarray(v).view(np.uint32)).tobytes()).hexdigest()

    # loop of plain per-request calls: select + copy back + synchronise
    h = D.Handle(dev.index or 0)
    kmax = max(r[3] for r in reqs)
    kth = torch.zeros(1, dtype=torch.int32, device=dev)
    vals = torch.zeros(kmax, dtype=torch.int32, device=dev)
    hv = torch.zeros(kmax, dtype=torch.int32, pin_memory=True)
    hk = torch.zeros(1, dtype=torch.int32, pin_memory=True)
    ref = []

    def one(t, n, dt, k, keep):
        p = D.autotune(n, k, dt, D.params(alpha=-2))
        h.select_raw(t.data_ptr(), dt, n, k, p, kth.data_ptr(), vals.data_ptr(), None, stream.cuda_stream or None)
        hk.copy_(kth, non_blocking=True)
        hv[:k].copy_(vals[:k], non_blocking=True)
        torch.cuda.synchronize(dev)
        if keep:
            ref.append((int(hk.item()) & 0xFFFFFFFF, digest(hv[:k].numpy())))

    # warm-up over the whole request list, as the server's below: the
    # handle's workspace reaches its largest size and every kernel is loaded
    # before the timed loop
    for r in reqs:
        one(*r, keep=True)
    lat_loop = []
    t0 = time.perf_counter()
    for r in reqs:
        a = time.perf_counter()
        one(*r, keep=False)
        lat_loop.append((time.perf_counter() - a) * 1e3)
    loop_s = time.perf_counter() - t0
    h.close()
    loop_rps = R / loop_s
    out = {"config": "Poisson arrivals; N log-uniform 2^12..2^28 (u32 uniform / u32 normal / f32 normal); "
                     "k log-uniform 1..min(N,2^20); keys resident on the device; 120 GB budget; unsorted values; "
                     "max_inflight %d" % args.serve_inflight,
           "requests": R, "pool_arrays": npool, "loop_req_per_s": loop_rps,
           "loop_p50_ms": float(np.percentile(lat_loop, 50)), "loop_p99_ms": float(np.percentile(lat_loop, 99)),
           "rates": []}

    def run(lam):
        """Offer the request list at Poisson rate lam (None: all at once)."""
        srv = D.Server(dev.index or 0, hbm_budget_bytes=120 << 30, max_inflight=args.serve_inflight)
        arr = np.cumsum(rng.exponential(1.0 / lam, R)) if lam else np.zeros(R)
        ids = {}
        start = time.perf_counter()
        for i, (t, n, dt, k) in enumerate(reqs):
            while time.perf_counter() - start < arr[i]:
                pass
            ids[srv.submit(t, k, want_indices=False)] = i
        srv.drain(300000)
        res = []
        while True:
            got = srv.poll(R + 10)
            if not got:
                break
            res += got
        st = srv.stats()
        srv.close()
        lat = [r["t_done"] - r["t_submit"] for r in res]
        span = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
        exact = len(res) == R and all(r["status"] == 0 for r in res) and all(
            (int(np.asarray(r["kth"]).view(np.uint32)), digest(r["values"])) == ref[ids[r["id"]]] for r in res)
        first_done = min(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
        return {"offered_req_per_s": lam, "req_per_s": len(res) / (span * 1e-3),
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                "max_ms": float(max(lat)), "first_done_ms": float(first_done),
                "exact_vs_loop": bool(exact), "server_stats": st}

    run(None)  # warm-up: staging and output caches, memory pool growth
    sat = run(None)
    sat["offered"] = "all at once (saturation)"
    out["rates"].append(sat)
    cap = sat["req_per_s"]
    for f in args.serve_rates:
        r = run(cap * f)
        r["offered"] = f"{f} x saturation"
        out["rates"].append(r)
    out["saturation_req_per_s"] = cap
    out["speedup_vs_loop"] = cap / loop_rps
    out["exact_vs_loop"] = all(r["exact_vs_loop"] for r in out["rates"])
    return out


def bench_extras(D, torch, dev, stream, h, peak, log2n):
    """The other configurations BASELINE names, reported beside the headline
    (each: ms per call, keys/s, fraction of the measured HBM roofline over
    the algorithmic bytes 4N + output):
      C1   N=2^20 uint32 uniform, k=128: latency of one call, and the share of
           the phases after the sampler;
      C2b  N=2^30 normal(2^31, 2^28) uint32, k=2^0..2^24;
      C3   N=2^28 float32 uniform [0,1) and normal(0,1), and few-digits uint32
           (top 24 bits fixed), k in {16, 256, 4096, 65536}: radix (autotuned),
           bucket and bitonic (k <= 2048), sorted values with indices;
      sorted_idx  N=2^30 uint32 uniform, sorted top-k with int64 indices,
           k=2^0..2^24 (output bytes 12k counted)."""
    sp = stream.cuda_stream or None
    g = torch.Generator(device=dev)

    def timed(keys, dt, n, k, p, want_idx, reps):
        kth = torch.empty(1, dtype=torch.int32, device=dev)
        vals = torch.empty(k, dtype=torch.int32, device=dev)
        idx = torch.empty(k, dtype=torch.int64, device=dev) if want_idx else None
        ip = idx.data_ptr() if want_idx else None
        for _ in range(2):
            h.select_raw(keys.data_ptr(), dt, n, k, p, kth.data_ptr(), vals.data_ptr(), ip, sp)
        a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            h.select_raw(keys.data_ptr(), dt, n, k, p, kth.data_ptr(), vals.data_ptr(), ip, sp)
        b2.record(stream)
        torch.cuda.synchronize(dev)
        ms = a.elapsed_time(b2) / reps
        st = h.stats()
        outb = 4 * k + (8 * k if want_idx else 0)
        return {"ms": round(ms, 4), "keys_per_s": n / (ms * 1e-3),
                "frac_of_measured_hbm": round((4.0 * n + outb) / (ms * 1e-3) / (peak * 1e9), 4),
                "algo": st["algo"], "alpha": st["alpha"], "beta": st["beta"], "candidates": st["n_candidates"],
                "ms_sample": round(st["ms_sample"], 4), "ms_after_sampler": round(st["ms_total"] - st["ms_sample"], 4)}

    out = {}
    # C1
    g.manual_seed(1)
    n1 = 1 << 20
    k1 = torch.randint(-(1 << 31), 1 << 31, (n1,), dtype=torch.int32, device=dev, generator=g)
    r = timed(k1, D.U32, n1, 128, D.autotune(n1, 128, D.U32, D.params(alpha=-2)), False, 200)
    r["after_sampler_share"] = round(r["ms_after_sampler"] / max(1e-9, r["ms_sample"] + r["ms_after_sampler"]), 3)
    out["C1_n2^20_k128"] = r
    del k1
    # C2b
    if log2n == 30:
        g.manual_seed(2)
        n2 = 1 << 30
        z = torch.empty(n2, dtype=torch.int32, device=dev)
        for c in range(0, n2, 1 << 27):  # in slices: the float64 draw of 2^30 normals needs 8 GB
            zz = torch.randn(1 << 27, dtype=torch.float64, device=dev, generator=g)
            z[c:c + (1 << 27)] = (zz * 2.0 ** 28 + 2.0 ** 31).round().clamp(0, 2 ** 32 - 1).to(torch.int64).to(torch.int32)
        del zz
        rows = {}
        tot_ms = 0.0
        for i in range(25):
            k = 1 << i
            rr = timed(z, D.U32, n2, k, D.autotune(n2, k, D.U32, D.params(alpha=-2)), False, 3)
            rows[str(k)] = rr
            tot_ms += rr["ms"]
        out["C2b_normal_n2^30"] = {"keys_per_s_sweep": 25 * n2 / (tot_ms * 1e-3), "per_k": rows}
        del z
    # C3
    n3 = 1 << 28
    c3 = {}
    for dist in ("f32u", "f32n", "fewdigits"):
        g.manual_seed(3)
        if dist == "f32u":
            x = torch.rand(n3, dtype=torch.float32, device=dev, generator=g)
            dt = D.F32
        elif dist == "f32n":
            x = torch.randn(n3, dtype=torch.float32, device=dev, generator=g)
            dt = D.F32
        else:
            x = (torch.randint(0, 256, (n3,), dtype=torch.int32, device=dev, generator=g) | (0xABCDEF << 8)).to(
                torch.int32)
            dt = D.U32
        for k in (16, 256, 4096, 65536):
            for algo in ("radix", "radix-ref", "bucket", "bitonic"):
                if algo == "bitonic" and k > 2048:
                    continue
                if algo == "radix":  # autotuned
                    p = D.autotune(n3, k, dt, D.params(alpha=-2, sorted=True))
                elif algo == "radix-ref":  # the reference's own parameters (main.cu:83-89)
                    p = D.params(sorted=True)
                else:
                    p = D.params(algo=algo, sorted=True)
                c3[f"{dist}/k{k}/{algo}"] = timed(x, dt, n3, k, p, True, 5)
        del x
    out["C3_n2^28_sorted_idx"] = c3
    return out


METRIC = "keys/s (exact top-k over N=2^30 uint32 uniform keys, k sweep 2^0..2^24)"


def sweep_config(n, nks, world):
    """The workload both arms measure (identical dicts, so the two lines compare)."""
    return {"workload": "Dr.Top-k radix top-k, N=2^%d uint32 uniform over [0, 2^32-1], k=2^0..2^24 (one step = "
                        "the 25-k sweep), nbits=8, beta=2" % (n.bit_length() - 1),
            "n": n, "ks": nks, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "input 4 GiB >> 126 MB L2 (no flush needed)"}


def cpu_baseline(budget_s: float = 15.0):
    """The multi-threaded host top-k (oracle port: per-thread nth_element +
    merge + sort) on the box's host cores, on one bounded sample that both
    arms share: 2^26 seeded uniform uint32 keys, k in {1, 2^10, 2^16, 2^20}."""
    import numpy as np
    rng = np.random.default_rng(12345)
    sample = rng.integers(0, 1 << 32, size=1 << 26, dtype=np.uint64).astype(np.uint32)
    rate, threads, calls, dt = cpu_topk_rate(sample, [1, 1 << 10, 1 << 16, 1 << 20], budget_s)
    return {"value": rate, "unit": "keys/s", "cores": threads, "kind": "port",
            "sample": f"2^26 seeded uniform uint32 keys, k in {{1,2^10,2^16,2^20}}, {calls} calls in {dt:.1f} s "
                      "(oracle_topk_mt: per-thread nth_element + merge + sort; the reference has no CPU "
                      "implementation of the path)"}


def run_reference(args):
    """Reference arm (rank 0 only): the reference's own sample_radix_select
    (baseline+filter+beta+shuffle/radixselect.cuh:1782-1894), compiled from
    its sources for sm_100a into oracle/_ref/ref_harness, timed on this GPU
    over the same workload with its stock parameters (alpha from main.cu:83,
    8-bit digits, beta 2) and its stock blocking call.  Without the harness
    or a GPU, the CPU port stands in for it on a bounded sample."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    n = 1 << args.log2n
    ks = SWEEP if args.ks == "sweep" else [int(x) for x in args.ks.split(",")]
    ks = [k for k in ks if k <= n]
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    have_gpu = False
    try:
        have_gpu = subprocess.run(["nvidia-smi", "-L"], capture_output=True, timeout=60).returncode == 0
    except (OSError, subprocess.TimeoutExpired):
        pass
    out = {"impl": "reference", "metric": METRIC, "unit": "keys/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
           "config": sweep_config(n, len(ks), 1)}
    if os.access(harness, os.X_OK) and have_gpu:
        clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
        clocks.start()
        cmd = [harness, "--bench", "u32", str(args.log2n), ",".join(str(k) for k in ks), "8", "2", "1234",
               str(args.steps), str(max(3, args.warmup)), str(args.e2e_steps)]
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=3000)
        ck = clocks.stop()
        line = [ln for ln in p.stdout.splitlines() if ln.startswith("BENCH ")]
        if p.returncode != 0 or not line:
            out["unavailable"] = "reference harness failed: " + (p.stdout + p.stderr)[-300:].replace("\n", " ")
            print(json.dumps(out), flush=True)
            return 0
        r = json.loads(line[0][6:])
        calls = args.steps * len(ks)
        ms = r["ms_total"]
        value = calls * n / (ms * 1e-3)
        e2e_calls = args.e2e_steps * len(ks)
        out.update({
            "value": value, "ms_per_step": ms / args.steps,
            "data": "synthetic (seeded mt19937 uniform uint32 over [0, 2^32-1], generated on the host)",
            "params": "alpha per k from the reference formula (main.cu:83), 8-bit digits, beta 2, default path "
                      "when alpha > 5",
            "outputs": "the k-th value (the reference returns no top-k list)",
            "reference": {"kind": "the reference's own GPU code (sample_radix_select) built from its sources for "
                                  "sm_100a: oracle/_ref/ref_harness --bench",
                          "per_k": r["per_k"]},
            "e2e": {"value": e2e_calls * n / (r["e2e_ms_total"] * 1e-3), "unit": "keys/s",
                    "h2d_bytes_per_step": 4 * n * len(ks), "d2h_bytes_per_step": 4 * len(ks),
                    "ms_per_step": r["e2e_ms_total"] / max(1, args.e2e_steps),
                    "note": "per call: H2D of the keys from pinned memory + the reference's blocking call"},
            "clocks": ck,
        })
    else:
        # no harness or no GPU: the CPU port on a bounded sample of the workload
        import numpy as np
        n_sample = 1 << args.ref_log2n
        rng = np.random.default_rng(12345)
        sample = rng.integers(0, 1 << 32, size=n_sample, dtype=np.uint64).astype(np.uint32)
        sks = [k for k in ks if k <= n_sample]
        from oracle import oracle as O
        threads = os.cpu_count() or 1
        for i in range(args.warmup):
            O.topk_mt(sample, sks[i % len(sks)], threads)
        t0 = time.perf_counter()
        keys = 0
        for _ in range(args.steps):
            for k in sks:
                O.topk_mt(sample, k, threads)
                keys += sample.size
        dt = time.perf_counter() - t0
        value = keys / dt
        out.update({"value": value, "ms_per_step": dt * 1e3 / max(1, args.steps),
                    "data": "synthetic (seeded numpy uniform uint32)",
                    "reference": {"kind": f"CPU port on a 2^{args.ref_log2n}-key sample (no reference harness "
                                          "or no GPU on this host)"},
                    "e2e": {"value": value, "unit": "keys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    if not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline()
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--log2n", type=int, default=30)
    ap.add_argument("--ref-log2n", type=int, default=26)
    ap.add_argument("--ks", default="sweep")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--alpha-mode", choices=["auto", "ref", "emit"], default="auto",
                    help="auto: per-k parameters from the autotuner (headline); ref: the reference's alpha formula; "
                         "emit: the sampled-threshold path for every k")
    ap.add_argument("--no-table", action="store_true", help="skip the per-k tables after the timed region")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-form measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-form measurement")
    ap.add_argument("--no-extras", action="store_true", help="skip the other BASELINE configurations")
    ap.add_argument("--batch-segments", type=int, default=4096)
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-pool", type=int, default=48)
    ap.add_argument("--serve-inflight", type=int, default=256, help="server in-flight request limit")
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[0.5, 0.9],
                    help="offered loads (Poisson) as fractions of the server's measured saturation rate")
    args = ap.parse_args()

    if args.impl == "reference":
        return run_reference(args)

    import torch

    import drtopksc_b200 as D

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    n = 1 << args.log2n
    ks = SWEEP if args.ks == "sweep" else [int(x) for x in args.ks.split(",")]
    ks = [k for k in ks if k <= n]
    kmax = max(ks)
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    keys = torch.randint(-(1 << 31), 1 << 31, (n,), dtype=torch.int32, device=dev, generator=g)
    kth = torch.empty(len(ks), dtype=torch.int32, device=dev)
    vals = torch.empty(kmax, dtype=torch.int32, device=dev)
    h = D.Handle(local)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream or None
    # 8-bit digits, beta=2; alpha (and path / threshold digits) per k from the
    # autotuner, or the reference formula with --alpha-mode ref
    p_ref = D.params()
    if args.alpha_mode == "emit":
        plist = [D.params(path=4) for k in ks]
    else:
        plist = [D.autotune(n, k, D.U32, D.params(alpha=-2)) if args.alpha_mode == "auto" else p_ref for k in ks]

    def one_step():
        for i, k in enumerate(ks):
            h.select_raw(keys.data_ptr(), D.U32, n, k, plist[i], kth.data_ptr() + 4 * i, vals.data_ptr(), None, sp)

    for _ in range(args.warmup):
        one_step()
    h.sync_check(stream)

    # correctness guard (independent torch reductions): gt < k <= ge
    u = keys.to(torch.int64) & 0xFFFFFFFF
    kt = kth.to(torch.int64) & 0xFFFFFFFF
    for i in {0, len(ks) // 2, len(ks) - 1}:
        K, k = int(kt[i].item()), ks[i]
        gt, ge = int((u > K).sum().item()), int((u >= K).sum().item())
        if not (gt < k <= ge):
            print(json.dumps({"error": f"wrong k-th value for k={k}: gt={gt} ge={ge}"}), flush=True)
            return 3
    del u

    # ---------------- timed region
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    h.profile_begin(args.steps * len(ks))
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        one_step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ck = clocks.stop()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    ms_sample, ms_fused, ncalls = h.profile_end()
    h.sync_check(stream)
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    calls = args.steps * len(ks)
    value = world * calls * n / (ms * 1e-3)

    peak, peak_kind = load_peaks()
    sample_ms_per_launch = ms_sample / max(1, ncalls)
    achieved = 4.0 * n / (sample_ms_per_launch * 1e-3) / 1e9
    traffic = load_traffic()
    traffic_bytes = None
    if traffic and traffic.get("n") and traffic.get("dram_bytes_per_launch"):
        traffic_bytes = traffic["dram_bytes_per_launch"] * (n / traffic["n"])

    # ---------------- per-k tables (short, after the timed region)
    def table(params_for):
        out = {}
        for i, k in enumerate(ks):
            pk = params_for(i, k)
            # one untimed call (sizes the workspace for this configuration)
            h.select_raw(keys.data_ptr(), D.U32, n, k, pk, kth.data_ptr() + 4 * i, vals.data_ptr(), None, sp)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            reps = 3
            a.record(stream)
            for _ in range(reps):
                h.select_raw(keys.data_ptr(), D.U32, n, k, pk, kth.data_ptr() + 4 * i, vals.data_ptr(), None, sp)
            b.record(stream)
            torch.cuda.synchronize(dev)
            kms = a.elapsed_time(b) / reps
            st = h.stats()
            row = {"ms": round(kms, 4), "keys_per_s": n / (kms * 1e-3),
                   "frac_of_measured_hbm": (4.0 * n + 4.0 * k) / (kms * 1e-3) / (peak * 1e9),
                   "alpha": st["alpha"], "beta": st["beta"], "candidates": st["n_candidates"],
                   "ms_sample": round(st["ms_sample"], 4), "ms_first": round(st["ms_first"], 4),
                   "ms_concat": round(st["ms_concat"], 4), "ms_second": round(st["ms_second"], 4),
                   "launches": st["kernel_launches"]}
            if k in REF_V100S_MS and n == 1 << 30:
                row["reference_v100s_ms"] = REF_V100S_MS[k]
            out[str(k)] = row
        h.sync_check(stream)
        return out

    sweep, sweep_ref = {}, {}
    if not args.no_table:
        sweep = table(lambda i, k: plist[i])
        if args.alpha_mode == "auto":
            sweep_ref = table(lambda i, k: p_ref)
    # kernels one step launches (the same plans as the timed sweep)
    launches_per_step = sum(sweep[str(k)]["launches"] for k in ks) if sweep else None

    # sorted top-k with int64 indices over the same keys (12 output bytes per k)
    sorted_idx = {}
    if not args.no_extras and rank == 0 and world == 1:
        idx = torch.empty(kmax, dtype=torch.int64, device=dev)
        tot_ms = 0.0
        for i, k in enumerate(ks):
            pk = D.autotune(n, k, D.U32, D.params(alpha=-2, sorted=True))
            for _ in range(2):
                h.select_raw(keys.data_ptr(), D.U32, n, k, pk, kth.data_ptr(), vals.data_ptr(), idx.data_ptr(), sp)
            a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(3):
                h.select_raw(keys.data_ptr(), D.U32, n, k, pk, kth.data_ptr(), vals.data_ptr(), idx.data_ptr(), sp)
            b2.record(stream)
            torch.cuda.synchronize(dev)
            kms = a.elapsed_time(b2) / 3
            tot_ms += kms
            sorted_idx[str(k)] = {"ms": round(kms, 4), "frac_of_measured_hbm":
                                  round((4.0 * n + 12.0 * k) / (kms * 1e-3) / (peak * 1e9), 4)}
        h.sync_check(stream)
        sorted_idx = {"keys_per_s_sweep": len(ks) * n / (tot_ms * 1e-3), "per_k": sorted_idx}
        del idx

    # ---------------- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        host = torch.empty(n, dtype=torch.int32, pin_memory=True)
        host.copy_(keys)
        dkeys = torch.empty_like(keys)
        h_kth = torch.empty(len(ks), dtype=torch.int32, pin_memory=True)
        h_vals = torch.empty(kmax, dtype=torch.int32, pin_memory=True)
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        d2h = 0
        a.record(stream)
        for _ in range(args.e2e_steps):
            for i, k in enumerate(ks):
                dkeys.copy_(host, non_blocking=True)
                h.select_raw(dkeys.data_ptr(), D.U32, n, k, plist[i], kth.data_ptr() + 4 * i, vals.data_ptr(), None,
                             sp)
                h_kth[i:i + 1].copy_(kth[i:i + 1], non_blocking=True)
                h_vals[:k].copy_(vals[:k], non_blocking=True)
                d2h += 4 + 4 * k
        b.record(stream)
        torch.cuda.synchronize(dev)
        ems = a.elapsed_time(b)
        if dist:
            t = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e_calls = args.e2e_steps * len(ks)
        e2e = {"value": world * e2e_calls * n / (ems * 1e-3), "unit": "keys/s",
               "h2d_bytes_per_step": 4 * n * len(ks), "d2h_bytes_per_step": d2h // max(1, args.e2e_steps),
               "ms_per_step": ems / max(1, args.e2e_steps),
               "note": "per call: H2D of the 4 GiB keys from pinned memory + select + D2H of k-th and top-k values"}
        del host, dkeys

    # ---------------- CPU baseline (rank 0, N=1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline()

    batched = served = extras = None
    if rank == 0 and world == 1:
        del keys
        torch.cuda.empty_cache()
        if not args.no_extras:
            extras = bench_extras(D, torch, dev, stream, h, peak, args.log2n)
            torch.cuda.empty_cache()
        if not args.no_batch:
            batched = bench_batched(D, torch, dev, stream, args)
            torch.cuda.empty_cache()
        if not args.no_serve:
            served = bench_served(D, torch, dev, stream, args)
            torch.cuda.empty_cache()

    if rank == 0:
        out = {
            "metric": METRIC,
            "value": value, "unit": "keys/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32", "data": "synthetic (seeded torch Philox, uniform uint32 over [0, 2^32-1])",
            "config": sweep_config(n, len(ks), world),
            "params": "alpha, path and threshold digits per k: %s" % (
                {"auto": "autotuner (drtopk_autotune)", "ref": "reference formula (main.cu:83)",
                 "emit": "sampled-threshold path (path 4) for every k"}[args.alpha_mode]),
            "outputs": "the k-th value and the k largest values (unsorted), per call",
            "roofline": {"bound": "hbm", "kernel": "the streaming pass: k_sample (delegate sampler; sample passes + "
                                                    "k_emit on the sampled-threshold path)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic_bytes, "algorithmic_bytes_per_launch": 4 * n,
                         "ms_per_launch": sample_ms_per_launch,
                         "fused_ms_per_call": ms_fused / max(1, ncalls),
                         "whole_call_frac": (4.0 * n) / (ms / calls * 1e-3) / (peak * 1e9),
                         "per_k_ms": [sweep[str(k)]["ms"] for k in ks] if sweep else None,
                         "per_k_frac": [round(sweep[str(k)]["frac_of_measured_hbm"], 4) for k in ks] if sweep else None},
            "cpu_baseline": cpu,
            "clocks": ck,
            "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps if launches_per_step else None,
            "k_sweep": sweep,
            "k_sweep_reference_alpha": sweep_ref,
            "sorted_with_indices": sorted_idx,
            "extra_configs": extras,
            "batched": batched,
            "served": served,
        }
        print(json.dumps(out), flush=True)
    h.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
