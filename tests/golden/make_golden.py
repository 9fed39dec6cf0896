"""Generate the golden fixtures from the reference's own sample_radix_select
(oracle/_ref/ref_harness, compiled from the reference sources by
`make -C oracle ref`) on seeded inputs made by the oracle's generators.
Needs a CUDA GPU; run as

    python tests/golden/make_golden.py          -> tests/golden/ref_radix_kth.json
    python tests/golden/make_golden.py --big    -> tests/golden/ref_radix_big.json

The small set covers every input family, digit width and both paths at
N <= 2^24, with the CPU restatement's answer recorded beside each case
("oracle_kth") so the fixture also documents the pin.  The big set is the
headline configurations themselves: N = 2^30 uint32 uniform and normal
(mean 2^31, sd 2^28) for k = 2^0..2^24, and N = 2^28 float32 uniform,
float32 normal and few-digits keys for k in {16, 256, 4096, 65536}.  Every
case records the reference's k-th value and its three stage counters
(CountSelectedSubrange, CountLonelyElements, write_pos).
"""
import json
import os
import subprocess
import sys
from collections import OrderedDict

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
HERE = os.path.dirname(os.path.abspath(__file__))


def cases_small():
    out = []
    for seed in (1, 2):
        for k in (1, 2, 16, 128, 1000, 4096, 65536, 1 << 18, 1 << 19, 1 << 20):
            out.append(("u32", 20, k, 8, seed))
    for k in (1, 128, 4096, 1 << 17):
        out.append(("normal", 20, k, 8, 3))
    for k in (16, 256, 4096, 65536):
        out.append(("fewdigits", 20, k, 8, 4))
        out.append(("f32u", 20, k, 8, 5))
        out.append(("f32n", 20, k, 8, 6))
    for nbits in (1, 2, 4):
        for k in (1, 100, 4096):
            out.append(("u32", 16, k, nbits, 7))
    for k in (1, 1024, 1 << 20):
        out.append(("u32", 24, k, 8, 8))
    return out


# seeds of the headline inputs (the GPU parity tests regenerate them)
BIG_SEEDS = {"u32": 30, "normal": 31, "f32u": 32, "f32n": 33, "fewdigits": 34}


def cases_big():
    out = []
    for dist in ("u32", "normal"):
        for i in range(25):
            out.append((dist, 30, 1 << i, 8, BIG_SEEDS[dist]))
    for dist in ("f32u", "f32n", "fewdigits"):
        for k in (16, 256, 4096, 65536):
            out.append((dist, 28, k, 8, BIG_SEEDS[dist]))
    return out


def run_group(dist, log2n, nbits, seed, ks):
    """One harness process per generated input; returns {k: result}."""
    p = subprocess.run([HARNESS, dist, str(log2n), ",".join(str(k) for k in ks), str(nbits), "2", str(seed), "1"],
                       capture_output=True, text=True, timeout=1800)
    res = {}
    for ln in p.stdout.splitlines():
        if ln.startswith("RESULT "):
            r = json.loads(ln[7:])
            if "k" in r:
                res[r["k"]] = r
    for k in ks:
        if k not in res:
            res[k] = {"dist": dist, "log2n": log2n, "k": k, "nbits": nbits, "seed": seed,
                      "error": (p.stdout + p.stderr)[-300:]}
    return res


def main(big: bool, path: str):
    groups = OrderedDict()
    for dist, log2n, k, nbits, seed in (cases_big() if big else cases_small()):
        groups.setdefault((dist, log2n, nbits, seed), []).append(k)
    res = []
    for (dist, log2n, nbits, seed), ks in groups.items():
        out = run_group(dist, log2n, nbits, seed, ks)
        x = O.gen(dist, 1 << log2n, seed) if (not big and log2n <= 20) else None
        for k in ks:
            r = out[k]
            if x is not None and "kth" in r:
                r["oracle_kth"] = O.radix_final_kth(x, k, nbits)[0]
            res.append(r)
            print(json.dumps(r), flush=True)
    doc = {"source": "reference sample_radix_select (baseline+filter+beta+shuffle/radixselect.cuh) "
                     "compiled for sm_100a, run on a B200 by tests/golden/make_golden.py"
                     + (" --big" if big else ""),
           "cases": res}
    with open(path, "w") as f:
        json.dump(doc, f, indent=1)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    big = "--big" in sys.argv[1:]
    default = os.path.join(HERE, "ref_radix_big.json" if big else "ref_radix_kth.json")
    main(big, args[0] if args else default)
