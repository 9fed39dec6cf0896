"""Generate tests/golden/ref_radix_kth.json: k-th values produced by the
reference's own sample_radix_select (oracle/_ref/ref_harness, compiled from
the reference sources by `make -C oracle ref`) on seeded inputs made by the
oracle's generators.  Needs a CUDA GPU; run as

    python tests/golden/make_golden.py OUT.json

The CPU restatement's answer is recorded beside each case ("oracle_kth") so
the fixture also documents the pin.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def cases():
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


def main(path):
    res = []
    for dist, log2n, k, nbits, seed in cases():
        p = subprocess.run([HARNESS, dist, str(log2n), str(k), str(nbits), "2", str(seed), "1"],
                           capture_output=True, text=True, timeout=600)
        line = [ln for ln in p.stdout.splitlines() if ln.startswith("RESULT ")]
        if p.returncode != 0 or not line:
            res.append({"dist": dist, "log2n": log2n, "k": k, "nbits": nbits, "seed": seed,
                        "error": (p.stdout + p.stderr)[-300:]})
            continue
        r = json.loads(line[0][7:])
        if log2n <= 20:
            x = O.gen(dist, 1 << log2n, seed)
            r["oracle_kth"] = O.radix_final_kth(x, k, nbits)[0]
        res.append(r)
        print(json.dumps(r), flush=True)
    doc = {"source": "reference sample_radix_select (baseline+filter+beta+shuffle/radixselect.cuh) "
                     "compiled for sm_100a, run on a B200 by tests/golden/make_golden.py",
           "cases": res}
    with open(path, "w") as f:
        json.dump(doc, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(__file__), "ref_radix_kth.json"))
