"""The drop-in topk.bin (baseline+filter+beta+shuffle/main.cu:56-323 and the
real-dataset build RealDatasets/BinaryDataset/main.cu:56-148) run as the
reference's run*.bash sweeps run it: its result line must carry the oracle's
k-th value, --check must print Success!, and the CSV row must have the
reference's fields (main.cu:306-314)."""
import os
import re
import subprocess

import numpy as np
import pytest

import drtopksc_b200 as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CLI = os.path.join(os.path.dirname(D.LIB_PATH), "topk.bin")


def _run(args, csv):
    p = subprocess.run([CLI] + [str(a) for a in args] + ["--check"], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    out = p.stdout
    assert "Success!" in out and "Not Success!" not in out, out
    m = re.search(r"The kth element from top is:(\d+)", out)
    assert m, out
    rows = [r for r in open(csv).read().splitlines() if r.strip()]
    fields = rows[-1].split(";")
    assert len(fields) == 11, rows[-1]
    return int(m.group(1)), fields, out


@pytest.mark.parametrize("log2n,k,path", [(20, 128, "D"), (22, 1 << 20, "B"), (24, 1, "D"), (20, 1 << 15, "B")])
def test_cli_reference_argv_default_and_beta_paths(tmp_path, log2n, k, path):
    csv = tmp_path / "out.csv"
    kth, fields, out = _run([log2n, k, 8, 2, "--csv", csv], csv)
    x = O.gen("u32", 1 << log2n, 1)  # the CLI's default data: seeded mt19937 (seed 1)
    assert kth == O.topk_exact(x, k, False)[0]
    alpha = O.ref_alpha(log2n, k)
    assert fields[0] == path and int(fields[1]) == log2n and int(fields[2]) == k
    assert int(fields[3]) == alpha and int(fields[4]) == 2
    assert f"Calculated alpha: {alpha}" in out


def test_cli_real_dataset_text_and_binary(tmp_path):
    rng = np.random.default_rng(5)
    scores = rng.random(1 << 14, dtype=np.float32)
    txt = tmp_path / "scores.txt"
    with open(txt, "w") as f:
        f.write("\n".join("%.9g" % s for s in scores))
    n = 1 << 16
    keys, _ = D.load_dataset(str(txt), n, "txt")
    csv = tmp_path / "real.csv"
    for k in (1, 100, 4096):
        kth, fields, _ = _run([16, k, 8, 2, txt, csv], csv)  # the reference's six-argument form
        assert kth == O.topk_exact(keys, k, False)[0]
    bin_ = tmp_path / "scores.dat"
    vals = rng.integers(-(1 << 31), 1 << 31, size=n, dtype=np.int64).astype("<i4")
    vals.tofile(bin_)
    for k in (7, 5000):
        kth, _, _ = _run([16, k, 8, 2, bin_, csv, "--format", "bin"], csv)
        assert kth == O.topk_exact(vals.view(np.uint32), k, False)[0]
