"""GPU tests of the batched form: every segment of a persistent batched
launch equals the oracle's exact top-k (and the plain per-vector call), for
mixed lengths, k and dtypes; the CUDA-graph replay equals the direct run."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import expected

pytestmark = pytest.mark.gpu


def make_batch(seed, nseg, lo=10, hi=20, kmax=1024, f32_frac=0.8):
    rng = np.random.default_rng(seed)
    lens = np.exp2(rng.uniform(lo, hi, nseg)).astype(np.int64)
    kinds = rng.random(nseg) < f32_frac
    ks = np.array([int(np.exp2(rng.uniform(0, np.log2(min(L, kmax))))) for L in lens], dtype=np.uint32)
    segs = []
    for s in range(nseg):
        if kinds[s]:
            segs.append(O.gen("f32n", int(lens[s]), seed * 1000 + s))
        else:
            segs.append(O.gen("u32", int(lens[s]), seed * 1000 + s))
    bits = np.concatenate([x.view(np.uint32) for x in segs])
    offsets = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    dtypes = kinds.astype(np.int32)  # 1 = f32
    return segs, bits, offsets, ks, dtypes


def run_batch(bits, offsets, ks, dtypes, sorted=True, graph=False, reps=1):
    import torch

    import drtopksc_b200 as D
    b = D.Batch().plan(offsets, ks, dtypes, sorted=sorted)
    keys = torch.from_numpy(bits.view(np.int32)).cuda()
    kth = torch.zeros(len(ks), dtype=torch.int32, device="cuda")
    tot = int(ks.astype(np.int64).sum())
    vals = torch.zeros(tot, dtype=torch.int32, device="cuda")
    idx = torch.zeros(tot, dtype=torch.int64, device="cuda")
    for _ in range(reps):
        b.run(keys, kth, vals, idx, graph=graph)
    b.sync_check()
    return b, kth.cpu().numpy().view(np.uint32), vals.cpu().numpy().view(np.uint32), idx.cpu().numpy()


def check_segments(segs, ks, b, kth, vals, idx, sorted=True):
    oo = b.out_offsets
    for s, x in enumerate(segs):
        k = int(ks[s])
        ek, ev, ei = expected(x, k)
        v = vals[oo[s]:oo[s + 1]]
        i = idx[oo[s]:oo[s + 1]]
        if x.dtype == np.float32:
            v = v.view(np.float32)
            assert np.float32(ek).view(np.uint32) == kth[s], s
        else:
            assert ek == kth[s], s
        if not sorted:  # index order: compare as sets of (value, index)
            order = np.lexsort((i, -O.as_keys(np.asarray(v, dtype=x.dtype)).astype(np.int64)))
            v, i = v[order], i[order]
        assert np.array_equal(np.asarray(v).view(np.uint32), np.asarray(ev).view(np.uint32)), (s, k)
        assert np.array_equal(i, ei), (s, k)


@pytest.mark.parametrize("sorted", [True, False])
def test_batch_matches_oracle(sorted):
    segs, bits, offsets, ks, dtypes = make_batch(1, 60, 10, 20)
    b, kth, vals, idx = run_batch(bits, offsets, ks, dtypes, sorted=sorted)
    algo, alpha, beta = b.describe()
    assert (algo == 0).any()  # delegate segments present (short ones: plain or bitonic)
    kn = b.describe_params()
    assert all(q["nbits"] in (4, 8) and q["bucket"] in (0, 1) for q in kn)
    assert all(q["chunk_log2"] >= q["alpha"] for q in kn if q["algo"] == 0)
    check_segments(segs, ks, b, kth, vals, idx, sorted)


# every knob of drtopk_seg_params_t, forced per segment
KNOBS = ([{"algo": "plain", "nbits": nb, "bucket": bk} for nb in (4, 8) for bk in (0, 1)] +
         [{"algo": "radix", "alpha": al, "beta": be, "nbits": nb, "bucket": bk, "chunk_log2": ch}
          for al, ch in ((6, 13), (9, 15), (12, 17)) for be in (1, 2) for nb in (4, 8) for bk in (0, 1)] +
         [{"algo": "bitonic"}])


@pytest.mark.parametrize("sorted", [True, False])
def test_batch_every_forced_knob_matches_oracle(sorted):
    import torch

    import drtopksc_b200 as D
    rng = np.random.default_rng(7)
    segs, ks, params = [], [], []
    for i, q in enumerate(KNOBS):
        for dist in ("u32", "f32n", "fewdigits", "ties"):
            n = int(rng.integers(1500, 4096)) if q["algo"] == "bitonic" else int(rng.integers(40000, 300000))
            if dist == "ties":
                x = np.repeat(rng.integers(0, 40, (n + 999) // 1000).astype(np.uint32), 1000)[:n].copy()
            else:
                x = O.gen(dist, n, 100 * i + len(segs))
            kmax = 1365 if q.get("beta") == 2 else 4096
            k = int(min(n, kmax, np.exp2(rng.uniform(0, 12))))
            if q["algo"] == "radix":  # the delegate vector must hold k
                k = min(k, (n >> q["alpha"]) * q["beta"])
            segs.append(x)
            ks.append(max(1, k))
            params.append(q)
    ks = np.array(ks, dtype=np.uint32)
    bits = np.concatenate([x.view(np.uint32) for x in segs])
    offsets = np.concatenate([[0], np.cumsum([x.size for x in segs])]).astype(np.uint64)
    dtypes = np.array([1 if x.dtype == np.float32 else 0 for x in segs], dtype=np.int32)
    b = D.Batch().plan(offsets, ks, dtypes, sorted=sorted, params=params)
    got = b.describe_params()
    for q, g in zip(params, got):
        for f, v in q.items():
            if f == "algo":
                v = D._ALGOS[v]
            assert g[f] == v, (q, g)
    keys = torch.from_numpy(bits.view(np.int32)).cuda()
    kth = torch.zeros(len(ks), dtype=torch.int32, device="cuda")
    tot = int(ks.astype(np.int64).sum())
    vals = torch.zeros(tot, dtype=torch.int32, device="cuda")
    idx = torch.zeros(tot, dtype=torch.int64, device="cuda")
    b.run(keys, kth, vals, idx)
    b.sync_check()
    check_segments(segs, ks, b, kth.cpu().numpy().view(np.uint32), vals.cpu().numpy().view(np.uint32),
                   idx.cpu().numpy(), sorted)


def test_batch_graph_replay_and_heavy_ties():
    segs, bits, offsets, ks, dtypes = make_batch(2, 24, 12, 21, kmax=4096)
    # a few adversarial segments: all-equal and few distinct values
    segs[0] = np.full(segs[0].size, 7, dtype=np.uint32)
    segs[1] = O.gen("fewdigits", segs[1].size, 5)
    dtypes[0] = dtypes[1] = 0
    bits = np.concatenate([x.view(np.uint32) for x in segs])
    b, kth, vals, idx = run_batch(bits, offsets, ks, dtypes, graph=True, reps=3)
    check_segments(segs, ks, b, kth, vals, idx)


def test_batch_equals_plain_calls():
    import torch

    import drtopksc_b200 as D
    segs, bits, offsets, ks, dtypes = make_batch(3, 8, 15, 21)
    b, kth, vals, idx = run_batch(bits, offsets, ks, dtypes)
    h = D.Handle()
    for s, x in enumerate(segs):
        t = torch.from_numpy(x).cuda() if x.dtype == np.float32 else torch.from_numpy(x.view(np.int32)).cuda()
        pk, pv, pi = h.topk(t, int(ks[s]), sorted=True)
        assert np.array_equal(pi.cpu().numpy(), idx[b.out_offsets[s]:b.out_offsets[s + 1]])


def test_batch_argument_errors():
    import drtopksc_b200 as D
    b = D.Batch()
    with pytest.raises(D.DrTopKError) as e:  # bitonic segments hold at most 4096 keys
        b.plan([0, 10000], [5], [0], params=[{"algo": "bitonic"}])
    assert e.value.status == D.EINVAL
    with pytest.raises(D.DrTopKError) as e:  # beta 2 keeps up to 3k subranges: k <= 1365
        b.plan([0, 1 << 20], [2000], [0], params=[{"algo": "radix", "beta": 2}])
    assert e.value.status == D.EINVAL
    with pytest.raises(D.DrTopKError) as e:
        b.plan([0, 10], [11], [0])
    assert e.value.status == D.EINVAL
    with pytest.raises(D.DrTopKError) as e:
        b.plan([0, 100000], [5000], [0])
    assert e.value.status == D.EUNSUPPORTED
