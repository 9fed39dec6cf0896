"""The phases after the sampler run on the whole GPU (cooperative grid,
software grid barrier), inside one thread-block cluster (hardware cluster
barrier) or in one CTA with the sets in shared memory.  Every team must give
the oracle's exact answer on every path, key mode and tie pattern."""
import numpy as np
import pytest

import drtopksc_b200 as D
from oracle import oracle as O
from tests.helpers import expected, run_topk, same_bits

pytestmark = pytest.mark.gpu

# team parameter -> stats["team_cluster"] (team 4, the shared-GPU choice, is
# the one-CTA tail when the sets fit, else one cluster)
TEAM_KIND = {1: (0,), 2: (1,), 3: (3,), 4: (1, 3)}

CASES = [
    # (dist, log2n, k, extra params)
    ("u32", 20, 128, {}),
    ("u32", 20, 1, {"alpha": 10, "path": 1}),
    ("u32", 18, 4096, {"alpha": 4, "path": 2}),
    ("normal", 22, 64, {"alpha": -2}),
    ("normal", 20, 70000, {"alpha": -2}),
    ("fewdigits", 20, 300, {}),
    ("fewdigits", 20, 65536, {"alpha": 3, "path": 2}),
    ("f32n", 20, 1000, {"alpha": -2}),
    ("f32u", 19, 5000, {"alpha": 2, "path": 2}),
    ("u32", 15, 777, {"algo": "plain"}),
    ("u32", 17, 20000, {"algo": "plain"}),
    ("u32", 20, 256, {"algo": "bucket"}),
    ("normal", 19, 33, {"nbits": 4}),
    ("u32", 20, 9000, {"alpha": 6, "path": 1}),
    ("u32", 13, 3000, {"algo": "plain"}),
    ("f32n", 17, 2500, {"alpha": 5, "path": 2}),
]


@pytest.mark.parametrize("team", [1, 2, 3, 4])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_team_exact(case, team):
    dist, log2n, k, kw = CASES[case]
    x = O.gen(dist, (1 << log2n) + 3 * case, 500 + case)
    for largest in (True, False):
        for sorted_ in (True, False):
            try:
                kth, vals, idx, st = run_topk(x, k, largest=largest, sorted=sorted_, team=team, **kw)
            except D.DrTopKError as e:
                # the shared-memory tail only takes problems whose sets fit
                assert team == 3 and e.status == D.EUNSUPPORTED
                return
            ek, ev, ei = expected(x, k, largest)
            if not sorted_:
                keys = O.as_keys(vals)
                if not largest:
                    keys = ~keys
                order = np.lexsort((idx, -keys.astype(np.int64)))
                vals, idx = vals[order], idx[order]
            assert same_bits(kth, ek), (case, team, largest, st)
            assert same_bits(vals, ev), (case, team, largest, sorted_)
            assert np.array_equal(idx, ei), (case, team, largest, sorted_)
            assert st["device_error"] == 0
            assert st["team_cluster"] in TEAM_KIND[team], st


@pytest.mark.parametrize("team", [1, 2, 4])
def test_team_large_k_sorted(team):
    # k above the one-CTA sort: multi-CTA LSD sort inside the team
    x = O.gen("normal", 1 << 20, 77)
    k = 20000
    kth, vals, idx, st = run_topk(x, k, sorted=True, team=team)
    ek, ev, ei = expected(x, k)
    assert same_bits(kth, ek) and same_bits(vals, ev) and np.array_equal(idx, ei)
    assert st["team_cluster"] in TEAM_KIND[team]


def test_auto_team_small_problem_is_one_cta():
    x = O.gen("u32", 1 << 20, 5)
    kth, vals, idx, st = run_topk(x, 64, sorted=False, alpha=-2)
    assert st["team_cluster"] == 3 and st["team_ctas"] == 8  # one cluster, rank 0 works
    ek, ev, ei = expected(x, 64)
    assert same_bits(kth, ek)
    order = np.lexsort((idx, -O.as_keys(vals).astype(np.int64)))
    assert same_bits(vals[order], ev) and np.array_equal(idx[order], ei)


@pytest.mark.parametrize("log2n,k,kw", [(17, 100, {"alpha": 5, "path": 2}), (16, 3000, {"alpha": 4, "path": 2}),
                                        (16, 50, {"alpha": 6, "path": 1})])
def test_one_cta_overflow_falls_back_exact(log2n, k, kw):
    # heavy ties (top 24 bits shared): every key of a kept subrange passes the
    # threshold, the candidates outgrow shared memory and the cluster finishes
    # on the general path -- same exact answer
    x = O.gen("fewdigits", 1 << log2n, 42)
    for largest in (True, False):
        kth, vals, idx, st = run_topk(x, k, largest=largest, sorted=True, team=3, **kw)
        ek, ev, ei = expected(x, k, largest)
        assert same_bits(kth, ek) and same_bits(vals, ev) and np.array_equal(idx, ei), (log2n, k, kw, st)
        assert st["team_cluster"] == 3 and st["device_error"] == 0
