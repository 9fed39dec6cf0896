"""BMW experiment (BMW/radixselect.cuh:1746-1832, BMW/PQ.h) through the C
ABI: the device sampler's delegates guide a host heap scan that skips every
subrange whose Max is below the heap's minimum.  The k-th key must equal the
exact k-th and the count of skipped keys must equal the oracle's restatement
of the same scan (the delegates are exact, so the scan is the same)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import expected

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dist", ["u32", "normal", "fewdigits"])
def test_bmw_matches_oracle(dist):
    import torch

    import drtopksc_b200 as D
    n = (1 << 20) + 333
    x = O.gen(dist, n, 77)
    t = torch.from_numpy(x.view(np.int32)).cuda()
    h = D.Handle()
    for k in (1, 100, 5000):
        for alpha in (6, 9, 12):
            if (n + (1 << alpha) - 1) >> alpha < k:
                continue  # one delegate per subrange: at least k subranges
            kth, skipped, _, _ = h.bmw_select(t, x, k, alpha)
            ek, _, _ = expected(x, k)
            okth, oskip = O.bmw_kth(x, k, alpha)
            assert kth == ek == okth, (dist, k, alpha)
            assert skipped == oskip, (dist, k, alpha, skipped, oskip)
            if dist == "u32" and k <= 100 and alpha >= 9:
                assert skipped > n // 4  # uniform keys: many subranges fall below the heap early


def test_bmw_argument_errors():
    import torch

    import drtopksc_b200 as D
    x = O.gen("u32", 4096, 1)
    t = torch.from_numpy(x.view(np.int32)).cuda()
    h = D.Handle()
    with pytest.raises(D.DrTopKError):
        h.bmw_select(t, x, 10, 11)  # 2 subranges cannot hold k = 10 delegates
