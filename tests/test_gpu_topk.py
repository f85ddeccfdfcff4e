"""cpg_select_topk: the final select-and-sort step on its own, through the
C ABI on device buffers, against numpy."""
import numpy as np
import pytest

import cpg_b200

pytestmark = pytest.mark.gpu


def _costs(n, seed, zeros=0.1, ties=False):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-5.0, 500.0, size=n).astype(np.float32)
    if ties:
        c = np.round(c).astype(np.float32)
    c[rng.random(n) < zeros] = 0.0
    return c


@pytest.mark.parametrize("n,k,ties", [(1, 1, False), (1000, 10, False), (100_000, 4096, True),
                                      (3_000_000, 1_000_000, False), (50_000, 200_000, True)])
def test_select_topk_matches_numpy(n, k, ties):
    import torch
    c = _costs(n, n + k, ties=ties)
    d = torch.from_numpy(c).cuda()
    out = torch.empty(max(k, 1), dtype=torch.float32, device="cuda")
    got = cpg_b200.select_topk(d.data_ptr(), n, k, out.data_ptr())
    want = np.sort(c[c != 0.0])[:k]
    assert got == len(want)
    assert np.array_equal(out[:got].cpu().numpy().view(np.uint32), want.view(np.uint32))


def test_select_topk_all_zero_and_empty():
    import torch
    d = torch.zeros(1000, dtype=torch.float32, device="cuda")
    out = torch.empty(10, dtype=torch.float32, device="cuda")
    assert cpg_b200.select_topk(d.data_ptr(), 1000, 10, out.data_ptr()) == 0
    assert cpg_b200.select_topk(d.data_ptr(), 0, 10, out.data_ptr()) == 0
