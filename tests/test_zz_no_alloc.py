"""cpg_select_topk_noalloc against cpg_select_topk, through the C ABI.

The no-alloc entry point is for callers that cannot allocate device memory
(a pipeline whose other streams must not be stalled by cudaFree's device-wide
synchronisation, a memory pool that owns every byte).  It must return exactly
what the allocating entry point returns, call after call, although every call
reuses the same library-owned scratch.  This file is collected last on
purpose: a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

import cpg_b200

pytestmark = pytest.mark.gpu

MAX_K = 262144


def _run(fn, d, n, k, out):
    got = C.c_int64(-1)
    st = fn(d.data_ptr(), n, k, out.data_ptr(), C.byref(got), None)
    return st, got.value


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    rng = np.random.default_rng(7)
    # two calls in a row: the second is smaller than the first, so stale
    # scratch from the first call would show up in its result
    for n, k in ((2_000_000, MAX_K), (30_000, 1000)):
        c = rng.uniform(0.0, 100.0, size=n).astype(np.float32)
        c[rng.random(n) < 0.05] = 0.0
        c[rng.random(n) < 0.05] = 42.0        # a tie group
        d = torch.from_numpy(c).cuda()
        a = torch.full((k,), -1.0, dtype=torch.float32, device="cuda")
        b = torch.full((k,), -2.0, dtype=torch.float32, device="cuda")
        st_a, na = _run(cpg_b200.lib.cpg_select_topk, d, n, k, a)
        st_b, nb = _run(cpg_b200.lib.cpg_select_topk_noalloc, d, n, k, b)
        assert st_a == 0 and st_b == 0
        assert na == nb == min(k, int(np.count_nonzero(c)))
        # integer-ordered selection and sort: bit for bit
        assert torch.equal(a[:na].view(torch.int32), b[:nb].view(torch.int32))
        want = np.sort(c[c != 0.0])[:k]
        assert np.array_equal(b[:nb].cpu().numpy(), want)


def test_noalloc_rejects_k_above_its_limit():
    import torch
    d = torch.ones(16, dtype=torch.float32, device="cuda")
    out = torch.empty(16, dtype=torch.float32, device="cuda")
    st, n = _run(cpg_b200.lib.cpg_select_topk_noalloc, d, 16, MAX_K + 1, out)
    assert st == 4 and n == 0          # CPG_ERR_CAPACITY, nothing written


@pytest.mark.parametrize("case", ["n_below_k", "all_zero", "few_nonzero_at_max_k"])
def test_noalloc_edge_cases_match_numpy(case):
    """k above n (min(k, n) is selected), an all-zero input (nothing is
    returned), and fewer non-zero costs than k at the largest k (the sort
    runs on fewer keys than the scratch is laid out for); each against
    np.sort(c[c != 0])[:k] and against the allocating entry point."""
    import torch
    rng = np.random.default_rng(11)
    if case == "n_below_k":
        n, k = 5000, 20000
        c = rng.uniform(0.0, 10.0, size=n).astype(np.float32)
    elif case == "all_zero":
        n, k = 100_000, 5000
        c = np.zeros(n, np.float32)
    else:
        n, k = 1_000_000, MAX_K
        c = np.zeros(n, np.float32)
        nz = rng.choice(n, size=70_000, replace=False)
        c[nz] = rng.uniform(0.5, 50.0, size=nz.size).astype(np.float32)
    d = torch.from_numpy(c).cuda()
    a = torch.full((k,), -1.0, dtype=torch.float32, device="cuda")
    b = torch.full((k,), -2.0, dtype=torch.float32, device="cuda")
    st_a, na = _run(cpg_b200.lib.cpg_select_topk, d, n, k, a)
    st_b, nb = _run(cpg_b200.lib.cpg_select_topk_noalloc, d, n, k, b)
    want = np.sort(c[c != 0.0])[:k]
    assert st_a == 0 and st_b == 0
    assert na == nb == want.size
    assert np.array_equal(b[:nb].cpu().numpy(), want)
    assert torch.equal(a[:na].view(torch.int32), b[:nb].view(torch.int32))
