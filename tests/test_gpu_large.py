"""Full-size parity: the 1,000,000-pin / 200-level workload (fp32 and integer
delays, K = 1e6) and the density sweep on the same generator (mean degree 10 /
30 / 40 / 50 at K = 1e6 / 2e5 / 2e5 / 1e5), against the CPU oracle.

The oracle's answers at these sizes are committed as pins
(tests/golden/oracle_pins.npz, made by tests/golden/make_oracle_pins.py):
per prefix P in {1e3, 1e4, 1e5, 1e6} the sha256 of the first P float32 costs
and their sum, every 100th cost, and the sha256 of the suffix-tree arrays.

Bars:
- IEEE division: every prefix bit-exact (sha256 equal), suffix tree bit-exact;
- the reference's fast division: within rtol 1e-5, atol 0 of the pinned
  costs for fp32 delays; bit-exact at every prefix for integer delays;
- the engine, the host-stepped phase loop and the level-synchronous suffix
  tree give the same answer; a smaller K gives the prefix of a larger one.
"""
import hashlib
import os

import numpy as np
import pytest

import cases
import cpg_b200

pytestmark = pytest.mark.gpu

RTOL = 1e-5  # fp32 delays, reference (fast) division
PREFIXES = [1_000, 10_000, 100_000, 1_000_000]
PINS = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                            "oracle_pins.npz"))


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _answer(n, src, dst, w, k, division=cpg_b200.DIV_IEEE, **kw):
    with cpg_b200.CpGen(division=division, root_seeding=cpg_b200.ROOTS_ALL, **kw) as g:
        g.load_edges(n, src, dst, w)
        g.report_paths(k)
        return g.get_slacks(k), g.get_sfxt(), g.stats()


def _assert_pinned(name, costs):
    """costs bit-exact against the oracle's pins at every prefix."""
    k = int(PINS[f"{name}/k"])
    assert costs.size == int(PINS[f"{name}/n_costs"]) == k
    assert np.array_equal(costs[::100].view(np.uint32), PINS[f"{name}/every100"].view(np.uint32))
    for p in PREFIXES:
        if p > k:
            continue
        assert _sha(costs[:p]) == str(PINS[f"{name}/p{p}_sha"]), (name, p)
        assert costs[:p].astype(np.float64).sum() == float(PINS[f"{name}/p{p}_sum"])


def _assert_sfxt_pinned(name, sfxt):
    d, s, lv = sfxt
    assert _sha(d) == str(PINS[f"{name}/sfxt_sha_dist"])
    assert _sha(s) == str(PINS[f"{name}/sfxt_sha_succ"])
    assert _sha(lv) == str(PINS[f"{name}/sfxt_sha_level"])


@pytest.fixture(scope="module", params=["large1m_f32", "large1m_int"])
def large(request):
    name = request.param
    n, src, dst, w = cases.load_case(name)
    full, sfxt, st = _answer(n, src, dst, w, 1_000_000)
    return name, (n, src, dst, w), full, sfxt, st


def test_full_size_ieee_pinned_at_every_prefix(large):
    name, _, full, sfxt, st = large
    assert np.all(np.diff(full) >= 0)
    assert st["paths_accepted"] >= full.size
    _assert_pinned(name, full)
    _assert_sfxt_pinned(name, sfxt)
    if name.endswith("_int"):
        # integer delays: every cost is a whole number of delay units
        assert np.array_equal(full, np.round(full))


def test_full_size_reference_division(large):
    name, (n, src, dst, w), full, _, _ = large
    ref_div, _, _ = _answer(n, src, dst, w, 1_000_000, cpg_b200.DIV_REFERENCE)
    if name.endswith("_int"):
        _assert_pinned(name, ref_div)
    else:
        np.testing.assert_allclose(ref_div, full, rtol=RTOL, atol=0)
        np.testing.assert_allclose(ref_div[::100], PINS[f"{name}/every100"], rtol=RTOL, atol=0)


def test_full_size_prefixes_equal_smaller_queries(large):
    _, (n, src, dst, w), full, _, _ = large
    for k in PREFIXES[:3]:
        got, _, _ = _answer(n, src, dst, w, k)
        assert np.array_equal(got.view(np.uint32), full[:k].view(np.uint32)), k


def test_full_size_engine_agrees_with_host_stepped_and_level_sync(large):
    _, (n, src, dst, w), full, _, _ = large
    k = 100_000
    a, _, _ = _answer(n, src, dst, w, k, host_stepped=True)
    b, _, _ = _answer(n, src, dst, w, k, sfxt_level_sync=True)
    assert np.array_equal(a.view(np.uint32), full[:k].view(np.uint32))
    assert np.array_equal(b.view(np.uint32), full[:k].view(np.uint32))


@pytest.mark.parametrize("name", sorted(cases.SWEEP))
def test_density_sweep_pinned(name):
    n, src, dst, w = cases.load_case(name)
    k = cases.SWEEP[name][1]
    full, sfxt, _ = _answer(n, src, dst, w, k)
    assert np.all(np.diff(full) >= 0)
    _assert_pinned(name, full)
    _assert_sfxt_pinned(name, sfxt)
    ref_div, _, _ = _answer(n, src, dst, w, k, cpg_b200.DIV_REFERENCE)
    np.testing.assert_allclose(ref_div, full, rtol=RTOL, atol=0)
