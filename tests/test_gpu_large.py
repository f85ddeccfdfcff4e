"""Full-size parity: the 1,000,000-pin / 200-level workload (fp32 and integer
delays, K = 1e6) and the density sweep on the same generator (mean degree 10 /
30 / 40 / 50).

At these sizes the oracle runs at K = 1e4 (the SEQUENTIAL heap restated on the
CPU, seconds); the rest are size-independent properties: every prefix of the
K = 1e6 answer equals the answer at that K (1e3, 1e4, 1e5), costs ascend, the
first cost is the shortest path, integer delays give integer costs, the
suffix tree matches the oracle's, and the device engine agrees with the
host-stepped split raises and with the level-synchronous suffix tree.
"""
import numpy as np
import pytest

import cases
import cpg_b200
import oracle

pytestmark = pytest.mark.gpu

PREFIXES = [1_000, 10_000, 100_000]
ORACLE_K = 10_000


def _graph(name):
    return cases.load_case(name)


def _answer(n, src, dst, w, k, **kw):
    with cpg_b200.CpGen(division=cpg_b200.DIV_IEEE, root_seeding=cpg_b200.ROOTS_ALL, **kw) as g:
        g.load_edges(n, src, dst, w)
        g.report_paths(k)
        return g.get_slacks(k), g.get_sfxt(), g.stats()


@pytest.fixture(scope="module", params=["large1m_f32", "large1m_int"])
def large(request):
    name = request.param
    n, src, dst, w = _graph(name)
    full, sfxt, st = _answer(n, src, dst, w, 1_000_000)
    return name, (n, src, dst, w), full, sfxt, st


def test_full_size_answer_shape(large):
    name, _, full, _, st = large
    assert full.size == 1_000_000
    assert np.all(np.diff(full) >= 0)
    assert st["paths_accepted"] >= full.size
    if name.endswith("_int"):
        # integer delays: every cost is a whole number of delay units
        assert np.array_equal(full, np.round(full))


def test_full_size_prefixes_equal_smaller_queries(large):
    _, (n, src, dst, w), full, _, _ = large
    for k in PREFIXES:
        got, _, _ = _answer(n, src, dst, w, k)
        assert np.array_equal(got.view(np.uint32), full[:k].view(np.uint32)), k


def test_full_size_sfxt_and_head_match_oracle(large):
    _, (n, src, dst, w), full, (d, s, lv), _ = large
    og = oracle.OracleGraph.from_edges(n, src, dst, w)
    od, os_, ol = og.sfxt()
    np.testing.assert_array_equal(d, od)
    np.testing.assert_array_equal(s, os_)
    np.testing.assert_array_equal(lv, ol)
    want = og.sequential(ORACLE_K)["slack"]
    assert np.array_equal(full[:ORACLE_K].view(np.uint32), want.view(np.uint32))


def test_full_size_reference_division_within_tolerance(large):
    _, (n, src, dst, w), full, _, _ = large
    with cpg_b200.CpGen(division=cpg_b200.DIV_REFERENCE, root_seeding=cpg_b200.ROOTS_ALL) as g:
        g.load_edges(n, src, dst, w)
        g.report_paths(1_000_000)
        ref_div = g.get_slacks(1_000_000)
    np.testing.assert_allclose(ref_div, full, rtol=1e-5, atol=0)


def test_full_size_engine_agrees_with_host_stepped_and_level_sync(large):
    _, (n, src, dst, w), full, _, _ = large
    k = 100_000
    a, _, _ = _answer(n, src, dst, w, k, host_stepped=True)
    b, _, _ = _answer(n, src, dst, w, k, sfxt_level_sync=True)
    assert np.array_equal(a.view(np.uint32), full[:k].view(np.uint32))
    assert np.array_equal(b.view(np.uint32), full[:k].view(np.uint32))


@pytest.mark.parametrize("name", sorted(cases.SWEEP))
def test_density_sweep(name):
    n, src, dst, w = _graph(name)
    k = cases.SWEEP[name][1]
    full, (d, s, _), st = _answer(n, src, dst, w, k)
    assert full.size == k and np.all(np.diff(full) >= 0)
    got, _, _ = _answer(n, src, dst, w, 1_000)
    assert np.array_equal(got.view(np.uint32), full[:1_000].view(np.uint32))
    og = oracle.OracleGraph.from_edges(n, src, dst, w)
    od, os_, _ = og.sfxt()
    np.testing.assert_array_equal(d, od)
    np.testing.assert_array_equal(s, os_)
    want = og.sequential(1_000)["slack"]
    assert np.array_equal(full[:1_000].view(np.uint32), want.view(np.uint32))
