"""Failure detection without a GPU fault.

The reference exits on any CUDA error (cudaCheckErrors, gpucpg.cu:87-98) and
its cooperative loop waits on grid.sync() without a bound (gpucpg.cu:9152-
9415).  Here every device wait is a bounded poll that records a timeout and
returns, and allocation failures come back as statuses.  These tests make the
failures happen on purpose, in forms that neither fault nor hang a GPU:

- a poll limit of one makes the suffix tree's and the engine's waits run out
  (a queue slot or a barrier that is not ready on the first poll); the call
  returns CPG_ERR_TIMEOUT and the same handle then answers correctly;
- a host-side cap on device buffer sizes (cpg_debug_fail_allocs_above) makes
  allocations fail as out of memory, in a query, at server start and inside
  the server's request loop; each returns CPG_ERR_OOM, and the same handle or
  server answers correctly once the cap is lifted.
"""
import numpy as np
import pytest

import cases
import cpg_b200
import oracle

pytestmark = pytest.mark.gpu

TIMEOUT, OOM = 5, 3


@pytest.fixture
def no_alloc_cap():
    yield
    cpg_b200.debug_fail_allocs_above(0)


def _want(name, k):
    n, src, dst, w = cases.load_case(name)
    return (n, src, dst, w), oracle.OracleGraph.from_edges(n, src, dst, w).closure_topk(k)[0]["slack"]


def test_suffix_tree_wait_runs_out_then_handle_recovers():
    (n, src, dst, w), want = _want("single20k_f32", 3000)
    with cpg_b200.CpGen(division=cpg_b200.DIV_IEEE, spin_limit=1) as g:
        g.load_edges(n, src, dst, w)
        with pytest.raises(cpg_b200.CpgError) as e:
            g.levelize()
        assert e.value.status == TIMEOUT
        g.set_spin_limit(0)
        g.report_paths(3000)
        got = g.get_slacks(3000)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_engine_wait_runs_out_then_handle_recovers():
    (n, src, dst, w), want = _want("small_f32_s11", 5000)
    with cpg_b200.CpGen(division=cpg_b200.DIV_IEEE) as g:
        g.load_edges(n, src, dst, w)
        g.levelize()
        g.set_spin_limit(1)
        with pytest.raises(cpg_b200.CpgError) as e:
            g.report_paths(5000)      # the suffix tree is current: the engine runs
        assert e.value.status == TIMEOUT
        g.set_spin_limit(0)
        g.report_paths(5000)
        got = g.get_slacks(5000)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_allocation_failure_in_a_query_then_handle_recovers(no_alloc_cap):
    k = 200_000
    (n, src, dst, w), want = _want("single20k_f32", k)
    with cpg_b200.CpGen(division=cpg_b200.DIV_IEEE) as g:
        g.load_edges(n, src, dst, w)
        g.levelize()
        cpg_b200.debug_fail_allocs_above(1 << 20)   # the query's piles need more
        with pytest.raises(cpg_b200.CpgError) as e:
            g.report_paths(k)
        assert e.value.status == OOM
        cpg_b200.debug_fail_allocs_above(0)
        g.report_paths(k)
        got = g.get_slacks(k)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def _small_dags():
    return [cpg_b200.generate(cpg_b200.gen_params(seed=70 + i, n_pins=3000, n_levels=20,
                                                  n_first=16, n_last=16, level_span=3,
                                                  degree_kind=1, deg_mean=4.0, deg_cap=32))
            for i in range(3)]


def _alone(dag, k):
    with cpg_b200.CpGen() as h:
        h.load_dag(dag)
        h.report_paths(k)
        return h.get_slacks(k)


def test_allocation_failure_at_server_start_then_start_succeeds(no_alloc_cap):
    dags = _small_dags()
    with cpg_b200.Server(max_batch=8) as s:
        for d in dags:
            s.add_dag(d)
        # the graphs and suffix trees fit under 32 MiB; the engine piles the
        # start sizes for a 4M-path launch do not
        cpg_b200.debug_fail_allocs_above(32 << 20)
        with pytest.raises(cpg_b200.CpgError) as e:
            s.start()
        assert e.value.status == OOM
        cpg_b200.debug_fail_allocs_above(0)
        s.start()
        ts = [s.submit(i % 3, 1000) for i in range(6)]
        res = [s.wait(t, timeout_ms=120000)[0] for t in ts]
        st = s.stats()
        s.stop()
    for i, r in enumerate(res):
        assert np.array_equal(r.view(np.uint32), _alone(dags[i % 3], 1000).view(np.uint32))
    assert st["loop_allocs"] == 0 and st["retries"] == 0


def test_allocation_failure_inside_the_server_loop_then_next_query_succeeds(no_alloc_cap):
    dags = _small_dags()
    big = 300_000
    # a 1 GiB admission budget presizes the piles for 262,144 paths, so a
    # query for 300,000 paths must grow them inside the loop
    with cpg_b200.Server(max_batch=8, hbm_budget_bytes=1 << 30) as s:
        for d in dags:
            s.add_dag(d)
        s.start()
        cpg_b200.debug_fail_allocs_above(1 << 20)
        t = s.submit(0, big)
        with pytest.raises(cpg_b200.CpgError) as e:
            s.wait(t, timeout_ms=120000)
        assert e.value.status == OOM
        cpg_b200.debug_fail_allocs_above(0)
        t = s.submit(0, big)
        got, _ = s.wait(t, timeout_ms=120000)
        t = s.submit(1, 1000)
        small, _ = s.wait(t, timeout_ms=120000)
        st = s.stats()
        s.stop()
    assert np.array_equal(got.view(np.uint32), _alone(dags[0], big).view(np.uint32))
    assert np.array_equal(small.view(np.uint32), _alone(dags[1], 1000).view(np.uint32))
    assert st["loop_allocs"] >= 1
