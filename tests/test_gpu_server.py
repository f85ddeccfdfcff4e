"""Served form: queries answered by the continuous-batching request loop are
the same as each query answered alone on its graph's state at arrival
(delay updates applied in arrival order), whatever the batching."""
import numpy as np
import pytest

import cpg_b200

pytestmark = pytest.mark.gpu


def _dags(count, seed=21):
    out = []
    for i in range(count):
        p = cpg_b200.gen_params(seed=seed + i, n_pins=3000 + 500 * i, n_levels=20 + 3 * i,
                                n_first=16, n_last=16, level_span=3, degree_kind=1,
                                deg_mean=3.0 + i, deg_cap=32)
        out.append(cpg_b200.generate(p))
    return out


def _csr(dag):
    order = np.argsort(dag.src, kind="stable")
    adjp = np.zeros(dag.n + 1, np.int64)
    np.add.at(adjp, dag.src + 1, 1)
    return np.cumsum(adjp).astype(np.int32), dag.dst[order].astype(np.int32), dag.w[order].copy()


def _stream(dags, n, seed=5):
    rng = np.random.default_rng(seed)
    qs = []
    for _ in range(n):
        g = int(rng.integers(len(dags)))
        k = int(np.exp(rng.uniform(np.log(100), np.log(3000))))
        upd = None
        if rng.random() < 0.2:
            m = dags[g].m
            e = rng.choice(m, size=max(1, m // 100), replace=False).astype(np.int32)
            upd = (e, rng.uniform(0.1, 10.0, size=e.size).astype(np.float32))
        qs.append((g, k, upd))
    return qs


def _serve(dags, qs, max_batch):
    with cpg_b200.Server(max_batch=max_batch) as s:
        for d in dags:
            s.add_dag(d)
        s.start()
        tickets = [s.submit(g, k, *(upd if upd else (None, None))) for g, k, upd in qs]
        out = [s.wait(t, timeout_ms=120000)[0] for t in tickets]
        st = s.stats()
        s.stop()
    return out, st


def test_server_mix_equals_alone():
    dags = _dags(4)
    qs = _stream(dags, 48)
    mixed, st = _serve(dags, qs, max_batch=64)
    assert st["completed"] == len(qs) and st["max_batch_seen"] > 1
    # the mix stays inside what cpg_server_start allocated: nothing is
    # allocated in the loop and no launch reruns after a buffer grew
    assert st["loop_allocs"] == 0 and st["retries"] == 0
    n_upd = sum(1 for q in qs if q[2] is not None)
    assert 1 <= st["sfxt_rebuilds"] <= n_upd
    one, _ = _serve(dags, qs, max_batch=1)
    csr = [_csr(d) for d in dags]
    for i, (g, k, upd) in enumerate(qs):
        adjp, adj, w = csr[g]
        if upd is not None:
            w[upd[0]] = upd[1]               # the graph's state from now on
        with cpg_b200.CpGen() as h:
            h.load_csr(dags[g].n, adjp, adj, w)
            h.report_paths(k)
            alone = h.get_slacks(k)
        assert np.array_equal(mixed[i].view(np.uint32), alone.view(np.uint32)), i
        assert np.array_equal(one[i].view(np.uint32), alone.view(np.uint32)), i


def test_server_admission_budget_splits_launches():
    dags = _dags(2, seed=40)
    qs = [(i % 2, 2000, None) for i in range(16)]
    per_query = 2000 * 700                    # about two queries per launch
    with cpg_b200.Server(max_batch=64, hbm_budget_bytes=2 * per_query) as s:
        for d in dags:
            s.add_dag(d)
        s.start()
        ts = [s.submit(g, k) for g, k, _ in qs]
        res = [s.wait(t, timeout_ms=120000)[0] for t in ts]
        st = s.stats()
    assert all(r.size == 2000 for r in res)
    assert st["max_batch_seen"] <= 2 and st["launches"] >= 8


def test_server_many_updates_rebuild_only_changed_graphs():
    """Every query updates delays: per-graph incremental rebuilds append to the
    chain-heap pool until it overflows and a full rebuild compacts it; results
    stay equal to each query answered alone."""
    dags = _dags(3, seed=60)
    rng = np.random.default_rng(8)
    qs = []
    for _ in range(90):
        g = int(rng.integers(len(dags)))
        m = dags[g].m
        e = rng.choice(m, size=max(1, m // 50), replace=False).astype(np.int32)
        qs.append((g, 500, (e, rng.uniform(0.1, 10.0, size=e.size).astype(np.float32))))
    mixed, st = _serve(dags, qs, max_batch=16)
    assert st["completed"] == len(qs)
    # the diagnostics: every rebuild is counted, the pool filled at least
    # once, and the longest step is a real duration
    assert 1 <= st["sfxt_rebuilds"] <= len(qs)
    assert st["pool_rebuilds"] >= 1 and st["retries"] == 0
    assert 0.0 < st["max_step_ms"] < 60_000.0
    csr = [_csr(d) for d in dags]
    for i, (g, k, upd) in enumerate(qs):
        adjp, adj, w = csr[g]
        w[upd[0]] = upd[1]
        with cpg_b200.CpGen() as h:
            h.load_csr(dags[g].n, adjp, adj, w)
            h.report_paths(k)
            alone = h.get_slacks(k)
        assert np.array_equal(mixed[i].view(np.uint32), alone.view(np.uint32)), i
