"""Batched form: many (graph, k) queries answered by one captured launch
sequence return exactly what each query returns alone."""
import numpy as np
import pytest

import cpg_b200

pytestmark = pytest.mark.gpu


def _dags(count, seed=100):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(1500, 6000))
        levels = int(rng.integers(12, 40))
        p = cpg_b200.gen_params(seed=seed + i, n_pins=n, n_levels=levels,
                                n_first=max(8, n // (2 * levels)),
                                n_last=max(8, n // (2 * levels)), level_span=3,
                                degree_kind=1, deg_mean=float(rng.uniform(2, 8)), deg_cap=64,
                                weight_kind=int(i % 5 == 4))
        out.append(cpg_b200.generate(p))
    return out


def _alone(dag, k, division):
    with cpg_b200.CpGen(division=division) as g:
        g.load_dag(dag)
        g.report_paths(k)
        return g.get_slacks(k)


@pytest.mark.parametrize("division", [cpg_b200.DIV_REFERENCE, cpg_b200.DIV_IEEE])
def test_batch_matches_single_queries(division):
    dags = _dags(12)
    rng = np.random.default_rng(3)
    ks = [int(x) for x in np.exp(rng.uniform(np.log(100), np.log(20000), size=16))]
    gids = [i % len(dags) for i in range(len(ks))]      # some graphs asked twice
    want = [_alone(dags[g], k, division) for g, k in zip(gids, ks)]
    with cpg_b200.Batch(division=division) as b:
        for d in dags:
            b.add_dag(d)
        b.commit()
        b.set_queries(gids, ks)
        for step in range(3):                             # capture, then replays
            b.run(rebuild_sfxt=True)
            for q in range(len(ks)):
                got = b.costs(q)
                assert np.array_equal(got.view(np.uint32), want[q].view(np.uint32)), (step, q)
        st = b.stats()
        assert st["paths_accepted"] > 0


def test_batch_replay_without_rebuild_and_autotune():
    dags = _dags(6, seed=7)
    ks = [500, 2000, 50, 8000, 1000, 300]
    with cpg_b200.Batch() as b:
        for d in dags:
            b.add_dag(d)
        b.commit()
        b.set_queries(list(range(6)), ks)
        b.run(rebuild_sfxt=True)
        first = [b.costs(q) for q in range(6)]
        b.run(rebuild_sfxt=False)
        again = [b.costs(q) for q in range(6)]
        b.autotune()
        b.run(rebuild_sfxt=True)
        tuned = [b.costs(q) for q in range(6)]
    for a, c, t in zip(first, again, tuned):
        assert np.array_equal(a, c) and np.array_equal(a, t)


@pytest.mark.parametrize("caller_order", [False, True])
@pytest.mark.parametrize("roots", [cpg_b200.ROOTS_REFERENCE, cpg_b200.ROOTS_ALL])
def test_batch_of_reference_fixtures_matches_alone(roots, caller_order):
    """A batch renumbers each graph's vertices in level order.  On the
    reference's fixtures -- unit delays, so many heads tie for a vertex's
    distance and the successor tie-break decides, and many sources, so the
    root order decides -- every query still returns exactly what its graph
    returns alone, and a delay update names the caller's edge ids.
    caller_order keeps the callers' numbering (the A/B check)."""
    import cases
    names = ["tv80_unit_wgts", "simple", "dac21_paper_example", "small_int_s13"]
    graphs = [cases.load_case(nm) for nm in names]
    ks = [10_000, 1_000, 1_000, 5_000]
    rng = np.random.default_rng(5)
    upd = []  # (input edge indices, new delays) per graph
    for n, src, dst, w in graphs:
        e = rng.choice(src.size, size=max(1, src.size // 10), replace=False).astype(np.int64)
        upd.append((e, np.round(rng.uniform(1.0, 9.0, size=e.size)).astype(np.float32)))

    def alone(i):
        n, src, dst, w = graphs[i]
        with cpg_b200.CpGen(division=cpg_b200.DIV_IEEE, root_seeding=roots) as g:
            g.load_edges(n, src, dst, w)
            g.report_paths(ks[i])
            return g.get_slacks(ks[i])

    def csr(n, src, dst, w):
        order = np.argsort(src, kind="stable")
        adjp = np.zeros(n + 1, np.int64)
        np.add.at(adjp, src + 1, 1)
        return np.cumsum(adjp).astype(np.int32), dst[order], w[order]

    with cpg_b200.Batch(division=cpg_b200.DIV_IEEE, root_seeding=roots,
                        caller_order=caller_order) as b:
        for n, src, dst, w in graphs:
            b.add_graph(n, *csr(n, src, dst, w))
        b.commit()
        b.set_queries(list(range(len(graphs))), ks)
        b.run(True)
        for i in range(len(graphs)):
            want = alone(i)
            assert np.array_equal(b.costs(i).view(np.uint32), want.view(np.uint32)), names[i]
    # the served form holds the batch: re-asks with delay updates by the
    # caller's edge ids (positions in the graph's own CSR)
    with cpg_b200.Server(division=cpg_b200.DIV_IEEE, root_seeding=roots) as s:
        for n, src, dst, w in graphs:
            s.add_graph(n, *csr(n, src, dst, w))
        s.start()
        for i in range(len(graphs)):
            n, src, dst, w = graphs[i]
            # the caller's edge ids are positions in its CSR (rows in file order)
            order = np.argsort(src, kind="stable")
            pos = np.empty(src.size, np.int64)
            pos[order] = np.arange(src.size)
            e, nw = upd[i]
            got, _ = s.wait(s.submit(i, ks[i], pos[e].astype(np.int32), nw))
            want = alone_csr_update(graphs[i], pos[e].astype(np.int32), nw, ks[i], roots)
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), names[i]


def alone_csr_update(graph, eids, nw, k, roots):
    """One graph alone, its CSR edges eids given delays nw."""
    n, src, dst, w = graph
    with cpg_b200.CpGen(division=cpg_b200.DIV_IEEE, root_seeding=roots) as g:
        g.load_edges(n, src, dst, w)
        g.report_paths(k)          # levels known: the update rebuilds incrementally
        g.update_delays(eids, nw)
        g.report_paths(k)
        return g.get_slacks(k)
