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
