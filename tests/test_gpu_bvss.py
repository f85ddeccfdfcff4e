"""BVSS on the GPU: pull BFS levels and deviation pair discovery against the
oracle and the reference's known answers (unittests/tc_sfxt_bvss.cu:153-189,
unittests/tc_pfxt_bvss.cu:58-70), tensor-core tiles against scalar popc, and
the suffix tree built with the BVSS pull against the CSR push (bit-exact)."""
import numpy as np
import pytest

import bvss_graphs as bg
import cases
import cpg_b200
import oracle

pytestmark = pytest.mark.gpu

TILES = [cpg_b200.TILES_TENSOR, cpg_b200.TILES_SCALAR, cpg_b200.TILES_DENSITY]


@pytest.mark.parametrize("tiles", TILES)
def test_levels_known_answer(tiles):
    b = cpg_b200.Bvss(8, bg.REF8_ROW_PTR, bg.REF8_COL_IDX)
    lv, st = b.levels(bg.REF8_SINKS, tiles=tiles)
    assert lv.tolist() == bg.REF8_LEVELS
    assert st["levels"] == 4
    if tiles == cpg_b200.TILES_TENSOR:
        assert st["tiles_tensor"] > 0 and st["tiles_scalar"] == 0 and st["mma_issued"] > 0
    if tiles == cpg_b200.TILES_SCALAR:
        assert st["tiles_tensor"] == 0 and st["mma_issued"] == 0


def _sinks(adjp):
    return np.nonzero(np.diff(adjp) == 0)[0].astype(np.int32)


@pytest.mark.parametrize("seed", [3, 4])
def test_levels_local_dag_tensor_equals_scalar_equals_oracle(seed):
    n, src, dst, _ = bg.local_dag(seed, levels=60, width=700)
    adjp, adj = bg.to_csr(n, src, dst)
    want = oracle.bfs_levels(n, adjp, adj, _sinks(adjp))
    b = cpg_b200.Bvss(n, adjp, adj)
    got = {}
    for tiles in TILES:
        got[tiles], st = b.levels(None, tiles=tiles)
        np.testing.assert_array_equal(got[tiles], want)
    # dense slices: the density test sends tiles to the tensor cores
    _, st = b.levels(None, tiles=cpg_b200.TILES_DENSITY)
    assert st["tiles_tensor"] > 0


def test_levels_generated_dag_and_partial_sinks():
    n, src, dst, w = cases.load_case("single20k_f32")
    adjp, adj = bg.to_csr(n, src, dst)
    b = cpg_b200.Bvss(n, adjp, adj)
    sinks = _sinks(adjp)
    lv, _ = b.levels(sinks, tiles=cpg_b200.TILES_TENSOR)
    np.testing.assert_array_equal(lv, oracle.bfs_levels(n, adjp, adj, sinks))
    part = sinks[: max(1, sinks.size // 3)]
    lv, _ = b.levels(part, tiles=cpg_b200.TILES_SCALAR)
    np.testing.assert_array_equal(lv, oracle.bfs_levels(n, adjp, adj, part))
    assert (lv == -1).any() or part.size == sinks.size


@pytest.mark.parametrize("tiles", TILES)
def test_pairs_known_answer(tiles):
    b = cpg_b200.Bvss(10, bg.REF10_ROW_PTR, bg.REF10_COL_IDX, bg.REF10_SUCCS)
    pairs, _ = b.discover_pairs([0, 1, 2], max_pairs=16, tiles=tiles)
    assert pairs.tolist() == [[0, 1], [2, 9]]


@pytest.mark.parametrize("tiles", TILES)
def test_pairs_local_dag(tiles):
    n, src, dst, _ = bg.local_dag(7, levels=30, width=400)
    adjp, adj = bg.to_csr(n, src, dst)
    rng = np.random.default_rng(1)
    succ = np.array([adj[adjp[u]] if adjp[u + 1] > adjp[u] else -1 for u in range(n)], np.int32)
    b = cpg_b200.Bvss(n, adjp, adj, succ)
    sources = rng.choice(n, size=n // 3, replace=False).astype(np.int32)
    want = oracle.adev_pairs(n, adjp, adj, succ, sources)
    got, st = b.discover_pairs(sources, max_pairs=want.shape[0] + 10, tiles=tiles)
    np.testing.assert_array_equal(got, want)


def test_pairs_overflow_reports_capacity():
    n, src, dst, _ = bg.local_dag(8, levels=10, width=200)
    adjp, adj = bg.to_csr(n, src, dst)
    succ = np.full(n, -1, np.int32)
    b = cpg_b200.Bvss(n, adjp, adj, succ)
    with pytest.raises(cpg_b200.CpgError) as e:
        b.discover_pairs(np.arange(n, dtype=np.int32), max_pairs=10)
    assert e.value.status == 4  # CPG_ERR_CAPACITY


def _sfxt_and_costs(n, src, dst, w, k, **kw):
    with cpg_b200.CpGen(division=cpg_b200.DIV_IEEE, **kw) as g:
        g.load_edges(n, src, dst, w)
        g.report_paths(k)
        return g.get_sfxt(), g.get_slacks(k), g.stats()


@pytest.mark.parametrize("tiles", TILES)
def test_sfxt_bvss_pull_equals_csr_push_local_dag(tiles):
    n, src, dst, w = bg.local_dag(11, levels=80, width=600)
    (d0, s0, l0), c0, st0 = _sfxt_and_costs(n, src, dst, w, 2000, frontier=cpg_b200.FRONTIER_CSR)
    (d1, s1, l1), c1, st1 = _sfxt_and_costs(n, src, dst, w, 2000, frontier=cpg_b200.FRONTIER_BVSS,
                                             bvss_tiles=tiles)
    assert st0["frontier_used"] == cpg_b200.FRONTIER_CSR
    assert st1["frontier_used"] == cpg_b200.FRONTIER_BVSS
    np.testing.assert_array_equal(l1, l0)
    np.testing.assert_array_equal(d1, d0)
    np.testing.assert_array_equal(s1, s0)
    assert np.array_equal(c1.view(np.uint32), c0.view(np.uint32))
    if tiles == cpg_b200.TILES_TENSOR:
        assert st1["bvss_tiles_tensor"] > 0 and st1["bvss_tiles_scalar"] == 0
    if tiles == cpg_b200.TILES_SCALAR:
        assert st1["bvss_tiles_tensor"] == 0 and st1["bvss_tiles_scalar"] > 0


def test_sfxt_auto_picks_bvss_on_dense_and_csr_on_sparse():
    n, src, dst, w = bg.local_dag(12, levels=30, width=300)
    (_, _, _), _, st = _sfxt_and_costs(n, src, dst, w, 100)
    assert st["frontier_used"] == cpg_b200.FRONTIER_BVSS
    assert st["bvss_bits_per_slice"] >= 2.0
    n, src, dst, w = cases.load_case("single20k_f32")
    (_, _, _), _, st = _sfxt_and_costs(n, src, dst, w, 100)
    assert st["frontier_used"] == cpg_b200.FRONTIER_CSR


@pytest.mark.parametrize("name", ["simple", "tv80_unit_wgts", "single20k_f32", "single20k_int"])
def test_sfxt_bvss_forced_matches_oracle(name):
    n, src, dst, w = cases.load_case(name)
    od, os_, ol = oracle.OracleGraph.from_edges(n, src, dst, w).sfxt()
    with cpg_b200.CpGen(frontier=cpg_b200.FRONTIER_BVSS, bvss_tiles=cpg_b200.TILES_TENSOR) as g:
        g.load_edges(n, src, dst, w)
        g.levelize()
        d, s, lvl = g.get_sfxt()
        assert g.stats()["frontier_used"] == cpg_b200.FRONTIER_BVSS
    np.testing.assert_array_equal(lvl, ol)
    np.testing.assert_array_equal(d, od)
    np.testing.assert_array_equal(s, os_)


def test_sfxt_bvss_repeat_and_incremental():
    n, src, dst, w = bg.local_dag(13, levels=40, width=500)
    rng = np.random.default_rng(0)
    with cpg_b200.CpGen(division=cpg_b200.DIV_IEEE, frontier=cpg_b200.FRONTIER_BVSS) as g, \
         cpg_b200.CpGen(division=cpg_b200.DIV_IEEE, frontier=cpg_b200.FRONTIER_CSR) as h:
        g.load_edges(n, src, dst, w)
        h.load_edges(n, src, dst, w)
        for _ in range(3):
            g.levelize()
            h.levelize()
            for a, b in zip(g.get_sfxt(), h.get_sfxt()):
                np.testing.assert_array_equal(a, b)
            eids = rng.choice(src.size, size=src.size // 100, replace=False).astype(np.int32)
            nw = rng.uniform(0.1, 10.0, size=eids.size).astype(np.float32)
            g.update_delays(eids, nw)
            h.update_delays(eids, nw)
        g.report_paths(500)
        h.report_paths(500)
        assert np.array_equal(g.get_slacks(500).view(np.uint32), h.get_slacks(500).view(np.uint32))
