"""BVSS packing on the host (no GPU): the reference's known answers
(unittests/tc_sfxt_bvss.cu:12-51, unittests/tc_pfxt_bvss.cu:9-100), decode and
verify round trips on seeded graphs, and the oracle's BFS and pair restatements
against the reference's expected outputs."""
import numpy as np
import pytest

import bvss_graphs as bg
import cpg_b200
import oracle


def test_fanout_packing_known_answer():
    b = cpg_b200.Bvss(10, bg.REF10_ROW_PTR, bg.REF10_COL_IDX)
    i = b.info()
    assert (i["sigma"], i["slices_per_thread"], i["slice_capacity"]) == (8, 4, 128)
    assert i["n_intervals"] == 2
    assert i["unpadded_slices"] == 6 and i["total_set_bits"] == 6
    assert i["compression_ratio"] == pytest.approx(6.0 / 48.0)
    a = b.arrays()
    assert a["real_ptrs"].tolist() == [0, 1, 2]
    assert a["virtual_to_real"].tolist() == [0, 1]
    assert a["row_ids"].size == 256 and a["masks"].size == 64
    assert b.decode_row(0) == [1, 9]
    assert b.decode_row(1) == [8]
    assert b.decode_row(2) == [0, 9]
    assert b.decode_row(4) == [2]


def test_verify_rejects_mismatched_csr():
    b = cpg_b200.Bvss(4, [0, 1, 2, 2, 2], [1, 2])
    assert b.verify(4, [0, 1, 2, 2, 2], [1, 2])
    assert not b.verify(4, [0, 1, 2, 2, 2], [1, 3])


def test_adev_packing_known_answer():
    b = cpg_b200.Bvss(10, bg.REF10_ROW_PTR, bg.REF10_COL_IDX, bg.REF10_SUCCS)
    i = b.info()
    assert i["n_intervals"] == 2
    assert i["unpadded_slices"] == 2 and i["total_set_bits"] == 2
    assert i["compression_ratio"] == pytest.approx(2.0 / 16.0)
    assert b.decode_row(0) == []
    assert b.decode_row(1) == [0]
    assert b.decode_row(2) == []
    assert b.decode_row(9) == [2]
    assert b.verify(10, bg.REF10_ROW_PTR, bg.REF10_COL_IDX, bg.REF10_SUCCS)
    assert not b.verify(10, bg.REF10_ROW_PTR, bg.REF10_COL_IDX, [-1] * 10)


def test_adev_rejects_bad_succs():
    with pytest.raises(cpg_b200.CpgError):
        cpg_b200.Bvss(2, [0, 1, 1], [1], [1, 5])


def test_compact_packing_known_answer():
    b = cpg_b200.Bvss(10, None, None, compact_offsets=[0, 2, 3, 3, 3, 3, 3, 3, 3, 5, 5])
    i = b.info()
    assert i["n_intervals"] == 2 and i["unpadded_slices"] == 5 and i["total_set_bits"] == 5
    a = b.arrays()
    rec = []
    for vss in range(i["n_vss"]):
        iv = int(a["virtual_to_real"][vss])
        for lane in range(32):
            packed = int(a["masks"][vss * 32 + lane])
            for ch in range(4):
                d = int(a["row_ids"][vss * 128 + lane * 4 + ch])
                if d < 0:
                    continue
                m = (packed >> (8 * ch)) & 0xFF
                assert m != 0
                rec.append((iv * 8 + (m & -m).bit_length() - 1, d))
    assert sorted(rec) == [(0, 0), (0, 1), (1, 2), (8, 3), (8, 4)]


def _layout_ok(a, n_intervals):
    """Slices of every VSS fill lanes first (slice s at lane s % 32, chunk s // 32)."""
    cnt = a["slice_counts"].astype(int)
    rows = a["row_ids"].reshape(-1, 32, 4)
    for vss, c in enumerate(cnt):
        filled = np.zeros(128, bool)
        for s in range(128):
            filled[s] = rows[vss, s % 32, s // 32] >= 0
        assert filled[:c].all() and not filled[c:].any()
    assert a["real_ptrs"][-1] == cnt.size and a["real_ptrs"].size == n_intervals + 1


@pytest.mark.parametrize("seed", [1, 2])
def test_round_trip_local_dag(seed):
    n, src, dst, _ = bg.local_dag(seed, levels=12, width=200)
    adjp, adj = bg.to_csr(n, src, dst)
    b = cpg_b200.Bvss(n, adjp, adj)
    assert b.verify(n, adjp, adj)
    i = b.info()
    assert i["total_set_bits"] == adj.size  # no duplicate edges here
    assert i["total_set_bits"] / i["unpadded_slices"] >= 2.0  # dense slices
    _layout_ok(b.arrays(), i["n_intervals"])
    # slices of an interval keep row order (the reference's ordering)
    a = b.arrays()
    rows = a["row_ids"].reshape(-1, 32, 4)
    for iv in range(min(i["n_intervals"], 50)):
        seq = []
        for vss in range(a["real_ptrs"][iv], a["real_ptrs"][iv + 1]):
            for s in range(int(a["slice_counts"][vss])):
                seq.append(int(rows[vss, s % 32, s // 32]))
        assert seq == sorted(seq)


def test_round_trip_generated_dag_with_duplicates():
    dag = cpg_b200.generate(cpg_b200.gen_params(seed=5, n_pins=3000, n_levels=20, n_first=40,
                                                n_last=40, level_span=3, degree_kind=0,
                                                deg_lo=1, deg_hi=4))
    src = np.concatenate([dag.src, dag.src[:50]])  # repeated edges collapse to one bit
    dst = np.concatenate([dag.dst, dag.dst[:50]])
    adjp, adj = bg.to_csr(dag.n, src, dst)
    b = cpg_b200.Bvss(dag.n, adjp, adj)
    assert b.verify(dag.n, adjp, adj)
    assert b.info()["total_set_bits"] == dag.src.size
    succ = np.full(dag.n, -1, np.int32)
    for u in range(dag.n):
        if adjp[u + 1] > adjp[u]:
            succ[u] = adj[adjp[u]]
    ad = cpg_b200.Bvss(dag.n, adjp, adj, succ)
    assert ad.verify(dag.n, adjp, adj, succ)


def test_oracle_bfs_levels_known_answer():
    got = oracle.bfs_levels(8, bg.REF8_ROW_PTR, bg.REF8_COL_IDX, bg.REF8_SINKS)
    assert got.tolist() == bg.REF8_LEVELS


def test_oracle_pairs_known_answer():
    got = oracle.adev_pairs(10, bg.REF10_ROW_PTR, bg.REF10_COL_IDX, bg.REF10_SUCCS, [0, 1, 2])
    assert got.tolist() == [[0, 1], [2, 9]]
