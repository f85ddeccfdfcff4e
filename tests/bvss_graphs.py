"""Seeded graphs for the BVSS tests: a level-local DAG whose rows have several
heads in one interval of 8 (dense slices), and the reference's unit-test
fixtures (unittests/tc_sfxt_bvss.cu:12-189, unittests/tc_pfxt_bvss.cu:9-100)."""
import numpy as np

# unittests/tc_sfxt_bvss.cu:14-16 and unittests/tc_pfxt_bvss.cu:11-13
REF10_ROW_PTR = [0, 2, 3, 5, 5, 6, 6, 6, 6, 6, 6]
REF10_COL_IDX = [1, 9, 8, 0, 9, 2]
REF10_SUCCS = [9, 8, 0, -1, 2, -1, -1, -1, -1, -1]
# unittests/tc_sfxt_bvss.cu:153-189
REF8_ROW_PTR = [0, 2, 3, 4, 5, 6, 7, 7, 7]
REF8_COL_IDX = [2, 4, 2, 3, 6, 5, 6]
REF8_SINKS = [6, 7]
REF8_LEVELS = [3, 3, 2, 1, 2, 1, 0, 0]


def local_dag(seed, levels=40, width=512, deg=6, span=12, int_weights=False):
    """Edges from level i to a window of `span` consecutive pins of level i+1
    (ids level-major), so a row's heads share intervals of 8."""
    rng = np.random.default_rng(seed)
    n = levels * width
    src, dst = [], []
    for lv in range(levels - 1):
        base = lv * width
        nxt = (lv + 1) * width
        for i in range(width):
            u = base + i
            off = rng.integers(0, width - span + 1)
            heads = nxt + off + rng.choice(span, size=min(deg, span), replace=False)
            src.extend([u] * len(heads))
            dst.extend(heads.tolist())
    src = np.asarray(src, np.int32)
    dst = np.asarray(dst, np.int32)
    if int_weights:
        w = rng.integers(1, 101, size=src.size).astype(np.float32)
    else:
        w = rng.uniform(0.1, 10.0, size=src.size).astype(np.float32)
    return n, src, dst, w


def to_csr(n, src, dst):
    order = np.argsort(src, kind="stable")
    adj = np.asarray(dst, np.int32)[order]
    adjp = np.zeros(n + 1, np.int64)
    np.add.at(adjp, np.asarray(src, np.int64) + 1, 1)
    return np.cumsum(adjp).astype(np.int32), adj
