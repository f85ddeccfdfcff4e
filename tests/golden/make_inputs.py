"""Extract the reference's own small benchmark graphs into npz fixtures.

Runs in the build container only (it reads the reference tree, which is not
present where the GPU tests run).  Each fixture keeps the edge list in the
row order the reference's read_input builds (edges grouped by tail vertex in
file order, gpucpg/gpucpg.cu:500-541), parsed by the oracle's restatement of
read_input.  Output: tests/golden/inputs/<name>.npz with n, src, dst, w.

    python tests/golden/make_inputs.py REFERENCE_DIR    (or CPG_REFERENCE=...)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

NAMES = ["simple", "dac21_paper_example", "tv80_unit_wgts"]


def main(ref):
    out = os.path.join(HERE, "inputs")
    os.makedirs(out, exist_ok=True)
    for name in NAMES:
        g = oracle.OracleGraph.from_text(os.path.join(ref, "benchmarks", name + ".txt"))
        adjp, adj, w = g.csr()
        src = np.repeat(np.arange(g.n, dtype=np.int32), np.diff(adjp))
        np.savez_compressed(os.path.join(out, name + ".npz"), n=np.int32(g.n), src=src,
                            dst=adj.astype(np.int32), w=w.astype(np.float32))
        print(name, g.n, adj.size)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CPG_REFERENCE")
    if not ref:
        sys.exit("usage: make_inputs.py REFERENCE_DIR (or set CPG_REFERENCE)")
    main(ref)
