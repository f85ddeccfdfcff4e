"""Pack the reference's raw golden outputs into tests/golden/ref_goldens.npz.

Record of how the fixture was made: the reference library (gpucpg/gpucpg.cu,
compiled from its own sources with its own flags: --use_fast_math, RDC,
C++20) was linked to a small driver that called CpGen exactly as the
reference's golden writer does (examples/tc-pfxt-gate5.cu:15-44: reset(),
report_paths(k, 10, true, LEVELIZE_THEN_RELAX, SHORT_LONG, false, 0.005f,
5.0f, 8, false, false, false, true, CsrReorderMethod::NONE, false),
get_slacks(k), costs written with 9 significant digits) and dumped
dump_succ_dists / dump_sfxt_by_vertex.  It ran once on a B200.  The
reference finished simple, dac21_paper_example and tv80_unit_wgts (suffix
tree and costs) and the suffix tree of single20k_f32, then died with
cudaErrorIllegalAddress ("device free failed") in G-PathGen on single20k_f32
at K=10000.  The reference's GPU code is not run again, and the driver and
its runner are no longer part of the repository; this packer and the
fixture it wrote remain.

Input: a directory of raw outputs: <case>.sfxt.txt ("succ dist" per vertex)
and <case>.k<K>.txt (get_slacks(K), 9 significant digits).

Small cases keep full arrays.  Large cases keep, per prefix K in
{1e3, 1e4, 1e5, 1e6} that fits: the sha256 of the float32 costs of that
prefix, their float64 sum, and every 100th cost; plus the sha256 of the
suffix-tree arrays.  That keeps the fixture small while still pinning every
prefix bit for bit.

    python tests/golden/pack_goldens.py RAW_DIR
"""
import glob
import hashlib
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
import cases  # noqa: E402

PREFIXES = [1000, 10_000, 100_000, 1_000_000]
FULL_LIMIT = 20_000


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main(raw):
    out_path = os.path.join(HERE, "ref_goldens.npz")
    data = dict(np.load(out_path)) if os.path.exists(out_path) else {}
    for name, c in cases.CASES.items():
        sf = os.path.join(raw, name + ".sfxt.txt")
        if not os.path.exists(sf):
            continue
        arr = np.loadtxt(sf, dtype=np.int64, ndmin=2)
        succ = arr[:, 0].astype(np.int32)
        dist = arr[:, 1].astype(np.int64)
        dist = np.where(dist > 2**31 - 1, 2**31 - 1, dist).astype(np.int32)
        large = c.get("large", False)
        if large:
            data[f"{name}/sfxt_sha_dist"] = np.array(sha(dist))
            data[f"{name}/sfxt_sha_succ"] = np.array(sha(succ))
        else:
            data[f"{name}/sfxt_dist"] = dist
            data[f"{name}/sfxt_succ"] = succ
        for f in glob.glob(os.path.join(raw, name + ".k*.txt")):
            k = int(re.search(r"\.k(\d+)\.txt$", f).group(1))
            costs = np.loadtxt(f, dtype=np.float32, ndmin=1)
            data[f"{name}/k"] = np.int64(k)
            if costs.size <= FULL_LIMIT:
                data[f"{name}/costs"] = costs
            else:
                for p in PREFIXES:
                    if p <= costs.size:
                        data[f"{name}/p{p}_sha"] = np.array(sha(costs[:p]))
                        data[f"{name}/p{p}_sum"] = np.float64(costs[:p].astype(np.float64).sum())
                data[f"{name}/n_costs"] = np.int64(costs.size)
                data[f"{name}/every100"] = costs[::100].copy()
                data[f"{name}/head"] = costs[:FULL_LIMIT].copy()
        print(name, "packed")
    np.savez_compressed(out_path, **data)
    print("wrote", out_path, os.path.getsize(out_path), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: pack_goldens.py RAW_DIR")
    main(sys.argv[1])
