"""Pin the full-size workloads to the CPU oracle: tests/golden/oracle_pins.npz.

Runs on the CPU only (the oracle, no GPU and no product library): for the
1,000,000-pin / 200-level workload with fp32 and integer delays (K = 1e6) and
the density sweep on the same generator (mean degree 10 / 30 / 40 / 50 at
K = 1e6 / 2e5 / 2e5 / 1e5), it builds the graph with the oracle's generator,
computes the suffix tree and the K cheapest paths with the oracle's
closure-at-split (IEEE division, every source seeded), and keeps, per prefix
P in {1e3, 1e4, 1e5, 1e6} up to K:

  p<P>_sha   sha256 of the float32 costs of the first P paths
  p<P>_sum   their float64 sum
  every100   every 100th cost of the whole answer
  head       the first 1,000 costs
  sfxt_sha_dist / _succ / _level   sha256 of the suffix-tree arrays

which pins every prefix bit for bit in a few KB.

    python tests/golden/make_oracle_pins.py [--only NAME,...]
"""
import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)
import cases  # noqa: E402
import oracle  # noqa: E402

PREFIXES = [1000, 10_000, 100_000, 1_000_000]
PINNED = ["large1m_f32", "large1m_int", *sorted(cases.SWEEP)]
OUT = os.path.join(HERE, "oracle_pins.npz")


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def pin(name: str) -> dict:
    c = cases.CASES[name]
    k = c["ks"][0]
    t0 = time.time()
    og = oracle.OracleGraph.from_edges(*oracle.generate(**c["gen"]))
    dist, succ, level = og.sfxt()
    t1 = time.time()
    nodes, split = og.closure_topk(k, ref_roots=False)
    t2 = time.time()
    costs = nodes["slack"].astype(np.float32)
    out = {f"{name}/k": np.int64(k), f"{name}/n_costs": np.int64(costs.size),
           f"{name}/split": np.float32(split),
           f"{name}/every100": costs[::100].copy(), f"{name}/head": costs[:1000].copy(),
           f"{name}/sfxt_sha_dist": np.array(sha(dist)),
           f"{name}/sfxt_sha_succ": np.array(sha(succ)),
           f"{name}/sfxt_sha_level": np.array(sha(level))}
    for p in PREFIXES:
        if p <= costs.size:
            out[f"{name}/p{p}_sha"] = np.array(sha(costs[:p]))
            out[f"{name}/p{p}_sum"] = np.float64(costs[:p].astype(np.float64).sum())
    print(f"{name}: n={og.n} k={k} paths={costs.size} split={split:.6f} "
          f"sfxt {t1 - t0:.1f}s closure {t2 - t1:.1f}s", flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    only = [x for x in a.only.split(",") if x] or PINNED
    data = dict(np.load(OUT)) if os.path.exists(OUT) else {}
    for name in only:
        data = {k: v for k, v in data.items() if not k.startswith(name + "/")}
        data.update(pin(name))
    np.savez_compressed(OUT, **data)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
