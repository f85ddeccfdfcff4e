"""Run the reference gpu-cpg's G-PathGen on every golden case (GPU box).

Needs oracle/_ref/ref_driver (the reference library built from its own
sources by `make -C oracle ref`).  For each case it writes the graph in the
reference's text format, then calls the driver in `sfxt` mode (per-vertex
successor and fixed-point distance) and `gpg` mode (the K smallest costs as
get_slacks returns them, 9 significant digits), and keeps the raw outputs in
OUT (default gpurun_out/goldens).  pack_goldens.py turns them into the
committed fixture tests/golden/ref_goldens.npz.

    python tests/golden/make_goldens.py [--large] [--sweep] [--only NAME,...]

Record: this script ran once on a B200.  The reference's G-PathGen finished
simple, dac21_paper_example and tv80_unit_wgts (suffix tree and costs) and the
suffix tree of single20k_f32, then died with cudaErrorIllegalAddress ("device
free failed") in G-PathGen on single20k_f32 at K=10000.  The reference's GPU
code is not run again on this pool, so the script now refuses to run unless
--i-know-the-reference-faulted is given.
"""
import argparse
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gpu-cpg_b200"))
sys.path.insert(0, HERE)
import cases  # noqa: E402
import cpg_b200  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "gpurun_out", "goldens"))
    ap.add_argument("--large", action="store_true")
    ap.add_argument("--sweep", action="store_true")
    ap.add_argument("--only", default="")
    ap.add_argument("--trials", type=int, default=1)
    ap.add_argument("--i-know-the-reference-faulted", action="store_true")
    a = ap.parse_args()
    if not a.i_know_the_reference_faulted:
        sys.exit("the reference G-PathGen faulted on single20k_f32; not running it again")
    os.makedirs(a.out, exist_ok=True)
    only = set(filter(None, a.only.split(",")))
    tmp = tempfile.mkdtemp(prefix="cpg_golden_")
    for name, c in cases.CASES.items():
        if only and name not in only:
            continue
        if not only:
            if c.get("sweep") and not a.sweep:
                continue
            if c.get("large") and not c.get("sweep") and not a.large:
                continue
        n, src, dst, w = cases.load_case(name)
        path = os.path.join(tmp, name + ".txt")
        cpg_b200.write_text(cpg_b200.Dag(n, src, dst, w), path) if n < 200000 else _fast_text(c, path)
        log = open(os.path.join(a.out, name + ".log"), "w")
        t0 = time.time()
        subprocess.run([DRIVER, "sfxt", path, os.path.join(a.out, name + ".sfxt.txt")],
                       check=True, stdout=log, stderr=subprocess.STDOUT)
        for k in c["ks"]:
            subprocess.run([DRIVER, "gpg", path, str(k),
                            os.path.join(a.out, f"{name}.k{k}.txt"), str(a.trials)],
                           check=True, stdout=log, stderr=subprocess.STDOUT)
        print(f"{name}: n={n} m={src.size} done in {time.time() - t0:.1f}s", flush=True)
        os.remove(path)


def _fast_text(c, path):
    cpg_b200.generate(cpg_b200.gen_params(**c["gen"]), text_path=path)


if __name__ == "__main__":
    main()
