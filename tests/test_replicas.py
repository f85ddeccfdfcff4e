"""The multi-GPU form is replicas only (the path has no exchange step): each
rank runs its own query and the ranks share only the timing maximum.  These
tests run that host logic as world-size-2 gloo process groups on the CPU."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup(n_gpus=0)
    assert dist.get_backend() == "gloo"
    # rank r took (r + 1) * 10 ms for its 1,000 paths: the job time is the max
    ms = bench.max_over_ranks(10.0 * (rank + 1), w)
    bench.barrier(w)
    out[rank] = bench.replica_value(1000, ms, w)
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks_gloo():
    world = 2
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
        vals = dict(out)
    # 2 ranks x 1,000 paths over the slower rank's 20 ms
    assert vals == {0: pytest.approx(100_000.0), 1: pytest.approx(100_000.0)}


def test_reference_arm_under_torchrun_prints_on_rank0_only():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "0", "--cpu-k", "500"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] >= 1
