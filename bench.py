#!/usr/bin/env python3
"""Benchmark: K-paths/sec of the plain single-query critical-path generator.

Workload: the seeded levelised timing DAG with 1,000,000 pins in 200 levels,
geometric out-degree of mean 20 (capped at 256, level span 4, 2,000 sources and
2,000 sinks behind a virtual super-source/super-sink), fp32 delays uniform in
[0.1, 10.0]; one query reports the K = 1,000,000 cheapest paths.

A step is one full query on the device-resident graph: suffix tree (levelise,
relax, successors, deviation heaps) + prefix-tree enumeration + top-K select
and sort.  `value` is K / step time with the graph resident in HBM; `e2e` is
the same query through the C ABI from pinned host buffers, each step's CSR
upload, query and cost download inside the timed region: steps streamed
through two handles on two host threads, so that one step's upload overlaps
the previous step's query (`e2e.serial`: one handle, each step in turn).

The same JSON line carries the rest of the metric, measured in the same run
on the same GPU (N = 1 only): `batched` (256 queries in one captured launch
against plain per-graph handles), `served` (the 5,000-query Poisson stream:
open-loop p50/p99 and saturation capacity, each against plain), `density`
(mean degree 10/30/40/50) and `config1` (the 20,000-pin query at K = 1,000
beside the CPU port of the reference's SEQUENTIAL path).  --plain-only skips
them.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank runs an independent replica of the query on
its own GPU (replicas only: the path has no exchange step); value = all
ranks' paths / max-over-ranks time.

--impl reference times the reference's CPU implementation of the path (the
oracle port of its SEQUENTIAL heap; the reference's GPU code is not run,
because its G-PathGen faulted on this hardware) on the same workload at a
bounded K, without loading the product library.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _sub in ("gpu-cpg_b200", os.path.join("tests", "golden")):
    _p = os.path.join(ROOT, _sub)
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

WORKLOAD = "large1m_f32"
WORKLOAD_DESC = ("levelised DAG, 1,000,000 pins / 200 levels, geometric out-degree mean 20 "
                 "(cap 256), fp32 delays U[0.1,10], 2,000 sources / 2,000 sinks, K=1e6")
METRIC = "K-paths/sec"
# DRAM bytes (read + write) per query of the dominant kernels on this
# workload, from the one-pass ncu capture summarised in
# profiles/sfxt_dataflow_kernel_large400k.md (the suffix-tree build does not
# depend on K; the engine's figure is its two launches at K = 1e6).
KERNEL_TRAFFIC = {"sfxt_dataflow_kernel": 708_980_736 + 625_738_752,
                  "engine_kernel": 757_760 + 102_573_056 + 188_904_960}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML (read-only
    queries) every 2 ms during the timed region, so even a timed region of a
    few tens of milliseconds holds samples; nvidia-smi at 200 ms when the NVML
    bindings are missing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []  # (sm_mhz, max_mhz, set of reason names)
        self.proc = None
        self.thread = None
        self.nvml = None
        self.stop_flag = threading.Event()

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _nvml_sample(self):
        nv, h = self.nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        masks = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                 nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        self.rows.append((float(sm), float(mx),
                          {n for n, m in zip(self.NAMES, masks) if bits & m}))

    def _nvml_loop(self):
        while not self.stop_flag.wait(0.002):
            try:
                self._nvml_sample()
            except Exception:
                return

    def start(self):
        try:
            self.nvml = self._nvml_handle()
            self._nvml_sample()
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            if len(r) >= 9 and r[1].replace(".", "").isdigit():
                self.rows.append((float(r[1]), float(r[2]) if r[2].replace(".", "").isdigit()
                                  else float("nan"),
                                  {n for n, v in zip(self.NAMES, r[5:9]) if v.lower() == "active"}))

    def stop(self):
        if self.nvml is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            try:
                self._nvml_sample()
            except Exception:
                pass
            source = "nvml, 2 ms"
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.thread:
                self.thread.join(timeout=5)
            source = "nvidia-smi, 200 ms"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        sm = [r[0] for r in self.rows]
        mx = [r[1] for r in self.rows if r[1] == r[1]]
        reasons = set().union(*[r[2] for r in self.rows]) if self.rows else set()
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows), "source": source}


def ranks():
    """(world, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def dist_setup(n_gpus):
    """Process group for N > 1 replicas: NCCL between GPUs, gloo without a
    GPU (the host-side logic is exercised that way).  The replicas exchange
    only the timing maximum and barriers; the path itself has no exchange."""
    world, rank, local = ranks()
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if (n_gpus > 0 and torch.cuda.is_available()) else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def max_over_ranks(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = device if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(paths_per_rank, ms_max, world):
    """Whole-job K-paths/sec of N independent replicas: every rank's paths
    over the slowest rank's time."""
    return world * paths_per_rank / (ms_max / 1000.0)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_reference(k_sample, dag=None, name=WORKLOAD):
    """The reference's CPU path restated (oracle port): the SEQUENTIAL
    priority-queue enumeration (gpucpg.cu:21230-21300) on one host thread,
    timed alone as the reference's expand_time times it; the CPU suffix tree
    it needs (the reference builds that on the GPU) is timed separately.
    The graph comes from the oracle's generator unless one is given, so this
    leg never loads the product library.  Returns (paths, heap seconds,
    suffix-tree seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import cases
    if dag is None:
        n, src, dst, w = oracle.generate(**cases.CASES[name]["gen"])
    else:
        n, src, dst, w = dag.n, dag.src, dag.dst, dag.w
    og = oracle.OracleGraph.from_edges(n, src, dst, w)
    t0 = time.perf_counter()
    og.sfxt()
    t1 = time.perf_counter()
    out = og.sequential(k_sample)
    t2 = time.perf_counter()
    return len(out), t2 - t1, t1 - t0


def run_reference(args):
    # rank 0 alone times the reference's CPU path; the other ranks exit
    # without work (no process group is needed for that)
    world, rank, _ = ranks()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import cases
    k_sample = args.cpu_k
    n, src, dst, w = oracle.generate(**cases.CASES[WORKLOAD]["gen"])
    og = oracle.OracleGraph.from_edges(n, src, dst, w)
    t0 = time.perf_counter()
    og.sfxt()
    sfxt_s = time.perf_counter() - t0
    vals, got = [], 0
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        got = og.sequential(k_sample).size
        sec = time.perf_counter() - t0
        if i >= args.warmup:
            vals.append(got / sec)
    v = float(np.median(vals))
    sample = (f"oracle port of the reference CPU path: the SEQUENTIAL heap (gpucpg.cu:21230-"
              f"21300) on one host thread, timed alone as expand_time is, on the same graph at "
              f"K={k_sample} (the full K=1e6 would take about 2e9 heap pushes); its CPU suffix "
              f"tree, which the reference builds on the GPU, took {sfxt_s:.2f} s and is not in "
              f"the value")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "paths/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * got / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "desc": WORKLOAD_DESC, "k": args.k,
                   "sample_k": k_sample, "paths_per_step": got},
        "cpu_baseline": {"value": v, "unit": "paths/s", "cores": 1, "kind": "port",
                         "sample": sample, "sfxt_s": sfxt_s},
        "e2e": {"value": v, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    world, rank, local = dist_setup(args.gpus)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    import cpg_b200
    import cases

    c = cases.CASES[WORKLOAD]
    dag = cpg_b200.generate(cpg_b200.gen_params(**c["gen"]))
    K = args.k
    stream = torch.cuda.Stream(device=device)
    g = cpg_b200.CpGen(device=local, stream=stream.cuda_stream)
    g.load_dag(dag)
    adjp, adj, w = g.get_csr()
    N, M = g.num_verts(), g.num_edges()

    def step():
        g.levelize()
        g.report_paths(K)

    for _ in range(args.warmup):
        step()
    st0 = g.stats()
    # ---- device-resident timed region
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    sfxt_ms, sfxt_k_ms, pfxt_ms, sel_ms, launches = [], [], [], [], 0
    ev0.record(stream)
    for _ in range(args.steps):
        step()
        s = g.stats()
        sfxt_ms.append(s["sfxt_ms"])
        sfxt_k_ms.append(s["sfxt_kernel_ms"])
        pfxt_ms.append(s["pfxt_ms"])
        sel_ms.append(s["select_ms"])
        launches += s["kernel_launches"]
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(ms, world, device)
    n_out = int(g.get_slacks(K).size)
    value = replica_value(n_out, ms, world)
    stats = g.stats()

    # ---- end-to-end through the C ABI from pinned host buffers: every step
    # uploads the CSR (the library builds the device graph from it), answers
    # the query and reads the K costs back into host memory
    def pinned(a):
        t = torch.empty(a.size, dtype={np.int32: torch.int32, np.float32: torch.float32}[a.dtype.type],
                        pin_memory=True)
        t.numpy()[:] = a
        return t, t.numpy()
    keep = [pinned(adjp), pinned(adj), pinned(w), pinned(np.zeros(K, np.float32))]
    p_adjp, p_adj, p_w, costs_host = (x[1] for x in keep)
    e2e_ms = []
    for i in range(max(1, args.steps)):
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.load_csr(N, p_adjp, p_adj, p_w)
        g.report_paths(K)
        got = g.get_slacks(K, out=costs_host)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    e2e = max_over_ranks(float(np.median(e2e_ms)), world, device)
    h2d = adjp.nbytes + adj.nbytes + w.nbytes  # the CSR handed to cpg_load_csr
    d2h = 4 * int(got.size)
    serial_costs = np.array(got, copy=True)

    # ---- the same steps streamed through two handles, one host thread each
    # (one handle per thread is the library's threading model): while one
    # handle answers its query, the other's CSR upload is in flight.  Every
    # step still uploads its CSR from pinned host memory and reads its K
    # costs back; a lock keeps the queries themselves one at a time, so the
    # persistent kernels never share the GPU.
    stream2 = torch.cuda.Stream(device=device)
    g2 = cpg_b200.CpGen(device=local, stream=stream2.cuda_stream)
    keep.append(pinned(np.zeros(K, np.float32)))
    costs_host2 = keep[-1][1]
    g2.load_csr(N, p_adjp, p_adj, p_w)  # sizes its device buffers (untimed)
    g2.report_paths(K)
    n_pipe = max(2, args.steps)          # steps per handle
    lock = threading.Lock()
    fails = []

    def stream_queries(h, out):
        try:
            for _ in range(n_pipe):
                h.load_csr(N, p_adjp, p_adj, p_w)
                with lock:
                    h.report_paths(K)
                if h.get_slacks(K, out=out).size != n_out:
                    raise RuntimeError("pipelined query returned a different path count")
        except Exception as ex:  # reported after the join
            fails.append(ex)

    barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    workers = [threading.Thread(target=stream_queries, args=a)
               for a in ((g, costs_host), (g2, costs_host2))]
    for t in workers:
        t.start()
    for t in workers:
        t.join()
    # every call above returns after its device work, so e1 runs at the join
    e1.record(stream)
    torch.cuda.synchronize()
    if fails:
        raise fails[0]
    for out in (costs_host, costs_host2):
        if not np.array_equal(out[:n_out].view(np.uint32), serial_costs.view(np.uint32)):
            raise RuntimeError("pipelined costs differ from the serial step's")
    e2e_pipe = max_over_ranks(e0.elapsed_time(e1) / (2 * n_pipe), world, device)
    g2.close()

    # ---- roofline of the dominant kernel
    hbm, src = peaks()
    sfxt = float(np.mean(sfxt_ms))
    sfxt_k = float(np.mean(sfxt_k_ms))
    pfxt = float(np.mean(pfxt_ms))
    sel = float(np.mean(sel_ms))
    b_sfxt = 36 * M + 32 * N            # algorithmic bytes of one suffix-tree build
    acc = stats["paths_accepted"]
    items = stats["items_generated"]
    b_pfxt = 16 * acc + 20 * acc + 16 * items + 36 * items
    # the dominant kernel's average launch, timed with CUDA events on the
    # handle's stream around that launch alone; both kernels are listed
    per_kernel = {
        "sfxt_dataflow_kernel": {"kernel_ms": sfxt_k, "algorithmic_bytes": b_sfxt,
                                 "achieved": b_sfxt / (sfxt_k * 1e-3) / 1e9},
        "engine_kernel": {"kernel_ms": pfxt, "algorithmic_bytes": b_pfxt,
                          "achieved": b_pfxt / (pfxt * 1e-3) / 1e9},
    }
    for name_k, r in per_kernel.items():
        r["frac"] = r["achieved"] / hbm
        r["traffic"] = KERNEL_TRAFFIC.get(name_k)
    kern = "sfxt_dataflow_kernel" if sfxt_k >= pfxt else "engine_kernel"
    ach, k_ms = per_kernel[kern]["achieved"], per_kernel[kern]["kernel_ms"]
    traffic = KERNEL_TRAFFIC.get(kern)

    line = {
        "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "desc": WORKLOAD_DESC, "k": K, "n": N, "m": M,
                   "paths_returned": n_out, "l2": "inputs larger than L2 (CSR 240 MB, "
                   "deviations 320 MB > 126 MB)", "sfxt": "recomputed every step",
                   "parallelism": f"replicas x{world}"},
        "breakdown_ms": {"sfxt": sfxt, "pfxt": pfxt, "select_sort": sel,
                         "phases": stats["phases"], "rounds": stats["rounds"],
                         "paths_accepted": acc, "items_generated": items,
                         "engine_stages": dict(zip(
                             ["seed", "decide", "select", "promote", "closure", "out_select",
                              "out_sort", "emit"], stats["engine_stage_ms"]))},
        "roofline": {"bound": "hbm", "kernel": kern, "achieved": ach, "peak": hbm,
                     "peak_source": src, "unit": "GB/s", "frac": ach / hbm,
                     "traffic": traffic, "kernel_ms": k_ms,
                     "algorithmic_bytes": per_kernel[kern]["algorithmic_bytes"],
                     "kernels": per_kernel},
        "e2e": {"value": replica_value(n_out, e2e_pipe, world), "unit": "paths/s",
                "ms_per_step": e2e_pipe, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": d2h,
                "mode": "steps streamed through two handles on two host threads: one step's "
                        "CSR upload overlaps the previous step's query",
                "serial": {"value": replica_value(n_out, e2e, world), "ms_per_step": e2e,
                           "mode": "one handle, each step's upload, query and read-back in turn"}},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nk, sec, sfxt_s = cpu_reference(args.cpu_k, dag)
        line["cpu_baseline"] = {
            "value": nk / sec, "unit": "paths/s", "cores": 1, "kind": "port",
            "sample": f"oracle port of the reference CPU path: SEQUENTIAL heap alone (as "
                      f"expand_time), one host thread, same graph, K={args.cpu_k}, {sec:.2f} s; "
                      f"CPU suffix tree {sfxt_s:.2f} s, not in the value",
            "sfxt_s": sfxt_s}
    g.close()
    if world == 1 and not args.plain_only:
        # the rest of the metric, measured in the same run on the same GPU:
        # batched and served forms against plain, the density sweep, and the
        # 20,000-pin query the reference's CPU path runs in full
        line["batched"] = batched_record(steps=5, warmup=2, autotune=args.autotune)
        line["served"] = served_record(args.served_queries)
        line["density"] = density_record(steps=3, warmup=2)
        line["config1"] = config1_record(steps=20, warmup=3, cpu=not args.no_cpu_baseline)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------- batched form
BATCH_DESC = ("256 seeded DAGs, pins log-uniform 5,000-200,000, levels U{40..150}, geometric "
              "out-degree mean U[2,8] (cap 64), fp32 delays U[0.1,10], K log-uniform 100-100,000")


def batch_workload(seed=4, count=256):
    """The batched-form workload: graph generator settings and K per query."""
    import cpg_b200
    rng = np.random.default_rng(seed)
    dags, ks = [], []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(5_000), np.log(200_000))))
        levels = int(rng.integers(40, 151))
        side = max(8, n // (2 * levels))
        p = cpg_b200.gen_params(seed=seed * 100_000 + i, n_pins=n, n_levels=levels,
                                n_first=side, n_last=side, level_span=3, degree_kind=1,
                                deg_mean=float(rng.uniform(2.0, 8.0)), deg_cap=64,
                                weight_kind=0, w_lo=0.1, w_hi=10.0)
        dags.append(cpg_b200.generate(p))
        ks.append(int(np.exp(rng.uniform(np.log(100), np.log(100_000)))))
    return dags, ks


def batched_record(steps, warmup, autotune=True):
    """K-paths/sec of the batched form (one captured step answers all 256
    queries, suffix trees rebuilt each step) against the plain form answering
    the same queries one at a time on resident graphs."""
    import torch
    import cpg_b200
    dags, ks = batch_workload()
    stream = torch.cuda.Stream()
    with cpg_b200.Batch(stream=stream.cuda_stream) as b:
        for d in dags:
            b.add_dag(d)
        b.commit()
        b.set_queries(list(range(len(dags))), ks)
        b.run(True)
        if autotune:
            b.autotune()
        for _ in range(warmup):
            b.run(True)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            b.run(True)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        total = sum(int(b.costs(q).size) for q in range(len(ks)))
        st = b.stats()
    # plain form: the same queries one at a time (graphs resident, suffix
    # tree rebuilt per query as in report_paths)
    handles = []
    for d in dags:
        g = cpg_b200.CpGen(stream=stream.cuda_stream)
        g.load_dag(d)
        handles.append(g)
    for g, k in zip(handles, ks):
        g.levelize()
        g.report_paths(k)
    torch.cuda.synchronize()
    e0.record(stream)
    for g, k in zip(handles, ks):
        g.levelize()
        g.report_paths(k)
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1)
    for g in handles:
        g.close()
    return {
        "form": "batched", "metric": METRIC, "value": total / (ms / 1e3), "unit": "paths/s",
        "n_gpus": 1, "steps": steps, "warmup": warmup, "ms_per_step": ms,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batch256", "desc": BATCH_DESC, "queries": len(ks),
                   "paths_returned": total, "pins": int(sum(d.n for d in dags)),
                   "edges": int(sum(d.m for d in dags))},
        "plain_sequential": {"value": total / (plain_ms / 1e3), "unit": "paths/s",
                             "ms": plain_ms},
        "speedup_vs_plain": plain_ms / ms,
        "autotune": {"ran": bool(autotune),
                     "choice": {k: st[k] for k in ("sfxt_mode", "frontier_used",
                                                   "select_schedule", "sfxt_ctas_per_sm",
                                                   "engine_ctas_per_sm") if k in st}},
        "batch_stats": st,
    }


def run_batched(args):
    print(json.dumps(batched_record(args.steps, args.warmup, args.autotune)), flush=True)


# ---------------------------------------------------------------- served form
SERVED_DESC = ("open-loop Poisson stream of 5,000 queries at 500/s over 32 resident graphs from the "
               "batched-form generator, K log-uniform 100-100,000, 20% re-ask with 1% of the "
               "graph's delays re-sampled; HBM admission budget 150 GB")


def served_stream(n_graphs, sizes, count=5000, rate=500.0, seed=9):
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    t = np.cumsum(gaps)
    qs = []
    for i in range(count):
        g = int(rng.integers(n_graphs))
        k = int(np.exp(rng.uniform(np.log(100), np.log(100_000))))
        upd = None
        if rng.random() < 0.2:
            m = sizes[g]
            e = rng.choice(m, size=max(1, m // 100), replace=False).astype(np.int32)
            upd = (e, rng.uniform(0.1, 10.0, size=e.size).astype(np.float32))
        qs.append((float(t[i]), g, k, upd))
    return qs


def _serve_replay(dags, qs, open_loop=True, max_batch=256):
    """The served form: submit at the stream's arrival times (open loop) or
    all at once (saturation), then collect every result."""
    import cpg_b200
    with cpg_b200.Server(max_batch=max_batch, hbm_budget_bytes=150 << 30) as s:
        for d in dags:
            s.add_dag(d)
        s.start()
        t0 = time.perf_counter()
        tickets = []
        for at, g, k, upd in qs:
            delay = at - (time.perf_counter() - t0)
            if open_loop and delay > 0:
                time.sleep(delay)
            tickets.append(s.submit(g, k, *(upd if upd else (None, None))))
        for tk in tickets:
            s.wait(tk, timeout_ms=600000)
        st = s.stats()
        s.stop()
    return st


def _plain_replay(dags, qs, open_loop=True):
    """The plain form on the same stream: one resident handle per graph, one
    query at a time in arrival order (update delays, report_paths, read the
    costs back).  Latency is arrival to result, as for the server."""
    import cpg_b200
    handles = []
    for d in dags:
        h = cpg_b200.CpGen()
        h.load_dag(d)
        h.levelize()
        handles.append(h)
    lat, paths = [], 0
    t0 = time.perf_counter()
    done = 0.0
    for at, g, k, upd in qs:
        arrive = at if open_loop else 0.0
        delay = arrive - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        h = handles[g]
        if upd is not None:
            h.update_delays(*upd)
        h.report_paths(k)
        paths += int(h.get_slacks(k).size)
        done = time.perf_counter() - t0
        lat.append((done - arrive) * 1e3)
    for h in handles:
        h.close()
    lat = np.sort(np.asarray(lat))
    first = qs[0][0] if open_loop else 0.0
    wall = done - first
    pick = lambda f: float(lat[min(lat.size - 1, int(np.ceil(f * lat.size)) - 1)])
    return {"completed": len(qs), "paths": paths, "p50_ms": pick(0.50), "p99_ms": pick(0.99),
            "mean_ms": float(lat.mean()), "max_ms": float(lat[-1]), "wall_s": wall,
            "paths_per_s": paths / wall}


def served_record(n_queries):
    """The served form on the config-5 stream: open-loop Poisson arrivals
    (latency) and the same queries submitted at once (capacity), each beside
    the plain form answering the stream one query at a time."""
    dags, _ = batch_workload(seed=5, count=32)
    qs = served_stream(len(dags), [d.m for d in dags], count=n_queries)
    served = _serve_replay(dags, qs, open_loop=True)
    plain = _plain_replay(dags, qs, open_loop=True)
    served_sat = _serve_replay(dags, qs, open_loop=False)
    plain_sat = _plain_replay(dags, qs, open_loop=False)
    return {
        "form": "served", "metric": METRIC, "value": served["paths_per_s"], "unit": "paths/s",
        "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "served5000", "desc": SERVED_DESC, "queries": len(qs),
                   "graphs": len(dags)},
        "p50_ms": served["p50_ms"], "p99_ms": served["p99_ms"],
        "served": served,
        "plain_sequential": {"value": plain["paths_per_s"], "p50_ms": plain["p50_ms"],
                             "p99_ms": plain["p99_ms"], "stats": plain},
        "speedup_vs_plain": served["paths_per_s"] / max(plain["paths_per_s"], 1e-9),
        # the same queries submitted at once: the largest K-paths/sec each
        # form sustains on this mix (the open-loop arrival rate caps the above)
        "capacity": {"served": served_sat["paths_per_s"], "plain": plain_sat["paths_per_s"],
                     "speedup_vs_plain": served_sat["paths_per_s"] /
                     max(plain_sat["paths_per_s"], 1e-9),
                     "served_p50_ms": served_sat["p50_ms"], "served_p99_ms": served_sat["p99_ms"],
                     "plain_p50_ms": plain_sat["p50_ms"], "plain_p99_ms": plain_sat["p99_ms"],
                     "served_stats": served_sat, "plain_stats": plain_sat},
    }


def run_served(args):
    print(json.dumps(served_record(args.served_queries)), flush=True)


# ---------------------------------------------------------------- density sweep
def density_record(steps, warmup):
    """The density sweep on the 1M-pin generator (mean degree 10 / 30 / 40 /
    50 at K = 1e6 / 2e5 / 2e5 / 1e5): K-paths/sec per degree with the
    suffix tree rebuilt each query, and the split into suffix tree and
    engine."""
    import torch
    import cpg_b200
    import cases
    hbm, _ = peaks()
    out = {}
    for name in sorted(cases.SWEEP, key=lambda x: cases.SWEEP[x][0]):
        deg, k = cases.SWEEP[name]
        dag = cpg_b200.generate(cpg_b200.gen_params(**cases.CASES[name]["gen"]))
        stream = torch.cuda.Stream()
        with cpg_b200.CpGen(stream=stream.cuda_stream) as g:
            g.load_dag(dag)
            n, m = g.num_verts(), g.num_edges()
            for _ in range(warmup):
                g.levelize()
                g.report_paths(k)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            sf, sfk, pf = [], [], []
            e0.record(stream)
            for _ in range(steps):
                g.levelize()
                g.report_paths(k)
                st = g.stats()
                sf.append(st["sfxt_ms"])
                sfk.append(st["sfxt_kernel_ms"])
                pf.append(st["pfxt_ms"])
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            got = int(g.get_slacks(k).size)
            st = g.stats()
        sfk_ms = float(np.mean(sfk))
        out[name] = {
            "mean_degree": deg, "k": k, "n": n, "m": m, "paths_returned": got,
            "value": got / (ms / 1e3), "unit": "paths/s", "ms_per_query": ms,
            "sfxt_ms": float(np.mean(sf)), "engine_ms": float(np.mean(pf)),
            "paths_accepted": st["paths_accepted"], "items_generated": st["items_generated"],
            "phases": st["phases"], "rounds": st["rounds"],
            "sfxt_kernel_ms": sfk_ms,
            "sfxt_frac_of_hbm": (36 * m + 32 * n) / (sfk_ms * 1e-3) / 1e9 / hbm,
        }
        del dag
    return {"config": "density sweep, 1,000,000 pins / 200 levels, fp32 delays U[0.1,10]",
            "steps": steps, "warmup": warmup, "graphs": out}


# ---------------------------------------------------------------- config 1
def config1_record(steps, warmup, cpu=True):
    """The 20,000-pin / 60-level single query at K = 1,000 (the workload the
    reference's CPU path runs in full): the GPU plain form beside the CPU port
    of the reference's SEQUENTIAL heap on the same graph."""
    import torch
    import cpg_b200
    import cases
    name, k = "single20k_f32", 1000
    dag = cpg_b200.generate(cpg_b200.gen_params(**cases.CASES[name]["gen"]))
    stream = torch.cuda.Stream()
    with cpg_b200.CpGen(stream=stream.cuda_stream) as g:
        g.load_dag(dag)
        for _ in range(warmup):
            g.levelize()
            g.report_paths(k)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            g.levelize()
            g.report_paths(k)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        got = int(g.get_slacks(k).size)
        st = g.stats()
    rec = {"workload": name, "desc": "20,000 pins / 60 levels, out-degree U{1..4}, fp32 delays "
                                     "U[0.1,10], 64 sources / 64 sinks, K=1,000",
           "k": k, "paths_returned": got, "value": got / (ms / 1e3), "unit": "paths/s",
           "ms_per_query": ms, "sfxt_ms": st["sfxt_ms"], "engine_ms": st["pfxt_ms"],
           "steps": steps, "warmup": warmup}
    if cpu:
        reps, secs, nk, sfxt_s = 20, [], 0, 0.0
        for _ in range(reps):
            nk, sec, sfxt_s = cpu_reference(k, dag)
            secs.append(sec)
        sec = float(np.median(secs))
        rec["cpu_baseline"] = {"value": nk / sec, "unit": "paths/s", "cores": 1, "kind": "port",
                               "sample": f"SEQUENTIAL heap alone, one host thread, K={k}, median "
                                         f"of {reps} runs ({sec * 1e3:.2f} ms); CPU suffix tree "
                                         f"{sfxt_s * 1e3:.2f} ms, not in the value"}
    return rec


# ---------------------------------------------------------------- BVSS
def local_dag_np(seed, levels, width, deg, span):
    """A levelised DAG whose rows put `deg` heads in a window of `span`
    consecutive pins of the next level (dense BVSS slices), vectorised."""
    rng = np.random.default_rng(seed)
    n = levels * width
    src, dst = [], []
    for lv in range(levels - 1):
        off = rng.integers(0, width - span + 1, size=width)
        pick = np.argsort(rng.random((width, span)), axis=1)[:, :deg]
        src.append(np.repeat(np.arange(lv * width, (lv + 1) * width, dtype=np.int32), deg))
        dst.append(((lv + 1) * width + off[:, None] + pick).astype(np.int32).ravel())
    src = np.concatenate(src)
    dst = np.concatenate(dst)
    w = rng.uniform(0.1, 10.0, size=src.size).astype(np.float32)
    return n, src, dst, w


def _csr_np(n, src, dst):
    order = np.argsort(src, kind="stable")
    adjp = np.zeros(n + 1, np.int64)
    np.add.at(adjp, src.astype(np.int64) + 1, 1)
    return np.cumsum(adjp).astype(np.int32), dst[order].astype(np.int32)


def run_bvss(args):
    """BVSS pull BFS levels (tensor-core tiles vs scalar popc) and the suffix
    tree with the BVSS pull against the CSR push, on the sparse 1M-pin
    workload and on a dense level-local graph of the same size."""
    import cpg_b200
    import cases
    out = {"form": "bvss", "graphs": {}}
    graphs = {}
    if args.bvss_graphs in ("both", "sparse"):
        c = cases.CASES[WORKLOAD]
        dag = cpg_b200.generate(cpg_b200.gen_params(**c["gen"]))
        graphs["large1m_f32 (sparse slices)"] = (dag.n, dag.src, dag.dst, dag.w)
    if args.bvss_graphs in ("both", "dense"):
        graphs["local1m (dense slices: 16 heads in a 24-pin window, 200 x 5000 pins)"] = \
            local_dag_np(3, 200, 5000, 16, 24)
    for name, (n, src, dst, w) in graphs.items():
        adjp, adj = _csr_np(n, src, dst)
        b = cpg_b200.Bvss(n, adjp, adj)
        info = b.info()
        g = {"n": int(n), "m": int(src.size), "n_vss": info["n_vss"],
             "bits_per_slice": info["total_set_bits"] / max(info["unpadded_slices"], 1),
             "levels": {}}
        sinks = np.nonzero(np.diff(adjp) == 0)[0].astype(np.int32)
        ref = None
        for tname, tiles in (("tensor", cpg_b200.TILES_TENSOR), ("scalar", cpg_b200.TILES_SCALAR),
                             ("density", cpg_b200.TILES_DENSITY)):
            times = []
            for _ in range(args.warmup + args.steps):
                lv, st = b.levels(sinks, tiles=tiles)
                times.append(st["device_ms"])
            if ref is None:
                ref = lv
            assert np.array_equal(lv, ref)
            ms = float(np.median(times[args.warmup:]))
            # slice bytes pulled: 128 B masks + 512 B rows + 1 B count per VSS
            # tile, plus the 4 B level write per row
            tiles_done = st["tiles_tensor"] + st["tiles_scalar"]
            g["levels"][tname] = {"ms": ms, "bfs_levels": st["levels"],
                                  "tiles_tensor": st["tiles_tensor"],
                                  "tiles_scalar": st["tiles_scalar"], "mma": st["mma_issued"],
                                  "slice_gbs": (641 * tiles_done + 4 * n) / (ms * 1e-3) / 1e9,
                                  "b1_tops": st["mma_issued"] * 2 * 8 * 8 * 128 / (ms * 1e-3) / 1e12}
        b.close()
        sf = {}
        for fname, fr in (("csr_push", cpg_b200.FRONTIER_CSR), ("bvss_pull", cpg_b200.FRONTIER_BVSS)):
            with cpg_b200.CpGen(frontier=fr) as h:
                h.load_edges(n, src, dst, w)
                times = []
                for _ in range(args.warmup + args.steps):
                    h.levelize()  # a full build every time
                    times.append(h.stats()["sfxt_ms"])
                st = h.stats()
                sf[fname] = {"ms": float(np.median(times[args.warmup:])),
                             "frontier_used": st["frontier_used"],
                             "tiles_tensor": st["bvss_tiles_tensor"],
                             "tiles_scalar": st["bvss_tiles_scalar"]}
        g["sfxt"] = sf
        out["graphs"][name] = g
    print(json.dumps(out), flush=True)


def run_ingest(args):
    """Graph ingestion on the 1M-pin workload: the text file parsed on the host
    threads, read_input to a device graph, the binary CSR file to a device
    graph, and the oracle's sequential text parser beside them."""
    import tempfile
    import cpg_b200
    import cases
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    c = cases.CASES[WORKLOAD]
    with tempfile.TemporaryDirectory() as tmp:
        txt, binp = os.path.join(tmp, "g.txt"), os.path.join(tmp, "g.bin")
        dag = cpg_b200.generate(cpg_b200.gen_params(**c["gen"]), text_path=txt, csr_bin_path=binp)
        out = {"form": "ingest", "workload": WORKLOAD, "n": dag.n, "m": dag.m,
               "text_bytes": os.path.getsize(txt), "bin_bytes": os.path.getsize(binp),
               "host_threads": os.cpu_count()}

        def timed(fn):
            ts = []
            for _ in range(args.warmup + args.steps):
                t0 = time.perf_counter()
                fn()
                ts.append(time.perf_counter() - t0)
            return float(np.median(ts[args.warmup:]))

        t = timed(lambda: cpg_b200.read_text(txt))
        out["text_parse"] = {"s": t, "medges_per_s": dag.m / t / 1e6}
        with cpg_b200.CpGen() as g:
            def load_text():
                g.read_input(txt)
                g.sync()

            def load_bin():
                g.load_csr_bin(binp)
                g.sync()
            t = timed(load_text)
            out["read_input_to_device"] = {"s": t, "medges_per_s": dag.m / t / 1e6}
            t = timed(load_bin)
            out["csr_bin_to_device"] = {"s": t, "medges_per_s": dag.m / t / 1e6,
                                        "gb_per_s": out["bin_bytes"] / t / 1e9}
        t0 = time.perf_counter()
        oracle.OracleGraph.from_text(txt)
        t = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": dag.m / t / 1e6, "unit": "M edges/s", "cores": 1,
                               "kind": "port", "sample": "the whole text file, once",
                               "s": t}
    print(json.dumps(out), flush=True)


def run_profile_case(args):
    """A short fixed sequence for ncu: one warm-up query, then one query
    (suffix tree + engine) on the same workload at --k.  --profile-pins N
    scales the workload's generator down to N pins (same levels, degree and
    delays; sources and sinks in proportion), for captures that must stay
    small; --form batched runs one warm-up and one measured batched step;
    --form e2e runs two end-to-end steps (CSR upload from pinned host buffers,
    query, cost read-back), the first a warm-up."""
    import cpg_b200
    import cases
    if args.form == "e2e":
        import torch
        c = cases.CASES[WORKLOAD]
        dag = cpg_b200.generate(cpg_b200.gen_params(**c["gen"]))
        with cpg_b200.CpGen() as g:
            g.load_dag(dag)
            adjp, adj, w = g.get_csr()
            n = g.num_verts()
            keep = []
            for a in (adjp, adj, w, np.zeros(args.k, np.float32)):
                t = torch.empty(a.size, dtype={np.int32: torch.int32,
                                               np.float32: torch.float32}[a.dtype.type],
                                pin_memory=True)
                t.numpy()[:] = a
                keep.append(t)
            p_adjp, p_adj, p_w, out = (t.numpy() for t in keep)
            for _ in range(2):
                g.load_csr(n, p_adjp, p_adj, p_w)
                g.report_paths(args.k)
                g.get_slacks(args.k, out=out)
            print(json.dumps({"profile_case": "e2e", "n": n, "m": int(adj.size), "k": args.k,
                              **g.stats()}))
        return
    if args.form == "batched":
        # the batch with the level-synchronous build, the autotuner's pick
        dags, ks = batch_workload()
        with cpg_b200.Batch(sfxt_level_sync=True) as b:
            for d in dags:
                b.add_dag(d)
            b.commit()
            b.set_queries(list(range(len(dags))), ks)
            for _ in range(2):
                b.run(True)
            print(json.dumps({"profile_case": "batch256", **b.stats()}))
        return
    gen = dict(cases.CASES[WORKLOAD]["gen"])
    if args.profile_pins:
        side = max(8, gen["n_first"] * args.profile_pins // gen["n_pins"])
        gen.update(n_pins=args.profile_pins, n_first=side, n_last=side)
    dag = cpg_b200.generate(cpg_b200.gen_params(**gen))
    with cpg_b200.CpGen() as g:
        g.load_dag(dag)
        for _ in range(2):
            g.levelize()
            g.report_paths(args.k)
        g.sync()
        print(json.dumps({"profile_case": WORKLOAD, "pins": gen["n_pins"], "n": dag.n,
                          "m": dag.m, "k": args.k, **g.stats()}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--k", type=int, default=1_000_000)
    ap.add_argument("--cpu-k", type=int, default=100_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-case", action="store_true",
                    help="one warm-up and one measured query only (for ncu)")
    ap.add_argument("--profile-pins", type=int, default=0,
                    help="profile case: scale the workload down to this many pins")
    ap.add_argument("--form", default="plain",
                    choices=["plain", "batched", "served", "density", "config1", "bvss", "ingest",
                             "e2e"])
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="batched form: skip cpg_batch_autotune before timing")
    ap.add_argument("--served-queries", type=int, default=5000)
    ap.add_argument("--plain-only", action="store_true",
                    help="skip the batched, served, density and config-1 records")
    ap.add_argument("--bvss-graphs", default="both", choices=["both", "sparse", "dense"])
    args = ap.parse_args()
    if args.profile_case:
        run_profile_case(args)
    elif args.form == "batched":
        run_batched(args)
    elif args.form == "served":
        run_served(args)
    elif args.form == "density":
        print(json.dumps(density_record(args.steps, args.warmup)), flush=True)
    elif args.form == "config1":
        print(json.dumps(config1_record(args.steps, args.warmup, not args.no_cpu_baseline)),
              flush=True)
    elif args.form == "bvss":
        run_bvss(args)
    elif args.form == "ingest":
        run_ingest(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
