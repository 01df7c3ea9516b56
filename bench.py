"""Benchmark of the B200 Vamana hot path (batched build + query beam search).

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

A step is one full batched (prefix-doubling) build of the workload: beam
search + robustPrune for every point, then reverse-edge semisort + append /
prune, round after round.  Default workload: 10,000,000 x 128 uint8 (seeded,
skewed non-negative values from a 10,000-centre mixture), L2, R=64, L=128,
alpha=1.2 -- the BIGANN-10M shape.

value : build points/s with the points already resident in HBM (device time,
        CUDA events, max over ranks).
e2e   : the same build through the C ABI with host buffers: pinned-host upload
        of the points, build, download of the graph, all inside the timed region.
Also reported: the query sweep (L in {10,20,50,100,200}, k=10, recall@10 with
ties against a GPU brute-force ground truth), the roofline of the dominant
kernel and the reference's own CPU build timed on a sample.

With N > 1 ranks (torchrun), each rank builds an independent partition of the
same size (no data-path collective): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "build pts/s; QPS@recall10>=0.95, BF16/INT8+rerank vs exact plain, 1 B200"


def log(msg):
    """Progress on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench] {msg}", file=sys.stderr, flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="bigann-u8")
    ap.add_argument("--n", type=int, default=0, help="override the number of base points")
    ap.add_argument("--nq", type=int, default=0)
    ap.add_argument("--no-queries", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU-baseline work budget")
    ap.add_argument("--no-cpu-queries", action="store_true",
                    help="skip the reference's query QPS in the CPU baseline")
    ap.add_argument("--cpu-nq", type=int, default=2000,
                    help="queries of the reference's timed query sweep")
    ap.add_argument("--plain-steps", type=int, default=3,
                    help="timed builds of the plain exact form (capped by --steps)")
    ap.add_argument("--nvtx-build", action="store_true",
                    help="profiling run: calibrate the fast form's shapes on a 100k-point index "
                         "of the workload, then one instrumented fast build of --n points inside "
                         "the NVTX range 'target' (for ncu --nvtx-include target/); prints stats")
    ap.add_argument("--sharded", action="store_true",
                    help="with N ranks: one build spread over the N GPUs (the reference's "
                         "distributed build; NCCL all-gathers), instead of N independent builds")
    return ap.parse_args()


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    """DRAM bytes per inserted point of k_search, from the ncu capture
    summarised in profiles/ (None if no capture was made)."""
    p = os.path.join(ROOT, "profiles", "k_search_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v == "Active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": rows[0][1],
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------- reference CPU arm
def reference_cpu_build(base, w, budget_s, max_points=2_000_000):
    """Times the reference's own BSP build (oracle/_ref/ref_harness: the
    reference sources compiled unmodified) on a leading sample of the workload,
    sized to about `budget_s` seconds of CPU work.  Returns (pts/s, sample, secs)."""
    from oracle import oracle as O

    if not os.path.exists(O.REF_HARNESS):
        raise RuntimeError("reference CPU build missing (oracle/_ref/ref_harness)")
    cores = os.cpu_count() or 1
    n = min(20_000, base.shape[0])
    while True:
        _, secs = O.ref_build(base[:n], w.R, w.L, w.alpha, metric=w.metric, threads=cores)
        if secs >= budget_s / 3 or n >= min(max_points, base.shape[0]):
            return n / secs, n, secs
        n = int(min(max_points, base.shape[0], n * max(2.0, budget_s / max(secs, 1e-3) / 1.5)))


def run_reference(args, rank):
    if rank != 0:
        return
    from distributed_diskann_b200 import datasets as D

    w = D.WORKLOADS[args.workload]
    cores = os.cpu_count() or 1
    n_total = min(w.n, 2_000_000) if not args.n else args.n
    base, _ = D.make_workload(w, n=n_total, nq=1)
    # calibrate one step to a few seconds of CPU work, then W warm-up + K timed steps
    per_step = max(2.0, min(20.0, 150.0 / max(1, args.warmup + args.steps)))
    rate, n_s, _ = reference_cpu_build(base, w, per_step)
    from oracle import oracle as O

    for _ in range(args.warmup):
        O.ref_build(base[:n_s], w.R, w.L, w.alpha, metric=w.metric, threads=cores)
    secs = [O.ref_build(base[:n_s], w.R, w.L, w.alpha, metric=w.metric, threads=cores)[1]
            for _ in range(args.steps)]
    value = n_s * len(secs) / sum(secs)
    sample = (f"first {n_s} points of the {w.n}x{w.d} {w.dtype} workload per step "
              f"(reference BSP build, np=1, PARLAY_NUM_THREADS={cores})")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "points/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * sum(secs) / len(secs), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8" if w.dtype == "u8" else w.dtype,
        "data": "synthetic",
        "config": {"workload": f"{w.name} sample", "n": n_s, "d": w.d, "R": w.R, "L": w.L,
                   "alpha": w.alpha},
        "cpu_baseline": {"value": value, "unit": "points/s", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": "points/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reference_cpu_queries(base, graph, queries, gt_i, gt_d, w, nq):
    """The reference's searchAll timed like checkRecall (untimed pass, then a
    timed one) at each beam width of the sweep, on the built graph (identical
    to the reference's own build) with the first `nq` queries, all host
    threads; recall@10 with ties against the brute-force ground truth (the
    GPU's exact one, which the tests pin to the oracle's)."""
    from oracle import oracle as O

    cores = os.cpu_count() or 1
    nq = min(nq, queries.shape[0])
    q = np.ascontiguousarray(queries[:nq])
    res = O.ref_qps(base, graph, q, 10, list(w.sweep_L), cut=1.35, metric=w.metric,
                    threads=cores)
    gt_i, gt_d = gt_i[:nq], gt_d[:nq]
    sweep = []
    for L in w.sweep_L:
        ids, secs = res[L]
        sweep.append({"L": L, "qps": nq / secs,
                      "recall10": D_recall(ids, gt_i, gt_d)})
    ok = [s for s in sweep if s["recall10"] >= 0.95]
    return {"qps_at_recall10_0.95": max(s["qps"] for s in ok) if ok else None,
            "sweep": sweep, "unit": "queries/s", "cores": cores, "kind": "reference",
            "sample": f"first {nq} of the {queries.shape[0]} queries on the full built graph "
                      f"(reference searchAll, PARLAY_NUM_THREADS={cores})"}


def D_recall(ids, gt_i, gt_d):
    from distributed_diskann_b200 import datasets as D

    return D.recall_with_ties(ids, gt_i, gt_d, 10)


# ---------------------------------------------------------------------- sharded build
def run_sharded(args, rank, world, local_rank):
    """One build of the workload spread over the ranks (strong scaling): each
    round's batch split by rank, reverse edges owned by target % N, two NCCL
    all-gathers per round (distributed_diskann_b200/sharded.py)."""
    import torch
    import torch.distributed as dist

    from distributed_diskann_b200 import datasets as D
    from distributed_diskann_b200.index import GpuIndex
    from distributed_diskann_b200.sharded import ShardRankGpu, TorchExchange, run_rank

    dev = torch.device("cuda", local_rank)
    w = D.WORKLOADS[args.workload]
    n = args.n or w.n
    base, _ = D.make_workload(w, n=n, nq=1)  # every rank holds the same points
    base_t = torch.from_numpy(base).pin_memory()
    gi = GpuIndex(base.dtype, w.metric, n, w.d, w.R, device=local_rank)
    gi.upload_points(base)
    sr = ShardRankGpu(gi, w.L, w.alpha, mode="fast", world=world)
    ex = TorchExchange()
    stream = torch.cuda.current_stream(dev)

    def build():
        sr.begin()
        run_rank(sr, ex, rank, world, sr.rounds)

    def timed(fn, steps):
        dist.barrier()
        torch.cuda.synchronize(dev)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            fn()
        ev1.record(stream)
        ev1.synchronize()
        t = torch.tensor([ev0.elapsed_time(ev1) / 1000.0], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        build()
    t = timed(build, args.steps)
    graph_host = torch.empty((n, w.R + 1), dtype=torch.int32).pin_memory()

    def e2e_step():
        gi.lib.dd_upload_points(gi.h, base_t.data_ptr(), base_t.stride(0) * base_t.element_size())
        build()
        gi.lib.dd_download_graph(gi.h, graph_host.data_ptr())

    t_e2e = timed(e2e_step, args.steps)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": n * args.steps / t, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": w.dtype,
            "data": "synthetic",
            "config": {"workload": f"{w.name}: {n}x{w.d} {w.dtype} {w.metric}, R={w.R}, L={w.L}, "
                                   f"alpha={w.alpha} (one build spread over the GPUs)",
                       "n": n, "parallelism": f"sharded build over {world} GPUs (NCCL all-gathers)",
                       "l2_flush": "inputs larger than L2 (points + graph > 126 MB)"},
            "e2e": {"value": n * args.steps / t_e2e, "unit": "points/s",
                    "h2d_bytes_per_step": base.nbytes, "d2h_bytes_per_step": n * (w.R + 1) * 4},
        }), flush=True)
    gi.close()


# ---------------------------------------------------------------------- profiling run
def run_nvtx_build(args):
    """Calibrates the autotuner on a 100k-point index of the same shape (its
    shapes are cached per shape, not per n), then runs one fast build with
    statistics inside the NVTX range 'target': the build's k_search launch of
    round r is then the r-th k_search launch of that range."""
    import torch

    from distributed_diskann_b200 import datasets as D
    from distributed_diskann_b200.index import GpuIndex

    w = D.WORKLOADS[args.workload]
    b0, _ = D.make_workload(w, n=min(100_000, w.n), nq=1)
    g0 = GpuIndex(b0.dtype, w.metric, b0.shape[0], w.d, w.R)
    g0.upload_points(b0)
    g0.build(w.L, w.alpha, mode="fast")
    g0.close()
    n = args.n or w.n
    base, _ = D.make_workload(w, n=n, nq=1)
    gi = GpuIndex(base.dtype, w.metric, n, w.d, w.R)
    gi.upload_points(base)
    torch.cuda.nvtx.range_push("target")
    st = gi.build(w.L, w.alpha, mode="fast", collect_stats=True)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    print(json.dumps({"nvtx_build": st, "n": n, "workload": w.name}), flush=True)
    gi.close()


# ---------------------------------------------------------------------- our arm
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.nvtx_build:
        run_nvtx_build(args)
        return

    import torch
    import torch.distributed as dist

    from distributed_diskann_b200 import datasets as D
    from distributed_diskann_b200 import multirank as MR
    from distributed_diskann_b200.index import GpuIndex

    torch.cuda.set_device(local_rank)
    if world > 1 or args.sharded:
        from datetime import timedelta

        if "MASTER_ADDR" not in os.environ:  # one rank outside torchrun
            import socket

            with socket.socket() as sk:
                sk.bind(("127.0.0.1", 0))
                os.environ["MASTER_PORT"] = str(sk.getsockname()[1])
            os.environ["MASTER_ADDR"] = "127.0.0.1"
            os.environ.setdefault("RANK", "0")
            os.environ.setdefault("WORLD_SIZE", "1")

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    if args.sharded:
        run_sharded(args, rank, world, local_rank)
        dist.barrier()
        dist.destroy_process_group()
        return
    dev = torch.device("cuda", local_rank)
    w = D.WORKLOADS[args.workload]
    n = args.n or w.n
    nq = args.nq or w.nq
    # each rank builds its own partition (different seed) of the same size
    wr = MR.rank_workload(w, rank)
    t0 = time.time()
    base, queries = D.make_workload(wr, n=n, nq=nq)
    gen_s = time.time() - t0
    base_t = torch.from_numpy(base).pin_memory()
    graph_host = torch.empty((n, w.R + 1), dtype=torch.int32).pin_memory()

    gi = GpuIndex(base.dtype, w.metric, n, w.d, w.R, device=local_rank)
    stream = torch.cuda.current_stream(dev)
    gi.set_stream(stream.cuda_stream)
    gi.upload_points(base)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x):
        return MR.max_over_ranks(x, dev, world > 1)

    # ---- warm-up (the first fast build calibrates the CTA shapes; the next one
    # captures the build as a CUDA graph, which the timed builds replay)
    for _ in range(args.warmup):
        gi.build(w.L, w.alpha, collect_stats=False, mode="fast")
    barrier()

    # ---- timed builds, inputs resident in HBM
    clocks = ClockSampler(MR.gpu_index(local_rank))
    clocks.start()
    launches = 0
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        gi.build(w.L, w.alpha, collect_stats=False, mode="fast")
        launches += gi.launches()
    ev1.record(stream)
    ev1.synchronize()
    t_dev = ev0.elapsed_time(ev1) / 1000.0
    clk = clocks.stop()
    t_max = max_over_ranks(t_dev)
    value = MR.whole_job_rate(world, n, args.steps, t_max)
    log(f"fast build: {value:.4g} points/s, {1000 * t_max / args.steps:.1f} ms per build")

    # ---- e2e through the C ABI with host buffers
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        gi.lib.dd_upload_points(gi.h, base_t.data_ptr(), base_t.stride(0) * base_t.element_size())
        gi.build(w.L, w.alpha, collect_stats=False, mode="fast")
        gi.lib.dd_download_graph(gi.h, graph_host.data_ptr())
    ev1.record(stream)
    ev1.synchronize()
    t_e2e = max_over_ranks(ev0.elapsed_time(ev1) / 1000.0)
    e2e_value = MR.whole_job_rate(world, n, args.steps, t_e2e)
    h2d = base.nbytes
    d2h = n * (w.R + 1) * 4

    # ---- the plain exact form (CUDA-core distances, grid-stride kernels launched
    # round by round): same graph; timed on min(steps, plain_steps) builds
    graph_fast = gi.graph()
    ksp = max(1, min(args.steps, args.plain_steps))
    gi.build(w.L, w.alpha, collect_stats=False, mode="plain")
    barrier()
    ev0.record(stream)
    for _ in range(ksp):
        gi.build(w.L, w.alpha, collect_stats=False, mode="plain")
    ev1.record(stream)
    ev1.synchronize()
    t_plain = max_over_ranks(ev0.elapsed_time(ev1) / 1000.0)
    plain_value = MR.whole_job_rate(world, n, ksp, t_plain)
    plain_same = bool(np.array_equal(gi.graph(), graph_fast))
    log(f"plain build: {plain_value:.4g} points/s, same graph as fast: {plain_same}")
    st_plain = gi.build(w.L, w.alpha, collect_stats=True, mode="plain")

    # ---- one instrumented build: statistics + per-kernel device times
    st = gi.build(w.L, w.alpha, collect_stats=True, mode="fast")
    g = gi.graph()
    log(f"stats fast: {st}")
    log(f"stats plain: {st_plain}")
    deg = g[:, 0]
    es = 4 if w.dtype == "f32" else 1
    dsz = w.d * es
    # algorithmic bytes of the dominant kernel, k_search (per inserted point p):
    #   V_p*4(R+1) graph rows + C_p*d*s neighbour vectors + d*s own vector,
    # with V_p, C_p the reference's visited.size() and dist_cmps: the plain
    # form's counts, which replay the reference's lossy filter exactly (the
    # fast form's own filter makes a few fewer distance computations, which
    # earns no credit).  The time is the fast form's: the sum of CUDA-event
    # intervals around each k_search launch.
    alg_bytes = (st_plain["visited"] * 4 * (w.R + 1) + st_plain["dist_cmps"] * dsz + n * dsz)
    peak, peak_kind = load_peaks()
    search_s = st["search_ms"] / 1000.0
    achieved = alg_bytes / search_s / 1e9
    n_launch = st["rounds"]
    tr = load_traffic()
    traffic = None
    if tr:  # DRAM bytes per inserted point from the capture (its case is named there)
        traffic = tr["dram_bytes_per_point"] * n / n_launch
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "kernel": "k_search (batched beam search of the insert round)",
                "alg_bytes_per_launch": alg_bytes / n_launch, "launches": n_launch,
                "ms_per_launch": st["search_ms"] / n_launch,
                "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind}, copy burst)",
                "traffic_source": tr.get("case") if tr else None}

    # ---- queries: GPU ground truth, sweep of beam widths, one mixed-L launch
    qres = None
    if not args.no_queries and rank == 0:
        k = 10
        t_gt = time.time()
        gt_i, gt_d = gi.groundtruth(queries, 32)
        t_gt = time.time() - t_gt
        tdt = {"u8": torch.uint8, "i8": torch.int8, "f32": torch.float32}[w.dtype]
        row_elems = int(gi.lib.dd_device_row_stride(gi.h)) // es
        qpad = torch.zeros((nq, row_elems), dtype=tdt, device=dev)  # padded device rows
        qpad[:, : w.d] = torch.from_numpy(queries).to(dev)
        qstride = qpad.stride(0) * qpad.element_size()
        ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
        dd = torch.empty((nq, k), dtype=torch.float32, device=dev)
        def timed_search(Ls, Lmax):
            for _ in range(2):  # first run warms up; the second is timed (checkRecall)
                torch.cuda.synchronize(dev)  # rank 0 only: no collective here
                ev0.record(stream)
                gi.search_device(qpad.data_ptr(), nq, qstride, Ls.data_ptr(), Lmax, k,
                                 ids.data_ptr(), dd.data_ptr())
                ev1.record(stream)
                ev1.synchronize()
            gi.check_errors()  # the device error word of the asynchronous search
            return ev0.elapsed_time(ev1) / 1000.0

        Lmix = torch.tensor(np.array(w.sweep_L, np.int32)[np.arange(nq) % len(w.sweep_L)],
                            device=dev)
        qres = {"nq": nq, "k": k, "cut": 1.35,
                "groundtruth_s": t_gt,  # host wall time of dd_groundtruth, k = 32, copies included
                "groundtruth_form": "tensor-core Gram tiles" if w.dtype != "f32" else "FP64"}
        for form in ("fast", "plain"):
            gi.set_search_mode(form)
            sweep = []
            for L in w.sweep_L:
                Ls = torch.full((nq,), L, dtype=torch.int32, device=dev)
                t = timed_search(Ls, L)
                rec = D.recall_with_ties(ids.cpu().numpy().astype(np.uint32), gt_i, gt_d, k)
                sweep.append({"L": L, "qps": nq / t, "recall10": rec})
                log(f"{form} L={L}: {nq / t:.4g} QPS, recall@10 {rec:.4f}")
            t = timed_search(Lmix, max(w.sweep_L))
            log(f"{form} mixed L: {nq / t:.4g} QPS")
            ok = [s for s in sweep if s["recall10"] >= 0.95]
            qres[form] = {"sweep": sweep, "mixed_L_qps": nq / t,
                          "qps_at_recall10_0.95": max(s["qps"] for s in ok) if ok else None}
        gi.set_search_mode("fast")
        qres["qps_at_recall10_0.95"] = qres["fast"]["qps_at_recall10_0.95"]
        qres["mixed_L_qps"] = qres["fast"]["mixed_L_qps"]

    # ---- CPU baseline: the reference's own build on a sample, rank 0, N = 1
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            rate, n_s, secs = reference_cpu_build(base, w, args.cpu_seconds)
            cpu = {"value": rate, "unit": "points/s", "cores": os.cpu_count(),
                   "kind": "reference",
                   "sample": f"first {n_s} of the {n} points ({secs:.1f} s reference BSP build, "
                             f"PARLAY_NUM_THREADS={os.cpu_count()})"}
        except Exception as e:  # reported, never fatal for the GPU numbers
            cpu = {"value": None, "unit": "points/s", "cores": os.cpu_count(),
                   "kind": "reference", "sample": f"unavailable: {e}"}
        if qres is not None and not args.no_cpu_queries:
            try:
                cpu["queries"] = reference_cpu_queries(base, g, queries, gt_i, gt_d, w,
                                                       args.cpu_nq)
            except Exception as e:  # reported, never fatal for the GPU numbers
                cpu["queries"] = {"unavailable": str(e)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "points/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": w.dtype, "data": "synthetic",
            "config": {"workload": f"{w.name}: {n}x{w.d} {w.dtype} {w.metric}, R={w.R}, "
                                   f"L={w.L}, alpha={w.alpha} (full batched build per step)",
                       "n": n, "d": w.d, "R": w.R, "L": w.L, "alpha": w.alpha,
                       "form": "fast (INT8 tensor-core prune tiles, set-associative seen "
                               "filter and register step merges in the build search, "
                               "persistent work-queue kernels, CUDA-graph build replay, "
                               "autotuned CTA shapes); graph bit-exact vs the reference build",
                       "l2_flush": "inputs larger than L2 (points + graph > 126 MB)",
                       "parallelism": f"{world} independent partitions" if world > 1 else "1 GPU"},
            "e2e": {"value": e2e_value, "unit": "points/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clk,
            "build_stats": {k2: st[k2] for k2 in ("rounds", "visited", "dist_cmps", "groups",
                                                 "reverse_prunes", "prune_cands", "big_groups",
                                                 "build_ms", "search_prune_ms", "search_ms", "reverse_ms")},
            "graph": {"avg_degree": float(deg.mean()), "max_degree": int(deg.max())},
            "plain": {"value": plain_value, "unit": "points/s", "steps": ksp,
                      "ms_per_step": 1000.0 * t_plain / ksp,
                      "same_graph_as_fast": plain_same,
                      "build_stats": {k2: st_plain[k2] for k2 in ("build_ms", "search_ms",
                                                                  "search_prune_ms", "reverse_ms")},
                      "form": "plain exact (CUDA-core distances, grid-stride kernels launched "
                              "round by round)"},
            "fast_over_plain": {"build": value / plain_value,
                                "qps_at_recall10_0.95": (
                                    qres["fast"]["qps_at_recall10_0.95"]
                                    / qres["plain"]["qps_at_recall10_0.95"]
                                    if qres and qres["plain"]["qps_at_recall10_0.95"] else None),
                                "mixed_L_qps": (qres["fast"]["mixed_L_qps"]
                                                / qres["plain"]["mixed_L_qps"] if qres else None)},
            "tuned": {k2: st[k2] for k2 in ("search_warps_per_cta", "prune_warps_per_cta",
                                            "search_queue", "prune_queue")},
            "queries": qres,
            "setup_s": {"datagen": gen_s},
        }
        print(json.dumps(line), flush=True)
    gi.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
