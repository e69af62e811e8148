"""Benchmark: HashGraph build + intersect on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload large|large_zipf|small|capacity_lf1|capacity_lf05|capacity_lf2]

One step = build table A from n keys resident in HBM, then intersect n query
keys against it (pairs emitted; count only for large_zipf, whose output would
be about 1.4e15 pairs).  Metric: build & intersect keys/s = n (keys
per set) / (t_build + t_intersect).  Default workload (N=1): A = 2^28 uint64
keys uniform (seed 3), queries = 2^28 uint64 keys with 25% drawn from A,
n_buckets = 2^28.  Under torchrun every rank runs its own replica (weak
scaling; no data-path collective); the step time is the max over ranks.

Prints ONE JSON line on rank 0.  `--impl reference` times the CPU
implementation of the same algorithm (the oracle's multithreaded build +
probe, on all host threads) on the same workload (a 2^28-key sample of the
2^30-key capacity workloads).  On the large and small workloads our arm also
times, outside its own timed region, the reference's own MultiHashGraph
(built for sm_100a from its sources into oracle/_ref/) on the same inputs
(`reference_gpu`).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "build & intersect keys/sec on 1 B200, % of HBM roofline; batched/served p50/p99"
UNIT = "keys/s"

WORKLOADS = {
    # name: (key_bytes, n, n_buckets_fn, kind, seed_a, seed_q, overlap, with_index)
    "large": (8, 1 << 28, lambda n: n, "uniform", 3, 30, 0.25, False),
    # skewed variant of the large workload: Zipf(1.1) over one 2^24-key universe, count only
    "large_zipf": (8, 1 << 28, lambda n: n, "zipf", 3, 30, 0.0, False),
    "small": (4, 1 << 20, lambda n: n, "uniform", 1, 2, 0.5, False),
    "capacity_lf1": (4, 1 << 30, lambda n: n, "uniform", 4, 40, 0.1, True),
    "capacity_lf05": (4, 1 << 30, lambda n: 2 * n, "uniform", 4, 40, 0.1, True),
    "capacity_lf2": (4, 1 << 30, lambda n: n // 2, "uniform", 4, 40, 0.1, True),
}


def describe(name, kb, n, B, kind, overlap, with_index):
    kt = "u64" if kb == 8 else "u32"
    lg = n.bit_length() - 1
    if kind == "zipf":
        q = f"queries 2^{lg} {kt} Zipf(1.1) over a 2^24-key universe (independent seed), count only"
        a = f"A = 2^{lg} {kt} Zipf(1.1) over a 2^24-key universe"
    else:
        q = f"queries 2^{lg} {kt} with {int(overlap * 100)}% drawn from A, pairs emitted"
        a = f"A = 2^{lg} {kt} uniform"
    return (f"{name}: build {a}{' + index' if with_index else ''} into {B} buckets, then intersect "
            f"{q}")


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per key of each
# partition kernel, from one ncu capture at 2^25 u64 keys, 2^25 buckets,
# table without index, 25% overlap, same per-CTA geometry as 2^28 (the
# capture summarised under profiles/).  Traffic grows with the keys
# processed, so a full launch's traffic is this figure times its keys.
MEASURED_TRAFFIC_PER_KEY = {
    (8, False): {"multisplit": 14.5, "split": 14.4, "fine_build": 18.5,
                 "probe_multisplit": 18.3, "probe_split": 22.4, "fine_probe_emit": 25.8,
                 "coarse_probe_emit": 26.1},
}


def measured_traffic(phase, kb, with_index, n, nq, B):
    """Per-launch DRAM traffic of `phase` scaled from the capture, or None
    when the workload's shape differs from the captured one."""
    per = MEASURED_TRAFFIC_PER_KEY.get((kb, with_index), {}).get(phase)
    if per is None or n != nq or B != n:
        return None
    return per * n


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# distributed plumbing (replicas; barrier and max-over-ranks only)
# ---------------------------------------------------------------------------
def dist_setup(n_gpus):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        if torch.cuda.is_available():
            torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(x, world, op):
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, world):
    """Slowest rank's time: the job's step time."""
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.MAX if world > 1 else None)


def sum_over_ranks(x, world):
    """Units processed by all ranks together."""
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.SUM if world > 1 else None)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def algorithmic_bytes(phase, kb, n, nq, B, with_index, pairs):
    """Bytes each kernel's role must move (its inputs read once, its outputs
    written once): per key, K read and K (+4 index) written by a partition
    pass; the fine passes add the 4-byte offsets and the 8-byte pairs."""
    rec = kb + (4 if with_index else 0)
    qrec = kb + 4
    if phase.startswith("fallback_"):  # the gated direct kernels do the same role's work
        phase = phase[len("fallback_"):]
    return {
        # build
        "multisplit": n * kb + n * rec,
        "split": 2 * n * rec,
        "fine_build": 2 * n * rec + 4 * (B + 1),
        "count": n * kb,
        "scan": 8 * B,
        "scatter": n * kb + n * rec,
        # intersect
        "probe_multisplit": nq * kb + nq * qrec,
        "probe_split": 2 * nq * qrec,
        "fine_probe_emit": nq * qrec + n * rec + 4 * (B + 1) + 8 * pairs,
        "fine_probe_count": nq * qrec + n * rec + 4 * (B + 1),
        # the coarse probe reads every query record once, the table once (each
        # bucket range's slice comes from HBM into L2 once) and writes the pairs
        "coarse_probe_emit": nq * qrec + n * rec + 4 * (B + 1) + 8 * pairs,
        "coarse_probe_count": nq * qrec + n * rec + 4 * (B + 1),
        "probe_emit": nq * kb + n * rec + 4 * (B + 1) + 8 * pairs,
        "probe_count": nq * kb + n * rec + 4 * (B + 1),
        # the heavy-key count reads at most every key of A once
        "heavy_keys": n * kb,
    }.get(phase)


def is_probe_phase(name):
    return "probe" in name


def run_ours(args, rank, world, local):
    import numpy as np
    import torch

    import hashgraph_b200 as hg

    kb, n, bfn, kind, seed_a, seed_q, overlap, with_index = WORKLOADS[args.workload]
    n = args.n or n
    B = bfn(n)
    emit = kind != "zipf"
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    hg.lib()
    # inputs, generated on the device (same definitions as the oracle)
    if kind == "zipf":
        cdf = hg.zipf_cdf(1 << 24, 1.1, device=dev)
        a_keys = hg.gen_zipf(n, kb, cdf, seed_a)
        q_keys = hg.gen_zipf(n, kb, cdf, seed_q)
        del cdf
    else:
        a_keys = hg.gen_uniform(n, kb, seed_a, device=dev)
        q_keys = hg.gen_overlap(n, a_keys, overlap, seed_q)
    nq = q_keys.numel()
    paths = {"auto": hg.PATH_AUTO, "direct": 0, "partitioned": 1}
    build_path, probe_path = paths[args.build_path], paths[args.probe_path]
    table = hg.Table(B, kb, with_index, n, dev, build_path)
    pair_cap = nq if emit else 0
    import ctypes
    table.n = n  # the probe plan depends on the table's size
    ws = torch.empty(max(hg.intersect_workspace_bytes(table, nq, emit, probe_path), 1), dtype=torch.uint8,
                     device=dev)
    count = torch.zeros(1, dtype=torch.int64, device=dev)
    pairs = torch.empty((max(pair_cap, 1), 2), dtype=torch.int32, device=dev) if emit else None
    L = hg.lib()
    sptr = ctypes.c_void_p(stream.cuda_stream)

    def step(a_src, q_src):
        table.rebuild(a_src, stream)
        hg.check(L.hg_intersect_into_path(
            ctypes.c_void_p(table.offsets.data_ptr()), ctypes.c_void_p(table.keys.data_ptr()),
            ctypes.c_void_p(table.idx.data_ptr()) if table.idx is not None else None, table.n, B, kb,
            ctypes.c_void_p(q_src.data_ptr()), nq, None,
            ctypes.c_void_p(pairs.data_ptr()) if emit else None, pair_cap,
            ctypes.c_void_p(count.data_ptr()), ctypes.c_void_p(ws.data_ptr()), ws.numel(), probe_path, sptr),
            "intersect")

    for _ in range(args.warmup):
        step(a_keys, q_keys)
    torch.cuda.synchronize(dev)
    n_matches = int(count.item())
    if hg.device_error() != 0:
        raise RuntimeError("device error during warm-up")

    # ---- timed region: inputs resident in HBM.  Sets larger than L2 (126 MB)
    # need no flush; smaller ones get L2 flushed (a 256 MiB buffer written)
    # before every timed step, outside the step's events.
    l2_bytes = 126 << 20
    flush = None
    if (n + nq) * kb < 2 * l2_bytes:
        flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
        l2_note = ("inputs fit in L2 (each set %.1f MiB vs 126 MB L2): L2 flushed before every timed step by "
                   "writing a 256 MiB buffer (outside the step's events)" % (n * kb / 2**20))
    else:
        l2_note = "inputs larger than L2 (each set %d MiB vs 126 MB L2); no flush" % (n * kb >> 20)
    hg.profile_enable(True)
    hg.profile_read()
    clocks = ClockSampler(local)
    launches0 = hg.launch_count()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps)]
    barrier(world)
    torch.cuda.synchronize(dev)
    clocks.start()
    time.sleep(0.3)
    for k in range(args.steps):
        if flush is not None:
            flush.fill_(k & 0xFF)
        ev[2 * k].record(stream)
        step(a_keys, q_keys)
        ev[2 * k + 1].record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    launches = hg.launch_count() - launches0
    clk = clocks.stop()
    phases = hg.profile_read()
    hg.profile_enable(False)
    del flush
    step_ms = [ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(args.steps)]
    total_ms = sum(step_ms)
    total_ms_max = max_over_ranks(total_ms, world)
    if hg.device_error() != 0:
        raise RuntimeError("device error during timed steps")

    per_phase = {}
    for name, ms in phases:
        per_phase.setdefault(name, []).append(ms)
    phase_avg = {k: sum(v) / len(v) for k, v in per_phase.items()}
    phase_share = {k: sum(v) / max(total_ms, 1e-9) for k, v in per_phase.items()}
    dom = max(per_phase, key=lambda k: sum(per_phase[k]))
    peak, peak_kind = load_peaks()
    alg = algorithmic_bytes(dom, kb, n, nq, B, with_index, n_matches)
    achieved = alg / (phase_avg[dom] * 1e-3) / 1e9 if alg else None
    build_ms = sum(sum(v) for k, v in per_phase.items() if not is_probe_phase(k)) / args.steps
    probe_ms = sum(sum(v) for k, v in per_phase.items() if is_probe_phase(k)) / args.steps
    # compulsory bytes of the step (build + probe form of intersect)
    rec = kb + (4 if with_index else 0)
    build_bytes = n * kb + n * rec + 4 * (B + 1)
    isect_bytes = nq * kb + n * rec + 4 * (B + 1) + (8 * n_matches if emit else 0) + 8
    step_s = total_ms / args.steps * 1e-3
    value = sum_over_ranks(n * args.steps, world) / (total_ms_max * 1e-3)

    # ---- end to end through the public API from pinned host buffers: every
    # step uploads its keys and queries, builds, probes and downloads the count
    # and the pairs; HostPipeline overlaps step k+1's upload with step k's
    # build + probe and step k-1's download
    e2e = None
    if not args.skip_e2e:
        from hashgraph_b200.pipeline import HostPipeline
        h_a = torch.empty(a_keys.shape, dtype=a_keys.dtype, pin_memory=True)
        h_q = torch.empty(q_keys.shape, dtype=q_keys.dtype, pin_memory=True)
        h_a.copy_(a_keys)
        h_q.copy_(q_keys)
        h_pairs = torch.empty((max(pair_cap, 1), 2), dtype=torch.int32, pin_memory=True) if emit else None
        del table, ws, pairs
        pipe = HostPipeline(n, nq, B, key_bytes=kb, with_index=with_index, emit=emit, pair_cap=pair_cap,
                            device=dev, build_path=build_path, probe_path=probe_path)
        pipe.run([(h_a, h_q)], [h_pairs])  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world)
        torch.cuda.synchronize(dev)
        counts = pipe.run([(h_a, h_q)] * args.steps, [h_pairs] * args.steps, start_event=e0, end_event=e1)
        torch.cuda.synchronize(dev)
        if any(c != n_matches for c in counts):
            raise RuntimeError(f"end-to-end counts {set(counts)} != {n_matches}")
        d2h = sum(8 + (8 * min(c, pair_cap) if emit else 0) for c in counts)
        e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
        e2e = {"value": sum_over_ranks(n * args.steps, world) / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(a_keys.numel() * kb + q_keys.numel() * kb),
               "d2h_bytes_per_step": int(d2h // args.steps),
               "api": "hashgraph_b200.pipeline.HostPipeline (hg_build_into + hg_intersect_into on its streams)"}
        del h_a, h_q, h_pairs, pipe

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        cpu = cpu_baseline(args.workload, n_sample=cpu_sample_size(args, n))

    # the reference's own GPU build + intersect on the same inputs, outside our
    # timed region, with this process's device memory released first
    ref_gpu = None
    if rank == 0 and world == 1 and not args.skip_ref_gpu and kind == "uniform":
        table = ws = pairs = count = a_keys = q_keys = None  # noqa: F841 (releases the device buffers)
        import gc
        gc.collect()
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()
        ref_gpu = reference_gpu(args.workload, n, value)

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64" if kb == 8 else "u32",
        "data": "synthetic (seeded splitmix64 keys generated on the device; definitions shared with the oracle)",
        "config": {"workload": describe(args.workload, kb, n, B, kind, overlap, with_index), "n": n, "nq": nq,
                   "n_buckets": B, "key_bytes": kb, "with_index": with_index, "emit_pairs": emit,
                   "matches": n_matches, "build_path": args.build_path, "probe_path": args.probe_path,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": l2_note},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": measured_traffic(dom, kb, with_index, n, nq, B),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum at 2^25, scaled by keys",
                     "peak_source": peak_kind, "algorithmic_bytes": alg,
                     "avg_launch_ms": phase_avg[dom]},
        "step_roofline": {"compulsory_bytes": build_bytes + isect_bytes,
                          "achieved_gbs": (build_bytes + isect_bytes) / step_s / 1e9,
                          "frac_of_measured_hbm": (build_bytes + isect_bytes) / step_s / 1e9 / peak,
                          "frac_of_8tbs": (build_bytes + isect_bytes) / step_s / 1e9 / 8000.0,
                          "build_ms": build_ms, "intersect_ms": probe_ms,
                          "build_keys_per_s": n / (build_ms * 1e-3) if build_ms else None,
                          "build_frac_of_measured_hbm": build_bytes / (build_ms * 1e-3) / 1e9 / peak if build_ms else None,
                          "intersect_frac_of_measured_hbm": isect_bytes / (probe_ms * 1e-3) / 1e9 / peak if probe_ms else None},
        "phases_ms": phase_avg, "phase_share": phase_share,
        "clocks": clk, "e2e": e2e, "gpu_launches": launches, "cpu_baseline": cpu,
        "reference_gpu": ref_gpu,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


def reference_gpu(workload, n, our_value, repeats=3):
    """Times the reference's own MultiHashGraph with gpuCount = 1 (built for
    sm_100a from its unmodified sources into oracle/_ref/ by oracle/Makefile)
    on the same seeded inputs as our arm, through its public API as its test
    main drives it: construct A and B, build A, build B, intersect, timed with
    CUDA events (oracle/ref_multi_driver.cu).  The sequence runs `repeats`
    times in one process; the first run is what the reference's test main
    times (it includes the first touch of its managed memory), the best run
    is its steady state, against which our ratio is taken."""
    import tempfile

    import numpy as np

    import oracle
    if workload.startswith("capacity"):
        # 2^30 u32 keys into 2^30 and 2^31 buckets: the reference printed
        # "ERROR: NOT ENOUGH TEMP SPACE ALLOCATED" (src/MultiHashGraph.cu:
        # 331-361; its scan scratch is max(2048, tableSize / 10) bytes, :178)
        # and then made an illegal memory access, so it is not run at the
        # capacity sizes at all
        return {"unavailable": "the reference faulted at these sizes (NOT ENOUGH TEMP SPACE ALLOCATED, then an "
                               "illegal memory access at 2^30 u32 keys with B = 2^30 and 2^31); not run"}
    kb, _, bfn, kind, seed_a, seed_q, overlap, with_index = WORKLOADS[workload]
    exe = oracle.ref_binary("ref_multi" if kb == 8 else "ref_multi32")
    if exe is None:
        return {"unavailable": "oracle/_ref/ref_multi* not built (the reference sources were absent at build time)"}
    B = bfn(n)
    a = oracle.gen_uniform(n, kb, seed_a)
    q = oracle.gen_overlap(n, a, overlap, seed_q)
    with tempfile.TemporaryDirectory() as td:
        fa, fq = os.path.join(td, "a.bin"), os.path.join(td, "q.bin")
        a.tofile(fa)
        q.tofile(fq)
        del a, q
        try:
            r = subprocess.run([exe, fa, str(n), fq, str(n), str(B), "-", "1", str(repeats)], capture_output=True,
                               text=True, timeout=900)
        except subprocess.TimeoutExpired:
            return {"unavailable": "reference run exceeded 900 s"}
    if r.returncode != 0:
        return {"unavailable": f"reference run failed (rc {r.returncode}): {r.stderr.strip()[-300:]}"}
    runs = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    if not runs:
        return {"unavailable": "reference run printed no timing"}
    best = min(runs, key=lambda x: x["total_s"])
    first = runs[0]

    def summary(x):
        bi = x["build_a_s"] + x["intersect_s"]
        return {"build_a_ms": x["build_a_s"] * 1e3, "build_b_ms": x["build_b_s"] * 1e3,
                "intersect_ms": x["intersect_s"] * 1e3, "composite_ms": x["total_s"] * 1e3,
                "build_a_plus_intersect_keys_per_s": n / bi if bi > 0 else None,
                "composite_keys_per_s": n / x["total_s"] if x["total_s"] > 0 else None}

    b = summary(best)
    return {"impl": "reference MultiHashGraph (gpuCount 1, sm_100a, unmodified sources; oracle/_ref)",
            "workload": "same seeded inputs as our arm; the reference builds both sets into tables "
                        "(its intersect joins two tables) and emits the matched keys",
            "runs": len(runs), "composite_ms_per_run": [x["total_s"] * 1e3 for x in runs],
            "first_run": summary(first), "best_run": b,
            "ours_over_reference_build_a_plus_intersect": (our_value / b["build_a_plus_intersect_keys_per_s"]
                                                           if b["build_a_plus_intersect_keys_per_s"] else None),
            "ours_over_reference_composite": (our_value / b["composite_keys_per_s"]
                                              if b["composite_keys_per_s"] else None)}


def cpu_sample_size(args, n):
    """Keys per set the CPU arm processes: the whole workload up to 2^28 keys
    per set (about 3 s per step on 16 host threads), a 2^28 sample beyond."""
    return min(n, args.cpu_sample) if args.cpu_sample else min(n, 1 << 28)


# ---------------------------------------------------------------------------
# batched build + intersect (many independent pairs per step)
# ---------------------------------------------------------------------------
def batched_sizes(n_pairs, lo_log2, hi_log2, seed=4):
    """Pair i: n_i = floor(2^U(lo, hi)) keys (log-uniform), B_i = n_i buckets,
    n_i queries with overlap fraction U(0, 1); seeded."""
    import numpy as np
    rng = np.random.default_rng(seed)
    sizes = np.floor(2.0 ** rng.uniform(lo_log2, hi_log2, n_pairs)).astype(np.int64)
    fracs = rng.uniform(0.0, 1.0, n_pairs)
    return sizes, fracs


def batch_kernel_launches(hg, batch):
    """Kernels one run of `batch` launches (the library's launch counter over
    one direct run)."""
    import torch
    c0 = hg.launch_count()
    batch.run()
    torch.cuda.synchronize()
    return hg.launch_count() - c0


def run_batched(args, rank, world, local):
    import ctypes

    import numpy as np
    import torch

    import hashgraph_b200 as hg

    kb = 8
    sizes, fracs = batched_sizes(args.pairs, 6, 20)
    n_total = int(sizes.sum())
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    L = hg.lib()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    # every pair's keys and queries are views of two arena tensors
    a_all = torch.empty(n_total, dtype=torch.int64, device=dev)
    q_all = torch.empty(n_total, dtype=torch.int64, device=dev)
    starts = np.concatenate([[0], np.cumsum(sizes)])
    a_views = [a_all[starts[i]:starts[i + 1]] for i in range(args.pairs)]
    q_views = [q_all[starts[i]:starts[i + 1]] for i in range(args.pairs)]
    for i in range(args.pairs):
        n = int(sizes[i])
        check = hg._capi.check
        check(L.hg_gen_uniform(ctypes.c_void_p(a_views[i].data_ptr()), n, kb, 100_000 + i, sptr), "gen")
        m = hg.overlap_count(n, n, float(fracs[i]))
        check(L.hg_gen_overlap(ctypes.c_void_p(q_views[i].data_ptr()), n, kb,
                               ctypes.c_void_p(a_views[i].data_ptr()), n, m, 200_000 + i, sptr), "gen")
    B = [int(x) for x in sizes]
    batch = hg.Batch(a_views, q_views, B, with_index=False, pair_caps=B)
    # size classes picked by the autotuner on this batch, outside the timed region
    size_classes, tune_ms = batch.autotune()
    for _ in range(args.warmup):
        batch.run()
    torch.cuda.synchronize(dev)
    if hg.device_error() != 0:
        raise RuntimeError("device error during warm-up")
    matches = int(batch.counts[: args.pairs].sum().item())
    # the whole batch (its memset and its fixed kernel sequence) captured once
    # into a CUDA graph: each timed step is ONE graph launch
    graph = torch.cuda.CUDAGraph()
    cap = torch.cuda.Stream(dev)  # capture needs a stream other than the default one
    cap.wait_stream(stream)
    with torch.cuda.graph(graph, stream=cap):
        batch.run(stream=cap)
    graph.replay()
    torch.cuda.synchronize(dev)
    if int(batch.counts[: args.pairs].sum().item()) != matches or hg.device_error() != 0:
        raise RuntimeError("the captured batch disagrees with the direct run")

    hg.profile_enable(True)
    hg.profile_read()
    clocks = ClockSampler(local)
    launches0 = hg.launch_count()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps)]
    barrier(world)
    torch.cuda.synchronize(dev)
    clocks.start()
    time.sleep(0.3)
    for k in range(args.steps):
        ev[2 * k].record(stream)
        graph.replay()
        ev[2 * k + 1].record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    # kernels inside a replayed graph are not counted by the library's launch
    # counter: each replay runs the captured batch's kernels
    launches = (hg.launch_count() - launches0) + args.steps * batch_kernel_launches(hg, batch)
    clk = clocks.stop()
    hg.profile_read()
    hg.profile_enable(False)
    total_ms = sum(ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(args.steps))
    # per-kernel phases from one direct (uncaptured) run with the library's events
    hg.profile_enable(True)
    hg.profile_read()
    batch.run(stream=stream)
    torch.cuda.synchronize(dev)
    phases = hg.profile_read()
    hg.profile_enable(False)
    total_ms_max = max_over_ranks(total_ms, world)
    if hg.device_error() != 0:
        raise RuntimeError("device error during timed steps")
    value = sum_over_ranks(n_total * args.steps, world) / (total_ms_max * 1e-3)
    per_phase = {}
    for name, ms in phases:
        per_phase.setdefault(name, []).append(ms)
    phase_avg = {k: sum(v) for k, v in per_phase.items()}  # ms per batch run (one run profiled)
    dom = max(per_phase, key=lambda k: sum(per_phase[k]))
    peak, peak_kind = load_peaks()
    sum_b = n_total + args.pairs  # buckets + 1 per pair
    # the L2 form of the probe takes the pairs of >= 2^14 queries (tables of at most 2^20 u64 keys fit its
    # 24 MB budget): their queries once, their tables once, their pairs
    large = sizes >= (1 << 14)
    l2_n = int(sizes[large].sum())
    l2_m = int(batch.counts[: args.pairs].cpu().numpy()[large].sum())
    alg = {"batch_count": n_total * kb, "batch_scan": 8 * sum_b, "batch_scatter": 2 * n_total * kb,
           "batch_probe": n_total * kb * 2 + 4 * sum_b + 8 * matches, "batch_clear": 4 * sum_b,
           "batch_l2_probe": l2_n * kb * 2 + 4 * (l2_n + int(large.sum())) + 8 * l2_m}.get(dom)
    achieved = alg / (phase_avg[dom] * 1e-3) / 1e9 if alg else None
    compulsory = n_total * kb * 2 + 4 * sum_b + (n_total * kb * 2 + 4 * sum_b + 8 * matches)
    step_s = total_ms / args.steps * 1e-3

    # the same pairs as one build + intersect call each (the launch-bound
    # form), every call on the planner's own path choice, as a user would call
    ws_need = 1
    for nn in sorted(set(int(x) for x in sizes)):
        ws_b = ctypes.c_size_t(0)
        ws_q = ctypes.c_size_t(0)
        hg._capi.check(L.hg_build_workspace_size_path(nn, kb, nn, 0, -1, ctypes.byref(ws_b)), "ws")
        hg._capi.check(L.hg_intersect_workspace_size_path(nn, 0, nn, nn, kb, 1, -1, ctypes.byref(ws_q)), "ws")
        ws_need = max(ws_need, ws_b.value, ws_q.value)
    ws = torch.empty(ws_need, dtype=torch.uint8, device=dev)

    def plain_step():
        for i in range(args.pairs):
            n = int(sizes[i])
            hg._capi.check(L.hg_build_into_path(
                ctypes.c_void_p(a_views[i].data_ptr()), n, kb, n, ctypes.c_void_p(batch.offsets[i].data_ptr()),
                ctypes.c_void_p(batch.table_keys[i].data_ptr()), None, ctypes.c_void_p(ws.data_ptr()),
                ws.numel(), -1, sptr), "plain build")
            hg._capi.check(L.hg_intersect_into_path(
                ctypes.c_void_p(batch.offsets[i].data_ptr()), ctypes.c_void_p(batch.table_keys[i].data_ptr()),
                None, n, n, kb, ctypes.c_void_p(q_views[i].data_ptr()), n, None,
                ctypes.c_void_p(batch.pairs[i].data_ptr()), n,
                ctypes.c_void_p(batch.counts.data_ptr() + 8 * i), ctypes.c_void_p(ws.data_ptr()), ws.numel(),
                -1, sptr), "plain intersect")

    plain_step()
    torch.cuda.synchronize(dev)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    plain_step()
    p1.record(stream)
    torch.cuda.synchronize(dev)
    plain_ms = p0.elapsed_time(p1)
    if int(batch.counts[: args.pairs].sum().item()) != matches:
        raise RuntimeError("plain calls and the batch disagree on the match count")

    e2e = None
    if not args.skip_e2e:
        h_a = torch.empty(n_total, dtype=torch.int64, pin_memory=True)
        h_q = torch.empty(n_total, dtype=torch.int64, pin_memory=True)
        h_a.copy_(a_all)
        h_q.copy_(q_all)
        h_counts = torch.empty(args.pairs, dtype=torch.int64, pin_memory=True)
        h_pairs = torch.empty((n_total, 2), dtype=torch.int32, pin_memory=True)
        pstart = starts
        d2h = 0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(args.steps):
            a_all.copy_(h_a, non_blocking=True)
            q_all.copy_(h_q, non_blocking=True)
            batch.run()
            h_counts.copy_(batch.counts[: args.pairs], non_blocking=True)
            stream.synchronize()
            d2h += 8 * args.pairs
            cnt = h_counts.numpy()
            for i in range(args.pairs):
                c = int(cnt[i])
                if c:
                    h_pairs[pstart[i]:pstart[i] + c].copy_(batch.pairs[i][:c], non_blocking=True)
                    d2h += 8 * c
        e1.record(stream)
        torch.cuda.synchronize(dev)
        e2e_ms = max_over_ranks(e0.elapsed_time(e1), world)
        e2e = {"value": sum_over_ranks(n_total * args.steps, world) / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(2 * n_total * kb), "d2h_bytes_per_step": int(d2h // args.steps)}

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded splitmix64 keys generated on the device; definitions shared with the oracle)",
        "config": {"workload": f"batched: {args.pairs} pairs, A_i = 2^U(6,20) u64 uniform keys into B_i = n_i "
                               f"buckets, n_i queries with U(0,1) drawn from A_i, pairs emitted; one "
                               f"hg_batch_run captured into a CUDA graph, one graph launch per step",
                   "pairs": args.pairs, "keys_total": n_total, "matches": matches,
                   "size_classes": size_classes, "autotune_best_ms": tune_ms,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs (%d MiB per set) larger than L2; no flush" % (n_total * kb >> 20)},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": None,
                     "peak_source": peak_kind, "algorithmic_bytes": alg, "avg_launch_ms": phase_avg[dom]},
        "step_roofline": {"compulsory_bytes": compulsory, "achieved_gbs": compulsory / step_s / 1e9,
                          "frac_of_measured_hbm": compulsory / step_s / 1e9 / peak},
        "plain_calls": {"ms_per_step": plain_ms, "value": n_total / (plain_ms * 1e-3), "unit": UNIT,
                        "calls": 2 * args.pairs,
                        "note": "one hg_build_into + hg_intersect_into per pair (the planner's path), same buffers"},
        "phases_ms": phase_avg, "clocks": clk, "e2e": e2e, "gpu_launches": launches, "cpu_baseline": None,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# serving: Poisson arrivals of build / intersect requests against resident tables
# ---------------------------------------------------------------------------
def serving_requests(n_req, rate, arena_keys, lo_log2=10, hi_log2=24, seed=5):
    """Request list: Poisson arrivals at `rate`/s, 30% builds (table ids in
    order) and 70% intersects against one of the last 128 built tables;
    sizes 2^U(lo, hi).  A build takes the key-arena slice [off, off+n); an
    intersect's queries are the slice starting half-way into its table's
    slice (so about half of them, up to the table's size, match)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    t, reqs, built = 0.0, [], []
    for k in range(n_req):
        t += rng.exponential(1.0 / rate)
        size = int(2 ** rng.uniform(lo_log2, hi_log2))
        if k < 16 or rng.uniform() < 0.3:
            off = int(rng.integers(0, arena_keys - size))
            built.append((len(built), off, size))
            reqs.append(("build", len(built) - 1, t, off, size))
        else:
            tid, toff, tn = built[int(rng.integers(max(0, len(built) - 128), len(built)))]
            qoff = (toff + tn // 2) % max(1, arena_keys - size)
            reqs.append(("intersect", tid, t, qoff, size))
    return reqs


# table memory mapped into the serving engine's pool before the run (the
# resident tables of the default request mix peak near 13 GB)
RESERVE_BYTES = 32 << 30


def run_serving(args, rank, world, local):
    import torch

    import hashgraph_b200 as hg
    from hashgraph_b200.serve import Request, Server, latency_summary, now, run_open_loop

    dev = torch.device("cuda", local)
    arena_keys = 1 << 27
    arena = hg.gen_uniform(arena_keys, 8, 6, device=dev)
    specs = serving_requests(args.requests, args.rate, arena_keys)

    def make(spec):
        kind, tid, t, off, size = spec
        sl = arena[off:off + size]
        if kind == "build":
            return Request("build", tid, t, keys=sl, n_buckets=size)
        return Request("intersect", tid, t, queries=sl, pair_cap=size)

    torch.cuda.synchronize(dev)
    server = Server(budget_bytes=120 << 30, max_tables=512, n_streams=args.streams, max_keys=1 << 24, device=dev)
    server.reserve(RESERVE_BYTES)
    # warm-up: one build and one intersect of each size decade, outside the timed run
    for lg in range(10, 25, 2):
        server.submit(Request("build", -1, 0.0, keys=arena[: 1 << lg], n_buckets=1 << lg))
        server.submit(Request("intersect", -1, 0.0, queries=arena[: 1 << lg], pair_cap=1 << lg))
        server.drain()
    torch.cuda.synchronize(dev)
    reqs = [make(sp) for sp in specs]
    clocks = ClockSampler(local)
    launches0 = hg.launch_count()
    clocks.start()
    makespan = run_open_loop(server, reqs)
    clk = clocks.stop()
    launches = hg.launch_count() - launches0
    done = [r for r in reqs if r.latency_s is not None]
    keys_total = sum((r.keys.numel() if r.kind == "build" else r.queries.numel()) for r in reqs)
    value = keys_total / makespan
    by_kind = {k: latency_summary([r for r in done if r.kind == k]) for k in ("build", "intersect")}
    missed = sum(1 for r in reqs if r.missed)

    # each intersect's count against a serial run of the same request list
    st = server.stats()
    server.free()

    # saturated: every request submitted at once, served (1) with continuous
    # batching, (2) one launch per request on the same streams, (3) as plain
    # calls, one build or intersect call after another on one stream; the
    # counts (and misses) must be identical.  Once on the request mix above,
    # once on small requests only (2^U(10,16) keys), where launches dominate.
    def saturated_run(sp_list):
        out, counts = {}, {}
        total = sum(sp[4] for sp in sp_list)
        for mode, kw in (("batched", dict(batching=True, n_streams=args.streams)),
                         ("one_launch_per_request", dict(batching=False, n_streams=args.streams)),
                         ("plain_calls", dict(batching=False, n_streams=1))):
            srv = Server(budget_bytes=120 << 30, max_tables=512, max_keys=1 << 24, device=dev, **kw)
            srv.reserve(RESERVE_BYTES)
            for lg in range(10, 25, 2):
                srv.submit(Request("build", -1, 0.0, keys=arena[: 1 << lg], n_buckets=1 << lg))
                srv.submit(Request("intersect", -1, 0.0, queries=arena[: 1 << lg], pair_cap=1 << lg))
                srv.drain()
            torch.cuda.synchronize(dev)
            rq = [make(sp) for sp in sp_list]
            t0 = now()
            for r in rq:
                r.arrival = t0
            srv.submit_many(rq)  # one call for the whole burst: the host's per-call cost does not bound it
            srv.drain()
            span = now() - t0
            bst = srv.stats()
            srv.free()
            counts[mode] = [(r.count, r.missed) for r in rq if r.kind == "intersect"]
            out[mode] = {"makespan_ms": span * 1e3, "keys_per_s": total / span, "requests_per_s": len(rq) / span,
                         "batches": bst["batches"], "batched_requests": bst["batched_requests"]}
        if not (counts["batched"] == counts["one_launch_per_request"] == counts["plain_calls"]):
            raise RuntimeError("saturated runs disagree on the intersect counts")
        out["identical_counts"] = True
        out["batched_over_plain_calls"] = out["batched"]["keys_per_s"] / out["plain_calls"]["keys_per_s"]
        out["batched_over_one_launch_per_request"] = (out["batched"]["keys_per_s"] /
                                                      out["one_launch_per_request"]["keys_per_s"])
        return out

    saturated = {"mix": saturated_run(specs),
                 "small_requests": saturated_run(serving_requests(args.requests, args.rate, arena_keys, lo_log2=10,
                                                                  hi_log2=16, seed=7))}
    serial = Server(budget_bytes=1 << 50, max_tables=1 << 30, n_streams=1, max_keys=1 << 24, device=dev,
                    batching=False)
    mismatches, checked = 0, 0
    for sp, r in zip(specs, reqs):
        q = make(sp)
        serial.submit(q)
        serial.drain()
        if q.kind == "intersect" and not r.missed:
            checked += 1
            mismatches += int(q.count != r.count)
    if mismatches:
        raise RuntimeError(f"{mismatches} of {checked} served intersects differ from the serial run")

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": 1, "warmup": 1,
        "ms_per_step": makespan * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic (seeded splitmix64 key arena on the device; requests take slices)",
        "config": {"workload": f"serving: {args.requests} requests, Poisson arrivals at {args.rate}/s, 30% build / "
                               f"70% intersect, sizes 2^U(10,24) u64, <= 512 resident tables, 120 GB budget "
                               f"({RESERVE_BYTES >> 30} GB reserved), LRU, {args.streams} streams, continuous "
                               f"batching of requests up to 2^16 keys",
                   "requests": args.requests, "rate_per_s": args.rate, "keys_total": keys_total,
                   "offered_keys_per_s": keys_total / (specs[-1][2] - specs[0][2]) if len(specs) > 1 else None,
                   "parallelism": "single GPU"},
        "latency": by_kind, "latency_all": latency_summary(done), "missed_intersects": missed,
        "evictions": st["evictions"], "serial_check": {"intersects_checked": checked, "mismatches": 0},
        "batching": {"batches": st["batches"], "batched_requests": st["batched_requests"]},
        "saturated": saturated,
        "clocks": clk, "e2e": None, "gpu_launches": launches, "cpu_baseline": None,
        "note": "native serving engine (hg_server_*); value = keys of all requests / makespan (first arrival "
                "to last completion); latency = arrival to device completion of the request's last kernel",
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# sharded: one table over all ranks by bucket range (hashgraph_b200.shard)
# ---------------------------------------------------------------------------
def run_sharded(args, rank, world, local):
    """Each rank holds n u64 keys and n queries (25% drawn from its keys); one
    step = ShardedTable.build over all ranks' keys into n * world buckets
    (histogram, all-reduce, splits, route, all-to-all, shard build) + the
    intersect of all ranks' queries (route, all-to-all, shard probe with
    pairs, all-reduce of the count).  With one rank the all-to-alls move the
    routed keys to the rank itself; the collectives are NCCL."""
    import socket

    import torch
    import torch.distributed as dist

    import hashgraph_b200 as hg
    from hashgraph_b200.shard import ShardedTable

    dev = torch.device("cuda", local)
    own_group = False
    if not dist.is_initialized():
        sk = socket.socket()
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
        sk.close()
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                                device_id=dev)
        own_group = True
    try:
        kb = 8
        n = args.n or (1 << 28)
        B = n * world
        a = hg.gen_uniform(n, kb, 3 + 1000 * rank, device=dev)
        q = hg.gen_overlap(n, a, 0.25, 4 + 1000 * rank)
        torch.cuda.synchronize(dev)

        def step():
            t = ShardedTable.build(a, B, with_index=True)
            return t, t.intersect(q)

        for _ in range(args.warmup):
            t, r = step()
        torch.cuda.synchronize(dev)
        matches = r.count
        if world == 1:  # the one-shard table against the plain path
            plain = hg.Table.build(a, B, with_index=True)
            c, _ = plain.intersect(q, emit=False)
            if int(c.item()) != matches:
                raise RuntimeError(f"sharded count {matches} != plain count {int(c.item())}")
            del plain
        del t, r
        barrier(world)
        torch.cuda.synchronize(dev)
        clocks = ClockSampler(local)
        launches0 = hg.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        hg.profile_enable(True)
        hg.profile_read()
        clocks.start()
        e0.record()
        for _ in range(args.steps):
            t, r = step()
        e1.record()
        torch.cuda.synchronize(dev)
        clk = clocks.stop()
        phases = {}
        for name, pms in hg.profile_read():
            phases[name] = phases.get(name, 0.0) + pms / args.steps
        hg.profile_enable(False)
        launches = hg.launch_count() - launches0
        barrier(world)
        ms = max_over_ranks(e0.elapsed_time(e1), world) / args.steps
        value = sum_over_ranks(n, world) / (ms * 1e-3)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64",
            "data": "synthetic (seeded splitmix64 keys generated on each rank's device)",
            "config": {"workload": f"sharded: {n} u64 keys + {n} queries (25% overlap) per rank, one table of "
                                   f"{B} buckets over {world} rank(s) by bucket range, index + pairs",
                       "keys_per_rank": n, "n_buckets": B, "matches": matches, "splits": t.splits,
                       "parallelism": f"{world} shard(s), NCCL all-to-all",
                       "l2": "inputs larger than L2; no flush"},
            "phases_ms": phases, "library_ms": sum(phases.values()),
            "clocks": clk, "e2e": None, "gpu_launches": launches, "cpu_baseline": None,
            "note": "device time of whole steps (CUDA events), max over ranks; includes the host reads of the "
                    "route and exchange sizes each step; phases_ms: the library's kernels per step (the rest "
                    "is the collectives and the host round trips)",
        }
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if own_group:
            dist.destroy_process_group()


# ---------------------------------------------------------------------------
# CPU baseline / reference arm
# ---------------------------------------------------------------------------
def cpu_inputs(workload, n_sample):
    """The workload's inputs on the host (the oracle's generators, the same
    definitions as the device generators): n keys per set, at most the
    workload's own n, with the workload's load factor."""
    import oracle
    kb, n_full, bfn, kind, seed_a, seed_q, overlap, with_index = WORKLOADS[workload]
    n = min(n_sample, n_full)
    B = max(1, int(bfn(n_full) * n // n_full))
    if kind == "zipf":
        cdf = oracle.zipf_cdf(1 << 24, 1.1)
        a = oracle.gen_zipf(n, kb, cdf, seed_a)
        q = oracle.gen_zipf(n, kb, cdf, seed_q)
    else:
        a = oracle.gen_uniform(n, kb, seed_a)
        q = oracle.gen_overlap(n, a, overlap, seed_q)
    return n, B, a, q


def cpu_step(workload, B, a, q, threads):
    """One build + intersect on the host: the oracle's multithreaded stable
    build and probe (pairs emitted, as on the GPU).  Zipf sets are counted
    through a hash map of A's distinct keys instead of the probe, whose cost
    is the product of the multiplicities.  Returns (seconds, build s,
    intersect s, count)."""
    import oracle
    kind, with_index = WORKLOADS[workload][3], WORKLOADS[workload][7]
    t0 = time.perf_counter()
    off, k, i = oracle.build(a, B, with_index, threads=threads)
    t1 = time.perf_counter()
    if kind == "zipf":
        c = oracle.join_count_hashed(k, q, max_distinct=1 << 24, threads=threads)
    else:
        c, _ = oracle.intersect(off, k, i, q, pair_cap=q.size, threads=threads)
    t2 = time.perf_counter()
    return t2 - t0, t1 - t0, t2 - t1, c


def cpu_note(workload):
    return ("zipf: build by the oracle's stable counting sort, count through a hash map of A's distinct keys"
            if WORKLOADS[workload][3] == "zipf" else
            "the oracle's multithreaded stable build and probe, pairs emitted")


def cpu_baseline(workload, n_sample, repeats=2):
    import oracle
    threads = oracle.max_threads()
    n, B, a, q = cpu_inputs(workload, n_sample)
    best = min((cpu_step(workload, B, a, q, threads) for _ in range(repeats)), key=lambda x: x[0])
    dt, tb, ti, c = best
    return {"value": n / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} keys per set into {B} buckets (the same seeded inputs"
                      f"{'' if n == WORKLOADS[workload][1] else ', a sample with the same load factor'}), "
                      f"best of {repeats}; build {tb:.3f} s + intersect {ti:.3f} s; {cpu_note(workload)}"}


def run_reference_batched(args):
    """The oracle's multithreaded build + probe over the batched workload's
    pairs, in order, until about --cpu-sample keys (a bounded sample)."""
    import oracle
    sizes, fracs = batched_sizes(args.pairs, 6, 20)
    cores = oracle.max_threads()
    inputs, total = [], 0
    for i in range(args.pairs):
        n = int(sizes[i])
        a = oracle.gen_uniform(n, 8, 100_000 + i)
        q = oracle.gen_overlap(n, a, float(fracs[i]), 200_000 + i)
        inputs.append((a, q, n))
        total += n
        if total >= (args.cpu_sample or 1 << 26) // 4:
            break
    times = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for a, q, n in inputs:
            off, kk, ii = oracle.build(a, n, False, threads=cores)
            oracle.intersect(off, kk, ii, q, pair_cap=n, threads=cores)
        if k >= args.warmup:
            times.append(time.perf_counter() - t0)
    value = total * len(times) / sum(times)
    sample = (f"the first {len(inputs)} of {args.pairs} pairs ({total} keys per set), each built and "
              "probed by the oracle's multithreaded restatement (the reference has no CPU path)")
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sum(times) / len(times) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded splitmix64 keys; same generators as our arm)",
        "config": {"workload": f"batched: {args.pairs} pairs, A_i = 2^U(6,20) u64 uniform keys into B_i = n_i "
                               "buckets, n_i queries with U(0,1) drawn from A_i, pairs emitted",
                   "pairs": args.pairs},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_reference_serving(args):
    """The oracle's multithreaded build + probe over the serving request list,
    serially (no arrivals), until about --cpu-sample keys."""
    import numpy as np

    import oracle
    arena_keys = 1 << 27
    specs = serving_requests(args.requests, args.rate, arena_keys)
    cores = oracle.max_threads()
    need = max(s[3] + s[4] for s in specs)
    arena = oracle.gen_uniform(min(need, arena_keys), 8, 6)
    tables, total, t_sum, k = {}, 0, 0.0, 0
    for kind, tid, _, off, size in specs:
        sl = arena[off:off + size]
        t0 = time.perf_counter()
        if kind == "build":
            tables[tid] = oracle.build(sl, size, False, threads=cores)
        elif tid in tables:
            o, kk, ii = tables[tid]
            oracle.intersect(o, kk, ii, sl, pair_cap=size, threads=cores)
        t_sum += time.perf_counter() - t0
        total += size
        k += 1
        if total >= (args.cpu_sample or 1 << 26):
            break
    value = total / t_sum
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": 1, "steps": 1,
        "warmup": 0, "ms_per_step": t_sum * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded splitmix64 key arena; same request list)",
        "config": {"workload": f"serving: {args.requests} requests at {args.rate}/s, 30% build / 70% intersect, "
                               "sizes 2^U(10,24) u64", "requests": args.requests},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"the first {k} requests ({total} keys), run back to back by the oracle's "
                                   "multithreaded restatement (the reference has no CPU path)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_reference(args, rank, world):
    if rank != 0:
        return
    if args.workload == "batched":
        run_reference_batched(args)
        return
    if args.workload == "serving":
        run_reference_serving(args)
        return
    if args.workload == "sharded":  # the same per-rank work on one host: build + probe of 2^28 u64
        args.workload = "large"
    import oracle
    kb, n, bfn, kind, seed_a, seed_q, overlap, with_index = WORKLOADS[args.workload]
    n = args.n or n
    B = bfn(n)
    cores = oracle.max_threads()
    ns, BB, a, q = cpu_inputs(args.workload, cpu_sample_size(args, n))
    times = []
    for k in range(args.warmup + args.steps):
        dt, tb, ti, c = cpu_step(args.workload, BB, a, q, cores)
        if k >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = ns * len(times) / total
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / len(times) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64" if kb == 8 else "u32",
        "data": "synthetic (seeded splitmix64 keys; same generators as our arm)",
        "config": {"workload": describe(args.workload, kb, n, B, kind, overlap, with_index), "n": n,
                   "n_buckets": B, "key_bytes": kb, "with_index": with_index},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{ns} keys per set into {BB} buckets per step"
                                   f"{' (the whole workload)' if ns == n else ' (a sample with the same load factor)'}; "
                                   f"{cpu_note(args.workload)} (the reference has no CPU build/intersect; this is "
                                   "the oracle's multithreaded restatement of its algorithm)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batched", "serving", "sharded"], default="large")
    ap.add_argument("--requests", type=int, default=3000, help="requests of the serving workload")
    ap.add_argument("--rate", type=float, default=20000.0, help="serving arrivals per second")
    ap.add_argument("--streams", type=int, default=4, help="serving CUDA streams")
    ap.add_argument("--pairs", type=int, default=4096, help="pairs of the batched workload")
    ap.add_argument("--n", type=int, default=0, help="override keys per set (parity/profiling runs)")
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="keys per set of the CPU arm (0: the workload's own, at most 2^28)")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-ref-gpu", action="store_true", help="do not time the reference's GPU build")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--build-path", choices=["auto", "direct", "partitioned"], default="auto")
    ap.add_argument("--probe-path", choices=["auto", "direct", "partitioned"], default="auto")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        run_reference(args, rank, world)
        return
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.workload == "batched":
            run_batched(args, rank, world, local)
        elif args.workload == "serving":
            run_serving(args, rank, world, local)
        elif args.workload == "sharded":
            run_sharded(args, rank, world, local)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
