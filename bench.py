#!/usr/bin/env python
"""Benchmark of the batched rotated photon-pair correlator.

Workload (the configuration the headline metric is quoted on): 1024x512
two-panel detector, 5 % masked, 100 000 frames whose photon counts are
Poisson(lambda_f) with lambda_f log-normal (median 80, sigma 0.8), uniform SO(3)
orientation per frame, 201^3 uint64 mesh (MeshSize 199), nearest/nearest with
double mapping, Multiplicator 1000.  Seeded synthetic data of that shape.

One step = the whole batch through the hot path: clear the half mesh, plan the
work queue, bin every photon pair (persistent kernel), fold into the full mesh.
`value` times steps with inputs resident in HBM; `e2e` times the C-ABI host
entry point (pinned host photon lists in, full mesh out) per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank bins its own 100 000 frames (weak scaling)
and the per-rank meshes are summed on rank 0 with one NCCL reduce per step.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "pixel pairs/s into 3D q-mesh"
UNIT = "pairs/s"
WORKLOAD = "rotated correlator: 1024x512 two-panel detector, 100k log-normal frames, SO(3), 201^3 u64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=100_000)
    ap.add_argument("--cpu-frames", type=int, default=1500,
                    help="frames per CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world, local, backend="nccl"):
    import datetime

    import torch
    import torch.distributed as dist
    if world > 1 and not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world > 1


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

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
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's route for these frames on the host cores
# ---------------------------------------------------------------------------
def cpu_baseline(cfg, nframes: int, repeats: int = 1):
    """The reference sends frames with fewer than 1 % hit pixels through its
    OpenMP CPU route (ACMesh::Atomic_Add_q_Entry, IAC/Detector.cpp:1025-1050);
    every frame of this workload qualifies.  That route is timed here in its C
    restatement (the reference's ACMesh.cpp needs Boost/Eigen/HDF5/OpenCL
    headers and does not build on its own), on all host cores, on the first
    `nframes` frames.  Best of `repeats`."""
    import oracle
    from incohautocorrelate_b200 import capi
    shape = oracle.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    off = cfg["offsets"][: nframes + 1]
    ph = cfg["photons"][: int(off[-1])]
    rot = cfg["rot"][:nframes]
    pairs = _pairs(off)
    best = None
    for _ in range(repeats):
        t0 = time.perf_counter()
        oracle.sparse_batch(ph, off, rot, shape, cpu_gpu=-1, det_pixels=cfg["npix"])
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    del capi
    return pairs / best, best, pairs


def _pairs(off):
    n = np.diff(np.asarray(off, np.int64))
    return int((n * (n + 1) // 2).sum())


def cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    from incohautocorrelate_b200 import workloads as W
    cfg = W.rotated_config(nframes=args.cpu_frames * max(1, args.steps + args.warmup) + 1, seed=2)
    nthreads = cores()
    os.environ.setdefault("OMP_NUM_THREADS", str(nthreads))
    import oracle
    shape = oracle.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    f = args.cpu_frames
    times, pairs = [], []
    for s in range(args.warmup + args.steps):
        off = cfg["offsets"][s * f: (s + 1) * f + 1]
        ph = cfg["photons"][int(off[0]): int(off[-1])]
        rot = cfg["rot"][s * f: (s + 1) * f]
        t0 = time.perf_counter()
        oracle.sparse_batch(ph, off - off[0], rot, shape, cpu_gpu=-1, det_pixels=cfg["npix"])
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
            pairs.append(_pairs(off))
    value = sum(pairs) / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32+u64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_frames_per_step": f, "mesh": 201},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": f"{f} frames per step of the 100k-frame workload through the "
                                   "reference's CPU route (its choice for <1% hit pixels), "
                                   "OpenMP on all host threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def committed_traffic():
    """dram bytes per launch of the pair kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "sparse_pairs_rotated.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return d.get("dram_bytes_per_full_launch")
    return None


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    distributed = init_dist(world, local)
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    import torch.distributed as dist

    from incohautocorrelate_b200 import capi
    from incohautocorrelate_b200 import workloads as W

    cfg = W.rotated_config(nframes=args.frames, seed=2 + 7919 * rank)
    ph_h, off_h, rot_h = cfg["photons"], cfg["offsets"], cfg["rot"]
    nframes = len(off_h) - 1
    pairs = _pairs(off_h)
    ctx = capi.Context(dev)
    shape = capi.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    S = shape.size_ab
    params = capi.sparse_params(shape, capi.NEAREST, capi.NEAREST, True, 1000.0)

    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    ph = torch.from_numpy(ph_h).cuda()
    off = torch.from_numpy(off_h.view(np.int64)).cuda()
    rot = torch.from_numpy(rot_h).cuda()
    half = torch.zeros(capi.half_mesh_words(S), dtype=torch.int64, device="cuda")
    full = torch.zeros(capi.full_mesh_words(S), dtype=torch.int64, device="cuda")

    # -- the L2 atomic rate the pair kernel is bound by (same footprint) ------
    def scatter_rate(bits):
        scratch = torch.zeros(capi.half_mesh_words(S), dtype=torch.int64, device="cuda")
        upd = 1 << 30
        ctx.bench_scatter_add(scratch, scratch.numel(), bits, upd // 8, 1, sptr)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.bench_scatter_add(scratch, scratch.numel(), bits, upd, 2, sptr)
        e1.record(stream)
        torch.cuda.synchronize()
        return upd / (e0.elapsed_time(e1) * 1e-3)
    atomic_peak = scatter_rate(64)
    atomic_peak_u32 = scatter_rate(32)

    ev = []

    def step(record=False):
        half.zero_()
        full.zero_()
        if record:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
        ctx.sparse_ac_batch(ph, off, rot, nframes, params, half, sptr)
        if record:
            b.record(stream)
            ev.append((a, b))
        ctx.sparse_fold(half, S, full, sptr)
        if distributed:
            dist.reduce(full, dst=0)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if distributed:
        dist.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    l0 = ctx.launches()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if distributed:
        dist.barrier()
    t_start.record(stream)
    for _ in range(args.steps):
        step(record=True)
    t_end.record(stream)
    torch.cuda.synchronize()
    if distributed:
        dist.barrier()
    launches = ctx.launches() - l0
    clk = clocks.stop()
    ms = t_start.elapsed_time(t_end)
    ms_kernel = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
    oob = ctx.check(sptr)
    if distributed:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_pairs = pairs * world
    value = total_pairs * args.steps / (ms * 1e-3)

    # -- end to end through the C-ABI host entry point (pinned host buffers) --
    ph_p = torch.from_numpy(ph_h).pin_memory()
    off_p = torch.from_numpy(off_h.view(np.int64)).pin_memory()
    rot_p = torch.from_numpy(rot_h).pin_memory()
    mesh_p = torch.zeros(capi.full_mesh_words(S), dtype=torch.int64).pin_memory()
    for _ in range(max(1, args.warmup // 2)):
        ctx.sparse_ac_frames_host(ph_p, off_p, rot_p, nframes, params, mesh_p)
    e2e_times = []
    for _ in range(max(2, args.steps // 2)):
        mesh_p.zero_()
        t0 = time.perf_counter()
        ctx.sparse_ac_frames_host(ph_p, off_p, rot_p, nframes, params, mesh_p)
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = statistics.median(e2e_times)
    if distributed:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = ph_h.nbytes + off_h.nbytes + rot_h.nbytes + 8 * capi.full_mesh_words(S)
    d2h = 8 * capi.full_mesh_words(S)

    # -- roofline of the pair kernel --------------------------------------
    # algorithmic bytes per launch: one 8-byte read-modify-write (16 B) per
    # mesh update (pairs off the ss = 0 plane update once, on it twice; self
    # pairs of a frame are summed into one update) plus 16 B per photon read.
    hbm_peak, peak_kind = measured_peaks()
    updates = pairs - int(len(ph_h))  # distinct pairs: ~one update each
    alg_bytes = 16.0 * updates + 16.0 * len(ph_h)
    achieved = alg_bytes / (ms_kernel * 1e-3) / 1e9
    traffic = committed_traffic()
    upd_rate = updates / (ms_kernel * 1e-3)

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32+u64", "data": "synthetic (seeded; shapes of the rotated-correlator "
                                              "configuration)",
            "config": {"workload": WORKLOAD, "frames_per_gpu": nframes, "pairs_per_gpu": pairs,
                       "photons_per_gpu": int(len(ph_h)), "mesh": S,
                       "interpolation": "nearest/nearest, double mapping",
                       "l2": "inputs larger than L2 (photon lists 176 MB > 126 MB)",
                       "parallelism": f"frame-sharded dp{world}" if world > 1 else "1 GPU",
                       "tuning": ctx.sparse_tuning(S)},
            "clocks": clk, "gpu_launches": launches,
            "out_of_mesh_writes": oob,
            "e2e": {"value": total_pairs / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "seconds_per_step": e2e_s},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic,
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "kernel": "sparse_pairs_kernel (+ planner)",
                         "kernel_ms": ms_kernel,
                         "limiter": "L2 64-bit atomic adds",
                         "atomic_updates_per_s": upd_rate,
                         "atomic_peak_per_s": atomic_peak,
                         "atomic_frac": upd_rate / atomic_peak,
                         "atomic_peak_u32_per_s": atomic_peak_u32,
                         "atomic_peak_source": "measured in this run: 2^30 scattered u64 atomic "
                                               "adds into a buffer of the half-mesh size"},
        }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nthreads = cores()
        v, secs, cp = cpu_baseline(cfg, min(args.cpu_frames, nframes))
        line["cpu_baseline"] = {
            "value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"first {min(args.cpu_frames, nframes)} frames ({cp} pairs, {secs:.1f} s) "
                      "through the reference's CPU route, OpenMP on all host threads"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if distributed:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
