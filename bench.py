#!/usr/bin/env python
"""Benchmark of the batched rotated photon-pair correlator and the rest of
the pair-correlation path.

Workload of the headline metric: 1024x512 two-panel detector, 5 % masked,
100 000 frames whose photon counts are Poisson(lambda_f) with lambda_f
log-normal (median 80, sigma 0.8), uniform SO(3) orientation per frame, 201^3
uint64 mesh (MeshSize 199), nearest/nearest with double mapping,
Multiplicator 1000.  Seeded synthetic data of that shape.

One step = the whole batch through the hot path: clear the half mesh, plan the
work queue, bin every photon pair (persistent kernel), fold into the full mesh.
`value` times steps with inputs resident in HBM; `e2e` times the C-ABI host
entry point with pinned host photon lists, the batches of a run accumulating
into a device-resident mesh that is folded and read back once at the end of
the run.  On one GPU the line also carries `parts`: one timed step of each
other part of the path on its configuration (dense C(q) and AC1D C(q) on
1024^2, the C(q) merge, AC1D of sparse frames with the reference's route
choice, the simulator feeding the correlator, the denoiser's training step and
a frames-to-error check of the committed denoiser weights).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--scaling weak|strong] [--no-parts] [--kernel PART]

Under torchrun (N > 1) every rank bins its own 100 000 frames (--scaling weak)
or a pair-balanced share of one 100 000-frame batch (--scaling strong), and
the per-rank meshes are summed on rank 0 with one NCCL reduce per step.
"""
from __future__ import annotations

import argparse
import ctypes as C
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
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="multi-GPU runs: weak = 100 000 frames per rank, strong = one 100 000-frame "
                         "batch shared by the ranks")
    ap.add_argument("--cpu-frames", type=int, default=1500,
                    help="frames per step of the --impl reference arm")
    ap.add_argument("--cpu-baseline-frames", type=int, default=100_000,
                    help="frames of the cpu_baseline sample (all 100 000: about 8 s on 16 host threads)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parts", action="store_true",
                    help="headline only: skip the timed step of every other part of the path")
    ap.add_argument("--f2e-crystals", type=int, default=4,
                    help="held-out crystals of the frames-to-error part")
    ap.add_argument("--det", type=int, default=1024,
                    help="edge of the square detector of the dense kernels (1024 = their config)")
    ap.add_argument("--backend", type=int, default=0,
                    help="denoiser convolutions: 0 = tcgen05 + TMEM, 1 = mma.sync")
    ap.add_argument("--dn-batch", type=int, default=8,
                    help="denoiser training patches per step (8 = the training configuration)")
    ap.add_argument("--no-layers", action="store_true",
                    help="--kernel denoise: skip timing every layer shape alone")
    ap.add_argument("--kernel", default="sparse",
                    choices=["sparse", "cq_small", "ac1d_cq", "cq_merge", "ac1d_sparse", "ac1d_uw", "simulate",
                             "denoise", "frames_to_error", "average"],
                    help="sparse is the headline; the others print one line for that part of the path "
                         "on its configuration")
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
    """SM clock and clock-event reasons of the device, polled through NVML every
    10 ms from a thread while the timed region runs (reads only; nvidia-smi
    polling as the fallback when NVML is unavailable)."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []
        self.nvml = None
        self.samples = []
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            try:
                import torch
                pr = torch.cuda.get_device_properties(device_index)
                h = pynvml.nvmlDeviceGetHandleByPciBusId(
                    f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0")
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self.nvml, self.handle = pynvml, h
        except Exception:
            self.nvml = None

    def start(self):
        if self.nvml is not None:
            self.samples, self._stop = [], threading.Event()

            def poll():
                n = self.nvml
                while not self._stop.is_set():
                    try:
                        self.samples.append((n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM),
                                             n.nvmlDeviceGetCurrentClocksEventReasons(self.handle)))
                    except Exception:
                        pass
                    self._stop.wait(0.01)

            self._t = threading.Thread(target=poll, daemon=True)
            self._t.start()
            return
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
        if self.nvml is not None:
            n = self.nvml
            try:  # one more sample at the end of the timed region
                self.samples.append((n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM),
                                     n.nvmlDeviceGetCurrentClocksEventReasons(self.handle)))
            except Exception:
                pass
            self._stop.set()
            self._t.join(timeout=2)
            sm = [c for c, _ in self.samples]
            reasons = set()
            for _, r in self.samples:
                for name, const in self.REASONS:
                    if r & getattr(self.nvml, const, 0):
                        reasons.add(name)
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, 10 ms"}
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
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 100 ms"}


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


def measured_bf16_tflops():
    """(sustained dense bf16 TFLOP/s, source) from MEASURED_PEAKS.json."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        if "bf16_tflops_sustained" in d:
            return float(d["bf16_tflops_sustained"]), "measured bf16_tflops_sustained"
    return 1400.0, "fallback (1.4 PFLOP/s sustained)"


def pair_box_radius(C, ctas_per_sm):
    """Half-width of the pair kernel's shared-memory box around q = 0 for a
    tuning row (the library's rule: 10, shrunk until ctas_per_sm boxes of
    (R + 1)(2R + 1)^2 words fit in 200 KB, at most the mesh centre)."""
    budget = (200 << 10) // max(1, ctas_per_sm)
    r = min(10, C)
    while r > 0 and 8 * (r + 1) * (2 * r + 1) ** 2 > budget:
        r -= 1
    return r


def box_value_share(half, S, R, self_sum):
    """Share of the distinct pairs' mesh value that lands in the box of
    half-width R around q = 0 (ss <= R, |fs - C| <= R, |ms - C| <= R); the
    self pairs (all at the centre) are left out.  With photon counts mostly 1
    this is close to the share of the pair kernel's updates the box takes."""
    import torch
    C = (S - 1) // 2
    h = half.view(-1)[: S * S * ((S + 1) // 2)].view((S + 1) // 2, S, S)
    tot = float(h.double().sum().item()) - self_sum
    box = float(h[: R + 1, C - R: C + R + 1, C - R: C + R + 1].double().sum().item()) - self_sum
    return box / tot if tot > 0 else 0.0


def run_ours(args):
    import torch
    rank, world, local = dist_env()
    distributed = init_dist(world, local)
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    import torch.distributed as dist

    from incohautocorrelate_b200 import capi, shard

    ph_h, off_h, rot_h, cfg = shard.rank_workload(rank, world, args.scaling, args.frames, seed=2)
    nframes = len(off_h) - 1
    pairs = _pairs(off_h)
    ctx = capi.Context(dev)
    shape = capi.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    S = shape.size_ab
    params = capi.sparse_params(shape, capi.NEAREST, capi.NEAREST, True, 1000.0)
    total_pairs = pairs
    if distributed:
        t = torch.tensor([pairs], dtype=torch.int64, device="cuda")
        dist.all_reduce(t)
        total_pairs = int(t.item())

    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    ph = torch.from_numpy(ph_h).cuda()
    off = torch.from_numpy(off_h.view(np.int64)).cuda()
    rot = torch.from_numpy(rot_h).cuda()
    half = torch.zeros(capi.half_mesh_words(S), dtype=torch.int64, device="cuda")
    full = torch.zeros(capi.full_mesh_words(S), dtype=torch.int64, device="cuda")

    # -- the L2 atomic rate the pair kernel is bound by (same footprint) ------
    atomic_peak = scatter_rate(ctx, stream, capi.half_mesh_words(S), 64)
    atomic_peak_u32 = scatter_rate(ctx, stream, capi.half_mesh_words(S), 32)

    ev = []

    def step(record=False):
        full.zero_()  # clear the full mesh first so the half mesh is the L2-resident one
        half.zero_()
        if record:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
        ctx.sparse_ac_batch(ph, off, rot, nframes, params, half, sptr)
        if record:
            b.record(stream)
            ev.append((a, b))
        ctx.sparse_fold(half, S, full, sptr)
        if distributed:
            shard.reduce_mesh(full, dst=0)

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
    value = total_pairs * args.steps / (ms * 1e-3)

    # -- the same step captured once in a CUDA graph and replayed (1 GPU) --
    graph_ms = None
    if not distributed:
        cap = torch.cuda.Stream()
        cap.wait_stream(stream)

        def body():
            full.zero_()
            half.zero_()
            ctx.sparse_ac_batch(ph, off, rot, nframes, params, half, cap.cuda_stream)
            ctx.sparse_fold(half, S, full, cap.cuda_stream)

        with torch.cuda.stream(cap):  # the capture stream's scratch exists before capture
            body()
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=cap):
            body()
        graph.replay()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for _ in range(args.steps):
            graph.replay()
        g1.record(stream)
        torch.cuda.synchronize()
        graph_ms = g0.elapsed_time(g1) / args.steps
        del graph

    # -- roofline of the pair kernel: L2 64-bit atomic updates ---------------
    # one update per distinct pair (two on the ss = 0 plane, one per frame for
    # its summed self pairs); the denominator is the scattered-atomic rate
    # measured above on a buffer of the half mesh's size.  The voxels within R
    # of q = 0 go to each CTA's shared-memory box instead of L2.
    step()
    torch.cuda.synchronize()
    updates = pairs - int(len(ph_h))
    upd_rate = updates / (ms_kernel * 1e-3)
    tun = ctx.sparse_tuning(S)
    R = pair_box_radius((S - 1) // 2, tun["ctas_per_sm"])
    self_sum = 1000.0 * float((ph_h[:, 3].astype(np.float64) ** 2).sum())
    share = box_value_share(half, S, R, self_sum) if R > 0 else 0.0

    # -- end to end: pinned host photon lists -> device-resident mesh --------
    ph_p = torch.from_numpy(ph_h).pin_memory()
    off_p = torch.from_numpy(off_h.view(np.int64)).pin_memory()
    rot_p = torch.from_numpy(rot_h).pin_memory()
    mesh_p = torch.zeros(capi.full_mesh_words(S), dtype=torch.int64).pin_memory()
    e_half = torch.zeros_like(half)
    e_full = torch.zeros_like(full)

    def e2e_run(nsteps):
        e_half.zero_()
        e_full.zero_()
        for _ in range(nsteps):
            ctx.sparse_ac_frames_host_to_device(ph_p, off_p, rot_p, nframes, params, e_half, sptr)
        ctx.sparse_fold(e_half, S, e_full, sptr)
        if distributed:
            shard.reduce_mesh(e_full, dst=0)
        if rank == 0:
            mesh_p.copy_(e_full, non_blocking=True)
        torch.cuda.synchronize()

    e2e_run(1)
    if distributed:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_run(args.steps)
    e2e_s = time.perf_counter() - t0
    if distributed:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = ph_h.nbytes + off_h.nbytes + rot_h.nbytes
    d2h = 8 * capi.full_mesh_words(S) / args.steps if rank == 0 else 0

    # the reference's per-call contract: every call uploads the caller's host
    # mesh and reads it back (iac_sparse_ac_frames_host), median of 15 calls
    sync_call = None
    if not distributed:
        ctx.sparse_ac_frames_host(ph_p, off_p, rot_p, nframes, params, mesh_p)
        tt = []
        for _ in range(max(15, args.steps)):
            t0 = time.perf_counter()
            ctx.sparse_ac_frames_host(ph_p, off_p, rot_p, nframes, params, mesh_p)
            tt.append(time.perf_counter() - t0)
        sync_s = statistics.median(tt)
        sync_call = {"value": pairs / sync_s, "unit": UNIT, "seconds_per_call": sync_s,
                     "h2d_bytes_per_call": int(h2d + 8 * capi.full_mesh_words(S)),
                     "d2h_bytes_per_call": int(8 * capi.full_mesh_words(S)),
                     "note": "iac_sparse_ac_frames_host: the caller's 65 MB host mesh is uploaded and read "
                             "back on every call (+= semantics of ACMesh::Mesh per batch)"}

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": args.scaling, "vs_baseline": None,
            "dtype": "fp32+u64", "data": "synthetic (seeded; shapes of the rotated-correlator "
                                              "configuration)",
            "config": {"workload": WORKLOAD, "frames_per_gpu": nframes, "pairs_per_gpu": pairs,
                       "batch_frames": cfg["batch_frames"], "pairs_total": total_pairs,
                       "photons_per_gpu": int(len(ph_h)), "mesh": S,
                       "interpolation": "nearest/nearest, double mapping",
                       "l2": "inputs larger than L2 (photon lists 176 MB > 126 MB)",
                       "parallelism": (f"frame-sharded dp{world} ({args.scaling} scaling)" if world > 1
                                       else "1 GPU"),
                       "tuning": tun},
            "clocks": clk, "gpu_launches": launches,
            "graph": None if graph_ms is None else {
                "ms_per_step": graph_ms, "value": total_pairs / (graph_ms * 1e-3),
                "note": "the step (clear, plan, bin, fold) captured in one CUDA graph and replayed"},
            "out_of_mesh_writes": oob,
            "e2e": {"value": total_pairs * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "seconds_per_step": e2e_s / args.steps,
                    "frac_of_value": (total_pairs * args.steps / e2e_s) / value,
                    "note": f"{args.steps} batches of pinned host photon lists "
                            "(iac_sparse_ac_frames_host_to_device: chunked copies overlapping the binning) "
                            "accumulate into a device-resident mesh that is folded and read back once at "
                            "the end of the run; d2h per step = the 65 MB mesh / steps"},
            "e2e_sync_call": sync_call,
            "roofline": {"bound": "l2_atomic", "achieved": upd_rate, "peak": atomic_peak,
                         "unit": "updates/s", "frac": upd_rate / atomic_peak, "traffic": None,
                         "peak_source": "measured in this run: 2^30 scattered u64 atomic adds into a buffer "
                                        "of the half mesh's size (iac_bench_scatter_add)",
                         "kernel": "sparse_pairs_kernel (+ planner)", "kernel_ms": ms_kernel,
                         "updates_per_launch": updates,
                         "box": {"radius": R, "value_share": share,
                                 "l2_updates_per_s": upd_rate * (1 - share),
                                 "l2_frac": upd_rate * (1 - share) / atomic_peak,
                                 "note": "updates within R of q = 0 go to a per-CTA shared-memory box; "
                                         "l2_frac counts only the updates that reach L2 (box share "
                                         "estimated from the mesh value it holds)"},
                         "atomic_peak_u32_per_s": atomic_peak_u32,
                         "traffic_note": "DRAM bytes are not measured in the run; the half mesh stays in "
                                         "L2 and each photon is read once"},
        }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nthreads = cores()
        nb = min(args.cpu_baseline_frames, nframes)
        v, secs, cp = cpu_baseline(cfg, nb)
        line["cpu_baseline"] = {
            "value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"first {nb} frames ({cp} pairs, {secs:.1f} s) "
                      "through the reference's CPU route, OpenMP on all host threads"}
    if rank == 0 and world == 1 and not args.no_parts:
        line["parts"] = run_parts(args, ctx, stream, atomic_peak)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if distributed:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def scatter_rate(ctx, stream, words, bits):
    """Scattered atomic adds per second into a buffer of `words` words."""
    import torch
    scratch = torch.zeros(words, dtype=torch.int64, device="cuda")
    upd = 1 << 30
    sptr = stream.cuda_stream
    ctx.bench_scatter_add(scratch, scratch.numel(), bits, upd // 8, 1, sptr)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ctx.bench_scatter_add(scratch, scratch.numel(), bits, upd, 2, sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    return upd / (e0.elapsed_time(e1) * 1e-3)


# ---------------------------------------------------------------------------
# the other parts of the path, each on its configuration
# ---------------------------------------------------------------------------
def _fp32_peak_tflops(clock_mhz):
    """FP32 FMA peak of 148 SMs x 128 lanes x 2 flop at the sampled clock (no
    measured FP32 figure exists for this pool; derived, not measured)."""
    return 148 * 128 * 2 * clock_mhz * 1e6 / 1e12


def _time(fn, steps, warmup, stream):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def _dense_inputs(ny, nx, gap=None):
    from incohautocorrelate_b200 import workloads as W
    I = W.radial_mean_intensity(ny, nx, 300.0, 0.02, 0.05, seed=3)
    pm = W.flat_pixel_map(ny, nx, gap_x=2e-3 if gap else 0.0, gap_after=gap)
    km, mq = W.kmap_numpy(pm)
    return I, km, mq


def _fp32_roofline(rate, flops, clk, what):
    mhz = clk.get("sm_mhz") or 1965.0
    peak = _fp32_peak_tflops(mhz)
    return {"bound": "fp32", "achieved": rate * flops / 1e12, "peak": peak, "unit": "TFLOP/s",
            "frac": rate * flops / 1e12 / peak, "flop_per_unit": flops, "unit_of_work": what,
            "peak_source": "derived: 148 SM x 128 FP32 lanes x 2 at the sampled clock (no measured FP32 peak)"}


def part_dense(kind, args, ctx, stream, steps, warmup, nthreads):
    """All 5.5e11 unordered pixel pairs of the 1024^2 radial mean-intensity
    map: nearest-voxel C(q) on the 255-edge small mesh, or the 2 048-bin
    linear AC1D histogram."""
    import torch
    import oracle
    from incohautocorrelate_b200 import capi
    sp = stream.cuda_stream
    I, km, mq = _dense_inputs(args.det, args.det)
    npix = I.size
    dI, dk = torch.from_numpy(I).cuda(), torch.from_numpy(km).cuda()
    pairs = npix * (npix + 1) // 2
    if kind == "cq_small":
        sh = capi.small_cq_mesh_shape(mq, 253)
        mult = capi.cq_small_multiplicator(I)
        out = torch.zeros(sh.size_ab * sh.size_ab * sh.size_c, dtype=torch.int64, device="cuda")
        fn = lambda: (out.zero_(), ctx.cq_small(dI, dk, npix, sh, 0, mult, out, sp, fast_size=args.det))
        desc = f"small C(q) mesh {sh.size_ab}x{sh.size_ab}x{sh.size_c}, nearest"
        # diff 3, norm 5, product 1, scale 3
        flops = 12.0
    else:
        sh = capi.ac1d_shape(mq, 2048)
        mult = capi.ac1d_cq_multiplicator(I)
        out = torch.zeros(sh.size, dtype=torch.int64, device="cuda")
        fn = lambda: (out.zero_(), ctx.ac1d_cq(dI, dk, npix, sh, 1, mult, out, sp))
        desc = "AC1D 2048 bins, linear"
        # diff 3, norm 5, product 1, sqrt 1, divide 1
        flops = 11.0
    clocks = ClockSampler(0)
    clocks.start()
    ms = _time(fn, steps, warmup, stream)
    clk = clocks.stop()
    rate = pairs / (ms * 1e-3)
    res = {"metric": f"pixel pairs/s into {desc}", "value": rate, "unit": "pairs/s", "ms_per_step": ms,
           "steps": steps, "dtype": "fp32+u64",
           "config": {"workload": f"{args.det}x{args.det} radial mean intensity, 5% masked, "
                                  f"all {pairs:.3g} unordered pixel pairs", "pixels": npix},
           "clocks": clk, "roofline": _fp32_roofline(rate, flops, clk, "unordered pixel pair")}
    if not args.no_cpu_baseline:
        rows = 48
        t0 = time.perf_counter()
        if kind == "cq_small":
            so = oracle.small_cq_mesh_shape(mq, 253)
            m = np.zeros(so.size_ab * so.size_ab * so.size_c, np.uint64)
            oracle.lib().iaco_cq_small(oracle.p(I), oracle.p(km), npix, so, 0, mult, npix // 2, npix // 2 + rows,
                                       oracle.p(m))
        else:
            so = oracle.ac1d_shape(mq, 2048)
            m = np.zeros(so.size, np.uint64)
            oracle.lib().iaco_ac1d_cq(oracle.p(I), oracle.p(km), npix, so, 1, mult, npix // 2, npix // 2 + rows,
                                      oracle.p(m))
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": rows * npix / 2 / dt, "unit": "pairs/s", "cores": nthreads, "kind": "port",
                               "sample": f"{rows} work items (rows) x {npix} pixels of the reference's ordered-pair "
                                         f"loop ({dt:.1f} s, OpenMP over rows), counted as unordered pairs "
                                         "(2 ordered = 1)"}
    return res


def part_cq_merge(args, ctx, stream, steps, warmup, nthreads, atomic_peak):
    """Merge_CQ: every non-zero voxel of the 1024x512 detector's small C(q)
    mesh rotated by each of 100 000 SO(3) frames into the 201^3 mesh."""
    import torch
    import oracle
    from incohautocorrelate_b200 import capi
    from incohautocorrelate_b200 import workloads as W
    sp = stream.cuda_stream
    I, km, mq = _dense_inputs(512, 1024, gap=512)
    npix = I.size
    sh = capi.small_cq_mesh_shape(mq, 199)
    mult = capi.cq_small_multiplicator(I)
    small_u = torch.zeros(sh.size_ab * sh.size_ab * sh.size_c, dtype=torch.int64, device="cuda")
    ctx.cq_small(torch.from_numpy(I).cuda(), torch.from_numpy(km).cuda(), npix, sh, 0, mult, small_u, sp,
                 fast_size=1024)
    small = small_u.cpu().numpy().view(np.uint64).astype(np.float64) / mult
    nf = args.frames
    R = W.haar_rotations(nf, seed=3)
    MI = np.random.default_rng(4).uniform(0.5e-4, 4e-4, nf).astype(np.float32)
    rw, m = capi.cq_merge_weights(R, MI, small)
    d_small, d_rw = torch.from_numpy(small).cuda(), torch.from_numpy(rw).cuda()
    big = torch.zeros(sh.size_ab ** 3, dtype=torch.int64, device="cuda")
    nvox = int((small >= np.float32(1e-37)).sum())
    fn = lambda: (big.zero_(), ctx.cq_merge(d_small, d_rw, nf, sh, 0, m, big, sp))
    clocks = ClockSampler(0)
    clocks.start()
    ms = _time(fn, steps, warmup, stream)
    clk = clocks.stop()
    rate = nvox * nf / (ms * 1e-3)
    res = {"metric": "voxel-frame scatters/s (C(q) merge)", "value": rate, "unit": "scatters/s",
           "ms_per_step": ms, "steps": steps, "dtype": "fp32+u64",
           "config": {"workload": f"small C(q) {sh.size_ab}x{sh.size_ab}x{sh.size_c} ({nvox} non-zero voxels) "
                                  f"x {nf} SO(3) frames into {sh.size_ab}^3"},
           "clocks": clk,
           "roofline": {"bound": "l2_reduction", "achieved": rate, "unit": "updates/s", "peak": None, "frac": None,
                        "scattered_atomic_rate": atomic_peak, "vs_scattered_atomic_rate": rate / atomic_peak,
                        "note": "one 64-bit L2 reduction per (voxel, frame); updates of consecutive small-mesh "
                                "voxels coalesce into shared L2 reduction requests, so the rate can exceed the "
                                "scattered-atomic rate of this run (one request per update): no measured peak "
                                "applies, the fraction is left out"}}
    if not args.no_cpu_baseline:
        sub = min(nvox, 20000)
        so = oracle.small_cq_mesh_shape(mq, 199)
        out = np.zeros(sh.size_ab ** 3, np.uint64)
        nz = np.nonzero(small >= np.float32(1e-37))[0]
        v0 = int(nz[len(nz) // 2])
        t0 = time.perf_counter()
        oracle.lib().iaco_cq_merge(oracle.p(small), oracle.p(rw.reshape(-1)), min(nf, 2000), so, 0, m, v0, v0 + sub,
                                   oracle.p(out))
        dt = time.perf_counter() - t0
        done = int(((small[v0:v0 + sub]) >= np.float32(1e-37)).sum()) * min(nf, 2000)
        res["cpu_baseline"] = {"value": done / dt, "unit": "scatters/s", "cores": nthreads, "kind": "port",
                               "sample": f"{sub} voxels x {min(nf, 2000)} frames of the reference's Merge_CQ loop"}
    return res


def part_ac1d(kind, args, ctx, stream, steps, warmup, nthreads):
    """AC1D of the rotated-correlator frames (100 000 frames, 2 048 bins).
    "ac1d_uw": the reference's per-frame route choice; every frame of this
    workload has fewer than 0.75 % hits and takes the host loop (k >= j, factor
    2), run on the device, nearest binning.  "ac1d_sparse": the
    AutoCorr_sparseHL_AAV kernel's route forced on every frame, linear."""
    import torch
    import oracle
    from incohautocorrelate_b200 import capi
    from incohautocorrelate_b200 import workloads as W
    sp = stream.cuda_stream
    cfg = W.rotated_config(nframes=args.frames, seed=2)
    sh = capi.ac1d_shape(cfg["max_q"], 2048)
    ph = torch.from_numpy(cfg["photons"]).cuda()
    off = torch.from_numpy(cfg["offsets"].view(np.int64)).cuda()
    nf = len(cfg["offsets"]) - 1
    if kind == "ac1d_uw":
        acc = torch.zeros(capi.ac1d_uw_words(sh), dtype=torch.int64, device="cuda")
        uw = torch.zeros(sh.size, dtype=torch.float64, device="cuda")
        fn = lambda: (acc.zero_(), ctx.ac1d_uw_batch(ph, off, nf, cfg["npix"], sh, 0, acc, stream=sp),
                      ctx.ac1d_uw_finish(acc, sh, uw, sp))
        desc = "reference route choice (all frames: host loop, k >= j), nearest"
    else:
        vs = capi.ac1d_vecsize(sh.max_q, sh.dq_per_step)
        hist = torch.zeros(vs, dtype=torch.int64, device="cuda")
        fn = lambda: (hist.zero_(), ctx.ac1d_sparse_batch(ph, off, nf, sh.max_q, sh.dq_per_step, 1, 100.0, hist, sp))
        desc = "device route (ordered pairs), linear"
    clocks = ClockSampler(0)
    clocks.start()
    ms = _time(fn, steps, warmup, stream)
    clk = clocks.stop()
    pairs = _pairs(cfg["offsets"])
    rate = pairs / (ms * 1e-3)
    res = {"metric": "photon pairs/s into the AC1D histogram", "value": rate, "unit": "pairs/s", "ms_per_step": ms,
           "steps": steps, "dtype": "fp32+u64/f64", "clocks": clk,
           "config": {"workload": f"{nf} rotated-correlator frames (1024x512), 2048 bins, {desc}"},
           "roofline": _fp32_roofline(rate, 11.0, clk, "unordered photon pair (diff 3, norm 5, product 1, "
                                                       "sqrt 1, divide 1)")}
    if not args.no_cpu_baseline and kind == "ac1d_uw":
        f = 3000
        off_h = cfg["offsets"][: f + 1]
        ac = np.zeros(sh.size)
        t0 = time.perf_counter()
        oracle.lib().iaco_ac1d_uw_frames(oracle.p(cfg["photons"]), oracle.p(off_h), f, cfg["npix"], sh.max_q,
                                         sh.dq_per_step, sh.size, 0, -1, oracle.p(ac))
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": _pairs(off_h) / dt, "unit": "pairs/s", "cores": 1, "kind": "port",
                               "sample": f"first {f} frames through the reference's host loop "
                                         f"(Calculate_AC_UW_Mapped, one thread per frame range; {dt:.2f} s)"}
    return res


def part_average(args, ctx, stream, steps, warmup, nthreads):
    """LoadAndAverageIntensity on the device: 512 frames of the 1024x512
    detector (1.07 GB, > L2), photon discretisation, mask."""
    import torch
    sp = stream.cuda_stream
    ny, nx, nf = 1024, 512, 512
    rng = np.random.default_rng(5)
    frames = torch.from_numpy(rng.gamma(0.3, 1.0, (nf, ny * nx)).astype(np.float32)).cuda()
    mask = torch.from_numpy((rng.random(ny * nx) > 0.05).astype(np.int32)).cuda()
    discr = torch.zeros(ny * nx, dtype=torch.int64, device="cuda")
    mean = torch.zeros(nf, dtype=torch.float32, device="cuda")
    phs = torch.zeros(nf, dtype=torch.float32, device="cuda")
    fn = lambda: ctx.average_frames(frames, ny * nx, nf, mask, 0.2, 1.0, None, discr, mean, phs, sp)
    clocks = ClockSampler(0)
    clocks.start()
    ms = _time(fn, steps, max(3, warmup), stream)
    clk = clocks.stop()
    # the same batch without discretisation: the per-frame sums are then arbitrary FP32
    # values summed sequentially in pixel order, a chain of ny*nx dependent adds per frame
    fsum = torch.zeros(ny * nx, dtype=torch.float32, device="cuda")
    fn_f = lambda: ctx.average_frames(frames, ny * nx, nf, mask, 0.2, 0.0, fsum, None, mean, None, sp)
    ms_f = _time(fn_f, steps, max(3, warmup), stream)
    nbytes = frames.numel() * 4 + ny * nx * (4 + 16)  # frames read once, mask, counts read + written
    peak, kind = measured_peaks()
    res = {"metric": "frames/s averaged (LoadAndAverageIntensity, photon discretisation)",
           "value": nf / (ms * 1e-3), "unit": "frames/s", "ms_per_step": ms, "dtype": "fp32+i64", "clocks": clk,
           "config": {"workload": f"{nf} frames of {ny}x{nx} (1.07 GB), 5% masked, threshold 0.2, step 1.0"},
           "roofline": {"bound": "hbm", "achieved": nbytes / (ms * 1e-3) / 1e9, "peak": peak,
                        "unit": "GB/s", "frac": nbytes / (ms * 1e-3) / 1e9 / peak,
                        "peak_source": f"{kind} hbm_gbs",
                        "note": "one pass over the frames: per-pixel photon counts and the exact "
                                "integer per-frame photon totals in the same kernel"},
           "float_mode": {"ms_per_step": ms_f, "frames_per_s": nf / (ms_f * 1e-3),
                          "bound": "sequential FP32 sum per frame: a chain of "
                                   f"{ny * nx} dependent adds (4 cycles each)"}}
    if not args.no_cpu_baseline:
        import oracle
        sub = 16
        fh = frames[:sub].cpu().numpy()
        mh = mask.cpu().numpy()
        so = np.zeros(ny * nx, np.float32)
        do = np.zeros(ny * nx, np.int64)
        mo = np.zeros(sub, np.float32)
        po = np.zeros(sub, np.float32)
        t0 = time.perf_counter()
        oracle.lib().iaco_average_frames(oracle.p(fh), ny * nx, sub, oracle.p(mh), 0.2, 1.0, oracle.p(so),
                                         oracle.p(do), oracle.p(mo), oracle.p(po))
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": sub / dt, "unit": "frames/s", "cores": 1, "kind": "port",
                               "sample": f"{sub} of the {nf} frames"}
    return res


def part_frames_to_error(args, ctx, stream):
    """The second half of the headline metric: frames the plain mesh needs to
    reach the voxel-wise RMS error (against an independent 100 000-frame
    reference) that the committed denoiser reaches from 500 frames, on
    held-out random crystals simulated and correlated on the device."""
    import torch
    from incohautocorrelate_b200 import capi
    from incohautocorrelate_b200 import denoise as D
    params, meta = D.load_model(os.path.join(ROOT, "incohautocorrelate_b200", "weights", "denoiser_128.npz"))
    setup = D.SimSetup(**meta["setup"])
    sim = D.MeshSimulator(ctx, setup, stream=stream)
    E = setup.crop
    dn = capi.Denoiser(ctx, 1, E, E, E, backend=args.backend)
    dn.set_params(params)
    frames_in = int(meta["frames_in"])
    plain = [frames_in, 1000, 2000, 5000, 10000, 20000, 50000]
    clocks = ClockSampler(0)
    clocks.start()
    t0 = time.perf_counter()
    summary, rows = D.evaluate(ctx, sim, dn, meta["norm"], args.f2e_crystals, frames_in, plain, 100000,
                               seed=9001, log=None)
    secs = time.perf_counter() - t0
    clk = clocks.stop()
    dn.close()
    assert ctx.check() == 0
    return {"metric": "frames to set mesh error, denoised vs plain (median over held-out crystals)",
            "value": summary["median_gain"], "unit": "x fewer frames", "higher_is_better": True,
            "dtype": "bf16 network, fp32 accumulation; uint64 meshes",
            "config": {"workload": f"{args.f2e_crystals} held-out random crystals (a 3-6 A, 2-8 cells per axis, "
                                   "1-4 emitters per cell), 128x128 detector of 0.3 mm pixels at 0.1 m, 0.02 "
                                   "photons/pixel, 4 modes, 129^3 mesh; denoised 500-frame mesh vs plain meshes "
                                   "of 500-50 000 frames against an independent 100 000-frame reference",
                       "weights": "incohautocorrelate_b200/weights/denoiser_128.npz"},
            "min_gain": summary["min_gain"], "geomean_gain": summary["geomean_gain"],
            "gains": [r["gain"] for r in rows], "emitters": [r["emitters"] for r in rows],
            "seconds": secs, "frames_simulated": sim.frames,
            "frames_per_s": sim.frames / secs, "clocks": clk, "roofline": None,
            "cpu_baseline": None,
            "note": "no counterpart in the reference (its output of record is the plain mesh)"}


def run_parts(args, ctx, stream, atomic_peak):
    """One timed step (after one untimed) of every other part of the path."""
    nthreads = cores()
    parts = {}
    for name, fn in (("cq_small", lambda: part_dense("cq_small", args, ctx, stream, 1, 1, nthreads)),
                     ("ac1d_cq", lambda: part_dense("ac1d_cq", args, ctx, stream, 1, 1, nthreads)),
                     ("cq_merge", lambda: part_cq_merge(args, ctx, stream, 1, 1, nthreads, atomic_peak)),
                     ("ac1d_uw", lambda: part_ac1d("ac1d_uw", args, ctx, stream, 2, 1, nthreads)),
                     ("simulate", lambda: simulate_pipeline(args, ctx, stream, nthreads, steps=2, warmup=1)),
                     ("denoise", lambda: denoise_bench(args, ctx, stream, nthreads, layers=False)),
                     ("frames_to_error", lambda: part_frames_to_error(args, ctx, stream))):
        try:
            parts[name] = fn()
        except Exception as e:  # one part failing must not hide the headline
            parts[name] = {"error": f"{type(e).__name__}: {e}"}
    return parts


def run_kernel(args):
    import torch
    from incohautocorrelate_b200 import capi
    torch.cuda.set_device(0)
    ctx = capi.Context(0)
    stream = torch.cuda.current_stream()
    nthreads = cores()
    k = args.kernel
    if k in ("cq_small", "ac1d_cq"):
        res = part_dense(k, args, ctx, stream, args.steps, min(args.warmup, 1), nthreads)
    elif k == "cq_merge":
        peak = scatter_rate(ctx, stream, capi.half_mesh_words(201), 64)
        res = part_cq_merge(args, ctx, stream, args.steps, min(args.warmup, 1), nthreads, peak)
    elif k in ("ac1d_sparse", "ac1d_uw"):
        res = part_ac1d(k, args, ctx, stream, args.steps, args.warmup, nthreads)
    elif k == "simulate":
        res = simulate_pipeline(args, ctx, stream, nthreads, steps=args.steps, warmup=args.warmup)
    elif k == "denoise":
        res = denoise_bench(args, ctx, stream, nthreads, layers=not args.no_layers)
    elif k == "frames_to_error":
        res = part_frames_to_error(args, ctx, stream)
    else:
        res = part_average(args, ctx, stream, args.steps, args.warmup, nthreads)
    line = {"n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic", "kernel": k}
    line.update(res)
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


# multiply-adds per full-resolution voxel of the denoiser's forward pass:
# 3x3x3 layers 1->16, 16->16 at full resolution, 16->32, 32->32 at 1/8,
# 32->64, 64->64 at 1/64, 96->32, 32->32 at 1/8, 48->16, 16->16 at full
# resolution, and the 16->1 head
DENOISE_LAYERS = [(1, 16, 1), (16, 16, 1), (16, 32, 8), (32, 32, 8), (32, 64, 64), (64, 64, 64),
                  (96, 32, 8), (32, 32, 8), (48, 16, 1), (16, 16, 1)]
DENOISE_FWD_MACS = sum(27 * ci * co / d for ci, co, d in DENOISE_LAYERS) + 16
# training step: forward + data gradients (all but the first layer) + weight gradients
DENOISE_TRAIN_MACS = DENOISE_FWD_MACS + (DENOISE_FWD_MACS - 27 * 16 - 16) + DENOISE_FWD_MACS


def denoise_bench(args, ctx, stream, nthreads, layers=True):
    """The denoiser's training step (8 patches of 64^3, forward + loss +
    backward + AdamW) and its inference on a whole 128^3 mesh, plus (layers)
    each 3x3x3 layer shape alone in both tensor-core backends."""
    import torch
    from incohautocorrelate_b200 import capi
    sp = stream.cuda_stream
    rng = np.random.default_rng(11)
    B, P, E = args.dn_batch, 64, 128
    dn = capi.Denoiser(ctx, B, P, P, P, backend=args.backend)
    parts = []
    for ci, co, _ in DENOISE_LAYERS:
        parts += [rng.normal(0, (2.0 / (27 * ci)) ** 0.5, co * 27 * ci), rng.normal(0, 0.05, co)]
    parts += [rng.normal(0, 0.3, 16), [0.0]]
    dn.set_params(np.concatenate(parts).astype(np.float32))
    x = torch.from_numpy(rng.gamma(2.0, 0.5, (B, P, P, P)).astype(np.float32)).cuda()
    t = x * (1 + 0.2 * torch.randn_like(x))
    clocks = ClockSampler(0)
    clocks.start()

    def train_step():
        dn.backward(x, t, B, P, P, P, stream=sp, want_loss=False)
        dn.adamw_step(lr=1e-5, stream=sp)

    ms_train = _time(train_step, args.steps, max(3, args.warmup), stream)
    # the same step replayed from one captured CUDA graph (patches cut on the device)
    nm, Em = 4, 128
    meshes = torch.from_numpy(rng.gamma(2.0, 0.5, (nm, Em, Em, Em)).astype(np.float32)).to(torch.bfloat16)
    meshes = meshes.view(torch.int16).cuda()
    gsteps = max(args.steps, 4)
    plans = np.stack([rng.integers(0, nm, (gsteps, B)), rng.integers(0, Em - P + 1, (gsteps, B)),
                      rng.integers(0, Em - P + 1, (gsteps, B)), rng.integers(0, Em - P + 1, (gsteps, B)),
                      rng.integers(0, 48, (gsteps, B))], 2).astype(np.int32)
    d_plans = torch.from_numpy(plans).cuda()
    d_lrs = torch.full((gsteps,), 1e-5, dtype=torch.float32, device="cuda")
    for _ in range(2):  # capture + warm
        dn.train_steps(meshes, meshes, nm, Em, d_plans, d_lrs, gsteps, B, P, stream=sp)
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    dn.train_steps(meshes, meshes, nm, Em, d_plans, d_lrs, gsteps, B, P, stream=sp)
    g1.record(stream)
    torch.cuda.synchronize()
    ms_graph = g0.elapsed_time(g1) / gsteps
    xf = torch.from_numpy(rng.gamma(2.0, 0.5, (1, E, E, E)).astype(np.float32)).cuda()
    of = torch.zeros_like(xf)
    dn_inf = dn if B * P ** 3 >= E ** 3 else capi.Denoiser(ctx, 1, E, E, E, backend=args.backend)
    if dn_inf is not dn:
        dn_inf.set_params(dn.get_params())
    ms_fwd = _time(lambda: dn_inf.forward(xf, 1, E, E, E, of, sp), args.steps, max(3, args.warmup), stream)
    if dn_inf is not dn:
        dn_inf.close()
    # every 3x3x3 shape alone on the training batch's volume at its level (the
    # decoder's concatenated inputs are materialised by the network, so every
    # layer reads one plain tensor)
    layer_rows = []
    for ci, co, d in (DENOISE_LAYERS[1:] if layers else []):
        edge = P // round(d ** (1 / 3))
        nvox = B * edge ** 3
        s1 = torch.randn((B, edge, edge, edge, ci), device="cuda").to(torch.bfloat16).view(torch.int16)
        w = torch.from_numpy(capi.conv_weight_tiles(rng.normal(0, 0.1, (co, 27, ci)))).cuda()
        w = w.to(torch.bfloat16).view(torch.int16)
        b = torch.zeros(co, device="cuda")
        y = torch.zeros((nvox, co), dtype=torch.int16, device="cuda")
        row = {"cin": ci, "cout": co, "volume": f"{B}x{edge}^3"}
        for be, name in ((0, "tcgen05"), (1, "mma_sync")):
            ms = _time(lambda: capi.denoise_conv3x3(ctx, be, None, 0, 0, s1, ci, w, b, co, 1, B, edge, edge,
                                                    edge, y, sp), 10, 3, stream)
            row[name + "_ms"] = ms
            row[name + "_tflops"] = 2.0 * 27 * ci * co * nvox / (ms * 1e-3) / 1e12
        # the weight gradient of the same shape: tcgen05 (slabs 2) and mma.sync slabs (1)
        gq = torch.randn((nvox, co), device="cuda").to(torch.bfloat16).view(torch.int16)
        dw = torch.zeros((co, 27, ci), dtype=torch.float32, device="cuda")
        for sl, name in ((3, "wgrad_tcgen05_dz"), (2, "wgrad_tcgen05"), (1, "wgrad_mma_sync")):
            ms = _time(lambda: capi.denoise_wgrad3x3(ctx, None, 0, 0, s1, ci, gq, co, B, edge, edge, edge, dw,
                                                     None, sp, slabs=sl), 10, 3, stream)
            row[name + "_ms"] = ms
            row[name + "_tflops"] = 2.0 * 27 * ci * co * nvox / (ms * 1e-3) / 1e12
        layer_rows.append(row)
    clk = clocks.stop()
    peak, peak_src = measured_bf16_tflops()
    tf_train = 2.0 * DENOISE_TRAIN_MACS * B * P ** 3 / (ms_train * 1e-3) / 1e12
    tf_fwd = 2.0 * DENOISE_FWD_MACS * E ** 3 / (ms_fwd * 1e-3) / 1e12
    out = {"metric": f"denoiser training voxels/s ({B} x 64^3 patches, forward + backward + AdamW)",
           "value": B * P ** 3 / (ms_train * 1e-3), "unit": "voxels/s", "ms_per_step": ms_train,
           "dtype": "bf16 operands, fp32 accumulation",
           "config": {"workload": f"3-level 3D U-Net 16/32/64, 3x3x3 convs, batch {B} x 64^3 (activations "
                                  "> L2 per step)", "backend": ["tcgen05 slabs", "mma.sync", "tcgen05 per tap"][args.backend],
                      "params": capi.denoise_param_count(),
                      "train_flop_per_voxel": 2.0 * DENOISE_TRAIN_MACS,
                      "forward_flop_per_voxel": 2.0 * DENOISE_FWD_MACS},
           "graph_step": {"ms": ms_graph, "note": "patch crop + forward + backward + AdamW of one step "
                                                  "captured in a CUDA graph and replayed"},
           "inference": {"volume": f"1 x {E}^3", "ms": ms_fwd, "tflops": tf_fwd,
                         "meshes_per_s": 1e3 / ms_fwd},
           "layers": layer_rows, "clocks": clk,
           "roofline": {"bound": "tensor", "achieved": tf_train, "unit": "TFLOP/s", "peak": peak,
                        "frac": tf_train / peak, "peak_source": peak_src,
                        "kernel": "whole training step"}}
    if not args.no_cpu_baseline:
        import torch as T
        from oracle import denoise_oracle as O
        T.set_num_threads(nthreads)
        L = [(w.float(), b.float()) for w, b in O.unpack(dn.get_params())]
        xc = T.from_numpy(rng.gamma(2.0, 0.5, (1, 32, 32, 32)).astype(np.float32))
        t0 = time.perf_counter()
        with T.no_grad():
            O.forward(L, xc)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 32 ** 3 / dt, "unit": "voxels/s (forward only)", "cores": nthreads,
                               "kind": "port", "sample": f"torch fp32 CPU forward of the same network on 1 x "
                                                         f"32^3 ({dt:.2f} s)"}
    dn.close()
    return out


def simulate_pipeline(args, ctx, stream, nthreads, steps=3, warmup=1):
    """512x512 detector (75 um at 0.10 m), 5x5x8 simple-cubic crystal (a = 4 A,
    200 emitters), 4 modes, SuSa 0, lambda 1.55 A, I = sum_modes |Psi|^2, mean
    0.02 photons per pixel, random orientations: emitters -> intensity ->
    Poisson -> photon lists -> 201^3 pair mesh, all on the device, in chunks
    of frames."""
    import torch
    import oracle
    from incohautocorrelate_b200 import capi
    from incohautocorrelate_b200 import workloads as W
    sp = stream.cuda_stream
    n = 512
    pm_m = W.flat_pixel_map(n, n)
    pm = (pm_m * np.float32(1e10)).astype(np.float32)  # Angstrom
    km, mq = W.kmap_numpy(pm_m)
    cells = (5, 5, 8)
    atoms = np.array([[(x - cells[0] / 2.0 + 0.5) * 4.0, (y - cells[1] / 2.0 + 0.5) * 4.0,
                       (z - cells[2] / 2.0 + 0.5) * 4.0]
                      for x in range(cells[0]) for y in range(cells[1]) for z in range(cells[2])],
                     np.float64)
    na, nmodes = len(atoms), 4
    chunk = min(args.frames, 1000)
    npix = n * n
    d_pm, d_km = torch.from_numpy(pm).cuda(), torch.from_numpy(km).cuda()
    d_atoms = torch.from_numpy(atoms.reshape(-1)).cuda()
    em = torch.zeros((chunk, nmodes, na, 4), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(chunk * nmodes, dtype=torch.int32, device="cuda")
    rot = torch.zeros((chunk, 9), dtype=torch.float32, device="cuda")
    img = torch.zeros((chunk, npix), dtype=torch.float32, device="cuda")
    cap = int(chunk * npix * 0.05) + 100000
    phot = torch.zeros((cap, 4), dtype=torch.float32, device="cuda")
    offs = torch.zeros(chunk + 1, dtype=torch.int64, device="cuda")
    shape = capi.big_mesh_shape(mq, 199)
    S = shape.size_ab
    half = torch.zeros(capi.half_mesh_words(S), dtype=torch.int64, device="cuda")
    cp = capi.CrystalParams(1, 1.0, 1, 1.0)
    us = 75e-6 * 1e10
    simp = capi.SimParams(0, (C.c_double * 3)(us, 0, 0), (C.c_double * 3)(0, us, 0), 1.55, 1, 0)
    pp = capi.PhotonParams(0.02 * npix, 1, 0.0, 1.0)
    params = capi.sparse_params(shape)
    ev = {"intensity": []}

    def step(k):
        ctx.crystal_emitters(d_atoms, na, chunk, nmodes, cp, 1234 + k, em, cnt, rot, None, sp)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.simulate_intensity(d_pm, npix, em, cnt, na, nmodes, chunk, simp, img, sp)
        b.record(stream)
        ev["intensity"].append((a, b))
        ctx.simulate_photons(img, npix, chunk, k * chunk, pp, 99, sp)
        ctx.sparsify_frames(img, None, d_km, npix, chunk, 0.0, 1.0, 1, phot, cap, offs, sp,
                            want_total=False)
        ctx.sparse_ac_batch(phot, offs, rot, chunk, params, half, sp)

    for k in range(warmup):
        step(k)
    torch.cuda.synchronize()
    ev["intensity"].clear()
    clocks = ClockSampler(0)
    clocks.start()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for k in range(steps):
        step(warmup + k)
    b.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = a.elapsed_time(b) / steps
    ms_int = sum(x.elapsed_time(y) for x, y in ev["intensity"]) / len(ev["intensity"])
    terms = npix * na * nmodes * chunk
    mufu_peak = 148 * 16 * (clk["sm_mhz"] or 1965.0) * 1e6 / 2  # two SFU ops per term
    out = {"metric": "simulated frames/s into the 201^3 pair mesh", "value": chunk / (ms * 1e-3),
           "unit": "frames/s", "ms_per_step": ms, "steps": steps, "dtype": "fp32",
           "config": {"workload": "512x512, 5x5x8 crystal (200 emitters), 4 modes, SuSa 0, "
                                  "|Psi|^2, 0.02 photons/pixel, random orientation",
                      "frames_per_step": chunk},
           "clocks": clk,
           "roofline": {"bound": "sfu", "kernel": "simulate_kernel", "kernel_ms": ms_int,
                        "achieved": terms / (ms_int * 1e-3), "unit": "terms/s",
                        "peak": mufu_peak, "frac": terms / (ms_int * 1e-3) / mufu_peak,
                        "peak_source": "derived: 148 SM x 16 SFU results/clk / 2 (sin + cos) "
                                       "at the sampled clock"}}
    if not args.no_cpu_baseline:
        em_h = em[0].cpu().numpy()
        P = np.array([na, 1, 0, us, 0, 0, 0, us, 0, 1.55], np.float64)
        rows = 4096
        t = np.zeros(rows, np.float32)
        t0 = time.perf_counter()
        for m in range(nmodes):
            e = np.ascontiguousarray(em_h[m])
            oracle.lib().iaco_simulate_crystal(oracle.p(pm[: 3 * rows].copy()), rows, oracle.p(e),
                                               na, oracle.p(P), 1, oracle.p(t))
        dt = time.perf_counter() - t0
        cpu_terms = rows * na * nmodes / dt
        out["cpu_baseline"] = {"value": cpu_terms / (npix * na * nmodes), "unit": "frames/s",
                               "cores": nthreads, "kind": "port",
                               "sample": f"SimulateCrystal of {rows} pixels x 4 modes "
                                         f"({dt:.2f} s), scaled to a 512x512 frame; intensity "
                                         "only (no Poisson, no correlation)"}
    return out


def main():
    args = parse()
    if args.kernel != "sparse":
        return run_kernel(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
