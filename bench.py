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
    ap.add_argument("--cpu-frames", type=int, default=1500,
                    help="frames per step of the --impl reference arm")
    ap.add_argument("--cpu-baseline-frames", type=int, default=100_000,
                    help="frames of the cpu_baseline sample (all 100 000: about 8 s on 16 host threads)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--det", type=int, default=1024,
                    help="edge of the square detector of the dense kernels (1024 = their config)")
    ap.add_argument("--backend", type=int, default=0,
                    help="denoiser convolutions: 0 = tcgen05 + TMEM, 1 = mma.sync")
    ap.add_argument("--kernel", default="sparse",
                    choices=["sparse", "cq_small", "ac1d_cq", "cq_merge", "ac1d_sparse", "simulate",
                             "denoise", "average"],
                    help="sparse is the headline; the others measure the remaining kernels "
                         "of the path on their configurations")
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

    from incohautocorrelate_b200 import capi, shard
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
    total_pairs = pairs * world
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

    # -- end to end through the C-ABI host entry point (pinned host buffers) --
    ph_p = torch.from_numpy(ph_h).pin_memory()
    off_p = torch.from_numpy(off_h.view(np.int64)).pin_memory()
    rot_p = torch.from_numpy(rot_h).pin_memory()
    mesh_p = torch.zeros(capi.full_mesh_words(S), dtype=torch.int64).pin_memory()
    for _ in range(max(1, args.warmup // 2)):
        ctx.sparse_ac_frames_host(ph_p, off_p, rot_p, nframes, params, mesh_p)
    e2e_times = []
    # The host mesh accumulates over the steps, as ACMesh does over a run's
    # batches (Detector::AutoCorrelateSparseList adds to it).  It is not cleared
    # between steps: a 65 MB CPU memset just before the call leaves the pinned
    # buffer dirty in the CPU caches and slows the copies into and out of it by
    # 1-2 ms, a cost of the benchmark loop rather than of the path.
    for _ in range(max(15, args.steps)):
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
            "graph": None if graph_ms is None else {
                "ms_per_step": graph_ms, "value": total_pairs / (graph_ms * 1e-3),
                "note": "the step (clear, plan, bin, fold) captured in one CUDA graph and replayed"},
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
        nb = min(args.cpu_baseline_frames, nframes)
        v, secs, cp = cpu_baseline(cfg, nb)
        line["cpu_baseline"] = {
            "value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"first {nb} frames ({cp} pairs, {secs:.1f} s) "
                      "through the reference's CPU route, OpenMP on all host threads"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if distributed:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# the other kernels of the path, each on its configuration (one JSON line)
# ---------------------------------------------------------------------------
def _fp32_peak_tflops(clock_mhz):
    """FP32 FMA peak of 148 SMs x 128 lanes x 2 flop at the sampled clock (no
    measured FP32 figure exists for this pool; derived, not measured)."""
    return 148 * 128 * 2 * clock_mhz * 1e6 / 1e12


# thread instructions per unordered pixel pair (ncu smsp__inst_executed.sum x 32 / pairs;
# cq_small on the 1024^2 configuration itself, ac1d_cq on a 256^2 detector;
# profiles/cq_small_kernel.md, profiles/ac1d_cq_kernel.md)
INST_PER_PAIR = {"cq_small": 1582131114734 * 32 / (1048576 * 1048577 / 2),
                 "ac1d_cq": 8217131069 * 32 / (65536 * 65537 / 2)}


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


def run_kernel(args):
    import torch
    from incohautocorrelate_b200 import capi
    from incohautocorrelate_b200 import workloads as W
    torch.cuda.set_device(0)
    ctx = capi.Context(0)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    nthreads = cores()
    clocks = ClockSampler(0)
    line = {"metric": None, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "data": "synthetic",
            "kernel": args.kernel}
    import oracle
    if args.kernel in ("cq_small", "ac1d_cq"):
        I, km, mq = _dense_inputs(args.det, args.det)
        npix = I.size
        dI, dk = torch.from_numpy(I).cuda(), torch.from_numpy(km).cuda()
        pairs = npix * (npix + 1) // 2
        if args.kernel == "cq_small":
            sh = capi.small_cq_mesh_shape(mq, 253)
            mult = capi.cq_small_multiplicator(I)
            out = torch.zeros(sh.size_ab * sh.size_ab * sh.size_c, dtype=torch.int64, device="cuda")
            fn = lambda: (out.zero_(), ctx.cq_small(dI, dk, npix, sh, 0, mult, out, sp, fast_size=args.det))
            shape_desc = f"small C(q) mesh {sh.size_ab}x{sh.size_ab}x{sh.size_c}"
        else:
            sh = capi.ac1d_shape(mq, 2048)
            mult = capi.ac1d_cq_multiplicator(I)
            out = torch.zeros(sh.size, dtype=torch.int64, device="cuda")
            fn = lambda: (out.zero_(), ctx.ac1d_cq(dI, dk, npix, sh, 1, mult, out, sp))
            shape_desc = "AC1D 2048 bins, linear"
        clocks.start()
        ms = _time(fn, args.steps, min(args.warmup, 1), stream)
        clk = clocks.stop()
        rate = pairs / (ms * 1e-3)
        # FP32 work per unordered pair: diff 3, norm 5, product 1, scale 3 (3D) / div 1
        flops = 12.0
        mhz = clk["sm_mhz"] or 1965.0
        line.update(metric=f"pixel pairs/s into {shape_desc}", value=rate, unit="pairs/s",
                    ms_per_step=ms, dtype="fp32+u64",
                    config={"workload": f"{args.det}x{args.det} radial mean intensity, 5% masked, "
                                        f"all {pairs:.3g} unordered pixel pairs", "pixels": npix},
                    clocks=clk,
                    roofline={"bound": "fp32", "achieved": rate * flops / 1e12,
                              "peak": _fp32_peak_tflops(mhz), "unit": "TFLOP/s",
                              "frac": rate * flops / 1e12 / _fp32_peak_tflops(mhz),
                              "peak_source": "derived 148 SM x 128 FP32 lanes x 2 at the sampled "
                                             "clock (no measured FP32 peak)",
                              "flop_per_pair": flops,
                              # the binding resource: instruction issue.  Instructions per pair
                              # from the committed ncu capture of this kernel (256^2 detector)
                              "issue": {"inst_per_pair": INST_PER_PAIR[args.kernel],
                                        "achieved": rate * INST_PER_PAIR[args.kernel],
                                        "peak": 148 * 4 * 32 * mhz * 1e6,
                                        "frac": rate * INST_PER_PAIR[args.kernel] / (148 * 4 * 32 * mhz * 1e6),
                                        "unit": "thread instructions/s",
                                        "source": f"profiles/{args.kernel}_kernel.md"}})
        if not args.no_cpu_baseline:
            rows = 48
            Ih = np.ascontiguousarray(I)
            t0 = time.perf_counter()
            if args.kernel == "cq_small":
                so = oracle.small_cq_mesh_shape(mq, 253)
                m = np.zeros(so.size_ab * so.size_ab * so.size_c, np.uint64)
                oracle.lib().iaco_cq_small(oracle.p(Ih), oracle.p(km), npix, so, 0, mult,
                                           npix // 2, npix // 2 + rows, oracle.p(m))
            else:
                so = oracle.ac1d_shape(mq, 2048)
                m = np.zeros(so.size, np.uint64)
                oracle.lib().iaco_ac1d_cq(oracle.p(Ih), oracle.p(km), npix, so, 1, mult,
                                          npix // 2, npix // 2 + rows, oracle.p(m))
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": rows * npix / 2 / dt, "unit": "pairs/s",
                                    "cores": nthreads, "kind": "port",
                                    "sample": f"{rows} rows x {npix} pixels of the reference's "
                                              f"ordered-pair loop ({dt:.1f} s), counted as "
                                              "unordered pairs (2 ordered = 1)"}
    elif args.kernel == "cq_merge":
        I, km, mq = _dense_inputs(512, 1024, gap=512)
        npix = I.size
        sh = capi.small_cq_mesh_shape(mq, 199)
        mult = capi.cq_small_multiplicator(I)
        small_u = torch.zeros(sh.size_ab * sh.size_ab * sh.size_c, dtype=torch.int64, device="cuda")
        ctx.cq_small(torch.from_numpy(I).cuda(), torch.from_numpy(km).cuda(), npix, sh, 0, mult,
                     small_u, sp, fast_size=1024)
        small = (small_u.cpu().numpy().view(np.uint64).astype(np.float64) / mult)
        nf = args.frames
        R = W.haar_rotations(nf, seed=3)
        MI = np.random.default_rng(4).uniform(0.5e-4, 4e-4, nf).astype(np.float32)
        rw, m = capi.cq_merge_weights(R, MI, small)
        d_small, d_rw = torch.from_numpy(small).cuda(), torch.from_numpy(rw).cuda()
        big = torch.zeros(sh.size_ab ** 3, dtype=torch.int64, device="cuda")
        nvox = int((small >= np.float32(1e-37)).sum())
        fn = lambda: (big.zero_(), ctx.cq_merge(d_small, d_rw, nf, sh, 0, m, big, sp))
        clocks.start()
        ms = _time(fn, args.steps, min(args.warmup, 1), stream)
        clk = clocks.stop()
        rate = nvox * nf / (ms * 1e-3)
        line.update(metric="voxel-frame scatters/s (C(q) merge)", value=rate, unit="scatters/s",
                    ms_per_step=ms, dtype="fp32+u64",
                    config={"workload": f"small C(q) {sh.size_ab}x{sh.size_ab}x{sh.size_c} "
                                        f"({nvox} non-zero voxels) x {nf} SO(3) frames into "
                                        f"{sh.size_ab}^3"},
                    clocks=clk,
                    roofline={"bound": "l2-atomic", "achieved": rate, "unit": "updates/s",
                              "note": "one 64-bit L2 atomic per (voxel, frame)"})
        if not args.no_cpu_baseline:
            sub = min(nvox, 20000)
            so = oracle.small_cq_mesh_shape(mq, 199)
            out = np.zeros(sh.size_ab ** 3, np.uint64)
            nz = np.nonzero(small >= np.float32(1e-37))[0]
            v0 = int(nz[len(nz) // 2])
            t0 = time.perf_counter()
            oracle.lib().iaco_cq_merge(oracle.p(small), oracle.p(rw.reshape(-1)), min(nf, 2000), so,
                                       0, m, v0, v0 + sub, oracle.p(out))
            dt = time.perf_counter() - t0
            done = int(((small[v0:v0 + sub]) >= np.float32(1e-37)).sum()) * min(nf, 2000)
            line["cpu_baseline"] = {"value": done / dt, "unit": "scatters/s", "cores": nthreads,
                                    "kind": "port", "sample": f"{sub} voxels x {min(nf, 2000)} frames"}
    elif args.kernel == "ac1d_sparse":
        cfg = W.rotated_config(nframes=args.frames, seed=2)
        sh = capi.ac1d_shape(cfg["max_q"], 256)
        vs = capi.ac1d_vecsize(sh.max_q, sh.dq_per_step)
        ph = torch.from_numpy(cfg["photons"]).cuda()
        off = torch.from_numpy(cfg["offsets"].view(np.int64)).cuda()
        hist = torch.zeros(vs, dtype=torch.int64, device="cuda")
        nf = len(cfg["offsets"]) - 1
        fn = lambda: (hist.zero_(), ctx.ac1d_sparse_batch(ph, off, nf, sh.max_q, sh.dq_per_step, 1,
                                                          100.0, hist, sp))
        clocks.start()
        ms = _time(fn, args.steps, args.warmup, stream)
        clk = clocks.stop()
        pairs = _pairs(cfg["offsets"])
        line.update(metric="photon pairs/s into the AC1D histogram", value=pairs / (ms * 1e-3),
                    unit="pairs/s", ms_per_step=ms, dtype="fp32+u64", clocks=clk,
                    config={"workload": f"{nf} rotated-correlator frames, 256 bins, linear"})
    elif args.kernel == "simulate":
        line.update(simulate_pipeline(args, ctx, stream, clocks, nthreads))
    elif args.kernel == "denoise":
        line.update(denoise_bench(args, ctx, stream, clocks, nthreads))
    elif args.kernel == "average":
        # LoadAndAverageIntensity on the device: 512 frames of the 1024x512 detector (1.07 GB, > L2),
        # photon discretisation, mask
        ny, nx, nf = 1024, 512, 512
        rng = np.random.default_rng(5)
        frames = torch.from_numpy(rng.gamma(0.3, 1.0, (nf, ny * nx)).astype(np.float32)).cuda()
        mask = torch.from_numpy((rng.random(ny * nx) > 0.05).astype(np.int32)).cuda()
        discr = torch.zeros(ny * nx, dtype=torch.int64, device="cuda")
        mean = torch.zeros(nf, dtype=torch.float32, device="cuda")
        phs = torch.zeros(nf, dtype=torch.float32, device="cuda")
        fn = lambda: ctx.average_frames(frames, ny * nx, nf, mask, 0.2, 1.0, None, discr, mean, phs, sp)
        clocks.start()
        ms = _time(fn, args.steps, max(3, args.warmup), stream)
        clk = clocks.stop()
        # the same batch without discretisation: the per-frame sums are then arbitrary FP32
        # values summed sequentially in pixel order, a chain of ny*nx dependent adds per frame
        fsum = torch.zeros(ny * nx, dtype=torch.float32, device="cuda")
        fn_f = lambda: ctx.average_frames(frames, ny * nx, nf, mask, 0.2, 0.0, fsum, None, mean, None, sp)
        ms_f = _time(fn_f, args.steps, max(3, args.warmup), stream)
        nbytes = frames.numel() * 4 + ny * nx * (4 + 16)  # frames read once, mask, counts read + written
        peak, kind = measured_peaks()
        line.update(metric="frames/s averaged (LoadAndAverageIntensity, photon discretisation)",
                    value=nf / (ms * 1e-3), unit="frames/s", ms_per_step=ms, dtype="fp32+i64", clocks=clk,
                    config={"workload": f"{nf} frames of {ny}x{nx} (1.07 GB), 5% masked, threshold 0.2, "
                                        "step 1.0"},
                    roofline={"bound": "hbm", "achieved": nbytes / (ms * 1e-3) / 1e9, "peak": peak,
                              "unit": "GB/s", "frac": nbytes / (ms * 1e-3) / 1e9 / peak,
                              "peak_source": f"{kind} hbm_gbs",
                              "note": "one pass over the frames: per-pixel photon counts and the exact "
                                      "integer per-frame photon totals in the same kernel"},
                    float_mode={"ms_per_step": ms_f, "frames_per_s": nf / (ms_f * 1e-3),
                                "bound": "sequential FP32 sum per frame: a chain of "
                                         f"{ny * nx} dependent adds (4 cycles each)"})
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
            line["cpu_baseline"] = {"value": sub / dt, "unit": "frames/s", "cores": 1, "kind": "port",
                                    "sample": f"{sub} of the {nf} frames"}
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


def denoise_bench(args, ctx, stream, clocks, nthreads):
    """The denoiser's training step (8 patches of 64^3, forward + loss +
    backward + AdamW) and its inference on a whole 128^3 mesh, plus each
    3x3x3 layer shape alone in both tensor-core backends."""
    import torch
    from incohautocorrelate_b200 import capi
    sp = stream.cuda_stream
    rng = np.random.default_rng(11)
    B, P, E = 8, 64, 128
    dn = capi.Denoiser(ctx, B, P, P, P, backend=args.backend)
    parts = []
    for ci, co, _ in DENOISE_LAYERS:
        parts += [rng.normal(0, (2.0 / (27 * ci)) ** 0.5, co * 27 * ci), rng.normal(0, 0.05, co)]
    parts += [rng.normal(0, 0.3, 16), [0.0]]
    dn.set_params(np.concatenate(parts).astype(np.float32))
    x = torch.from_numpy(rng.gamma(2.0, 0.5, (B, P, P, P)).astype(np.float32)).cuda()
    t = x * (1 + 0.2 * torch.randn_like(x))
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
    ms_fwd = _time(lambda: dn.forward(xf, 1, E, E, E, of, sp), args.steps, max(3, args.warmup), stream)
    # every 3x3x3 shape alone on the training batch's volume at its level (the
    # decoder's concatenated inputs are materialised by the network, so every
    # layer reads one plain tensor)
    layers = []
    for ci, co, d in DENOISE_LAYERS[1:]:
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
        for sl, name in ((2, "wgrad_tcgen05"), (1, "wgrad_mma_sync")):
            ms = _time(lambda: capi.denoise_wgrad3x3(ctx, None, 0, 0, s1, ci, gq, co, B, edge, edge, edge, dw,
                                                     None, sp, slabs=sl), 10, 3, stream)
            row[name + "_ms"] = ms
            row[name + "_tflops"] = 2.0 * 27 * ci * co * nvox / (ms * 1e-3) / 1e12
        layers.append(row)
    clk = clocks.stop()
    peak, peak_src = measured_bf16_tflops()
    tf_train = 2.0 * DENOISE_TRAIN_MACS * B * P ** 3 / (ms_train * 1e-3) / 1e12
    tf_fwd = 2.0 * DENOISE_FWD_MACS * E ** 3 / (ms_fwd * 1e-3) / 1e12
    out = {"metric": "denoiser training voxels/s (8 x 64^3 patches, forward + backward + AdamW)",
           "value": B * P ** 3 / (ms_train * 1e-3), "unit": "voxels/s", "ms_per_step": ms_train,
           "dtype": "bf16 operands, fp32 accumulation",
           "config": {"workload": "3-level 3D U-Net 16/32/64, 3x3x3 convs, batch 8 x 64^3 (activations "
                                  "> L2 per step)", "backend": ["tcgen05 slabs", "mma.sync", "tcgen05 per tap"][args.backend],
                      "params": capi.denoise_param_count(),
                      "train_flop_per_voxel": 2.0 * DENOISE_TRAIN_MACS,
                      "forward_flop_per_voxel": 2.0 * DENOISE_FWD_MACS},
           "graph_step": {"ms": ms_graph, "note": "patch crop + forward + backward + AdamW of one step "
                                                  "captured in a CUDA graph and replayed"},
           "inference": {"volume": f"1 x {E}^3", "ms": ms_fwd, "tflops": tf_fwd,
                         "meshes_per_s": 1e3 / ms_fwd},
           "layers": layers, "clocks": clk,
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


def simulate_pipeline(args, ctx, stream, clocks, nthreads):
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

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    ev["intensity"].clear()
    clocks.start()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for k in range(args.steps):
        step(args.warmup + k)
    b.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = a.elapsed_time(b) / args.steps
    ms_int = sum(x.elapsed_time(y) for x, y in ev["intensity"]) / len(ev["intensity"])
    terms = npix * na * nmodes * chunk
    mufu_peak = 148 * 16 * (clk["sm_mhz"] or 1965.0) * 1e6 / 2  # two SFU ops per term
    out = {"metric": "simulated frames/s into the 201^3 pair mesh", "value": chunk / (ms * 1e-3),
           "unit": "frames/s", "ms_per_step": ms, "dtype": "fp32",
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
