"""Training data, training and evaluation of the mesh denoiser (no counterpart
in the reference).

The denoiser maps a pair mesh accumulated over few frames to an estimate of
the mesh's many-frame mean.  Everything runs on the device through the C ABI:

* random synthetic crystals (lattice constant 3-6 A, 2-8 cells per axis, 1-4
  emitters per cell at random fractional positions) are simulated frame by
  frame (random orientation, incoherent emitters with random phases per
  mode, I = sum_modes |Psi|^2, Poisson photons), turned into photon lists and
  correlated into a uint64 pair mesh (nearest/nearest, double mapping);
* the folded mesh is scaled to "pairs per frame / norm" and cropped to the
  network's volume (the leading 128^3 corner of the 129^3 mesh);
* the network is trained on (few-frame, many-frame) patch pairs with the MSE
  loss and AdamW (iac_denoise_backward / iac_denoise_adamw_step);
* evaluation: plain meshes of one frame stream at several frame counts and a
  reference mesh from an independent stream; the voxel-wise RMS error of the
  plain mesh follows sigma^2 (1/N + 1/N_ref), and the frame count at which it
  equals the denoised few-frame mesh's error is the denoiser's frame
  equivalent.

    python -m incohautocorrelate_b200.denoise --out DIR [--crystals 512 ...]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import time
from dataclasses import asdict, dataclass, field

import numpy as np

from . import capi
from . import workloads as W

MULT = 1000.0  # ACMesh Multiplicator of the pair meshes


@dataclass
class SimSetup:
    """Detector, beam and mesh of the training data: a 128 x 128 detector with
    0.3 mm pixels at 0.1 m (the angular range of 512 x 512 x 75 um), 1.55 A,
    0.02 photons per pixel per frame, 4 incoherent modes, 129^3 mesh."""
    det: int = 128
    pitch: float = 300e-6
    dist: float = 0.10
    wavelength: float = 1.55
    photons_per_pixel: float = 0.02
    modes: int = 4
    mesh_edge: int = 127  # MeshSize argument: the mesh is (edge + 2)^3
    crop: int = 128
    chunk: int = 2000
    max_emitters: int = 2048  # the largest crystal below: 8 x 8 x 8 cells x 4


def random_crystal(rng, max_emitters=2048):
    """Emitter positions (A, centred) of a random crystal: cubic lattice
    constant a in [3, 6], 2..8 cells per axis, 1..4 emitters per cell at
    random fractional positions (8 to 2048 emitters; a smaller max_emitters
    redraws the larger crystals)."""
    while True:
        a = float(rng.uniform(3.0, 6.0))
        cells = rng.integers(2, 9, size=3)
        per = int(rng.integers(1, 5))
        if int(cells.prod()) * per <= max_emitters:
            break
    basis = rng.uniform(0.0, 1.0, (per, 3))
    g = np.stack(np.meshgrid(*[np.arange(c) for c in cells], indexing="ij"), -1).reshape(-1, 3)
    pos = ((g[:, None, :] + basis[None]) * a).reshape(-1, 3)
    pos -= pos.mean(0)
    return pos.astype(np.float64), {"a": a, "cells": [int(c) for c in cells], "per_cell": per}


class MeshSimulator:
    """Device pipeline crystal -> frames -> photons -> pair mesh, in chunks."""

    def __init__(self, ctx, setup: SimSetup, stream=None):
        import torch
        self.ctx, self.s = ctx, setup
        self.stream = stream or torch.cuda.current_stream()
        self.sp = self.stream.cuda_stream
        s = setup
        pm = W.flat_pixel_map(s.det, s.det, pitch=s.pitch, dist=s.dist)
        km, mq = W.kmap_numpy(pm)
        self.npix = s.det * s.det
        self.d_pm = torch.from_numpy((pm * np.float32(1e10)).astype(np.float32)).cuda()
        self.d_km = torch.from_numpy(km).cuda()
        self.shape = capi.big_mesh_shape(mq, s.mesh_edge)
        self.S = self.shape.size_ab
        self.params = capi.sparse_params(self.shape, multiplicator=MULT)
        n = s.chunk
        self.em = torch.zeros((n, s.modes, s.max_emitters, 4), dtype=torch.float32, device="cuda")
        self.cnt = torch.zeros(n * s.modes, dtype=torch.int32, device="cuda")
        self.rot = torch.zeros((n, 9), dtype=torch.float32, device="cuda")
        self.img = torch.zeros((n, self.npix), dtype=torch.float32, device="cuda")
        self.cap = int(n * self.npix * s.photons_per_pixel * 2) + 200000
        self.phot = torch.zeros((self.cap, 4), dtype=torch.float32, device="cuda")
        self.offs = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
        self.half = torch.zeros(capi.half_mesh_words(self.S), dtype=torch.int64, device="cuda")
        self.full = torch.zeros(self.S ** 3, dtype=torch.int64, device="cuda")
        self.cp = capi.CrystalParams(1, 1.0, 1, 1.0)
        us = s.pitch * 1e10
        self.simp = capi.SimParams(0, (C.c_double * 3)(us, 0, 0), (C.c_double * 3)(0, us, 0),
                                   s.wavelength, 1, 0)
        self.pp = capi.PhotonParams(s.photons_per_pixel * self.npix, 1, 0.0, 1.0)
        self.frames = 0

    def run(self, atoms, nframes, seed, snapshots, on_snapshot):
        """Accumulate nframes frames of one crystal; at each frame count in
        `snapshots` fold the mesh into self.full and call on_snapshot(n)."""
        import torch
        d_atoms = torch.from_numpy(np.ascontiguousarray(atoms).reshape(-1)).cuda()
        na = len(atoms)
        assert na <= self.s.max_emitters
        self.half.zero_()
        snaps = sorted(set(int(x) for x in snapshots if 0 < x <= nframes))
        done, k = 0, 0
        while done < nframes:
            nxt = next((x for x in snaps if x > done), nframes)
            n = min(self.s.chunk, nxt - done)
            rseed = (int(seed) * 1000003 + k) & ((1 << 63) - 1)
            self.ctx.crystal_emitters(d_atoms, na, n, self.s.modes, self.cp, rseed, self.em, self.cnt,
                                      self.rot, None, self.sp)
            self.ctx.simulate_intensity(self.d_pm, self.npix, self.em, self.cnt, na, self.s.modes, n,
                                        self.simp, self.img, self.sp)
            self.ctx.simulate_photons(self.img, self.npix, n, done, self.pp, rseed ^ 0x5bd1e995,
                                      self.sp)
            self.ctx.sparsify_frames(self.img, None, self.d_km, self.npix, n, 0.0, 1.0, 1, self.phot,
                                     self.cap, self.offs, self.sp, want_total=False)
            self.ctx.sparse_ac_batch(self.phot, self.offs, self.rot, n, self.params, self.half, self.sp)
            done += n
            k += 1
            self.frames += n
            if done in snaps:
                self.full.zero_()  # the fold accumulates (full += mirror(half))
                self.ctx.sparse_fold(self.half, self.S, self.full, self.sp)
                on_snapshot(done)

    def mesh_input(self, nframes, norm, d_f32=None, d_bf16=None):
        """The folded mesh as network input: pairs per frame / norm, cropped."""
        capi.denoise_mesh_input(self.ctx, self.full, self.S, self.s.crop,
                                1.0 / (MULT * nframes * norm), d_f32=d_f32, d_bf16=d_bf16,
                                stream=self.sp)


def _bf16_zeros(shape):
    import torch
    return torch.zeros(shape, dtype=torch.int16, device="cuda")


def make_pairs(sim: MeshSimulator, n_crystals, frames_in, frames_target, seed, norm=None,
               log=print):
    """(inputs, targets) as bf16 [n, E, E, E] device tensors (int16 views),
    from n_crystals random crystals; the few-frame input is the first
    frames_in frames of the target's frame stream."""
    import torch
    E = sim.s.crop
    xin = _bf16_zeros((n_crystals, E, E, E))
    tgt = _bf16_zeros((n_crystals, E, E, E))
    rng = np.random.default_rng(seed)
    info = []
    if norm is None:
        # pairs per frame per voxel of a first target mesh sets the scale
        atoms, _ = random_crystal(np.random.default_rng(seed + 99991), sim.s.max_emitters)
        sim.run(atoms, min(frames_target, 5000), seed + 99991, [min(frames_target, 5000)],
                lambda n: None)
        m = sim.full.view(torch.int64).double().mean().item() / (MULT * min(frames_target, 5000))
        norm = float(m)
    t0 = time.perf_counter()
    for i in range(n_crystals):
        atoms, desc = random_crystal(rng, sim.s.max_emitters)
        cs = int(rng.integers(1 << 40))

        def snap(n, i=i):
            if n == frames_in:
                sim.mesh_input(n, norm, d_bf16=xin[i])
            if n == frames_target:
                sim.mesh_input(n, norm, d_bf16=tgt[i])

        sim.run(atoms, frames_target, cs, [frames_in, frames_target], snap)
        desc["emitters"] = len(atoms)
        info.append(desc)
        if log and (i + 1) % max(1, n_crystals // 8) == 0:
            torch.cuda.synchronize()
            log(f"  crystals {i + 1}/{n_crystals}  {time.perf_counter() - t0:.1f} s")
    torch.cuda.synchronize()
    return xin, tgt, norm, info


@dataclass
class TrainConfig:
    steps: int = 4000
    batch: int = 8
    patch: int = 64
    lr: float = 2e-3
    lr_min: float = 1e-4
    warmup: int = 100
    weight_decay: float = 1e-4
    seed: int = 7
    backend: int = capi.TCGEN05


def train(ctx, xin, tgt, cfg: TrainConfig, log=print, dn=None):
    """Train on random patches (any of the 48 axis permutations/reflections:
    the crystal ensemble is symmetric under them) of the mesh pairs.  Steps
    run as replays of one captured CUDA graph (iac_denoise_train_steps); the
    patch plans and the learning-rate schedule (linear warm-up, cosine decay)
    are uploaded once."""
    import torch
    n, E = xin.shape[0], xin.shape[1]
    P, B = cfg.patch, cfg.batch
    if dn is None:
        dn = capi.Denoiser(ctx, B, P, P, P, backend=cfg.backend)
        dn.init_params(cfg.seed)
    rng = np.random.default_rng(cfg.seed)
    plans = np.stack([rng.integers(0, n, (cfg.steps, B)), rng.integers(0, E - P + 1, (cfg.steps, B)),
                      rng.integers(0, E - P + 1, (cfg.steps, B)), rng.integers(0, E - P + 1, (cfg.steps, B)),
                      rng.integers(0, 48, (cfg.steps, B))], 2).astype(np.int32)
    step = np.arange(cfg.steps)
    f = np.clip((step - cfg.warmup) / max(1, cfg.steps - cfg.warmup), 0.0, 1.0)
    lrs = np.where(step < cfg.warmup, cfg.lr * (step + 1) / cfg.warmup,
                   cfg.lr_min + 0.5 * (cfg.lr - cfg.lr_min) * (1 + np.cos(np.pi * f))).astype(np.float32)
    chunk = 100
    stream = torch.cuda.current_stream()
    losses = torch.zeros(chunk, dtype=torch.float64, device="cuda")
    # fixed device buffers, so the captured step graph is reused by every chunk
    d_plans = torch.zeros((chunk, B, 5), dtype=torch.int32, device="cuda")
    d_lrs = torch.zeros(chunk, dtype=torch.float32, device="cuda")
    hist = []
    t0 = time.perf_counter()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    timed = 0
    for s0 in range(0, cfg.steps, chunk):
        k = min(chunk, cfg.steps - s0)
        d_plans[:k].copy_(torch.from_numpy(np.ascontiguousarray(plans[s0:s0 + k])))
        d_lrs[:k].copy_(torch.from_numpy(np.ascontiguousarray(lrs[s0:s0 + k])))
        if s0 == chunk:
            ev0.record(stream)
        dn.train_steps(xin, tgt, n, E, d_plans, d_lrs, k, B, P, d_losses=losses, stream=stream.cuda_stream,
                       weight_decay=cfg.weight_decay)
        if s0 >= chunk:
            timed += k
        mean = losses[:k].cpu().numpy() / (B * P ** 3)
        hist.append((s0, float(mean[0])))
        if log and (s0 // chunk) % 10 == 0:
            log(f"  step {s0:5d}  loss {mean[0]:.5f}  lr {lrs[s0]:.2e}  {time.perf_counter() - t0:.1f} s")
    ev1.record(stream)
    torch.cuda.synchronize()
    hist.append((cfg.steps - 1, float(losses[(cfg.steps - 1) % chunk].item() / (B * P ** 3))))
    ms_step = ev0.elapsed_time(ev1) / timed if timed else float("nan")
    return dn, hist, ms_step


def data_parallel_step(dn, d_x, d_t, nb, D, H, W, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=1e-4):
    """One data-parallel training step on several GPUs: every rank (one process
    per GPU, its own `Denoiser` with the same parameters) computes the
    gradients of its own nb patches, the ranks average the gradient vector in
    place (one all-reduce of iac_denoise_grad_buffer), and every rank then takes
    the same AdamW step, so the replicas stay identical.  With equal local
    batches the mean of the local mean-loss gradients is the gradient of the
    global batch's mean loss.  Returns the global mean loss.  Without an
    initialised process group (or with one rank) this is backward + adamw_step."""
    import torch
    import torch.distributed as dist
    loss = dn.backward(d_x, d_t, nb, D, H, W)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        world = dist.get_world_size()
        g = dn.grad_tensor()
        dist.all_reduce(g, op=dist.ReduceOp.SUM)
        g.div_(world)
        t = torch.tensor([loss], dtype=torch.float64, device=g.device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        loss = float(t.item()) / world
        if g.is_cuda:
            torch.cuda.synchronize()  # the reduced gradients are in place before the optimizer reads them
    dn.adamw_step(lr, beta1, beta2, eps, weight_decay)
    return loss


def denoise_volume(dn, d_x, d_out, E):
    dn.forward(d_x, 1, E, E, E, d_out)


def plain_error_model(frames, errs, n_ref):
    """Least-squares sigma^2 of err(N)^2 = sigma^2 (1/N + 1/n_ref)."""
    f = np.asarray(frames, np.float64)
    e2 = np.asarray(errs, np.float64) ** 2
    a = 1.0 / f + 1.0 / n_ref
    return float((a @ e2) / (a @ a))


def frames_equivalent(err, sigma2, n_ref):
    """Frames at which the plain mesh's RMS error (model) equals err."""
    d = err ** 2 - sigma2 / n_ref
    return float("inf") if d <= 0 else sigma2 / d


def evaluate(ctx, sim: MeshSimulator, dn, norm, n_crystals, frames_in, plain_frames, n_ref, seed,
             log=print):
    """Denoised few-frame mesh vs plain meshes against an independent
    n_ref-frame reference, per held-out crystal."""
    import torch
    E = sim.s.crop
    rng = np.random.default_rng(seed)
    xin = torch.zeros((E, E, E), dtype=torch.float32, device="cuda")
    out = torch.zeros_like(xin)
    plain = {}
    ref = torch.zeros_like(xin)
    rows = []
    snaps = sorted(set([frames_in] + list(plain_frames)))
    for c in range(n_crystals):
        atoms, desc = random_crystal(rng, sim.s.max_emitters)
        s_a, s_b = int(rng.integers(1 << 40)), int(rng.integers(1 << 40))
        buf = {n: torch.zeros_like(xin) for n in snaps}
        sim.run(atoms, max(snaps), s_a, snaps, lambda n: sim.mesh_input(n, norm, d_f32=buf[n]))
        sim.run(atoms, n_ref, s_b, [n_ref], lambda n: sim.mesh_input(n, norm, d_f32=ref))
        xin.copy_(buf[frames_in])
        denoise_volume(dn, xin, out, E)
        torch.cuda.synchronize()
        rms = lambda a: float(torch.sqrt(torch.mean((a.double() - ref.double()) ** 2)))
        e_plain = {n: rms(buf[n]) for n in snaps}
        e_dn = rms(out)
        s2 = plain_error_model(list(e_plain), list(e_plain.values()), n_ref)
        neq = frames_equivalent(e_dn, s2, n_ref)
        rows.append({"crystal": desc, "emitters": len(atoms), "err_plain": e_plain, "err_denoised": e_dn,
                     "sigma2": s2, "frames_equivalent": neq, "gain": neq / frames_in})
        if log:
            log(f"  crystal {c}: err plain@{frames_in} {e_plain[frames_in]:.4g}  denoised {e_dn:.4g}  "
                f"-> {neq:.4g} frames ({neq / frames_in:.1f}x)")
    gains = np.array([r["gain"] for r in rows])
    finite = gains[np.isfinite(gains)]
    summary = {
        "crystals": n_crystals, "frames_in": frames_in, "reference_frames": n_ref,
        "median_gain": float(np.median(gains)),
        "geomean_gain": float(np.exp(np.mean(np.log(finite)))) if len(finite) else float("inf"),
        "min_gain": float(gains.min()),
        "mean_err_plain_in": float(np.mean([r["err_plain"][frames_in] for r in rows])),
        "mean_err_denoised": float(np.mean([r["err_denoised"] for r in rows])),
    }
    return summary, rows


def save_model(path, dn, norm, setup: SimSetup, extra=None, optimizer_state=False):
    """Parameters and metadata; with optimizer_state also the AdamW moments and
    step count, so that training can resume where it stopped (resume_model)."""
    meta = {"norm": norm, "setup": asdict(setup)}
    if extra:
        meta.update(extra)
    if optimizer_state:
        params, m, v, step = dn.get_state()
        np.savez_compressed(path, params=params, meta=json.dumps(meta), adam_m=m, adam_v=v, adam_step=step)
    else:
        np.savez_compressed(path, params=dn.get_params(), meta=json.dumps(meta))


def load_model(path):
    z = np.load(path)
    return z["params"], json.loads(str(z["meta"]))


def resume_model(path, dn):
    """Restore parameters and, when saved, the optimizer state into `dn`;
    returns the metadata."""
    z = np.load(path)
    if "adam_m" in z.files:
        dn.set_state(z["params"], z["adam_m"], z["adam_v"], int(z["adam_step"]))
    else:
        dn.set_params(z["params"])
    return json.loads(str(z["meta"]))


def main(argv=None):
    import torch
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--crystals", type=int, default=512)
    ap.add_argument("--frames-in", type=int, default=500)
    ap.add_argument("--frames-target", type=int, default=50000)
    ap.add_argument("--eval-crystals", type=int, default=32)
    ap.add_argument("--eval-ref", type=int, default=100000)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--backend", type=int, default=capi.TCGEN05)
    ap.add_argument("--plain-frames", default="1000,2000,5000,10000,20000,50000")
    ap.add_argument("--seed", type=int, default=2024)
    a = ap.parse_args(argv)
    os.makedirs(a.out, exist_ok=True)
    logf = open(os.path.join(a.out, "train.log"), "a")

    def log(msg):
        print(msg, flush=True)
        logf.write(msg + "\n")
        logf.flush()

    torch.cuda.set_device(0)
    ctx = capi.Context(0)
    setup = SimSetup()
    sim = MeshSimulator(ctx, setup)
    log(f"mesh {sim.S}^3, crop {setup.crop}^3, detector {setup.det}^2")
    t0 = time.perf_counter()
    xin, tgt, norm, info = make_pairs(sim, a.crystals, a.frames_in, a.frames_target, a.seed, log=log)
    t_data = time.perf_counter() - t0
    log(f"training pairs: {a.crystals} crystals, {sim.frames} frames in {t_data:.1f} s; norm {norm:.6g}")
    cfg = TrainConfig(steps=a.steps, batch=a.batch, lr=a.lr, backend=a.backend, seed=a.seed + 1)
    t0 = time.perf_counter()
    dn, hist, ms_step = train(ctx, xin, tgt, cfg, log=log)
    t_train = time.perf_counter() - t0
    log(f"trained {cfg.steps} steps in {t_train:.1f} s ({ms_step:.2f} ms/step on the device)")
    del xin, tgt
    torch.cuda.empty_cache()
    # inference on whole meshes: a 1 x E^3 workspace
    E = setup.crop
    dn_full = capi.Denoiser(ctx, 1, E, E, E, backend=a.backend)
    dn_full.set_params(dn.get_params())
    plain_frames = [a.frames_in] + [int(v) for v in a.plain_frames.split(",") if v]
    summary, rows = evaluate(ctx, sim, dn_full, norm, a.eval_crystals, a.frames_in, plain_frames, a.eval_ref,
                             a.seed + 5, log=log)
    assert ctx.check() == 0
    res = {"summary": summary, "per_crystal": rows, "train": {**asdict(cfg), "loss": hist,
                                                              "ms_per_step": ms_step, "seconds": t_train},
           "data": {"crystals": a.crystals, "frames_in": a.frames_in, "frames_target": a.frames_target,
                    "seconds": t_data, "norm": norm}}
    with open(os.path.join(a.out, "denoise_eval.json"), "w") as f:
        json.dump(res, f, indent=1, default=float)
    save_model(os.path.join(a.out, "denoiser.npz"), dn, norm, setup,
               {"frames_in": a.frames_in, "frames_target": a.frames_target, "summary": summary})
    log(json.dumps(summary))


if __name__ == "__main__":
    main()
