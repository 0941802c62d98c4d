"""Frame sharding across ranks and the one reduction of the pair mesh.

The correlation path has no exchange until the end: frames are independent
and a mesh is an integer sum, so each rank bins a contiguous range of frames
into its own mesh and the meshes are summed once (NCCL over NVLink for GPUs,
gloo on CPU).  Integer sums commute, so the result is bit-identical to one
process binning every frame, for any partition.
"""
from __future__ import annotations

import numpy as np


def frame_pairs(offsets) -> np.ndarray:
    """Photon pairs n(n+1)/2 of every frame."""
    n = np.diff(np.asarray(offsets, np.int64))
    return n * (n + 1) // 2


def balanced_frame_ranges(offsets, world: int):
    """Contiguous frame ranges, one per rank, with about equal pair counts."""
    pairs = frame_pairs(offsets)
    nframes = len(pairs)
    cum = np.concatenate([[0], np.cumsum(pairs)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(cum, total * r / world, side="left")))
    cuts.append(nframes)
    cuts = np.maximum.accumulate(np.minimum(np.array(cuts), nframes))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world)]


def shard(photons, offsets, rot, rank: int, world: int):
    """This rank's frames: (photons, rebased offsets, rotations, frame range)."""
    f0, f1 = balanced_frame_ranges(offsets, world)[rank]
    off = np.asarray(offsets, np.uint64)
    p0, p1 = int(off[f0]), int(off[f1])
    return photons[p0:p1], off[f0:f1 + 1] - off[f0], rot[f0:f1], (f0, f1)


def rank_workload(rank: int, world: int, scaling: str, nframes: int, seed: int):
    """The rotated-correlator frames one rank bins in a multi-process run.

    scaling "weak": every rank bins its own `nframes` frames (seed offset by
    rank), so the work per rank stays fixed as ranks are added; "strong": the
    ranks share one batch of `nframes` frames, each binning a contiguous range
    of about equal pair count.  Returns (photons, offsets, rotations, info)."""
    from . import workloads as W
    if scaling == "weak":
        cfg = W.rotated_config(nframes=nframes, seed=seed + 7919 * rank)
        info = {"frames": (0, nframes), "batch_frames": nframes * world}
        return cfg["photons"], cfg["offsets"], cfg["rot"], dict(cfg, **info)
    if scaling != "strong":
        raise ValueError(f"scaling must be 'weak' or 'strong', not {scaling!r}")
    cfg = W.rotated_config(nframes=nframes, seed=seed)
    ph, off, rot, rng = shard(cfg["photons"], cfg["offsets"], cfg["rot"], rank, world)
    info = {"frames": rng, "batch_frames": nframes}
    return ph, off, rot, dict(cfg, **info)


def reduce_mesh(mesh, dst: int = 0):
    """Sum the ranks' uint64 meshes (held as int64 tensors) onto `dst`.  Two's
    complement addition makes the int64 sum the uint64 sum modulo 2^64."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.reduce(mesh, dst=dst, op=dist.ReduceOp.SUM)
    return mesh
