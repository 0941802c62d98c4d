"""Two ranks over gloo on the CPU: frames are sharded by pair count, every rank
bins its shard (the oracle stands in for the device kernel here), one
reduction sums the meshes, and the result is bit-identical to a single
process binning every frame."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    import oracle
    from incohautocorrelate_b200 import shard, workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg = W.rotated_config(nframes=120, seed=5)
        shape = oracle.big_mesh_shape(cfg["max_q"], 63)
        ph, off, rot, (f0, f1) = shard.shard(cfg["photons"], cfg["offsets"], cfg["rot"], rank, world)
        mesh, _ = oracle.sparse_batch(ph, off, rot, shape, cpu_gpu=-1, det_pixels=cfg["npix"])
        t = torch.from_numpy(mesh.view(np.int64).copy())
        shard.reduce_mesh(t, dst=0)
        if rank == 0:
            np.save(os.path.join(out_dir, "reduced.npy"), t.numpy().view(np.uint64))
        np.save(os.path.join(out_dir, f"range{rank}.npy"), np.array([f0, f1]))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_reduction_is_bit_exact(tmp_path, oracle_lib):
    import torch.multiprocessing as mp

    from incohautocorrelate_b200 import workloads as W
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r0 = np.load(tmp_path / "range0.npy")
    r1 = np.load(tmp_path / "range1.npy")
    assert r0[0] == 0 and r0[1] == r1[0] and r1[1] == 120
    cfg = W.rotated_config(nframes=120, seed=5)
    shape = oracle_lib.big_mesh_shape(cfg["max_q"], 63)
    want, _ = oracle_lib.sparse_batch(cfg["photons"], cfg["offsets"], cfg["rot"], shape, cpu_gpu=-1,
                                      det_pixels=cfg["npix"])
    np.testing.assert_array_equal(np.load(tmp_path / "reduced.npy"), want)


def test_balanced_ranges_cover_all_frames():
    from incohautocorrelate_b200 import shard, workloads as W
    cfg = W.rotated_config(nframes=5000, seed=3)
    for world in (1, 2, 3, 8):
        rng = shard.balanced_frame_ranges(cfg["offsets"], world)
        assert rng[0][0] == 0 and rng[-1][1] == 5000
        assert all(a[1] == b[0] for a, b in zip(rng, rng[1:]))
        pairs = shard.frame_pairs(cfg["offsets"])
        loads = [pairs[a:b].sum() for a, b in rng]
        assert max(loads) <= pairs.sum() / world + pairs.max()
