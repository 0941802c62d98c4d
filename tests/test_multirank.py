"""Two ranks over gloo on the CPU: each rank takes its frames exactly as the
multi-GPU benchmark does (shard.rank_workload: a pair-balanced share of one
batch for strong scaling, its own frames for weak scaling), bins them (the
oracle stands in for the device kernel here), and the int64 view of its uint64
mesh goes through the same shard.reduce_mesh call; the result is
bit-identical to a single process binning every rank's frames."""
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


NFRAMES, SEED = 120, 5


def _rank_main(rank, world, port, out_dir, scaling):
    import torch
    import torch.distributed as dist

    import oracle
    from incohautocorrelate_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ph, off, rot, cfg = shard.rank_workload(rank, world, scaling, NFRAMES, SEED)
        shape = oracle.big_mesh_shape(cfg["max_q"], 63)
        mesh, _ = oracle.sparse_batch(ph, off, rot, shape, cpu_gpu=-1, det_pixels=cfg["npix"])
        full = torch.from_numpy(mesh.view(np.int64).copy())  # the benchmark's int64 mesh tensor
        shard.reduce_mesh(full, dst=0)
        if rank == 0:
            np.save(os.path.join(out_dir, "reduced.npy"), full.numpy().view(np.uint64))
        np.save(os.path.join(out_dir, f"range{rank}.npy"), np.array(cfg["frames"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("scaling", ["strong", "weak"])
def test_two_rank_gloo_reduction_is_bit_exact(tmp_path, oracle_lib, scaling):
    import torch.multiprocessing as mp

    from incohautocorrelate_b200 import shard, workloads as W
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path), scaling), nprocs=2, join=True,
                       start_method="spawn")
    r0 = np.load(tmp_path / "range0.npy")
    r1 = np.load(tmp_path / "range1.npy")
    cfg = W.rotated_config(nframes=NFRAMES, seed=SEED)
    shape = oracle_lib.big_mesh_shape(cfg["max_q"], 63)
    if scaling == "strong":  # one batch, split at a frame boundary
        assert r0[0] == 0 and r0[1] == r1[0] and r1[1] == NFRAMES
        want, _ = oracle_lib.sparse_batch(cfg["photons"], cfg["offsets"], cfg["rot"], shape, cpu_gpu=-1,
                                          det_pixels=cfg["npix"])
    else:  # every rank its own batch: the sum of the two single-process meshes
        want = np.zeros(shape.size_ab ** 3, np.uint64)
        for r in range(2):
            ph, off, rot, c = shard.rank_workload(r, 2, "weak", NFRAMES, SEED)
            m, _ = oracle_lib.sparse_batch(ph, off, rot, shape, cpu_gpu=-1, det_pixels=c["npix"])
            want += m
    assert want.sum() > 0
    np.testing.assert_array_equal(np.load(tmp_path / "reduced.npy"), want)


def _dense_rank_main(rank, world, port, out_dir):
    """A rank of a sharded dense C(q): its share of the pixel pairs binned into
    its own uint64 small mesh (the oracle's work items [r0, r1) stand in for
    the device kernel's tile-pair share), then the one integer reduction."""
    import torch
    import torch.distributed as dist

    import oracle
    from incohautocorrelate_b200 import shard, workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        I = W.radial_mean_intensity(24, 32, 9.0, 0.02, 0.05, seed=3)
        km, mq = oracle.calc_kmap(W.flat_pixel_map(24, 32, pitch=8 * 75e-6))
        s = oracle.small_cq_mesh_shape(mq, 31)
        npix = I.size
        r0, r1 = npix * rank // world, npix * (rank + 1) // world
        m = np.zeros(s.size_ab * s.size_ab * s.size_c, np.uint64)
        oracle.lib().iaco_cq_small(oracle.p(I), oracle.p(km), npix, s, 0, 1e5, r0, r1, oracle.p(m))
        t = torch.from_numpy(m.view(np.int64).copy())
        shard.reduce_mesh(t, dst=0)
        if rank == 0:
            np.save(os.path.join(out_dir, "dense.npy"), t.numpy().view(np.uint64))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_dense_reduction_is_bit_exact(tmp_path, oracle_lib):
    import torch.multiprocessing as mp

    from incohautocorrelate_b200 import workloads as W
    mp.start_processes(_dense_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    I = W.radial_mean_intensity(24, 32, 9.0, 0.02, 0.05, seed=3)
    km, mq = oracle_lib.calc_kmap(W.flat_pixel_map(24, 32, pitch=8 * 75e-6))
    s = oracle_lib.small_cq_mesh_shape(mq, 31)
    want = np.zeros(s.size_ab * s.size_ab * s.size_c, np.uint64)
    oracle_lib.lib().iaco_cq_small(oracle_lib.p(I), oracle_lib.p(km), I.size, s, 0, 1e5, 0, I.size,
                                   oracle_lib.p(want))
    assert want.sum() > 0
    np.testing.assert_array_equal(np.load(tmp_path / "dense.npy"), want)


def _dp_inputs():
    from oracle import denoise_oracle as O
    rng = np.random.default_rng(11)
    parts = []
    for ci, co in O.SPECS:
        parts += [rng.normal(0, (2.0 / (27 * ci)) ** 0.5, co * 27 * ci), rng.normal(0, 0.05, co)]
    parts += [rng.normal(0, 0.3, 16), [0.0]]
    params = np.concatenate(parts)
    x = rng.gamma(2.0, 0.5, (2, 8, 8, 8))
    return params, x, x * 1.1 + rng.normal(0, 0.05, x.shape)


def _dp_rank_main(rank, world, port, out_dir):
    """A rank of data-parallel denoiser training: the gradient of its own
    volume's mean loss (the float64 oracle stands in for the device backward),
    summed over ranks in place and divided by the rank count, as
    denoise.data_parallel_step does with the device gradient buffer."""
    import torch
    import torch.distributed as dist

    from oracle import denoise_oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        params, x, t = _dp_inputs()
        loss, g, _ = O.loss_and_grads(params, x[rank:rank + 1], t[rank:rank + 1])
        gt = torch.from_numpy(np.asarray(g, np.float64).copy())
        dist.all_reduce(gt, op=dist.ReduceOp.SUM)
        gt.div_(world)
        lt = torch.tensor([float(loss)], dtype=torch.float64)
        dist.all_reduce(lt, op=dist.ReduceOp.SUM)
        if rank == 0:
            np.save(os.path.join(out_dir, "grad.npy"), gt.numpy())
            np.save(os.path.join(out_dir, "loss.npy"), lt.numpy() / world)
    finally:
        dist.destroy_process_group()


class _OracleDenoiser:
    """The calls data_parallel_step makes on a Denoiser, on the CPU: backward
    puts the float64 oracle's gradient of the local mean loss into a float32
    tensor (the device gradient buffer's stand-in), adamw_step records the
    gradient it would apply."""

    def __init__(self, params):
        import torch
        self.params = params
        self.g = torch.zeros(params.size, dtype=torch.float32)
        self.applied = None

    def backward(self, x, t, nb, D, H, W):
        import torch
        from oracle import denoise_oracle as O
        loss, g, _ = O.loss_and_grads(self.params, x, t)
        self.g.copy_(torch.from_numpy(np.asarray(g, np.float32)))
        return float(loss)

    def grad_tensor(self):
        return self.g

    def adamw_step(self, lr, *args):
        self.applied = self.g.numpy().copy()


def _dp_step_rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    from incohautocorrelate_b200 import denoise
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        params, x, t = _dp_inputs()
        dn = _OracleDenoiser(params)
        loss = denoise.data_parallel_step(dn, x[rank:rank + 1], t[rank:rank + 1], 1, 8, 8, 8, 1e-3)
        np.save(os.path.join(out_dir, f"applied{rank}.npy"), dn.applied)
        np.save(os.path.join(out_dir, f"loss{rank}.npy"), np.array([loss]))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_data_parallel_step(tmp_path):
    """denoise.data_parallel_step itself on two gloo ranks: both ranks hand the
    optimizer the same gradient, the whole batch's, and report the whole
    batch's loss (float32 gradient buffer)."""
    import torch.multiprocessing as mp

    from oracle import denoise_oracle as O
    mp.start_processes(_dp_step_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    params, x, t = _dp_inputs()
    loss, g, _ = O.loss_and_grads(params, x, t)
    g = np.asarray(g, np.float64)
    a0, a1 = np.load(tmp_path / "applied0.npy"), np.load(tmp_path / "applied1.npy")
    np.testing.assert_array_equal(a0, a1)
    np.testing.assert_allclose(a0, g, rtol=1e-5, atol=1e-6 * np.abs(g).max())
    for r in range(2):
        np.testing.assert_allclose(np.load(tmp_path / f"loss{r}.npy")[0], float(loss), rtol=1e-12)


def test_two_rank_gloo_data_parallel_gradient(tmp_path):
    """The mean of the ranks' local mean-loss gradients is the gradient of the
    whole batch's mean loss: the identity data-parallel denoiser training
    relies on (equal local batches)."""
    import torch.multiprocessing as mp

    from oracle import denoise_oracle as O
    mp.start_processes(_dp_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    params, x, t = _dp_inputs()
    loss, g, _ = O.loss_and_grads(params, x, t)
    g = np.asarray(g, np.float64)
    got = np.load(tmp_path / "grad.npy")
    assert np.abs(g).max() > 0
    np.testing.assert_allclose(got, g, rtol=1e-9, atol=1e-12 * np.abs(g).max())
    np.testing.assert_allclose(np.load(tmp_path / "loss.npy")[0], float(loss), rtol=1e-12)


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
