"""(a) sparse photon pairs -> uint64 mesh on the GPU, through the C ABI,
against the oracle.  Integer meshes must match bit for bit."""
import numpy as np
import pytest

from helpers import random_frames, small_detector, to_capi_shape

pytestmark = pytest.mark.gpu

MODES = [(d, i1, i2) for d in (0, 1) for i1 in (0, 1) for i2 in (0, 1) if d or i1 == 0]


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_full_mesh(ctx, photons, offsets, rot, shape, dmap=1, i1=0, i2=0, tuning=None):
    import torch
    from incohautocorrelate_b200 import capi
    S = shape.size_ab
    p = capi.sparse_params(to_capi_shape(shape), i1, i2, dmap, 1000.0)
    half = torch.zeros(capi.half_mesh_words(S), dtype=torch.int64, device="cuda")
    full = torch.zeros(capi.full_mesh_words(S), dtype=torch.int64, device="cuda")
    if tuning:
        ctx.set_sparse_tuning(**tuning)
    ph = _dev(photons if len(photons) else np.zeros((1, 4), np.float32))
    off = _dev(offsets.astype(np.uint64).view(np.int64))
    R = _dev(rot.astype(np.float32))
    ctx.sparse_ac_batch(ph, off, R, len(offsets) - 1, p, half)
    ctx.sparse_fold(half, S, full)
    oob = ctx.check()
    if tuning:
        ctx.set_sparse_tuning()
    return full.cpu().numpy().view(np.uint64), oob


@pytest.mark.parametrize("dmap,i1,i2", MODES)
def test_all_modes_bit_exact(ctx, oracle_lib, rng, dmap, i1, i2):
    from incohautocorrelate_b200 import workloads as W
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    sizes = [0, 1, 2, 3, 9, 31, 64, 65, 127, 200, 0, 5]
    ph, off = random_frames(km, sizes, rng, integer=(i1 == 0 and i2 == 0))
    rot = W.haar_rotations(len(sizes), seed=11)
    want, o1 = oracle_lib.sparse_batch(ph, off, rot, shape, i1, i2, dmap, cpu_gpu=1)
    got, o2 = gpu_full_mesh(ctx, ph, off, rot, shape, dmap, i1, i2)
    assert o1 == 0 and o2 == 0
    np.testing.assert_array_equal(got, want)


def test_small_config_matches_reference_route(ctx, oracle_lib):
    """128^2 detector, Poisson(0.01) frames, identity orientation, 65^3 mesh:
    the reference takes its CPU route for these frames (hits < 1 %)."""
    from incohautocorrelate_b200 import workloads as W
    cfg = W.small_config(nframes=300, seed=1)
    shape = oracle_lib.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    want, _ = oracle_lib.sparse_batch(cfg["photons"], cfg["offsets"], cfg["rot"], shape,
                                      cpu_gpu=-1, det_pixels=cfg["npix"])
    got, oob = gpu_full_mesh(ctx, cfg["photons"], cfg["offsets"], cfg["rot"], shape)
    assert oob == 0
    np.testing.assert_array_equal(got, want)


def test_rotated_config_subset_matches(ctx, oracle_lib):
    """1024x512 two-panel detector, log-normal photon counts, random SO(3)
    orientations, 201^3 mesh: 400 frames against the oracle."""
    from incohautocorrelate_b200 import workloads as W
    cfg = W.rotated_config(nframes=400, seed=2)
    shape = oracle_lib.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    want, _ = oracle_lib.sparse_batch(cfg["photons"], cfg["offsets"], cfg["rot"], shape,
                                      cpu_gpu=-1, det_pixels=cfg["npix"])
    got, oob = gpu_full_mesh(ctx, cfg["photons"], cfg["offsets"], cfg["rot"], shape)
    assert oob == 0
    np.testing.assert_array_equal(got, want)


def test_one_large_frame(ctx, oracle_lib, rng):
    """A 3000-photon frame (4.5 M pairs) spans many queue tiles.  On the
    512k-pixel detector it has < 1 % hit pixels, so the reference takes its
    CPU route (IAC/Detector.cpp:1025-1026)."""
    from incohautocorrelate_b200 import workloads as W
    pm, km, mq, mask = W.rotated_detector()
    shape = oracle_lib.big_mesh_shape(mq, 199)
    ph, off = random_frames(km, [3000, 4, 1500], rng)
    rot = W.haar_rotations(3, seed=4)
    want, _ = oracle_lib.sparse_batch(ph, off, rot, shape, cpu_gpu=-1, det_pixels=512 * 1024)
    got, oob = gpu_full_mesh(ctx, ph, off, rot, shape)
    assert oob == 0
    np.testing.assert_array_equal(got, want)


def test_forced_device_route_differs_only_by_the_fold_quirk(ctx, oracle_lib, rng):
    """Forced through the reference's device route, a frame that adds more than
    ~1.05e7 to one half-mesh voxel loses units in the per-frame fold
    FloatToInt(H / 1000) (float Step 0.001f, IAC/Detector.cpp:1156-1158).  The
    batched mesh equals the oracle everywhere else and, at those voxels,
    exceeds it by exactly H - FloatToInt(H / 1000)."""
    from incohautocorrelate_b200 import workloads as W
    o = oracle_lib
    pm, km, mq, mask = W.rotated_detector()
    shape = o.big_mesh_shape(mq, 199)
    ph, off = random_frames(km, [3000], rng)
    rot = W.haar_rotations(1, seed=4)
    want, _ = o.sparse_batch(ph, off, rot, shape, cpu_gpu=1)
    got, _ = gpu_full_mesh(ctx, ph, off, rot, shape)
    S = shape.size_ab
    half = np.zeros(o.half_words(S), np.uint64)
    P = o.sparse_params_array(shape, len(ph), 1, 0, 0)
    o.lib().iaco_sparse_ac_halfmesh(o.p(ph), len(ph), o.p(P), o.p(rot[0]), o.p(half))
    exact = np.zeros(S ** 3, np.uint64)
    o.lib().iaco_fold_halfmesh(o.p(half), S, 1.0, 1.0, 0.0, o.p(exact))  # identity fold
    np.testing.assert_array_equal(got, exact)
    diff = (got.astype(np.int64) - want.astype(np.int64))
    big = exact > 10_000_000
    assert (diff[~big] == 0).all()
    assert (diff[big] >= 0).all()


@pytest.mark.parametrize("tuning", [dict(tile_pairs=64, block_threads=64, ctas_per_sm=1),
                                    dict(tile_pairs=1000, block_threads=96, ctas_per_sm=3),
                                    dict(tile_pairs=65536, block_threads=256, ctas_per_sm=16)])
def test_tuning_does_not_change_the_mesh(ctx, oracle_lib, rng, tuning):
    from incohautocorrelate_b200 import workloads as W
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    ph, off = random_frames(km, [1, 70, 300, 2, 45], rng)
    rot = W.haar_rotations(5, seed=8)
    want, _ = oracle_lib.sparse_batch(ph, off, rot, shape)
    got, _ = gpu_full_mesh(ctx, ph, off, rot, shape, tuning=tuning)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("edge", [5, 7, 15])
@pytest.mark.parametrize("dmap,i1,i2", [(0, 0, 0), (1, 0, 0), (1, 1, 1)])
def test_tiny_meshes_inside_the_shared_box(ctx, oracle_lib, rng, edge, dmap, i1, i2):
    """Meshes of 7^3, 9^3 and 17^3 (the smallest MeshSize with a nonzero
    Voxel_per_dq for this detector is 5): the per-CTA shared-memory box around
    q = 0 shrinks to the mesh's centre C and covers whole planes; at 1 and 16
    CTAs per SM (largest and smallest box).  Frames of at most 25 photons keep
    every frame's sum in one voxel below the reference device route's fold
    quirk (about 1.05e7; all 300 pairs x 9 x 1000, twice on ss = 0, is 5.4e6)."""
    from incohautocorrelate_b200 import workloads as W
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, edge)
    ph, off = random_frames(km, [0, 2, 12, 25, 7, 25, 19], rng, integer=(i1 == 0 and i2 == 0))
    rot = W.haar_rotations(7, seed=13)
    want, o1 = oracle_lib.sparse_batch(ph, off, rot, shape, i1, i2, dmap, cpu_gpu=1)
    for tuning in (dict(ctas_per_sm=1), dict(ctas_per_sm=16, block_threads=128)):
        got, o2 = gpu_full_mesh(ctx, ph, off, rot, shape, dmap, i1, i2, tuning=tuning)
        assert o2 == o1
        np.testing.assert_array_equal(got, want)


def test_empty_inputs(ctx, oracle_lib):
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    off = np.zeros(4, np.uint64)  # three empty frames
    got, oob = gpu_full_mesh(ctx, np.zeros((0, 4), np.float32), off,
                             np.tile(np.eye(3, dtype=np.float32).reshape(1, 9), (3, 1)), shape)
    assert oob == 0 and not got.any()


def test_out_of_mesh_writes_are_counted(ctx, oracle_lib, rng):
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    ph, off = random_frames(km, [60], rng)
    R = np.array([[3, 0, 0, 0, 3, 0, 0, 0, 3]], np.float32)
    want, o1 = oracle_lib.sparse_batch(ph, off, R, shape)
    got, o2 = gpu_full_mesh(ctx, ph, off, R, shape)
    assert o1 > 0 and o2 == o1
    np.testing.assert_array_equal(got, want)


def test_host_entry_point_accumulates(ctx, oracle_lib, rng):
    """iac_sparse_ac_frames_host: host buffers in, ACMesh::Mesh += result."""
    from incohautocorrelate_b200 import capi, workloads as W
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    ph, off = random_frames(km, [10, 80, 33], rng)
    rot = W.haar_rotations(3, seed=1)
    want, _ = oracle_lib.sparse_batch(ph, off, rot, shape)
    p = capi.sparse_params(to_capi_shape(shape))
    mesh = np.zeros(capi.full_mesh_words(shape.size_ab), np.uint64)
    ctx.sparse_ac_frames_host(ph, off, rot, 3, p, mesh)
    np.testing.assert_array_equal(mesh, want)
    ctx.sparse_ac_frames_host(ph, off, rot, 3, p, mesh)
    np.testing.assert_array_equal(mesh, 2 * want)


def test_host_entry_point_pipelined_chunks(ctx, oracle_lib):
    """1 500 frames go through the host entry point in several copy/compute
    chunks; the mesh equals the device entry point's and the oracle's."""
    import torch
    from incohautocorrelate_b200 import capi, workloads as W
    cfg = W.rotated_config(nframes=1500, seed=31)
    shape = oracle_lib.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    want, _ = oracle_lib.sparse_batch(cfg["photons"], cfg["offsets"], cfg["rot"], shape, cpu_gpu=-1,
                                      det_pixels=cfg["npix"])
    p = capi.sparse_params(to_capi_shape(shape))
    ph = torch.from_numpy(cfg["photons"]).pin_memory()
    off = torch.from_numpy(cfg["offsets"].view(np.int64)).pin_memory()
    rot = torch.from_numpy(cfg["rot"]).pin_memory()
    mesh = torch.zeros(capi.full_mesh_words(shape.size_ab), dtype=torch.int64).pin_memory()
    ctx.sparse_ac_frames_host(ph, off, rot, 1500, p, mesh)
    np.testing.assert_array_equal(mesh.numpy().view(np.uint64), want)
    # a sub-range of frames: offsets that do not start at 0
    mesh.zero_()
    ctx.sparse_ac_frames_host(ph, off[700:].clone(), rot[700:].clone(), 800, p, mesh)
    part, _ = oracle_lib.sparse_batch(cfg["photons"][int(cfg["offsets"][700]):],
                                      cfg["offsets"][700:] - cfg["offsets"][700], cfg["rot"][700:], shape,
                                      cpu_gpu=-1, det_pixels=cfg["npix"])
    np.testing.assert_array_equal(mesh.numpy().view(np.uint64), part)


def test_host_entry_point_into_a_resident_device_mesh(ctx, oracle_lib):
    """iac_sparse_ac_frames_host_to_device: host photon lists of three batches
    (one of them a sub-range with non-zero first offset) accumulate into one
    device half mesh on a caller stream; folded once at the end, the mesh is
    the oracle's.  The host buffers are refilled between calls (the call
    returns once they have been read)."""
    import torch
    from incohautocorrelate_b200 import capi, workloads as W
    cfg = W.rotated_config(nframes=2400, seed=33)
    shape = oracle_lib.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    want, _ = oracle_lib.sparse_batch(cfg["photons"], cfg["offsets"], cfg["rot"], shape, cpu_gpu=-1,
                                      det_pixels=cfg["npix"])
    p = capi.sparse_params(to_capi_shape(shape))
    S = shape.size_ab
    stream = torch.cuda.Stream()
    half = torch.zeros(capi.half_mesh_words(S), dtype=torch.int64, device="cuda")
    full = torch.zeros(capi.full_mesh_words(S), dtype=torch.int64, device="cuda")
    off_all = cfg["offsets"]
    ph_buf = torch.zeros((len(cfg["photons"]), 4), dtype=torch.float32).pin_memory()
    off_buf = torch.zeros(2401, dtype=torch.int64).pin_memory()
    rot_buf = torch.zeros((2400, 9), dtype=torch.float32).pin_memory()
    for f0, f1, rebase in ((0, 1000, True), (1000, 1900, False), (1900, 2400, True)):
        p0, p1 = int(off_all[f0]), int(off_all[f1])
        # rebased offsets index the buffer from 0; the others from the batch's
        # place in the whole photon array
        at = 0 if rebase else p0
        ph_buf[at: at + p1 - p0].copy_(torch.from_numpy(cfg["photons"][p0:p1]))
        off_buf[: f1 - f0 + 1].copy_(torch.from_numpy(off_all[f0:f1 + 1].astype(np.int64) - p0 + at))
        rot_buf[: f1 - f0].copy_(torch.from_numpy(cfg["rot"][f0:f1]))
        ctx.sparse_ac_frames_host_to_device(ph_buf, off_buf, rot_buf, f1 - f0, p, half, stream.cuda_stream)
    ctx.sparse_fold(half, S, full, stream.cuda_stream)
    stream.synchronize()
    assert ctx.check() == 0
    np.testing.assert_array_equal(full.cpu().numpy().view(np.uint64), want)


def test_cache_hint_setting_does_not_change_the_mesh(ctx, oracle_lib, rng):
    from incohautocorrelate_b200 import workloads as W
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    ph, off = random_frames(km, [5, 90, 200, 1, 33], rng)
    rot = W.haar_rotations(5, seed=18)
    want, _ = oracle_lib.sparse_batch(ph, off, rot, shape)
    for hints in (1, 2):
        got, _ = gpu_full_mesh(ctx, ph, off, rot, shape, tuning=dict(cache_hints=hints))
        np.testing.assert_array_equal(got, want)


def test_full_size_properties(ctx):
    """100 000 rotated frames at 201^3: point symmetry of the full mesh, the
    batch is the sum of its halves (linearity), and the result does not depend
    on the work-queue tiling."""
    import torch
    from incohautocorrelate_b200 import workloads as W
    cfg = W.rotated_config(nframes=100_000, seed=2)
    from incohautocorrelate_b200 import capi
    shape = capi.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])

    class S:  # oracle-shaped shim for gpu_full_mesh
        pass
    s = S()
    for f, _ in capi.MeshShape._fields_:
        setattr(s, f, getattr(shape, f))
    ph, off, rot = cfg["photons"], cfg["offsets"], cfg["rot"]
    full, oob = gpu_full_mesh(ctx, ph, off, rot, s)
    assert oob == 0
    S_ = shape.size_ab
    m = full.reshape(S_, S_, S_)
    np.testing.assert_array_equal(m, m[::-1, ::-1, ::-1])
    h = len(off) // 2
    a, _ = gpu_full_mesh(ctx, ph[: off[h]], off[: h + 1], rot[:h], s)
    b, _ = gpu_full_mesh(ctx, ph[off[h]:], off[h:] - off[h], rot[h:], s,
                         tuning=dict(tile_pairs=777, block_threads=128, ctas_per_sm=2))
    np.testing.assert_array_equal(a + b, full)
    # every self pair lands on the centre voxel
    w = ph[:, 3].astype(np.int64)
    assert int(m[(S_ - 1) // 2, (S_ - 1) // 2, (S_ - 1) // 2]) >= 1000 * int((w * w).sum())
    del torch
