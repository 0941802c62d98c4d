"""Checkpoint and resume of a correlation run (incohautocorrelate_b200.checkpoint):
a run cut short after a few batches and resumed from its checkpoint, in a new
context, ends with the oracle's mesh bit for bit; a checkpoint of other binning
parameters is refused."""
import numpy as np
import pytest

from helpers import random_frames, small_detector, to_capi_shape

pytestmark = pytest.mark.gpu


def _frames(oracle_lib, rng):
    from incohautocorrelate_b200 import workloads as W
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    sizes = rng.integers(0, 90, 300)
    ph, off = random_frames(km, sizes, rng)
    rot = W.haar_rotations(len(sizes), seed=41)
    want, _ = oracle_lib.sparse_batch(ph, off, rot, shape, 0, 0, 1, cpu_gpu=1)
    return shape, ph, off, rot, want


def test_resumed_run_equals_the_oracle(tmp_path, oracle_lib, rng):
    from incohautocorrelate_b200 import capi
    from incohautocorrelate_b200.checkpoint import MeshRun
    shape, ph, off, rot, want = _frames(oracle_lib, rng)
    p = capi.sparse_params(to_capi_shape(shape), 0, 0, True, 1000.0)
    S = shape.size_ab
    path = str(tmp_path / "run.npz")
    ctx = capi.Context(0)
    run = MeshRun(ctx, p, S)
    cursor = run.bin_frames(ph, off, rot, batch=37, checkpoint=path, every=2, stop_after=5)
    assert cursor == 5 * 37
    run.bin_frames(ph, off, rot, batch=37, stop_after=1)  # binned after the last save: lost
    ctx.close()
    ctx2 = capi.Context(0)
    try:
        run2 = MeshRun.resume(ctx2, p, S, path)
        assert run2.cursor == 4 * 37  # the save after batch 4; batch 5 and the next one re-run
        assert run2.bin_frames(ph, off, rot, batch=37, checkpoint=path) == len(off) - 1
        np.testing.assert_array_equal(run2.full_mesh(), want)
        run3 = MeshRun.resume(ctx2, p, S, path)  # a finished run resumes with nothing to do
        assert run3.bin_frames(ph, off, rot, batch=37) == len(off) - 1
        np.testing.assert_array_equal(run3.full_mesh(), want)
    finally:
        ctx2.close()


def test_checkpoint_of_other_parameters_is_refused(tmp_path, oracle_lib, rng):
    from incohautocorrelate_b200 import capi
    from incohautocorrelate_b200.checkpoint import MeshRun
    shape, ph, off, rot, _ = _frames(oracle_lib, rng)
    p = capi.sparse_params(to_capi_shape(shape), 0, 0, True, 1000.0)
    S = shape.size_ab
    path = str(tmp_path / "run.npz")
    ctx = capi.Context(0)
    try:
        MeshRun(ctx, p, S).bin_frames(ph, off, rot, batch=100, checkpoint=path, stop_after=1)
        other = capi.sparse_params(to_capi_shape(shape), 0, 0, False, 1000.0)
        with pytest.raises(ValueError, match="other mesh or binning parameters"):
            MeshRun.resume(ctx, other, S, path)
        # the same parameters but another event list: reordered frames, or fewer
        run = MeshRun.resume(ctx, p, S, path)
        order = np.arange(len(off) - 1)[::-1]
        n = np.diff(off.astype(np.int64))[order]
        off2 = np.concatenate([[0], np.cumsum(n)]).astype(np.uint64)
        ph2 = np.concatenate([ph[int(off[f]):int(off[f + 1])] for f in order])
        for args in ((ph2, off2, rot[order]), (ph, off[:-5], rot[:-5])):
            with pytest.raises(ValueError, match="another event list"):
                run.bin_frames(*args, batch=100)
        assert run.bin_frames(ph, off, rot, batch=100) == len(off) - 1  # the saved list continues
    finally:
        ctx.close()


def test_denoiser_training_resumes_with_its_optimizer_state(rng):
    """The AdamW state round-trips exactly, and training resumed from it follows
    the uninterrupted run (only the order of the gradients' float atomics
    differs), far closer than a restart whose moments start again at zero."""
    import torch
    from incohautocorrelate_b200 import capi
    ctx = capi.Context(0)
    x = torch.from_numpy(rng.gamma(2.0, 0.5, (2, 16, 16, 16, 1)).astype(np.float32)).cuda()
    t = x * 1.1

    def steps(dn, n):
        for _ in range(n):
            dn.backward(x, t, 2, 16, 16, 16)
            dn.adamw_step(1e-3)
        return dn.get_params()

    try:
        dn = capi.Denoiser(ctx, 2, 16, 16, 16)
        dn.init_params(7)
        steps(dn, 5)
        p, m, v, step = dn.get_state()
        assert step == 5 and np.abs(m).max() > 0 and np.abs(v).max() > 0
        a = steps(dn, 4)
        dn2 = capi.Denoiser(ctx, 2, 16, 16, 16)
        dn2.set_state(p, m, v, step)
        p2, m2, v2, step2 = dn2.get_state()
        assert step2 == step
        np.testing.assert_array_equal(p2, p)
        np.testing.assert_array_equal(m2, m)
        np.testing.assert_array_equal(v2, v)
        b = steps(dn2, 4)
        dn3 = capi.Denoiser(ctx, 2, 16, 16, 16)
        dn3.set_params(p)  # parameters only: moments and step start again
        c = steps(dn3, 4)
        # L2 norms over all parameters: AdamW divides by sqrt(v), so the float
        # atomics' ordering noise can move a parameter whose gradient is near
        # zero by a visible amount; the run as a whole must still follow.
        moved = np.linalg.norm(a - p)
        resumed, restarted = np.linalg.norm(b - a), np.linalg.norm(c - a)
        assert resumed < 1e-2 * moved, (resumed, moved)
        assert restarted > 10 * resumed, (restarted, resumed)
        for d in (dn, dn2, dn3):
            d.close()
    finally:
        ctx.close()
