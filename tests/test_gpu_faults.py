"""Failure paths on the GPU that fault, trap or hang nothing.

The reference has no error recovery (its device-pool wait has no timeout,
IAC/Detector.cpp:1078-1081; errors end the process).  Here every device wait is
bounded and every failure comes back as an iac_status with a message:

* a device wait on a flag that nothing sets runs out, is counted, and the next
  iac_ctx_check reports IAC_ERR_TIMEOUT; the context then still computes a
  batch bit for bit;
* a scratch request beyond the context's limit fails with IAC_ERR_NO_MEMORY
  before any allocation (device-memory exhaustion, injected on the host), and
  the same call succeeds, bit-exact, once the limit is lifted.
"""
import numpy as np
import pytest

from helpers import random_frames, small_detector, to_capi_shape

pytestmark = pytest.mark.gpu


def _batch(ctx, oracle_lib, rng, seed):
    """One batch of rotated frames through the device correlator, with the
    oracle's mesh for it."""
    import torch
    from incohautocorrelate_b200 import capi, workloads as W
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    sizes = [3, 40, 0, 77, 12]
    ph, off = random_frames(km, sizes, rng)
    rot = W.haar_rotations(len(sizes), seed=seed)
    want, _ = oracle_lib.sparse_batch(ph, off, rot, shape, 0, 0, 1, cpu_gpu=1)
    S = shape.size_ab
    p = capi.sparse_params(to_capi_shape(shape), 0, 0, 1, 1000.0)
    half = torch.zeros(capi.half_mesh_words(S), dtype=torch.int64, device="cuda")
    full = torch.zeros(capi.full_mesh_words(S), dtype=torch.int64, device="cuda")
    args = (torch.from_numpy(ph).cuda(), torch.from_numpy(off.astype(np.uint64).view(np.int64)).cuda(),
            torch.from_numpy(rot.astype(np.float32)).cuda(), len(sizes), p, half)

    def run():
        half.zero_()
        full.zero_()
        ctx.sparse_ac_batch(*args)
        ctx.sparse_fold(half, S, full)
        assert ctx.check() == 0
        return full.cpu().numpy().view(np.uint64)

    return run, want


def test_bounded_wait_times_out_and_the_context_stays_usable(oracle_lib, rng):
    import torch
    from incohautocorrelate_b200 import capi
    ctx = capi.Context(0)
    try:
        flag = torch.zeros(1, dtype=torch.int32, device="cuda")
        ctx.wait_flag(flag, 2000)  # nothing sets it: about 2 ms, then counted
        with pytest.raises(capi.IacError) as err:
            ctx.check()
        assert err.value.status == capi.IAC_ERR_TIMEOUT
        assert "bounded device waits ran out" in str(err.value)
        assert "(flag wait)" in str(err.value)  # the report names the kernel whose wait gave up
        assert ctx.check() == 0  # the counter was cleared by the report
        flag.fill_(1)  # a set flag ends the wait at once, however long the limit
        ctx.wait_flag(flag, 10_000_000)
        assert ctx.check() == 0
        run, want = _batch(ctx, oracle_lib, rng, seed=21)
        np.testing.assert_array_equal(run(), want)
    finally:
        ctx.close()


def test_scratch_limit_fails_before_allocating_then_recovers(oracle_lib, rng):
    from incohautocorrelate_b200 import capi
    ctx = capi.Context(0)  # fresh scratch: nothing grown yet
    try:
        run, want = _batch(ctx, oracle_lib, rng, seed=22)
        ctx.set_scratch_limit(64)
        with pytest.raises(capi.IacError) as err:
            run()
        assert err.value.status == capi.IAC_ERR_NO_MEMORY
        assert "limit" in str(err.value)
        ctx.set_scratch_limit(0)
        np.testing.assert_array_equal(run(), want)
        np.testing.assert_array_equal(run(), want)  # and again, on the grown scratch
    finally:
        ctx.close()
