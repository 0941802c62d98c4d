"""iac_sparse_ac_batch_static, the batch correlator for callers that may not
allocate device memory while they run (it keeps its work queue in a fixed
device array of the library instead of a buffer grown with cudaMalloc).

Checked through the C ABI against iac_sparse_ac_batch on the same inputs, bit
for bit, on two calls in a row (the second call reuses the array the first
call left behind), plus its size limit.  Collected last so that a run which
stops at the first failure has run every other test first; it also passes on
its own in a fresh process."""
import numpy as np
import pytest

from helpers import to_capi_shape

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _run(ctx, entry, photons, offsets, rot, params, S):
    import torch
    from incohautocorrelate_b200 import capi
    half = torch.zeros(capi.half_mesh_words(S), dtype=torch.int64, device="cuda")
    full = torch.zeros(capi.full_mesh_words(S), dtype=torch.int64, device="cuda")
    entry(_dev(photons), _dev(offsets.view(np.int64)), _dev(rot), len(offsets) - 1, params, half)
    ctx.sparse_fold(half, S, full)
    assert ctx.check() == 0
    return full.cpu().numpy().view(np.uint64)


def test_static_scratch_entry_matches_allocating_entry(ctx):
    from incohautocorrelate_b200 import capi, workloads as W
    # first call: rotated detector, uneven log-normal frames; second call: a
    # different workload and mesh on the array the first call left behind
    cases = [W.rotated_config(nframes=3000, seed=21), W.small_config(nframes=900, seed=3)]
    cases[1]["rot"] = W.haar_rotations(900, seed=8)
    for cfg in cases:
        shape = capi.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])
        params = capi.sparse_params(shape)
        S = shape.size_ab
        want = _run(ctx, ctx.sparse_ac_batch, cfg["photons"], cfg["offsets"], cfg["rot"], params, S)
        got = _run(ctx, ctx.sparse_ac_batch_static, cfg["photons"], cfg["offsets"], cfg["rot"],
                   params, S)
        assert want.sum() > 0
        np.testing.assert_array_equal(got, want)


def test_static_scratch_entry_rejects_batches_beyond_its_array(ctx):
    from incohautocorrelate_b200 import capi
    shape = capi.big_mesh_shape([0.7, 0.4, 0.1], 31)
    params = capi.sparse_params(shape)
    # aligned placeholder pointers: the frame limit is checked before any launch
    with pytest.raises(capi.IacError) as e:
        ctx.sparse_ac_batch_static(256, 256, 256, 200001, params, 256)
    assert e.value.status == capi.IAC_ERR_INVALID_ARG
    assert "200000" in str(e.value)


def test_static_scratch_entry_needs_no_scratch_allocation(ctx):
    """With the context's scratch capped at 64 bytes, on a new stream (which
    has no scratch yet), the allocating entry point fails with
    IAC_ERR_NO_MEMORY before allocating, while the allocation-free one bins
    the batch, bit for bit as the allocating one did without the cap."""
    import torch
    from incohautocorrelate_b200 import capi, workloads as W
    cfg = W.rotated_config(nframes=1500, seed=23)
    shape = capi.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    params = capi.sparse_params(shape)
    S = shape.size_ab
    want = _run(ctx, ctx.sparse_ac_batch, cfg["photons"], cfg["offsets"], cfg["rot"], params, S)
    c = capi.Context(0)
    try:
        c.set_scratch_limit(64)
        s = torch.cuda.Stream()
        ph, off, rot = _dev(cfg["photons"]), _dev(cfg["offsets"].view(np.int64)), _dev(cfg["rot"])
        half = torch.zeros(capi.half_mesh_words(S), dtype=torch.int64, device="cuda")
        with pytest.raises(capi.IacError) as e:
            c.sparse_ac_batch(ph, off, rot, 1500, params, half, s.cuda_stream)
        assert e.value.status == capi.IAC_ERR_NO_MEMORY
        c.sparse_ac_batch_static(ph, off, rot, 1500, params, half, s.cuda_stream)
        full = torch.zeros(capi.full_mesh_words(S), dtype=torch.int64, device="cuda")
        c.sparse_fold(half, S, full, s.cuda_stream)
        assert c.check(s.cuda_stream) == 0
        np.testing.assert_array_equal(full.cpu().numpy().view(np.uint64), want)
    finally:
        c.close()
