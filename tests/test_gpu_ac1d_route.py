"""AC_UW of sparse photon lists with the reference's per-frame route choice
(AC1D::Calculate_AC_UW_Mapped, IAC/AC1D.cpp:201-391) on the GPU through the C
ABI, against the oracle's restatement of both routes.

The reference sends a frame with fewer than 0.75 % of the detector's pixels
hit through a host loop over k >= j with a factor 2 (self pairs counted twice,
float products summed in double, :254-293) and every other frame through the
AutoCorr_sparseHL_AAV kernel (:295-379).  Photon counts with nearest binning
make every summand a whole number, so AC_UW must match bit for bit; linear
binning sums fractional floats in double in another order, so it must match
within a relative 1e-12 per bin (the double rounding of ~1e6 summands of
similar size stays far below that)."""
import numpy as np
import pytest

from helpers import random_frames, small_detector

pytestmark = pytest.mark.gpu

RTOL_FLOAT_SUMS = 1e-12


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _gpu_acuw(ctx, photons, offsets, npix, shape, interp, route, batches=1):
    import torch
    from incohautocorrelate_b200 import capi
    acc = torch.zeros(capi.ac1d_uw_words(shape), dtype=torch.int64, device="cuda")
    out = torch.zeros(shape.size, dtype=torch.float64, device="cuda")
    nf = len(offsets) - 1
    cuts = np.linspace(0, nf, batches + 1).astype(int)
    for b in range(batches):  # several batches accumulate into one accumulator
        f0, f1 = cuts[b], cuts[b + 1]
        off = offsets[f0:f1 + 1].astype(np.int64)
        ph = photons[off[0]:off[-1]]
        ctx.ac1d_uw_batch(_dev(ph if len(ph) else np.zeros((1, 4), np.float32)), _dev(off - off[0]), f1 - f0,
                          npix, shape, interp, acc, route=route)
    ctx.ac1d_uw_finish(acc, shape, out)
    assert ctx.check() == 0
    return out.cpu().numpy()


def _oracle_acuw(o, photons, offsets, npix, shape, interp, route):
    ac = np.zeros(shape.size, np.float64)
    o.lib().iaco_ac1d_uw_frames(o.p(np.ascontiguousarray(photons)), o.p(np.ascontiguousarray(offsets, np.uint64)),
                                len(offsets) - 1, int(npix), shape.max_q, shape.dq_per_step, shape.size,
                                int(interp), int(route), o.p(ac))
    return ac


def _routes(offsets, npix):
    n = np.diff(offsets.astype(np.int64)).astype(np.float32)
    return (n / np.float32(npix)) < np.float32(0.0075)  # True: the reference's host loop


@pytest.mark.parametrize("interp", [0, 1])
def test_rotated_detector_frames_take_the_host_route(ctx, oracle_lib, interp):
    """Frames of the rotated-correlator workload (1024 x 512, ~80 photons):
    every one is below 0.75 % and takes the host loop, whose self pairs count
    twice at bin 0 -- unlike the device kernel."""
    from incohautocorrelate_b200 import capi, workloads as W
    o = oracle_lib
    cfg = W.rotated_config(nframes=400, seed=31)
    npix = cfg["npix"]
    assert _routes(cfg["offsets"], npix).all()
    sh = capi.ac1d_shape(cfg["max_q"], 2048)
    got = _gpu_acuw(ctx, cfg["photons"], cfg["offsets"], npix, sh, interp, capi.AC1D_ROUTE_REFERENCE, batches=3)
    want = _oracle_acuw(o, cfg["photons"], cfg["offsets"], npix, sh, interp, -1)
    assert want.sum() > 0
    # bin 0 carries 2 v^2 per photon (nearest: exactly; linear: plus the split of close pairs)
    self2 = 2.0 * float((cfg["photons"][:, 3].astype(np.float64) ** 2).sum())
    if interp == 0:
        np.testing.assert_array_equal(got, want)
        assert got[0] >= self2
    else:
        np.testing.assert_allclose(got, want, rtol=RTOL_FLOAT_SUMS, atol=0)
    # the device kernel alone would give half the self-pair weight at bin 0
    dev = _oracle_acuw(o, cfg["photons"], cfg["offsets"], npix, sh, interp, 1)
    # (the device kernel's bins past VecSize wrap onto the first bins, so allow a margin)
    assert want[0] - dev[0] >= 0.45 * self2


@pytest.mark.parametrize("interp", [0, 1])
def test_dense_frames_keep_the_device_route_bit_exact(ctx, oracle_lib, rng, interp):
    """Frames above 0.75 % take the device kernel: AC_UW = its integer totals
    / 100, identical to iac_ac1d_sparse_batch's."""
    import torch
    from incohautocorrelate_b200 import capi
    o = oracle_lib
    pm, km, mq = small_detector(40, 48, 6e-4)
    npix = 40 * 48
    ph, off = random_frames(km, rng.integers(40, 400, 30), rng, max_count=4)
    assert not _routes(off, npix).any()
    sh = capi.ac1d_shape(mq, 257)
    got = _gpu_acuw(ctx, ph, off, npix, sh, interp, capi.AC1D_ROUTE_REFERENCE)
    want = _oracle_acuw(o, ph, off, npix, sh, interp, -1)
    if interp == 0:
        np.testing.assert_array_equal(got, want)
    else:
        np.testing.assert_allclose(got, want, rtol=RTOL_FLOAT_SUMS, atol=0)
    vs = capi.ac1d_vecsize(sh.max_q, sh.dq_per_step)
    h = torch.zeros(vs, dtype=torch.int64, device="cuda")
    ctx.ac1d_sparse_batch(_dev(ph), _dev(off.view(np.int64)), len(off) - 1, sh.max_q, sh.dq_per_step, interp,
                          100.0, h)
    np.testing.assert_array_equal(got[:vs], h.cpu().numpy().view(np.uint64).astype(np.float64) / 100.0)
    assert (got[vs:] == 0).all()


@pytest.mark.parametrize("interp", [0, 1])
def test_mixed_batch_routes_frame_by_frame(ctx, oracle_lib, rng, interp):
    """One batch whose frames alternate between the two routes, including
    empty and one-photon frames."""
    from incohautocorrelate_b200 import capi
    o = oracle_lib
    pm, km, mq = small_detector(64, 80, 4e-4)
    npix = 64 * 80
    sizes = []
    for i in range(60):
        sizes.append([0, 1, 5, 20, 38, 39, 200, 700][i % 8])  # 0.0075 * 5120 = 38.4
    ph, off = random_frames(km, sizes, rng, max_count=5)
    r = _routes(off, npix)
    assert r.any() and not r.all()
    sh = capi.ac1d_shape(mq, 301)
    got = _gpu_acuw(ctx, ph, off, npix, sh, interp, capi.AC1D_ROUTE_REFERENCE, batches=2)
    want = _oracle_acuw(o, ph, off, npix, sh, interp, -1)
    if interp == 0:
        np.testing.assert_array_equal(got, want)
    else:
        np.testing.assert_allclose(got, want, rtol=RTOL_FLOAT_SUMS, atol=0)


@pytest.mark.parametrize("route", [0, 1])
@pytest.mark.parametrize("integer", [True, False])
def test_forced_routes_and_real_valued_lists(ctx, oracle_lib, rng, route, integer):
    """Either route forced on every frame, with photon counts and with real
    values (non-whole products take the double accumulator)."""
    from incohautocorrelate_b200 import capi
    o = oracle_lib
    pm, km, mq = small_detector(40, 56, 5e-4)
    npix = 40 * 56
    ph, off = random_frames(km, rng.integers(1, 120, 25), rng, max_count=3, integer=integer)
    sh = capi.ac1d_shape(mq, 129)
    for interp in (0, 1):
        got = _gpu_acuw(ctx, ph, off, npix, sh, interp, route)
        want = _oracle_acuw(o, ph, off, npix, sh, interp, route)
        assert want.sum() > 0
        if integer and interp == 0:
            np.testing.assert_array_equal(got, want)
        else:
            np.testing.assert_allclose(got, want, rtol=RTOL_FLOAT_SUMS, atol=1e-9)


def test_rejects_histograms_beyond_shared_memory(ctx):
    import torch
    from incohautocorrelate_b200 import capi
    sh = capi.ac1d_shape([0.5, 0.5, 0.1], 9000)
    acc = torch.zeros(8, dtype=torch.int64, device="cuda")
    ph = torch.zeros((1, 4), dtype=torch.float32, device="cuda")
    off = torch.zeros(2, dtype=torch.int64, device="cuda")
    with pytest.raises(capi.IacError) as e:
        ctx.ac1d_uw_batch(ph, off, 1, 100, sh, 0, acc)
    assert e.value.status == capi.IAC_ERR_INVALID_ARG
