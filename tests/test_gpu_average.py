"""Averaged intensity and per-event statistics on the device
(iac_average_frames / iac_average_finish) against the oracle's restatement of
Detector::LoadAndAverageIntensity (IAC/Detector.cpp:687-790): bit-exact in all
three modes (plain, threshold, photon discretisation), with and without a
mask, over several batches, for pixel counts that take the 4-byte and the
16-byte copy paths of the per-frame sums, and with frames bright enough
(2^24 photons and more) to leave the exact integer sums for the sequential
one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("thr,step", [(0.0, 0.0), (-1.0, 0.0), (0.35, 0.0), (0.2, 1.0), (0.5, 0.73)])
@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("npix", [37 * 53, 4 * 601, 64 * 48])
def test_average_frames_bit_exact(ctx, oracle_lib, rng, thr, step, masked, npix):
    import torch
    o = oracle_lib
    batches = [5, 1, 40]
    mask = (rng.random(npix) > 0.1).astype(np.int32) if masked else None
    sum_o = np.zeros(npix, np.float32)
    discr_o = np.zeros(npix, np.int64)
    d_sum = torch.zeros(npix, dtype=torch.float32, device="cuda")
    d_discr = torch.zeros(npix, dtype=torch.int64, device="cuda")
    d_mask = torch.from_numpy(mask).cuda() if masked else None
    total = 0
    for nf in batches:
        frames = rng.gamma(0.6, 1.3, (nf, npix)).astype(np.float32)
        frames[rng.random((nf, npix)) < 0.3] = 0.0
        if nf > 1:
            frames[nf // 2] *= 2.0 ** 26 / npix  # past 2^24 photons in the sum
        mean_o = np.zeros(nf, np.float32)
        ph_o = np.zeros(nf, np.float32)
        o.lib().iaco_average_frames(o.p(frames), npix, nf, o.p(mask) if masked else None, thr, step,
                                    o.p(sum_o), o.p(discr_o), o.p(mean_o), o.p(ph_o))
        d_mean = torch.zeros(nf, dtype=torch.float32, device="cuda")
        d_ph = torch.zeros(nf, dtype=torch.float32, device="cuda")
        ctx.average_frames(torch.from_numpy(frames).cuda(), npix, nf, d_mask, thr, step, d_sum, d_discr,
                           d_mean, d_ph)
        np.testing.assert_array_equal(d_mean.cpu().numpy(), mean_o)
        if step > 0:
            np.testing.assert_array_equal(d_ph.cpu().numpy(), ph_o)
        total += nf
    if step > 0:
        np.testing.assert_array_equal(d_discr.cpu().numpy(), discr_o)
    else:
        np.testing.assert_array_equal(d_sum.cpu().numpy(), sum_o)
    want = np.zeros(npix, np.float32)
    o.lib().iaco_average_finish(o.p(sum_o), o.p(discr_o) if step > 0 else None, npix, total, o.p(want))
    got = torch.zeros(npix, dtype=torch.float32, device="cuda")
    ctx.average_finish(d_sum, d_discr if step > 0 else None, npix, total, got)
    np.testing.assert_array_equal(got.cpu().numpy(), want)
    assert ctx.check() == 0


@pytest.mark.parametrize("nframes", [8 * 148 + 3, 16 * 148 + 5, 32 * 148 + 7])
@pytest.mark.parametrize("npix", [37 * 53, 4 * 601])
@pytest.mark.parametrize("thr,step", [(0.35, 0.0), (0.2, 1.0)])
def test_average_frames_many_frames(ctx, oracle_lib, rng, nframes, npix, thr, step):
    """Batches large enough for 8, 16 and 32 frames per block of the per-frame sums."""
    import torch
    o = oracle_lib
    mask = (rng.random(npix) > 0.1).astype(np.int32)
    frames = rng.gamma(0.6, 1.3, (nframes, npix)).astype(np.float32)
    frames[:: 97] *= 2.0 ** 26 / npix  # some frames past 2^24 photons
    sum_o = np.zeros(npix, np.float32)
    discr_o = np.zeros(npix, np.int64)
    mean_o = np.zeros(nframes, np.float32)
    ph_o = np.zeros(nframes, np.float32)
    o.lib().iaco_average_frames(o.p(frames), npix, nframes, o.p(mask), thr, step, o.p(sum_o), o.p(discr_o),
                                o.p(mean_o), o.p(ph_o))
    d_sum = torch.zeros(npix, dtype=torch.float32, device="cuda")
    d_discr = torch.zeros(npix, dtype=torch.int64, device="cuda")
    d_mean = torch.zeros(nframes, dtype=torch.float32, device="cuda")
    d_ph = torch.zeros(nframes, dtype=torch.float32, device="cuda")
    ctx.average_frames(torch.from_numpy(frames).cuda(), npix, nframes, torch.from_numpy(mask).cuda(), thr, step,
                       d_sum, d_discr, d_mean, d_ph)
    np.testing.assert_array_equal(d_mean.cpu().numpy(), mean_o)
    if step > 0:
        np.testing.assert_array_equal(d_ph.cpu().numpy(), ph_o)
        np.testing.assert_array_equal(d_discr.cpu().numpy(), discr_o)
    else:
        np.testing.assert_array_equal(d_sum.cpu().numpy(), sum_o)
    assert ctx.check() == 0
