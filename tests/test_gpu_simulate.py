"""(d) Simulator on the GPU through the C ABI against the oracle: emitter
generation, the emitter-phase intensity (FP32 reference arithmetic within a
stated tolerance, error against FP64 reported), Poisson photon draws (the same
counter-based streams: identical counts) and device photonisation (exact)."""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RNG_ROTATION = 0x02 << 56
RNG_PHASE = 0x03 << 56
RNG_YIELD = 0x04 << 56
RNG_POISSON = 0x01 << 56


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def lattice(o, cells=(5, 5, 8), a=4.0):
    LV = np.diag([a, a, a]).astype(np.float64).reshape(-1)
    n = cells[0] * cells[1] * cells[2]
    atoms = np.zeros(3 * n, np.float64)
    o.lib().iaco_crystal_lattice(o.p(LV), (C.c_uint32 * 3)(*cells), o.p(np.zeros(3)), 1,
                                 o.p(atoms))
    return atoms.reshape(-1, 3)


def oracle_emitters(o, atoms, f, mode, seed, yield_=1.0, iso=1.0, rand=True):
    """Crystal::GetEmitters (IAC/Crystal.cpp:29-120) with the device's
    counter-based draws, restated with the oracle's Philox."""
    U = lambda stream, idx, d: o.lib().iaco_uniform_double(seed, stream, idx, d)
    m = np.eye(3)
    if rand:
        for t in range(256):
            v0 = U(RNG_ROTATION | f, 2 * t, 0) * 2. - 1.
            v1 = (U(RNG_ROTATION | f, 2 * t, 1) * 2. - 1.) * iso
            v2 = (U(RNG_ROTATION | f, 2 * t + 1, 0) * 2. - 1.) * iso
            if not (v0 * v0 + v1 * v1 + v2 * v2 > 1) and (v0 or v1 or v2):
                break
        alpha = U(RNG_ROTATION | f, 1 << 20, 0) * 2 * math.pi
        R = (C.c_float * 9)()
        o.lib().iaco_rotation_axis_angle(alpha, (C.c_double * 3)(v0, v1, v2), R)
        ax = np.array([v0, v1, v2]) / math.sqrt(v0 * v0 + v1 * v1 + v2 * v2)
        c, s = math.cos(alpha), math.sin(alpha)
        m = np.array([[ax[0] * ax[0] * (1 - c) + c, ax[1] * ax[0] * (1 - c) - ax[2] * s,
                       ax[2] * ax[0] * (1 - c) + ax[1] * s],
                      [ax[0] * ax[1] * (1 - c) + ax[2] * s, ax[1] * ax[1] * (1 - c) + c,
                       ax[2] * ax[1] * (1 - c) - ax[0] * s],
                      [ax[0] * ax[2] * (1 - c) - ax[1] * s, ax[1] * ax[2] * (1 - c) + ax[0] * s,
                       ax[2] * ax[2] * (1 - c) + c]])
    Rf = m.astype(np.float32)
    inv = (C.c_float * 9)()
    o.lib().iaco_invert3((C.c_float * 9)(*Rf.reshape(-1)), inv)
    em = []
    for i, p in enumerate(atoms):
        if yield_ < 1 and not (U(RNG_YIELD | (mode << 32) | f, i, 0) <= float(np.float32(yield_))):
            continue
        ph = U(RNG_PHASE | (mode << 32) | f, i, 0) * 2.0 * math.pi
        x = m @ p
        em.append([x[0], x[1], x[2], ph])
    return np.array(em, np.float32), np.array(list(inv), np.float32), Rf.reshape(-1)


def gpu_emitters(ctx, atoms, nframes, nmodes, seed, yield_=1.0, iso=1.0, rand=True):
    import torch
    from incohautocorrelate_b200 import capi
    cp = capi.CrystalParams(1, yield_, int(rand), iso)
    na = len(atoms)
    em = torch.zeros((nframes, nmodes, na, 4), dtype=torch.float32, device="cuda")
    cnt = torch.zeros(nframes * nmodes, dtype=torch.int32, device="cuda")
    rot = torch.zeros((nframes, 9), dtype=torch.float32, device="cuda")
    rc = torch.zeros((nframes, 9), dtype=torch.float32, device="cuda")
    ctx.crystal_emitters(_dev(atoms.reshape(-1)), na, nframes, nmodes, cp, seed, em, cnt, rot, rc)
    torch.cuda.synchronize()
    return em, cnt, rot, rc


@pytest.mark.parametrize("yield_", [1.0, 0.6])
def test_crystal_emitters_match(ctx, oracle_lib, yield_):
    o = oracle_lib
    atoms = lattice(o)
    em, cnt, rot, rc = gpu_emitters(ctx, atoms, 6, 3, seed=42, yield_=yield_, iso=0.7)
    em, cnt, rot, rc = em.cpu().numpy(), cnt.cpu().numpy(), rot.cpu().numpy(), rc.cpu().numpy()
    for f in range(6):
        for m in range(3):
            want, inv, Rf = oracle_emitters(o, atoms, f, m, 42, yield_, 0.7)
            n = cnt[f * 3 + m]
            assert n == len(want)
            np.testing.assert_allclose(em[f, m, :n], want, rtol=2e-6, atol=2e-6)
        np.testing.assert_allclose(rot[f], inv, rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(rc[f], Rf, rtol=1e-6, atol=1e-7)
        R = rc[f].reshape(3, 3).astype(np.float64)
        np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-6)


def _sim_setup(o, npx=48, pitch=2e-3, dist=0.10):
    from incohautocorrelate_b200 import workloads as W
    pm = W.flat_pixel_map(npx, npx, pitch=pitch, dist=dist) * np.float32(1e10)  # Angstrom
    return pm


@pytest.mark.parametrize("susa,squared", [(0, 1), (0, 0), (1, 0)])
def test_simulated_intensity_against_reference_arithmetic(ctx, oracle_lib, susa, squared):
    """FP32 phase sums against the oracle's FP32 restatement of SimulateCrystal
    (same argument arithmetic, libm sin/cos) within 2e-5 of the image maximum;
    the error of both against FP64 is the FP32 argument's and is bounded too."""
    import torch
    from incohautocorrelate_b200 import capi
    o = oracle_lib
    pm = _sim_setup(o)
    npix = pm.size // 3
    atoms = lattice(o)
    nmodes, nframes = 4, 3
    em, cnt, rot, rc = gpu_emitters(ctx, atoms, nframes, nmodes, seed=7)
    us = 2e7 / (2 * susa + 1)
    sp = capi.SimParams(susa, (C.c_double * 3)(us, 0, 0), (C.c_double * 3)(0, us, 0), 1.55,
                        squared, 0)
    out = torch.zeros((nframes, npix), dtype=torch.float32, device="cuda")
    ctx.simulate_intensity(_dev(pm), npix, em, cnt, len(atoms), nmodes, nframes, sp, out)
    sp.accurate_sincos = 1
    out_acc = torch.zeros_like(out)
    ctx.simulate_intensity(_dev(pm), npix, em, cnt, len(atoms), nmodes, nframes, sp, out_acc)
    got, got_acc, emn = out.cpu().numpy(), out_acc.cpu().numpy(), em.cpu().numpy()
    P = np.array([len(atoms), 1, susa, us, 0, 0, 0, us, 0, 1.55], np.float64)
    for f in range(nframes):
        want = np.zeros(npix, np.float32)
        f64 = np.zeros(npix, np.float64)
        for m in range(nmodes):
            e = np.ascontiguousarray(emn[f, m])
            t = np.zeros(npix, np.float32)
            o.lib().iaco_simulate_crystal(o.p(pm), npix, o.p(e), len(e), o.p(P), squared, o.p(t))
            want += t
            t64 = np.zeros(npix, np.float64)
            o.lib().iaco_simulate_crystal_f64(o.p(pm), npix, o.p(e), len(e), o.p(P), squared,
                                              o.p(t64))
            f64 += t64
        scale = float(want.max())
        np.testing.assert_allclose(got[f], want, atol=2e-5 * scale, rtol=0)
        np.testing.assert_allclose(got_acc[f], want, atol=2e-5 * scale, rtol=0)
        np.testing.assert_allclose(want, f64, atol=1e-3 * scale, rtol=0)


@pytest.mark.parametrize("cells,nmodes", [((10, 10, 15), 2), ((10, 10, 10), 14)])
def test_large_crystals_stream_through_shared_memory(ctx, oracle_lib, cells, nmodes):
    """Crystals past the shared-memory stage (1 500 emitters; 14 modes x 1 000
    emitters) take the chunked kernel: same tolerance against the oracle."""
    import torch
    from incohautocorrelate_b200 import capi
    o = oracle_lib
    pm = _sim_setup(o, npx=24)
    npix = pm.size // 3
    atoms = lattice(o, cells=cells)
    nframes = 2
    em, cnt, rot, rc = gpu_emitters(ctx, atoms, nframes, nmodes, seed=9)
    us = 2e7
    sp = capi.SimParams(0, (C.c_double * 3)(us, 0, 0), (C.c_double * 3)(0, us, 0), 1.55, 1, 0)
    out = torch.zeros((nframes, npix), dtype=torch.float32, device="cuda")
    ctx.simulate_intensity(_dev(pm), npix, em, cnt, len(atoms), nmodes, nframes, sp, out)
    got, emn = out.cpu().numpy(), em.cpu().numpy()
    P = np.array([len(atoms), 1, 0, us, 0, 0, 0, us, 0, 1.55], np.float64)
    for f in range(nframes):
        want = np.zeros(npix, np.float32)
        for m in range(nmodes):
            e = np.ascontiguousarray(emn[f, m])
            t = np.zeros(npix, np.float32)
            o.lib().iaco_simulate_crystal(o.p(pm), npix, o.p(e), len(e), o.p(P), 1, o.p(t))
            want += t
        np.testing.assert_allclose(got[f], want, atol=2e-5 * float(want.max()), rtol=0)
    assert ctx.check() == 0


def test_poisson_draws_match_oracle(ctx, oracle_lib):
    """Rescaled intensity -> counter-based Poisson draws: the GPU counts equal
    the oracle's draws from the same streams (both evaluate exp/log/cos in
    double; at most a handful of boundary draws may differ)."""
    import torch
    from incohautocorrelate_b200 import capi
    o = oracle_lib
    rng = np.random.default_rng(5)
    nframes, npix = 4, 40000
    I = rng.gamma(0.5, 1.0, (nframes, npix)).astype(np.float32)
    I[1, :10] = 1e6  # means above 25 take the Box-Muller branch
    expected = 900.0
    d = _dev(I)
    pp = capi.PhotonParams(expected, 1, 0.0, 1.0)
    ctx.simulate_photons(d, npix, nframes, 100, pp, 99)
    got = d.cpu().numpy()
    mism = 0
    for f in range(nframes):
        sums = float(I[f].astype(np.float64).sum())
        factor = np.float32(expected / sums)
        lam = (I[f] * factor).astype(np.float32)
        want = np.zeros(npix, np.float32)
        o.lib().iaco_poisson_array(o.p(lam), npix, 99, RNG_POISSON | (100 + f), o.p(want))
        mism += int((want != got[f]).sum())
        assert abs(got[f].sum() - expected) < 6 * math.sqrt(expected) + 10
    assert mism <= 4


def test_sparsify_matches_create_sparse_hit_list(ctx, oracle_lib):
    import torch
    o = oracle_lib
    rng = np.random.default_rng(11)
    nframes, ny, nx = 5, 70, 130
    npix = ny * nx
    I = (rng.poisson(0.05, (nframes, npix)) * rng.uniform(0.8, 3.2, (nframes, npix))).astype(np.float32)
    mask = (rng.random(npix) > 0.05).astype(np.int32)
    from incohautocorrelate_b200 import workloads as W
    km, _ = W.kmap_numpy(W.flat_pixel_map(ny, nx))
    cap = npix * nframes
    d_ph = torch.zeros((cap, 4), dtype=torch.float32, device="cuda")
    d_off = torch.zeros(nframes + 1, dtype=torch.int64, device="cuda")
    for thr, step in [(0.0, 1.0), (0.5, 0.7)]:
        tot = ctx.sparsify_frames(_dev(I), _dev(mask), _dev(km), npix, nframes, thr, step, 1, d_ph,
                                  cap, d_off)
        ph = d_ph.cpu().numpy()
        off = d_off.cpu().numpy()
        assert off[-1] == tot
        for f in range(nframes):
            Im = (I[f] * mask.astype(np.float32)).astype(np.float32)
            out = np.zeros((npix, 4), np.float32)
            n = o.lib().iaco_sparse_hitlist(o.p(Im), o.p(km), npix, thr, step, 1, o.p(out))
            assert off[f + 1] - off[f] == n
            np.testing.assert_array_equal(ph[off[f]:off[f + 1]], out[:n])
