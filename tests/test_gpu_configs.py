"""The benchmark configurations at their full sizes, on the GPU through the C
ABI, against the oracle.

* Dense C(q) and AC1D on the 1024 x 1024 radial mean-intensity map (5 %
  masked; 255-edge small mesh; 2 048 |q| bins).  An FP64 oracle over all
  5.5e11 pairs is out of reach on the host, so (as the reference's work items
  are independent) the GPU evaluates the reference's own work items `ind` for
  80 rows -- the detector centre, its corners and edges, masked pixels and 64
  random pixels -- bit for bit against the oracle, with the FP64 error of
  C(q) on those rows reported; and the pair-symmetric production kernels must
  equal the sum of the work items over all 1 048 576 rows, bit for bit.
* The small photon-pair configuration in full: 2 000 frames of a 128 x 128
  detector at Poisson(0.01) into the 65^3 mesh, the C(q) of a uniform
  mean-intensity map and AC1D at 256 bins.
* The simulator configuration's detector: 512 x 512 pixels, a 5 x 5 x 8
  crystal (200 emitters), 4 modes, no sub-sampling, on a pixel subset of the
  full frames, with the FP64 error stated.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _zeros(n, dtype=None):
    import torch
    return torch.zeros(int(n), dtype=dtype or torch.int64, device="cuda")


def _u64(t):
    return t.cpu().numpy().view(np.uint64)


# ---------------------------------------------------------------------------
# dense 1024 x 1024
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def dense1024():
    from incohautocorrelate_b200 import workloads as W
    n = 1024
    I = W.radial_mean_intensity(n, n, 300.0, 0.02, 0.05, seed=3)
    km, mq = W.kmap_numpy(W.flat_pixel_map(n, n))
    rng = np.random.default_rng(77)
    yx = [(511, 511), (512, 512), (511, 512), (512, 511), (0, 0), (0, n - 1), (n - 1, 0), (n - 1, n - 1),
          (0, 512), (n - 1, 512), (512, 0), (512, n - 1)]
    rows = [y * n + x for y, x in yx]
    rows += [int(i) for i in rng.choice(np.nonzero(I == 0)[0], 4, replace=False)]
    rows += [int(i) for i in rng.choice(n * n, 64, replace=False)]
    return dict(I=I, km=km, mq=mq, npix=n * n, n=n, rows=np.array(rows, np.uint32))


def _fp64_cq_rows(I, km, rows, s):
    """C(q) of the listed work items with every pair value kept in double (no
    Multiplicator truncation): the reference's nearest voxel of each ordered
    pair (float arithmetic, round half away from zero), weight the float
    product I_ind * I_i as a double."""
    k = km.reshape(-1, 3)
    out = np.zeros(s.size_ab * s.size_ab * s.size_c, np.float64)
    cab, cc = (s.size_ab - 1) // 2, (s.size_c - 1) // 2
    maxq = np.float32(s.max_q)
    vp = np.float32(s.voxel_per_dq)
    for r in rows:
        pv = (I[r] * I).astype(np.float32)
        q = (k[r][None, :] - k).astype(np.float32)
        n2 = ((q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2]).astype(np.float32)
        ok = ~(pv < np.float32(1e-37)) & ~(np.sqrt(n2) > maxq)
        qs = (q[ok] * vp).astype(np.float32).astype(np.float64)
        rd = np.where(qs >= 0, np.floor(qs + 0.5), -np.floor(-qs + 0.5)).astype(np.int64)
        fs = rd[:, s.k_a] + cab
        ms = rd[:, s.k_b] + cab
        ss = rd[:, s.k_c] + cc
        out += np.bincount(fs + ms * s.size_ab + ss * s.size_ab * s.size_ab,
                           weights=pv[ok].astype(np.float64), minlength=out.size)
    return out


@pytest.mark.parametrize("interp", [0, 1])
def test_dense_1024_cq_rows_match_oracle(ctx, oracle_lib, dense1024, interp):
    from incohautocorrelate_b200 import capi
    o, d = oracle_lib, dense1024
    s = o.small_cq_mesh_shape(d["mq"], 253)
    assert s.size_ab == 255
    mult = capi.cq_small_multiplicator(d["I"])
    want = np.zeros(s.size_ab * s.size_ab * s.size_c, np.uint64)
    for r in d["rows"]:
        o.lib().iaco_cq_small(o.p(d["I"]), o.p(d["km"]), d["npix"], s, interp, mult, int(r), int(r) + 1,
                              o.p(want))
    sh = capi.small_cq_mesh_shape(d["mq"], 253)
    out = _zeros(want.size)
    ctx.cq_small_rows(_dev(d["I"]), _dev(d["km"]), d["npix"], _dev(d["rows"]), len(d["rows"]), sh, interp, mult,
                      out)
    assert ctx.check() == 0
    got = _u64(out)
    assert want.sum() > 0
    np.testing.assert_array_equal(got, want)
    if interp == 0:  # FP64 error of CQMesh = u64 / Mult on these rows
        f64 = _fp64_cq_rows(d["I"], d["km"], d["rows"], s)
        cq = got.astype(np.float64) / mult
        big = f64 > 1e-3 * f64.max()
        rel = np.abs(cq[big] - f64[big]) / f64[big]
        print(f"\nC(q) 1024^2 rows: max relative error vs FP64 {rel.max():.3e} over {big.sum()} voxels "
              f"(Multiplicator {mult:.3g})")
        assert rel.max() < 2e-4
        assert np.all(cq <= f64 * (1 + 1e-9))  # truncation only lowers a voxel


@pytest.mark.parametrize("interp", [0, 1])
def test_dense_1024_ac1d_rows_match_oracle(ctx, oracle_lib, dense1024, interp):
    from incohautocorrelate_b200 import capi
    o, d = oracle_lib, dense1024
    s = o.ac1d_shape(d["mq"], 2048)
    mult = capi.ac1d_cq_multiplicator(d["I"])
    want = np.zeros(s.size, np.uint64)
    for r in d["rows"]:
        o.lib().iaco_ac1d_cq(o.p(d["I"]), o.p(d["km"]), d["npix"], s, interp, mult, int(r), int(r) + 1,
                             o.p(want))
    sh = capi.ac1d_shape(d["mq"], 2048)
    out = _zeros(s.size)
    ctx.ac1d_cq_rows(_dev(d["I"]), _dev(d["km"]), d["npix"], _dev(d["rows"]), len(d["rows"]), sh, interp, mult,
                     out)
    assert ctx.check() == 0
    assert want.sum() > 0
    np.testing.assert_array_equal(_u64(out), want)


@pytest.mark.parametrize("interp", [0, 1])
def test_dense_1024_production_kernels_equal_the_sum_of_work_items(ctx, dense1024, interp):
    """iac_cq_small (unordered tile pairs, reflection, shared-memory windows)
    and iac_ac1d_cq (unordered pairs, doubled) at full size equal the sum of
    the reference's work items over every pixel, bit for bit."""
    from incohautocorrelate_b200 import capi
    d = dense1024
    dI, dk = _dev(d["I"]), _dev(d["km"])
    all_rows = _dev(np.arange(d["npix"], dtype=np.uint32))
    sh = capi.small_cq_mesh_shape(d["mq"], 253)
    mult = capi.cq_small_multiplicator(d["I"])
    words = sh.size_ab * sh.size_ab * sh.size_c
    prod, items = _zeros(words), _zeros(words)
    ctx.cq_small(dI, dk, d["npix"], sh, interp, mult, prod, fast_size=d["n"])
    ctx.cq_small_rows(dI, dk, d["npix"], all_rows, d["npix"], sh, interp, mult, items)
    assert ctx.check() == 0
    a, b = _u64(prod), _u64(items)
    assert a.sum() > 0
    np.testing.assert_array_equal(a, b)
    s1 = capi.ac1d_shape(d["mq"], 2048)
    m1 = capi.ac1d_cq_multiplicator(d["I"])
    h_prod, h_items = _zeros(s1.size), _zeros(s1.size)
    ctx.ac1d_cq(dI, dk, d["npix"], s1, interp, m1, h_prod)
    ctx.ac1d_cq_rows(dI, dk, d["npix"], all_rows, d["npix"], s1, interp, m1, h_items)
    assert ctx.check() == 0
    np.testing.assert_array_equal(_u64(h_prod), _u64(h_items))


# ---------------------------------------------------------------------------
# the small photon-pair configuration in full
# ---------------------------------------------------------------------------
def test_small_configuration_in_full(ctx, oracle_lib):
    """2 000 frames of 128 x 128 at Poisson(0.01) into the 65^3 mesh (the
    reference's route choice per frame); the uniform mean-intensity map's
    C(q) (nearest and linear) and its 256-bin AC1D; the frames' AC_UW at 256
    bins -- all bit for bit."""
    import torch
    from incohautocorrelate_b200 import capi, workloads as W
    o = oracle_lib
    cfg = W.small_config(nframes=2000, seed=1)
    npix = cfg["npix"]
    shape = capi.big_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    S = shape.size_ab
    assert S == 65
    half, full = _zeros(capi.half_mesh_words(S)), _zeros(capi.full_mesh_words(S))
    ctx.sparse_ac_batch(_dev(cfg["photons"]), _dev(cfg["offsets"].view(np.int64)), _dev(cfg["rot"]), 2000,
                        capi.sparse_params(shape), half)
    ctx.sparse_fold(half, S, full)
    assert ctx.check() == 0
    want, oob = o.sparse_batch(cfg["photons"], cfg["offsets"], cfg["rot"],
                               o.big_mesh_shape(cfg["max_q"], cfg["mesh_size"]), cpu_gpu=-1, det_pixels=npix)
    assert oob == 0 and want.sum() > 0
    np.testing.assert_array_equal(_u64(full), want)

    Iu = np.full(npix, 0.01, np.float32)  # uniform mean intensity: the frames' photon rate
    km = cfg["kmap"]
    s = o.small_cq_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    sh = capi.small_cq_mesh_shape(cfg["max_q"], cfg["mesh_size"])
    mult = capi.cq_small_multiplicator(Iu)
    for interp in (0, 1):
        w = np.zeros(s.size_ab * s.size_ab * s.size_c, np.uint64)
        o.lib().iaco_cq_small(o.p(Iu), o.p(km), npix, s, interp, mult, 0, npix, o.p(w))
        g = _zeros(w.size)
        ctx.cq_small(_dev(Iu), _dev(km), npix, sh, interp, mult, g, fast_size=128)
        assert ctx.check() == 0
        np.testing.assert_array_equal(_u64(g), w)

    a1 = capi.ac1d_shape(cfg["max_q"], 256)
    s1 = o.ac1d_shape(cfg["max_q"], 256)
    m1 = capi.ac1d_cq_multiplicator(Iu)
    for interp in (0, 1):
        w = np.zeros(256, np.uint64)
        o.lib().iaco_ac1d_cq(o.p(Iu), o.p(km), npix, s1, interp, m1, 0, npix, o.p(w))
        g = _zeros(256)
        ctx.ac1d_cq(_dev(Iu), _dev(km), npix, a1, interp, m1, g)
        assert ctx.check() == 0
        np.testing.assert_array_equal(_u64(g), w)

    acc = _zeros(capi.ac1d_uw_words(a1))
    uw = torch.zeros(256, dtype=torch.float64, device="cuda")
    ctx.ac1d_uw_batch(_dev(cfg["photons"]), _dev(cfg["offsets"].view(np.int64)), 2000, npix, a1, 0, acc)
    ctx.ac1d_uw_finish(acc, a1, uw)
    want_uw = np.zeros(256)
    o.lib().iaco_ac1d_uw_frames(o.p(cfg["photons"]), o.p(cfg["offsets"]), 2000, npix, s1.max_q, s1.dq_per_step,
                                256, 0, -1, o.p(want_uw))
    np.testing.assert_array_equal(uw.cpu().numpy(), want_uw)


# ---------------------------------------------------------------------------
# the simulator configuration's detector
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("squared", [1, 0])
def test_simulator_512_detector_200_emitters(ctx, oracle_lib, squared):
    """Full 512 x 512 frames on the GPU; 4 096 pixels (corners, centre and
    random) against the FP32 restatement of SimulateCrystal within 2e-5 of
    the frame maximum, and against FP64."""
    import torch
    from incohautocorrelate_b200 import capi, workloads as W
    from test_gpu_simulate import gpu_emitters, lattice
    o = oracle_lib
    n = 512
    pm = (W.flat_pixel_map(n, n) * np.float32(1e10)).astype(np.float32)  # Angstrom
    npix = n * n
    atoms = lattice(o, cells=(5, 5, 8), a=4.0)
    assert len(atoms) == 200
    nmodes, nframes = 4, 2
    em, cnt, rot, rc = gpu_emitters(ctx, atoms, nframes, nmodes, seed=2024)
    us = 75e-6 * 1e10
    sp = capi.SimParams(0, (C.c_double * 3)(us, 0, 0), (C.c_double * 3)(0, us, 0), 1.55, squared, 0)
    out = torch.zeros((nframes, npix), dtype=torch.float32, device="cuda")
    ctx.simulate_intensity(_dev(pm), npix, em, cnt, len(atoms), nmodes, nframes, sp, out)
    assert ctx.check() == 0
    got, emn = out.cpu().numpy(), em.cpu().numpy()
    rng = np.random.default_rng(4)
    idx = np.unique(np.concatenate([[0, n - 1, npix - n, npix - 1, (n // 2) * n + n // 2],
                                    rng.choice(npix, 4091, replace=False)]))
    sub = np.ascontiguousarray(pm.reshape(-1, 3)[idx].reshape(-1))
    P = np.array([len(atoms), 1, 0, us, 0, 0, 0, us, 0, 1.55], np.float64)
    worst = 0.0
    for f in range(nframes):
        want = np.zeros(len(idx), np.float32)
        f64 = np.zeros(len(idx), np.float64)
        for m in range(nmodes):
            e = np.ascontiguousarray(emn[f, m])
            t = np.zeros(len(idx), np.float32)
            o.lib().iaco_simulate_crystal(o.p(sub), len(idx), o.p(e), len(e), o.p(P), squared, o.p(t))
            want += t
            t64 = np.zeros(len(idx), np.float64)
            o.lib().iaco_simulate_crystal_f64(o.p(sub), len(idx), o.p(e), len(e), o.p(P), squared, o.p(t64))
            f64 += t64
        scale = float(got[f].max())
        assert scale > 0
        np.testing.assert_allclose(got[f][idx], want, atol=2e-5 * scale, rtol=0)
        err = float(np.abs(got[f][idx].astype(np.float64) - f64).max()) / scale
        worst = max(worst, err)
        assert err < 1e-3
    print(f"\nsimulator 512^2, 200 emitters x 4 modes ({'|Psi|^2' if squared else '|Psi|'}): "
          f"max |GPU - FP64| = {worst:.2e} of the frame maximum")
