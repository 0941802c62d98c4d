"""The oracle's restatement of the dense C(q), C(q) merge, AC1D and simulator
kernels against the reference's own kernel.cl compiled for the CPU."""
import numpy as np
import pytest

from helpers import random_frames, small_detector


def _det(ny=18, nx=22, pitch=6e-4):
    pm, km, mq = small_detector(ny, nx, pitch)
    return pm, km, mq


def _mean_intensity(npix, rng, masked=0.1):
    I = rng.uniform(0.2, 1.5, npix).astype(np.float32)
    I[rng.random(npix) < masked] = 0
    return I


@pytest.mark.parametrize("interp", [0, 1])
def test_cq_small_matches_reference(oracle_lib, ref_lib, rng, interp):
    o = oracle_lib
    pm, km, mq = _det()
    npix = km.size // 3
    I = _mean_intensity(npix, rng)
    s = o.small_cq_mesh_shape(mq, 21)
    mult = o.lib().iaco_cq_small_multiplicator(o.p(I), npix)
    n = s.size_ab * s.size_ab * s.size_c
    want = np.zeros(n, np.uint64)
    P = np.array([npix, s.voxel_per_dq, s.size_ab, s.size_c, s.k_a, s.k_b, s.k_c, interp,
                  s.max_q, mult], np.float64)
    ref_lib.iacref_AutoCorr_CQ_small(o.p(I), o.p(km), o.p(P), o.p(want), npix)
    got = np.zeros(n, np.uint64)
    oob = o.lib().iaco_cq_small(o.p(I), o.p(km), npix, s, interp, mult, 0, npix, o.p(got))
    assert oob == 0
    np.testing.assert_array_equal(got, want)


def test_cq_small_integer_for_photon_counts(oracle_lib, rng):
    """IAC/UnitTest.cpp:215-230: with nearest-neighbour binning the C(q) of
    one photonised frame holds integers (u64 / Multiplicator)."""
    o = oracle_lib
    pm, km, mq = _det()
    npix = km.size // 3
    I = rng.poisson(0.7, npix).astype(np.float32)
    s = o.small_cq_mesh_shape(mq, 21)
    mult = o.lib().iaco_cq_small_multiplicator(o.p(I), npix)
    m = np.zeros(s.size_ab * s.size_ab * s.size_c, np.uint64)
    o.lib().iaco_cq_small(o.p(I), o.p(km), npix, s, 0, mult, 0, npix, o.p(m))
    cq = m.astype(np.float64) / mult
    np.testing.assert_array_equal(cq, np.round(cq))


@pytest.mark.parametrize("interp", [0, 1])
def test_cq_merge_matches_reference(oracle_lib, ref_lib, rng, interp):
    from incohautocorrelate_b200 import workloads as W
    o = oracle_lib
    pm, km, mq = _det()
    npix = km.size // 3
    I = _mean_intensity(npix, rng)
    s = o.small_cq_mesh_shape(mq, 21)
    mult = o.lib().iaco_cq_small_multiplicator(o.p(I), npix)
    n = s.size_ab * s.size_ab * s.size_c
    small_u = np.zeros(n, np.uint64)
    o.lib().iaco_cq_small(o.p(I), o.p(km), npix, s, 0, mult, 0, npix, o.p(small_u))
    small = small_u.astype(np.float64) / mult
    nf = 37
    R = W.haar_rotations(nf, seed=21)
    MI = rng.uniform(0.01, 0.3, nf).astype(np.float32)
    rw = np.zeros(10 * nf, np.float32)
    import ctypes as C
    m = C.c_double()
    o.lib().iaco_cq_merge_weights(o.p(R), o.p(MI), nf, o.p(small), n, o.p(rw), C.byref(m))
    big_n = s.size_ab ** 3
    want = np.zeros(big_n, np.uint64)
    P = np.array([s.voxel_per_dq, s.size_ab, s.size_c, s.k_a, s.k_b, s.k_c, interp, m.value, nf],
                 np.float64)
    ref_lib.iacref_Merge_CQ(o.p(small), o.p(rw), o.p(P), o.p(want), n)
    got = np.zeros(big_n, np.uint64)
    oob = o.lib().iaco_cq_merge(o.p(small), o.p(rw), nf, s, interp, m.value, 0, n, o.p(got))
    assert oob == 0
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("interp", [0, 1])
def test_ac1d_cq_matches_reference(oracle_lib, ref_lib, rng, interp):
    o = oracle_lib
    pm, km, mq = _det()
    npix = km.size // 3
    I = _mean_intensity(npix, rng)
    s = o.ac1d_shape(mq, 97)
    mult = o.lib().iaco_ac1d_cq_multiplicator(o.p(I), npix)
    mar = 10000
    tmp = np.zeros(mar * s.size, np.uint64)
    P = np.array([npix, s.dq_per_step, s.size, interp, s.max_q, mult, mar, 0], np.float64)
    ref_lib.iacref_AutoCorr_CQ_AV(o.p(I), o.p(km), o.p(P), o.p(tmp), npix)
    want = tmp.reshape(mar, s.size).sum(axis=0, dtype=np.uint64)
    got = np.zeros(s.size, np.uint64)
    o.lib().iaco_ac1d_cq(o.p(I), o.p(km), npix, s, interp, mult, 0, npix, o.p(got))
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("interp", [0, 1])
def test_ac1d_sparse_matches_reference(oracle_lib, ref_lib, rng, interp):
    o = oracle_lib
    pm, km, mq = _det(40, 48)
    s = o.ac1d_shape(mq, 101)
    vs = o.lib().iaco_ac1d_vecsize(s.max_q, s.dq_per_step)
    ph, off = random_frames(km, [1, 9, 150, 300], rng)
    mar = 10000
    for f in range(len(off) - 1):
        hl = np.ascontiguousarray(ph[off[f]:off[f + 1]])
        n = len(hl)
        tmp = np.zeros(mar * vs, np.uint64)
        P = np.array([n, vs, s.max_q, s.dq_per_step, 100.0, mar, interp], np.float64)
        ref_lib.iacref_AutoCorr_sparseHL_AAV(o.p(hl), o.p(P), o.p(tmp), n)
        want = tmp.reshape(mar, vs).sum(axis=0, dtype=np.uint64)
        got = np.zeros(vs, np.uint64)
        o.lib().iaco_ac1d_sparse_frame(o.p(hl), n, s.max_q, s.dq_per_step, interp, 100.0, o.p(got))
        np.testing.assert_array_equal(got, want)


def _crystal(o, cells=(2, 2, 3), a=4.0):
    import ctypes as C
    LV = np.diag([a, a, a]).astype(np.float64).reshape(-1)
    uc = np.zeros(3, np.float64)
    n = cells[0] * cells[1] * cells[2]
    atoms = np.zeros(3 * n, np.float64)
    o.lib().iaco_crystal_lattice(o.p(LV), (C.c_uint32 * 3)(*cells), o.p(uc), 1, o.p(atoms))
    return atoms.reshape(-1, 3)


@pytest.mark.parametrize("susa", [0, 1])
def test_simulate_crystal_matches_reference(oracle_lib, ref_lib, rng, susa):
    o = oracle_lib
    from incohautocorrelate_b200 import workloads as W
    pm = W.flat_pixel_map(20, 24, pitch=2e-3, dist=0.1) * np.float32(1e10)  # in Angstrom
    atoms = _crystal(o)
    em = np.zeros((len(atoms), 4), np.float32)
    em[:, :3] = atoms
    em[:, 3] = rng.uniform(0, 2 * np.pi, len(atoms))
    npix = pm.size // 3
    us = 2e7 / (2 * susa + 1)
    P = np.array([len(em), 1, susa, us, 0, 0, 0, us, 0, 1.55], np.float64)
    want = np.zeros(npix, np.float32)
    ref_lib.iacref_SimulateCrystal(o.p(pm), o.p(em), o.p(P), o.p(want), npix)
    got = np.zeros(npix, np.float32)
    o.lib().iaco_simulate_crystal(o.p(pm), npix, o.p(em), len(em), o.p(P), 0, o.p(got))
    np.testing.assert_array_equal(got, want)
    f64 = np.zeros(npix, np.float64)
    o.lib().iaco_simulate_crystal_f64(o.p(pm), npix, o.p(em), len(em), o.p(P), 0, o.p(f64))
    np.testing.assert_allclose(got, f64, rtol=2e-4)


def test_poisson_statistics(oracle_lib):
    """Inversion below a mean of 25 and the clipped Box-Muller normal above
    (IAC/ArrayOperators.h:25-55): mean and variance of many draws."""
    o = oracle_lib
    for mean in (0.02, 0.7, 6.0, 40.0):
        m = np.full(200_000, mean, np.float32)
        out = np.zeros_like(m)
        o.lib().iaco_poisson_array(o.p(m), m.size, 77, 3, o.p(out))
        assert abs(out.mean() - mean) < 5 * np.sqrt(mean / m.size) + (0.51 if mean >= 25 else 0)
        assert abs(out.var() - mean) < 0.05 * mean + 0.01


def test_philox_known_answer(oracle_lib):
    """Philox4x32-10 known-answer vector (counter 0, key 0) from the
    Random123 distribution's kat_vectors."""
    import ctypes as C
    o = oracle_lib
    ctr = (C.c_uint32 * 4)(0, 0, 0, 0)
    key = (C.c_uint32 * 2)(0, 0)
    out = (C.c_uint32 * 4)()
    o.lib().iaco_philox4x32_10(ctr, key, out)
    assert list(out) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
