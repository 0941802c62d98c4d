"""(b) dense C(q), (b') C(q) merge and (c) AC1D on the GPU through the C ABI,
against the oracle.  The uint64 accumulators must match bit for bit; the
double outputs the reference derives from them (u64 / Multiplicator) then
match too, except the AC1D sparse sum, whose double accumulation order differs
(relative tolerance 1e-12)."""
import numpy as np
import pytest

from helpers import random_frames, small_detector, to_capi_shape

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _zeros(n):
    import torch
    return torch.zeros(int(n), dtype=torch.int64, device="cuda")


def _u64(t):
    return t.cpu().numpy().view(np.uint64)


def _intensity(npix, rng, masked=0.08):
    I = rng.uniform(0.05, 1.5, npix).astype(np.float32)
    I[rng.random(npix) < masked] = 0
    return I


def _oracle_cq_small(o, I, km, s, interp, mult, rows=None):
    npix = km.size // 3
    m = np.zeros(s.size_ab * s.size_ab * s.size_c, np.uint64)
    r0, r1 = (0, npix) if rows is None else rows
    o.lib().iaco_cq_small(o.p(I), o.p(km), npix, s, interp, mult, r0, r1, o.p(m))
    return m


@pytest.mark.parametrize("interp", [0, 1])
@pytest.mark.parametrize("patches", [False, True])
@pytest.mark.parametrize("ny,nx", [(40, 48), (33, 70), (1, 300)])
def test_cq_small_bit_exact(ctx, oracle_lib, rng, interp, patches, ny, nx):
    """Linear tiles (row length unknown) and 16 x 16 patches, including
    ragged patches at the detector edges and a single-row detector."""
    from incohautocorrelate_b200 import capi
    o = oracle_lib
    pm, km, mq = small_detector(ny, nx, 6e-4)
    npix = ny * nx
    I = _intensity(npix, rng)
    s = o.small_cq_mesh_shape(mq, 31)
    mult = capi.cq_small_multiplicator(I)
    assert mult == o.lib().iaco_cq_small_multiplicator(o.p(I), npix)
    want = _oracle_cq_small(o, I, km, s, interp, mult)
    out = _zeros(want.size)
    ctx.cq_small(_dev(I), _dev(km), npix, to_capi_shape(s), interp, mult, out,
                 fast_size=nx if patches else 0)
    assert ctx.check() == 0
    np.testing.assert_array_equal(_u64(out), want)


@pytest.mark.parametrize("mult", [1000.0, 1234.5, 3.0e9, 2.0 ** 29 - 1])
def test_cq_small_value_paths(ctx, oracle_lib, rng, mult):
    """Integer multiplicators below 2^29 take the exact integer product; the
    others the double product.  Both reproduce the reference's cast."""
    o = oracle_lib
    pm, km, mq = small_detector(24, 40, 6e-4)
    I = _intensity(km.size // 3, rng)
    I[::7] *= np.float32(37.25)
    s = o.small_cq_mesh_shape(mq, 31)
    for fast in (0, 40):
        want = _oracle_cq_small(o, I, km, s, 0, mult)
        out = _zeros(want.size)
        ctx.cq_small(_dev(I), _dev(km), I.size, to_capi_shape(s), 0, mult, out, fast_size=fast)
        assert ctx.check() == 0
        np.testing.assert_array_equal(_u64(out), want)


def test_cq_small_bright_pixels(ctx, oracle_lib, rng):
    """Products at and above 2^23 (|I| up to 4096) in some tiles: those tile
    pairs take the general integer value path, the others the packed one,
    within one launch."""
    o = oracle_lib
    pm, km, mq = small_detector(48, 64, 6e-4)
    I = _intensity(km.size // 3, rng)
    I[5] = np.float32(4096.0)
    I[1000] = np.float32(2896.31)
    I[2500] = np.float32(-3000.0)
    s = o.small_cq_mesh_shape(mq, 31)
    for mult in (1000.0, 2.0 ** 29 - 1):
        want = _oracle_cq_small(o, I, km, s, 0, mult)
        for fast in (0, 64):
            out = _zeros(want.size)
            ctx.cq_small(_dev(I), _dev(km), I.size, to_capi_shape(s), 0, mult, out, fast_size=fast)
            assert ctx.check() == 0
            np.testing.assert_array_equal(_u64(out), want)


def test_cq_small_dense_detector_region(ctx, oracle_lib):
    """The 1024x1024 radial mean-intensity map's geometry on a 128x128 crop,
    255-edge small mesh: exact against the oracle in full."""
    from incohautocorrelate_b200 import capi, workloads as W
    o = oracle_lib
    I = W.radial_mean_intensity(128, 128, 300.0 / 8, 0.02, 0.05, seed=3)
    pm = W.flat_pixel_map(128, 128, pitch=8 * 75e-6)
    km, mq = o.calc_kmap(pm)
    s = o.small_cq_mesh_shape(mq, 253)
    mult = capi.cq_small_multiplicator(I)
    want = _oracle_cq_small(o, I, km, s, 0, mult)
    for fast in (0, 128):
        out = _zeros(want.size)
        ctx.cq_small(_dev(I), _dev(km), I.size, to_capi_shape(s), 0, mult, out, fast_size=fast)
        assert ctx.check() == 0
        np.testing.assert_array_equal(_u64(out), want)


@pytest.mark.parametrize("interp", [0, 1])
def test_dense_shares_sum_to_the_whole(ctx, oracle_lib, rng, interp):
    """iac_cq_small_part / iac_ac1d_cq_part (the per-GPU shares of a run on
    several GPUs): for 2, 3 and 7 shares the shares' meshes and histograms sum
    to the single-launch result bit for bit, which is the oracle's."""
    import torch
    from incohautocorrelate_b200 import capi
    o = oracle_lib
    pm, km, mq = small_detector(48, 80, 6e-4)
    npix = km.size // 3
    I = _intensity(npix, rng)
    s = o.small_cq_mesh_shape(mq, 31)
    mult = capi.cq_small_multiplicator(I)
    want = _oracle_cq_small(o, I, km, s, interp, mult)
    dI, dk = _dev(I), _dev(km)
    for fast in (0, 80):
        for nparts in (2, 3, 7):
            total = _zeros(want.size)
            for part in range(nparts):
                share = _zeros(want.size)
                ctx.cq_small(dI, dk, npix, to_capi_shape(s), interp, mult, share, fast_size=fast, part=part,
                             nparts=nparts)
                total += share
            assert ctx.check() == 0
            np.testing.assert_array_equal(_u64(total), want)
    sa = capi.ac1d_shape(mq, 97)
    m1 = capi.ac1d_cq_multiplicator(I)
    whole = _zeros(sa.size)
    ctx.ac1d_cq(dI, dk, npix, sa, interp, m1, whole)
    for nparts in (2, 3, 7):
        total = _zeros(sa.size)
        for part in range(nparts):
            ctx.ac1d_cq(dI, dk, npix, sa, interp, m1, total, part=part, nparts=nparts)
        assert ctx.check() == 0
        np.testing.assert_array_equal(_u64(total), _u64(whole))
    with pytest.raises(capi.IacError) as e:
        ctx.cq_small(dI, dk, npix, to_capi_shape(s), interp, mult, total, part=3, nparts=3)
    assert e.value.status == capi.IAC_ERR_INVALID_ARG


def test_ac1d_cq_rejects_a_bin_coordinate_past_2_22(ctx, rng):
    """|q| / dq is floored on the FMA pipe, exact below 2^22: a shape whose
    MaxQ / dq reaches it is refused before any launch."""
    from incohautocorrelate_b200 import capi
    pm, km, mq = small_detector(8, 8, 6e-4)
    I = _intensity(64, rng)
    sh = capi.AC1DShape(2048, 1.0, 1.0 / 5e6)
    out = _zeros(2048)
    with pytest.raises(capi.IacError) as e:
        ctx.ac1d_cq(_dev(I), _dev(km), 64, sh, 1, 1e5, out)
    assert e.value.status == capi.IAC_ERR_INVALID_ARG


@pytest.mark.parametrize("interp", [0, 1])
def test_cq_merge_bit_exact(ctx, oracle_lib, rng, interp):
    from incohautocorrelate_b200 import capi, workloads as W
    o = oracle_lib
    pm, km, mq = small_detector(30, 36, 6e-4)
    npix = km.size // 3
    I = _intensity(npix, rng)
    s = o.small_cq_mesh_shape(mq, 31)
    mult = capi.cq_small_multiplicator(I)
    small = _oracle_cq_small(o, I, km, s, 0, mult).astype(np.float64) / mult
    nf = 300
    R = W.haar_rotations(nf, seed=31)
    MI = rng.uniform(0.01, 0.4, nf).astype(np.float32)
    rw, m = capi.cq_merge_weights(R, MI, small)
    import ctypes as C
    rw_o = np.zeros(10 * nf, np.float32)
    m_o = C.c_double()
    o.lib().iaco_cq_merge_weights(o.p(R), o.p(MI), nf, o.p(small), small.size, o.p(rw_o), C.byref(m_o))
    np.testing.assert_array_equal(rw.reshape(-1), rw_o)
    assert m == m_o.value
    want = np.zeros(s.size_ab ** 3, np.uint64)
    o.lib().iaco_cq_merge(o.p(small), o.p(rw_o), nf, s, interp, m, 0, small.size, o.p(want))
    out = _zeros(want.size)
    ctx.cq_merge(_dev(small), _dev(rw), nf, to_capi_shape(s), interp, m, out)
    assert ctx.check() == 0
    np.testing.assert_array_equal(_u64(out), want)


@pytest.mark.parametrize("interp", [0, 1])
@pytest.mark.parametrize("mult_of", ["reference", 1234.5])
def test_ac1d_cq_bit_exact(ctx, oracle_lib, rng, interp, mult_of):
    from incohautocorrelate_b200 import capi
    o = oracle_lib
    pm, km, mq = small_detector(40, 48, 6e-4)
    npix = km.size // 3
    I = _intensity(npix, rng)
    sh_o = o.ac1d_shape(mq, 257)
    sh = capi.ac1d_shape(mq, 257)
    mult = capi.ac1d_cq_multiplicator(I)
    assert mult == o.lib().iaco_ac1d_cq_multiplicator(o.p(I), npix)
    if mult_of != "reference":
        mult = mult_of
    want = np.zeros(sh.size, np.uint64)
    o.lib().iaco_ac1d_cq(o.p(I), o.p(km), npix, sh_o, interp, mult, 0, npix, o.p(want))
    out = _zeros(sh.size)
    ctx.ac1d_cq(_dev(I), _dev(km), npix, sh, interp, mult, out)
    assert ctx.check() == 0
    np.testing.assert_array_equal(_u64(out), want)


@pytest.mark.parametrize("interp", [0, 1])
def test_ac1d_sparse_bit_exact(ctx, oracle_lib, rng, interp):
    from incohautocorrelate_b200 import capi
    o = oracle_lib
    pm, km, mq = small_detector(60, 64, 6e-4)
    sh = capi.ac1d_shape(mq, 256)
    vs = capi.ac1d_vecsize(sh.max_q, sh.dq_per_step)
    assert vs == o.lib().iaco_ac1d_vecsize(sh.max_q, sh.dq_per_step)
    ph, off = random_frames(km, [0, 1, 2, 17, 160, 900, 33], rng)
    want = np.zeros(vs, np.uint64)
    for f in range(len(off) - 1):
        hl = np.ascontiguousarray(ph[off[f]:off[f + 1]])
        o.lib().iaco_ac1d_sparse_frame(o.p(hl), len(hl), sh.max_q, sh.dq_per_step, interp, 100.0,
                                       o.p(want))
    out = _zeros(vs)
    ctx.ac1d_sparse_batch(_dev(ph), _dev(off.view(np.int64)), len(off) - 1, sh.max_q,
                          sh.dq_per_step, interp, 100.0, out)
    np.testing.assert_array_equal(_u64(out), want)
    # AC_UW as the reference's double sum over frames, within 1e-12
    ref = np.zeros(vs)
    for f in range(len(off) - 1):
        h = np.zeros(vs, np.uint64)
        hl = np.ascontiguousarray(ph[off[f]:off[f + 1]])
        o.lib().iaco_ac1d_sparse_frame(o.p(hl), len(hl), sh.max_q, sh.dq_per_step, interp, 100.0,
                                       o.p(h))
        ref += h.astype(np.float64) / 100.0
    np.testing.assert_allclose(_u64(out).astype(np.float64) / 100.0, ref, rtol=1e-12)
