"""The denoiser's CPU oracle on its own (no GPU): parameter layout shared with
the C ABI, the operand-tile helpers, and its autograd gradients against
central finite differences in float64."""
import numpy as np


def test_param_layout_matches_the_c_abi():
    from incohautocorrelate_b200 import capi
    from oracle import denoise_oracle as O
    assert O.param_count() == capi.denoise_param_count() == 353281
    p = np.random.default_rng(1).normal(size=O.param_count())
    np.testing.assert_array_equal(O.pack(O.unpack(p)), p)


def test_weight_tiles():
    from incohautocorrelate_b200 import capi
    rng = np.random.default_rng(2)
    co, ci = 32, 48
    w = rng.normal(size=(co, 27, ci))
    t = capi.conv_weight_tiles(w)
    for _ in range(50):
        o, tap, i = rng.integers(co), rng.integers(27), rng.integers(ci)
        assert t[tap, i // 8, o, i % 8] == w[o, tap, i]
    d = capi.dgrad_weight_tiles(w)  # [27][co/8][ci][8]
    for _ in range(50):
        o, tap, i = rng.integers(co), rng.integers(27), rng.integers(ci)
        assert d[26 - tap, o // 8, i, o % 8] == w[o, tap, i]


def test_dgrad_tiles_are_the_adjoint_convolution():
    """<conv(x; W), g> == <x, conv(g; W')> with W' the data-gradient weights."""
    from incohautocorrelate_b200 import capi
    from oracle import denoise_oracle as O
    rng = np.random.default_rng(3)
    co, ci = 16, 8
    w = rng.normal(size=(co, 27, ci))
    x = rng.normal(size=(1, 4, 5, 6, ci))
    g = rng.normal(size=(1, 4, 5, 6, co))
    y = O.conv_layer(None, x, w, None, False, 0)
    wd = capi.dgrad_weight_tiles(w)  # [27][co/8][ci][8] -> W'[ci][27][co]
    wprime = wd.transpose(2, 0, 1, 3).reshape(ci, 27, co)
    gx = O.conv_layer(None, g, wprime, None, False, 0)
    assert abs((y * g).sum() - (x * gx).sum()) < 1e-9 * abs((y * g).sum())


def test_oracle_gradients_against_finite_differences():
    from oracle import denoise_oracle as O
    rng = np.random.default_rng(4)
    parts = []
    for ci, co in O.SPECS:
        parts.append(rng.normal(0, (2.0 / (27 * ci)) ** 0.5, co * 27 * ci))
        parts.append(rng.normal(0, 0.05, co))
    parts.append(rng.normal(0, 0.3, 16))
    parts.append([0.02])
    p = np.concatenate(parts)
    x = rng.gamma(2.0, 0.5, (1, 8, 8, 8))
    t = x * (1 + 0.1 * rng.normal(size=x.shape))
    loss, g, _ = O.loss_and_grads(p, x, t)
    idx = np.concatenate([rng.integers(0, p.size, 12), [p.size - 1, p.size - 5, 10, 450]])
    for i in idx:
        h = 1e-5 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (O.loss_and_grads(pp, x, t)[0] - O.loss_and_grads(pm, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1e-3, abs(g[i])) + 1e-9, (i, fd, g[i])


def test_training_crystals_span_the_whole_distribution():
    """denoise.random_crystal: lattice constant in [3, 6] A, 2-8 cells per axis,
    1-4 emitters per cell, so 8 to 2048 emitters, centred; a smaller
    max_emitters redraws the larger crystals."""
    from incohautocorrelate_b200 import denoise as DN
    rng = np.random.default_rng(5)
    counts = []
    for _ in range(3000):
        pos, desc = DN.random_crystal(rng)
        assert 3.0 <= desc["a"] <= 6.0
        assert all(2 <= c <= 8 for c in desc["cells"]) and 1 <= desc["per_cell"] <= 4
        n = int(np.prod(desc["cells"])) * desc["per_cell"]
        assert pos.shape == (n, 3)
        np.testing.assert_allclose(pos.mean(0), 0.0, atol=1e-9)
        counts.append(n)
    assert min(counts) >= 8 and max(counts) <= 2048
    assert max(counts) > 1024  # the tail past the simulator's shared-memory stage is drawn
    for _ in range(300):
        pos, _ = DN.random_crystal(rng, max_emitters=256)
        assert len(pos) <= 256
