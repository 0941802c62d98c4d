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
