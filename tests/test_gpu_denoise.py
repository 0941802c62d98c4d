"""The mesh denoiser's device kernels against the float64 CPU oracle
(oracle/denoise_oracle.py): every 3x3x3 layer shape of the network in both
tensor-core backends (tcgen05 + TMEM, mma.sync), the weight gradients, the
whole network's forward pass and parameter gradients, patch extraction, and
a short training run.

Tolerances follow from the BF16 operands: the kernels multiply bf16 values
exactly and accumulate in fp32, so a single layer's pre-rounding result is
within ~1e-6 of the float64 value and its bf16 output within 2^-8 relative;
whole-network outputs carry one bf16 rounding per layer (relative L2 error
of the residual below 3e-2) and so do the gradients (per layer: relative L2
error below 5e-2, cosine similarity above 0.998)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (c0, up0, c1, cout): the forward layers and the data-gradient layers of the network
FWD = [(0, 0, 16, 16), (0, 0, 16, 32), (0, 0, 32, 32), (0, 0, 32, 64), (0, 0, 64, 64), (64, 1, 32, 32),
       (32, 1, 16, 16), (0, 0, 96, 32), (0, 0, 48, 16)]
DGRAD = [(0, 0, 32, 16), (0, 0, 64, 32), (0, 0, 32, 96), (0, 0, 16, 48)]


def _bf16(a):
    """fp32 array -> (bf16 bits as int16 torch tensor on the GPU, the float64 values)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16)
    return t.view(torch.int16).cuda(), t.to(torch.float64).numpy()


def _from_bf16(t):
    import torch
    return t.view(torch.bfloat16).to(torch.float64).cpu().numpy()


BACKENDS = dict(argvalues=[0, 1, 2], ids=["tcgen05_slab", "mma_sync", "tcgen05_tap"])


@pytest.mark.parametrize("backend", **BACKENDS)
@pytest.mark.parametrize("c0,up0,c1,cout", FWD + DGRAD)
@pytest.mark.parametrize("dims", [(2, 8, 8, 16), (2, 4, 6, 10), (4, 16, 32, 64), (3, 2, 6, 14)])
def test_conv3x3_matches_oracle(ctx, rng, backend, c0, up0, c1, cout, dims):
    import torch
    from incohautocorrelate_b200 import capi
    from oracle import denoise_oracle as O
    nb, D, H, W = dims
    cin = c0 + c1
    s1_q, s1 = _bf16(rng.normal(0, 1, (nb, D, H, W, c1)))
    s0_q, s0 = (None, None)
    if c0:
        s0_q, s0 = _bf16(rng.normal(0, 1, (nb, D // 2, H // 2, W // 2, c0)))
    w = rng.normal(0, (2.0 / (27 * cin)) ** 0.5, (cout, 27, cin)).astype(np.float32)
    wt_q, wq = _bf16(capi.conv_weight_tiles(w))
    w64 = wq.reshape(27, cin // 8, cout, 8).transpose(2, 0, 1, 3).reshape(cout, 27, cin)
    b = rng.normal(0, 0.1, cout).astype(np.float32)
    want = O.conv_layer(s0, s1, w64, b.astype(np.float64), True, up0)
    y = torch.zeros((nb, D, H, W, cout), dtype=torch.int16, device="cuda")
    capi.denoise_conv3x3(ctx, backend, s0_q, c0, up0, s1_q, c1, wt_q, torch.from_numpy(b).cuda(), cout, 1,
                         nb, D, H, W, y)
    torch.cuda.synchronize()
    assert ctx.check() == 0
    got = _from_bf16(y)
    scale = np.abs(want).max()
    np.testing.assert_allclose(got, want, rtol=8e-3, atol=1e-5 * scale)


@pytest.mark.parametrize("c1,cout,W", [(48, 16, 128), (96, 32, 64), (16, 48, 128), (32, 96, 64)])
def test_conv3x3_wide_rows_match_oracle(ctx, rng, c1, cout, W):
    """The decoder layers at the row widths of whole-mesh inference (128^3:
    48 -> 16 on rows of 128, 96 -> 32 on rows of 64, and their data-gradient
    shapes), where the dz-concatenated kernel runs one CTA per SM with the
    stages that fit beside its weights."""
    import torch
    from incohautocorrelate_b200 import capi
    from oracle import denoise_oracle as O
    nb, D, H = 1, 5, 3
    s1_q, s1 = _bf16(rng.normal(0, 1, (nb, D, H, W, c1)))
    w = rng.normal(0, (2.0 / (27 * c1)) ** 0.5, (cout, 27, c1)).astype(np.float32)
    wt_q, wq = _bf16(capi.conv_weight_tiles(w))
    w64 = wq.reshape(27, c1 // 8, cout, 8).transpose(2, 0, 1, 3).reshape(cout, 27, c1)
    b = rng.normal(0, 0.1, cout).astype(np.float32)
    want = O.conv_layer(None, s1, w64, b.astype(np.float64), True, 0)
    y = torch.zeros((nb, D, H, W, cout), dtype=torch.int16, device="cuda")
    capi.denoise_conv3x3(ctx, 0, None, 0, 0, s1_q, c1, wt_q, torch.from_numpy(b).cuda(), cout, 1, nb, D, H, W, y)
    torch.cuda.synchronize()
    assert ctx.check() == 0
    got = _from_bf16(y)
    scale = np.abs(want).max()
    np.testing.assert_allclose(got, want, rtol=8e-3, atol=1e-5 * scale)


@pytest.mark.parametrize("slabs", [3, 2, 1, 0], ids=["tcgen05_dz_stacked", "tcgen05", "slabs", "per_tap"])
@pytest.mark.parametrize("c0,up0,c1,cout", [(0, 0, 16, 16), (0, 0, 16, 32), (0, 0, 32, 32), (0, 0, 32, 64),
                                            (0, 0, 64, 64), (64, 1, 32, 32), (32, 1, 16, 16), (0, 0, 48, 16),
                                            (0, 0, 96, 32)])
@pytest.mark.parametrize("dims", [(2, 8, 12, 16), (1, 6, 10, 64)])
def test_wgrad3x3_matches_oracle(ctx, rng, c0, up0, c1, cout, slabs, dims):
    import torch
    from incohautocorrelate_b200 import capi
    from oracle import denoise_oracle as O
    nb, D, H, W = dims
    cin = c0 + c1
    s1_q, s1 = _bf16(rng.normal(0, 1, (nb, D, H, W, c1)))
    s0_q, s0 = (None, None)
    if c0:
        s0_q, s0 = _bf16(rng.normal(0, 1, (nb, D // 2, H // 2, W // 2, c0)))
    g_q, g = _bf16(rng.normal(0, 1, (nb, D, H, W, cout)))
    want_w, want_b = O.wgrad_layer(s0, s1, g, up0)
    dw = torch.zeros((cout, 27, cin), dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    capi.denoise_wgrad3x3(ctx, s0_q, c0, up0, s1_q, c1, g_q, cout, nb, D, H, W, dw, db, slabs=slabs)
    torch.cuda.synchronize()
    sw = np.abs(want_w).max()
    np.testing.assert_allclose(dw.cpu().numpy(), want_w, rtol=1e-4, atol=1e-5 * sw)
    np.testing.assert_allclose(db.cpu().numpy(), want_b, rtol=1e-4, atol=1e-5 * np.abs(want_b).max())


def _random_params(rng, head_scale=0.3):
    from oracle import denoise_oracle as O
    parts = []
    for ci, co in O.SPECS:
        parts.append(rng.normal(0, (2.0 / (27 * ci)) ** 0.5, co * 27 * ci))
        parts.append(rng.normal(0, 0.05, co))
    parts.append(rng.normal(0, head_scale, 16))
    parts.append([0.01])
    return np.concatenate(parts).astype(np.float32)


def _volumes(rng, nb, E):
    x = rng.gamma(2.0, 0.5, (nb, E, E, E)).astype(np.float32)
    t = (x * (1 + 0.2 * rng.normal(size=x.shape))).astype(np.float32)
    return x, t


def _bf16_params(p):
    """The parameters as the device sees them: bf16 weights, fp32 biases and head."""
    import torch
    from oracle import denoise_oracle as O
    q = p.astype(np.float64).copy()
    o = 0
    for ci, co in O.SPECS:
        n = co * 27 * ci
        q[o:o + n] = torch.from_numpy(p[o:o + n]).to(torch.bfloat16).to(torch.float64).numpy()
        o += n + co
    return q


@pytest.mark.parametrize("backend", **BACKENDS)
def test_network_forward_and_gradients_match_oracle(ctx, rng, backend):
    import torch
    from incohautocorrelate_b200 import capi
    from oracle import denoise_oracle as O
    nb, E = 2, 16
    dn = capi.Denoiser(ctx, nb, E, E, E, backend=backend)
    p = _random_params(rng)
    dn.set_params(p)
    x, t = _volumes(rng, nb, E)
    dx, dt = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    out = torch.zeros_like(dx)
    loss = dn.backward(dx, dt, nb, E, E, E, d_out=out)
    g = dn.get_grads()
    assert ctx.check() == 0
    want_loss, want_g, want_out = O.loss_and_grads(_bf16_params(p), x, t)
    o = out.cpu().numpy()
    assert np.linalg.norm(o - want_out) / np.linalg.norm(want_out - x) < 3e-2
    assert abs(loss - want_loss) / want_loss < 3e-2
    off = 0
    for l, (ci, co) in enumerate(O.SPECS + [(16, 1)]):
        n = co * 27 * ci + co if l < 10 else 17
        a, b = g[off:off + n].astype(np.float64), want_g[off:off + n]
        rel = np.linalg.norm(a - b) / np.linalg.norm(b)
        cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
        assert rel < 5e-2 and cos > 0.998, (l, rel, cos)
        off += n
    dn.close()


def test_backends_agree_on_a_full_volume(ctx, rng):
    import torch
    from incohautocorrelate_b200 import capi
    nb, E = 1, 64
    x, _ = _volumes(rng, nb, E)
    dx = torch.from_numpy(x).cuda()
    p = _random_params(rng)
    outs = []
    for be in (0, 1, 2):
        dn = capi.Denoiser(ctx, nb, E, E, E, backend=be)
        dn.set_params(p)
        o = torch.zeros_like(dx)
        dn.forward(dx, nb, E, E, E, o)
        torch.cuda.synchronize()
        outs.append(o.cpu().numpy() - x)
        dn.close()
    assert ctx.check() == 0
    for o in (outs[0], outs[2]):
        assert np.linalg.norm(o - outs[1]) / np.linalg.norm(outs[1]) < 1e-2


def test_training_reduces_the_loss(ctx, rng):
    import torch
    from incohautocorrelate_b200 import capi
    nb, E = 2, 16
    dn = capi.Denoiser(ctx, nb, E, E, E)
    dn.init_params(seed=3)
    # target: a smoothed copy of the input
    x = rng.gamma(2.0, 0.5, (nb, E, E, E)).astype(np.float32)
    k = np.ones(3) / 3
    t = x.copy()
    for ax in (1, 2, 3):
        t = np.apply_along_axis(lambda v: np.convolve(v, k, mode="same"), ax, t)
    dx, dt = torch.from_numpy(x).cuda(), torch.from_numpy(t.astype(np.float32)).cuda()
    first = dn.backward(dx, dt, nb, E, E, E)
    for _ in range(100):
        dn.adamw_step(lr=3e-3)
        last = dn.backward(dx, dt, nb, E, E, E)
    assert ctx.check() == 0
    assert last < 0.5 * first, (first, last)
    dn.close()


def test_crop_patches_and_mesh_input(ctx, rng):
    import torch
    from incohautocorrelate_b200 import capi
    E, P, n = 12, 5, 3
    m = rng.normal(0, 1, (n, E, E, E)).astype(np.float32)
    mq, m64 = _bf16(m)
    plan = np.array([[0, 0, 0, 0, 0], [2, 7, 3, 1, 13], [1, 4, 7, 2, 47]], np.int32)
    out = torch.zeros((3, P, P, P), dtype=torch.float32, device="cuda")
    capi.denoise_crop_patches(ctx, mq, n, E, torch.from_numpy(plan).cuda(), 3, P, out)
    assert ctx.check() == 0
    got = out.cpu().numpy()
    for b, (i, z0, y0, x0, tr) in enumerate(plan):
        perm = [(0, 1, 2), (0, 2, 1), (1, 2, 0), (1, 0, 2), (2, 0, 1), (2, 1, 0)][tr % 6]
        flip = tr // 6
        for z in range(P):
            for y in range(P):
                for x in range(P):
                    c = (z, y, x)
                    s = [c[perm[k]] for k in range(3)]
                    s = [(P - 1 - s[k]) if flip & (1 << k) else s[k] for k in range(3)]
                    assert got[b, z, y, x] == np.float32(m64[i, s[0] + z0, s[1] + y0, s[2] + x0])
    S = 7
    full = rng.integers(0, 1 << 40, S ** 3, dtype=np.uint64)
    d_full = torch.from_numpy(full.view(np.int64)).cuda()
    o32 = torch.zeros(4 ** 3, dtype=torch.float32, device="cuda")
    capi.denoise_mesh_input(ctx, d_full, S, 4, 1e-9, d_f32=o32)
    want = (full.reshape(S, S, S)[:4, :4, :4].astype(np.float64) * 1e-9).astype(np.float32)
    np.testing.assert_array_equal(o32.cpu().numpy().reshape(4, 4, 4), want)


def _frames_to_error(ctx, setup, n_crystals, plain, n_ref, seed):
    import os

    from incohautocorrelate_b200 import capi
    from incohautocorrelate_b200 import denoise as DN
    path = os.path.join(os.path.dirname(capi.__file__), "weights", "denoiser_128.npz")
    params, meta = DN.load_model(path)
    sim = DN.MeshSimulator(ctx, setup)
    E = setup.crop
    dn = capi.Denoiser(ctx, 1, E, E, E)
    dn.set_params(params)
    summary, rows = DN.evaluate(ctx, sim, dn, meta["norm"], n_crystals, 500, plain, n_ref, seed=seed, log=None)
    assert ctx.check() == 0
    dn.close()
    return summary, rows


def test_trained_denoiser_needs_fewer_frames_than_the_plain_mesh(ctx):
    """The committed network (trained on 512 random crystals, 500 -> 50 000
    frames) on held-out crystals it never saw: the denoised 500-frame mesh
    against an independent 40 000-frame reference matches the plain mesh of
    at least 10 times more frames (median over four crystals; measured
    13-26x, median 19x, on 32 crystals with a 100 000-frame reference)."""
    import os

    from incohautocorrelate_b200 import capi
    from incohautocorrelate_b200 import denoise as DN
    _, meta = DN.load_model(os.path.join(os.path.dirname(capi.__file__), "weights", "denoiser_128.npz"))
    summary, rows = _frames_to_error(ctx, DN.SimSetup(**meta["setup"]), 4, [1000, 2000, 5000], 40000, seed=777)
    for r in rows:
        assert r["err_denoised"] < 0.5 * r["err_plain"][500], r
    assert summary["median_gain"] >= 10.0, summary


def test_trained_denoiser_gain_holds_on_the_512_pixel_detector(ctx):
    """The simulator configuration's detector -- 512 x 512 pixels of 75 um at
    0.1 m, the same angular range and 129^3 mesh as the 128 x 128 x 0.3 mm
    detector the network was trained on -- at the training's photon budget per
    frame (328 photons: 0.02 per 0.3 mm pixel): the finer pixel grid changes the
    k-vectors of every photon, and the denoised 500-frame mesh still needs at
    least 10 times fewer frames than the plain mesh (median of three held-out
    crystals against an independent 20 000-frame reference)."""
    import os

    from incohautocorrelate_b200 import capi
    from incohautocorrelate_b200 import denoise as DN
    _, meta = DN.load_model(os.path.join(os.path.dirname(capi.__file__), "weights", "denoiser_128.npz"))
    base = DN.SimSetup(**meta["setup"])
    setup = DN.SimSetup(**dict(meta["setup"], det=512, pitch=base.pitch * base.det / 512,
                               photons_per_pixel=base.photons_per_pixel * (base.det / 512) ** 2, chunk=500))
    summary, rows = _frames_to_error(ctx, setup, 3, [1000, 2000, 5000], 20000, seed=4242)
    for r in rows:
        assert r["err_denoised"] < 0.5 * r["err_plain"][500], r
    assert summary["median_gain"] >= 10.0, summary


def test_graph_replayed_training_matches_eager_steps(ctx, rng):
    """iac_denoise_train_steps (one captured step, replayed) follows the same
    trajectory as the same steps issued one call at a time (fp32 atomics make
    the sums order-dependent, hence a tolerance)."""
    import torch
    from incohautocorrelate_b200 import capi
    nmesh, E, nb, P, steps = 3, 32, 2, 16, 6
    m_in = rng.gamma(2.0, 0.5, (nmesh, E, E, E)).astype(np.float32)
    m_tg = (m_in * (1 + 0.1 * rng.normal(size=m_in.shape))).astype(np.float32)
    d_in = torch.from_numpy(m_in).to(torch.bfloat16).view(torch.int16).cuda()
    d_tg = torch.from_numpy(m_tg).to(torch.bfloat16).view(torch.int16).cuda()
    plans = np.stack([rng.integers(0, nmesh, (steps, nb)), rng.integers(0, E - P + 1, (steps, nb)),
                      rng.integers(0, E - P + 1, (steps, nb)), rng.integers(0, E - P + 1, (steps, nb)),
                      rng.integers(0, 48, (steps, nb))], 2).astype(np.int32)
    lrs = np.linspace(1e-3, 2e-4, steps).astype(np.float32)
    d_plans, d_lrs = torch.from_numpy(plans).cuda(), torch.from_numpy(lrs).cuda()
    p0 = _random_params(rng)
    eager = capi.Denoiser(ctx, nb, P, P, P)
    eager.set_params(p0)
    x = torch.zeros((nb, P, P, P), dtype=torch.float32, device="cuda")
    t = torch.zeros_like(x)
    want = []
    for i in range(steps):
        capi.denoise_crop_patches(ctx, d_in, nmesh, E, d_plans[i], nb, P, x)
        capi.denoise_crop_patches(ctx, d_tg, nmesh, E, d_plans[i], nb, P, t)
        want.append(eager.backward(x, t, nb, P, P, P) * nb * P ** 3)
        eager.adamw_step(lr=float(lrs[i]))
    graph = capi.Denoiser(ctx, nb, P, P, P)
    graph.set_params(p0)
    losses = torch.zeros(steps, dtype=torch.float64, device="cuda")
    graph.train_steps(d_in, d_tg, nmesh, E, d_plans, d_lrs, steps, nb, P, d_losses=losses)
    torch.cuda.synchronize()
    assert ctx.check() == 0
    np.testing.assert_allclose(losses.cpu().numpy(), want, rtol=2e-3)
    a, b = graph.get_params(), eager.get_params()
    assert np.linalg.norm(a - b) / np.linalg.norm(b - p0) < 1e-2
    # a second call reuses the graph and continues the optimizer's step count
    graph.train_steps(d_in, d_tg, nmesh, E, d_plans, d_lrs, steps, nb, P, d_losses=losses)
    torch.cuda.synchronize()
    assert np.isfinite(losses.cpu().numpy()).all()
    eager.close()
    graph.close()


def test_gradient_buffer_feeds_the_optimizer(ctx, rng):
    """iac_denoise_grad_buffer (the in-place all-reduce target of data-parallel
    training): its view holds the gradients iac_denoise_get_grads copies out,
    and what is written into it is what AdamW uses -- zeroed gradients leave
    only the weight decay, w <- w - lr wd w on the weights (biases keep their
    values) -- while data_parallel_step on
    one process is backward + AdamW."""
    import torch
    from incohautocorrelate_b200 import capi, denoise
    dn = capi.Denoiser(ctx, 1, 8, 8, 8)
    try:
        dn.init_params(3)
        x = torch.from_numpy(rng.gamma(2.0, 0.5, (1, 8, 8, 8)).astype(np.float32)).cuda()
        t = (x * 1.1).contiguous()
        dn.backward(x, t, 1, 8, 8, 8)
        g = dn.grad_tensor()
        assert g.numel() == dn.nparams
        np.testing.assert_array_equal(g.cpu().numpy(), dn.get_grads())
        assert float(g.abs().sum()) > 0
        p0 = dn.get_params()
        g.zero_()
        lr, wd = 1e-2, 1e-1
        dn.adamw_step(lr, weight_decay=wd)
        from oracle import denoise_oracle as O
        is_w = []
        for ci, co in O.SPECS:
            is_w += [True] * (co * 27 * ci) + [False] * co
        is_w = np.array(is_w + [True] * 16 + [False])  # the head's 16 weights and its bias
        assert is_w.size == p0.size
        want = np.where(is_w, p0 - np.float32(lr) * (np.float32(wd) * p0), p0)
        np.testing.assert_allclose(dn.get_params(), want, rtol=1e-6, atol=1e-9)
        # one process: the data-parallel step is backward + AdamW, bit for bit
        dn.set_params(p0)
        loss = denoise.data_parallel_step(dn, x, t, 1, 8, 8, 8, 1e-3)
        p1 = dn.get_params()
        dn.set_params(p0)
        loss2 = dn.backward(x, t, 1, 8, 8, 8)
        dn.adamw_step(1e-3)
        assert loss == loss2
        np.testing.assert_array_equal(dn.get_params(), p1)
    finally:
        dn.close()

