"""Golden fixtures (tests/golden/*.npz, made by make_golden.py from the
reference's own kernel.cl compiled for the CPU): the oracle's restatement and
the GPU kernels must reproduce them."""
import ctypes as C
import os

import numpy as np
import pytest

from helpers import to_capi_shape

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MODES = [(d, i1, i2) for d in (0, 1) for i1 in (0, 1) for i2 in (0, 1) if d or i1 == 0]


def load(name):
    return dict(np.load(os.path.join(G, name)))


# ---------------------------------------------------------------- oracle ---
@pytest.mark.parametrize("dmap,i1,i2", MODES)
def test_oracle_sparse_fixture(oracle_lib, dmap, i1, i2):
    o = oracle_lib
    g = load("sparse.npz")
    shape = o.big_mesh_shape(g["max_q"], int(g["edge"]))
    k = f"sparse_{dmap}{i1}{i2}"
    ph, off, rot = g[k + "_photons"], g[k + "_offsets"], g[k + "_rot"]
    half = np.zeros(o.half_words(shape.size_ab), np.uint64)
    for f in range(len(off) - 1):
        hl = np.ascontiguousarray(ph[off[f]:off[f + 1]])
        P = o.sparse_params_array(shape, len(hl), dmap, i1, i2)
        o.lib().iaco_sparse_ac_halfmesh(o.p(hl), len(hl), o.p(P), o.p(np.ascontiguousarray(rot[f])), o.p(half))
    np.testing.assert_array_equal(half, g[k + "_half"])


def test_oracle_dense_fixtures(oracle_lib):
    o = oracle_lib
    g = load("dense.npz")
    I, km = g["intensity"], g["kmap"]
    npix = I.size
    s = o.small_cq_mesh_shape(g["max_q"], int(g["perp"]))
    mult = float(g["mult"])
    assert o.lib().iaco_cq_small_multiplicator(o.p(I), npix) == mult
    for interp in (0, 1):
        m = np.zeros(g["cq_small_0"].size, np.uint64)
        o.lib().iaco_cq_small(o.p(I), o.p(km), npix, s, interp, mult, 0, npix, o.p(m))
        np.testing.assert_array_equal(m, g[f"cq_small_{interp}"])
    small = g["cq_small_0"].astype(np.float64) / mult
    nf = len(g["merge_mean_intensity"])
    rw = np.zeros(10 * nf, np.float32)
    mm = C.c_double()
    o.lib().iaco_cq_merge_weights(o.p(g["merge_rot"]), o.p(g["merge_mean_intensity"]), nf, o.p(small),
                                  small.size, o.p(rw), C.byref(mm))
    np.testing.assert_array_equal(rw, g["merge_rw"])
    assert mm.value == float(g["merge_mult"])
    for interp in (0, 1):
        big = np.zeros(g["merge_0"].size, np.uint64)
        o.lib().iaco_cq_merge(o.p(small), o.p(rw), nf, s, interp, mm.value, 0, small.size, o.p(big))
        np.testing.assert_array_equal(big, g[f"merge_{interp}"])
    sh = o.ac1d_shape(g["max_q"], 97)
    for interp in (0, 1):
        h = np.zeros(sh.size, np.uint64)
        o.lib().iaco_ac1d_cq(o.p(I), o.p(km), npix, sh, interp, float(g["ac1d_mult"]), 0, npix, o.p(h))
        np.testing.assert_array_equal(h, g[f"ac1d_cq_{interp}"])


def test_oracle_ac1d_sparse_and_simulate_fixtures(oracle_lib):
    o = oracle_lib
    g = load("ac1d_sparse.npz")
    sh = o.ac1d_shape(g["max_q"], 101)
    vs = o.lib().iaco_ac1d_vecsize(sh.max_q, sh.dq_per_step)
    ph, off = g["photons"], g["offsets"]
    for interp in (0, 1):
        h = np.zeros(vs, np.uint64)
        for f in range(len(off) - 1):
            hl = np.ascontiguousarray(ph[off[f]:off[f + 1]])
            o.lib().iaco_ac1d_sparse_frame(o.p(hl), len(hl), sh.max_q, sh.dq_per_step, interp, 100.0, o.p(h))
        np.testing.assert_array_equal(h, g[f"ac1d_sparse_{interp}"])
    g = load("simulate.npz")
    pm, em = g["pixel_map"], g["emitters"]
    for susa in (0, 1):
        r = np.zeros(pm.size // 3, np.float32)
        o.lib().iaco_simulate_crystal(o.p(pm), pm.size // 3, o.p(em), len(em), o.p(g[f"sim_params_{susa}"]), 0,
                                      o.p(r))
        np.testing.assert_array_equal(r, g[f"sim_{susa}"])


# ------------------------------------------------------------------- GPU ---
def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.gpu
@pytest.mark.parametrize("dmap,i1,i2", MODES)
def test_gpu_sparse_fixture(ctx, oracle_lib, dmap, i1, i2):
    import torch
    from incohautocorrelate_b200 import capi
    g = load("sparse.npz")
    shape = oracle_lib.big_mesh_shape(g["max_q"], int(g["edge"]))
    k = f"sparse_{dmap}{i1}{i2}"
    ph, off, rot = g[k + "_photons"], g[k + "_offsets"], g[k + "_rot"]
    p = capi.sparse_params(to_capi_shape(shape), i1, i2, dmap, 1000.0)
    half = torch.zeros(capi.half_mesh_words(shape.size_ab), dtype=torch.int64, device="cuda")
    ctx.sparse_ac_batch(_dev(ph), _dev(off.astype(np.uint64).view(np.int64)), _dev(rot), len(off) - 1, p, half)
    assert ctx.check() == 0
    np.testing.assert_array_equal(half.cpu().numpy().view(np.uint64), g[k + "_half"])


@pytest.mark.gpu
def test_gpu_dense_fixtures(ctx, oracle_lib):
    import torch
    from incohautocorrelate_b200 import capi
    g = load("dense.npz")
    I, km = g["intensity"], g["kmap"]
    s = to_capi_shape(oracle_lib.small_cq_mesh_shape(g["max_q"], int(g["perp"])))
    for interp in (0, 1):
        for fast in (0, 22):  # linear tiles, 16 x 16 patches of the 18 x 22 detector
            out = torch.zeros(g["cq_small_0"].size, dtype=torch.int64, device="cuda")
            ctx.cq_small(_dev(I), _dev(km), I.size, s, interp, float(g["mult"]), out, fast_size=fast)
            np.testing.assert_array_equal(out.cpu().numpy().view(np.uint64), g[f"cq_small_{interp}"])
    small = g["cq_small_0"].astype(np.float64) / float(g["mult"])
    nf = len(g["merge_mean_intensity"])
    for interp in (0, 1):
        big = torch.zeros(g["merge_0"].size, dtype=torch.int64, device="cuda")
        ctx.cq_merge(_dev(small), _dev(g["merge_rw"]), nf, s, interp, float(g["merge_mult"]), big)
        np.testing.assert_array_equal(big.cpu().numpy().view(np.uint64), g[f"merge_{interp}"])
    sh = capi.ac1d_shape(g["max_q"], 97)
    for interp in (0, 1):
        h = torch.zeros(sh.size, dtype=torch.int64, device="cuda")
        ctx.ac1d_cq(_dev(I), _dev(km), I.size, sh, interp, float(g["ac1d_mult"]), h)
        np.testing.assert_array_equal(h.cpu().numpy().view(np.uint64), g[f"ac1d_cq_{interp}"])
    assert ctx.check() == 0


@pytest.mark.gpu
def test_gpu_ac1d_sparse_fixture(ctx):
    import torch
    from incohautocorrelate_b200 import capi
    g = load("ac1d_sparse.npz")
    sh = capi.ac1d_shape(g["max_q"], 101)
    vs = capi.ac1d_vecsize(sh.max_q, sh.dq_per_step)
    for interp in (0, 1):
        h = torch.zeros(vs, dtype=torch.int64, device="cuda")
        ctx.ac1d_sparse_batch(_dev(g["photons"]), _dev(g["offsets"].astype(np.uint64).view(np.int64)),
                              len(g["offsets"]) - 1, sh.max_q, sh.dq_per_step, interp, 100.0, h)
        np.testing.assert_array_equal(h.cpu().numpy().view(np.uint64), g[f"ac1d_sparse_{interp}"])
