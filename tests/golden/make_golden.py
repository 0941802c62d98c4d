"""Generate the golden fixtures of tests/golden/ from the reference's own
kernels.

The reference ships no tests or fixtures for this path.  These fixtures are
produced by running the reference's kernel.cl, compiled for the CPU from the
reference checkout (oracle/_ref/libiacref.so, see oracle/Makefile), on small
seeded inputs; the inputs and outputs are stored together.  They pin the
oracle's restatement and the GPU kernels where the reference checkout is not
available.

    python tests/golden/make_golden.py        # rewrites tests/golden/*.npz
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from helpers import random_frames, small_detector  # noqa: E402
from incohautocorrelate_b200 import workloads as W  # noqa: E402

MODES = [(d, i1, i2) for d in (0, 1) for i1 in (0, 1) for i2 in (0, 1) if d or i1 == 0]


def main():
    ref = oracle.ref()
    if ref is None:
        raise SystemExit("oracle/_ref/libiacref.so is missing: run `make -C oracle` with the reference checkout")
    o = oracle
    p = o.p
    rng = np.random.default_rng(2024)

    # ---- sparse pairs (Autocor_sparseHL), half meshes summed over frames ----
    _, km, mq = small_detector()
    shape = o.big_mesh_shape(mq, 31)
    S = shape.size_ab
    sizes = [0, 1, 3, 40, 97]
    out = {"kmap": km, "max_q": np.array(mq, np.float32), "edge": np.array(31), "sizes": np.array(sizes)}
    for dmap, i1, i2 in MODES:
        ph, off = random_frames(km, sizes, rng, integer=(i1 == 0 and i2 == 0))
        rot = W.haar_rotations(len(sizes), seed=int(rng.integers(1 << 30)))
        half = np.zeros(o.half_words(S), np.uint64)
        for f in range(len(sizes)):
            hl = np.ascontiguousarray(ph[off[f]:off[f + 1]])
            P = o.sparse_params_array(shape, len(hl), dmap, i1, i2)
            if len(hl):
                ref.iacref_Autocor_sparseHL(p(hl), p(P), p(np.ascontiguousarray(rot[f])), p(half), len(hl))
        key = f"sparse_{dmap}{i1}{i2}"
        out[key + "_photons"], out[key + "_offsets"], out[key + "_rot"], out[key + "_half"] = ph, off, rot, half
    np.savez_compressed(os.path.join(HERE, "sparse.npz"), **out)

    # ---- dense C(q), merge, AC1D C(q) --------------------------------------
    _, km, mq = small_detector(18, 22, 6e-4)
    npix = km.size // 3
    I = rng.uniform(0.2, 1.5, npix).astype(np.float32)
    I[rng.random(npix) < 0.1] = 0
    s = o.small_cq_mesh_shape(mq, 21)
    mult = o.lib().iaco_cq_small_multiplicator(p(I), npix)
    out = {"kmap": km, "max_q": np.array(mq, np.float32), "intensity": I, "perp": np.array(21),
           "mult": np.array(mult)}
    n = s.size_ab * s.size_ab * s.size_c
    for interp in (0, 1):
        m = np.zeros(n, np.uint64)
        P = np.array([npix, s.voxel_per_dq, s.size_ab, s.size_c, s.k_a, s.k_b, s.k_c, interp, s.max_q, mult],
                     np.float64)
        ref.iacref_AutoCorr_CQ_small(p(I), p(km), p(P), p(m), npix)
        out[f"cq_small_{interp}"] = m
    small = out["cq_small_0"].astype(np.float64) / mult
    nf = 25
    R = W.haar_rotations(nf, seed=77)
    MI = rng.uniform(0.01, 0.3, nf).astype(np.float32)
    rw = np.zeros(10 * nf, np.float32)
    mm = C.c_double()
    o.lib().iaco_cq_merge_weights(p(R), p(MI), nf, p(small), small.size, p(rw), C.byref(mm))
    out.update(merge_rot=R, merge_mean_intensity=MI, merge_rw=rw, merge_mult=np.array(mm.value))
    for interp in (0, 1):
        big = np.zeros(s.size_ab ** 3, np.uint64)
        P = np.array([s.voxel_per_dq, s.size_ab, s.size_c, s.k_a, s.k_b, s.k_c, interp, mm.value, nf], np.float64)
        ref.iacref_Merge_CQ(p(small), p(rw), p(P), p(big), n)
        out[f"merge_{interp}"] = big
    sh = o.ac1d_shape(mq, 97)
    am = o.lib().iaco_ac1d_cq_multiplicator(p(I), npix)
    out["ac1d_mult"] = np.array(am)
    for interp in (0, 1):
        tmp = np.zeros(10000 * sh.size, np.uint64)
        P = np.array([npix, sh.dq_per_step, sh.size, interp, sh.max_q, am, 10000, 0], np.float64)
        ref.iacref_AutoCorr_CQ_AV(p(I), p(km), p(P), p(tmp), npix)
        out[f"ac1d_cq_{interp}"] = tmp.reshape(10000, sh.size).sum(axis=0, dtype=np.uint64)
    np.savez_compressed(os.path.join(HERE, "dense.npz"), **out)

    # ---- AC1D sparse (AutoCorr_sparseHL_AAV), folded modulo VecSize --------
    _, km, mq = small_detector(40, 48, 6e-4)
    sh = o.ac1d_shape(mq, 101)
    vs = o.lib().iaco_ac1d_vecsize(sh.max_q, sh.dq_per_step)
    ph, off = random_frames(km, [1, 9, 150, 310], rng)
    out = {"kmap": km, "max_q": np.array(mq, np.float32), "photons": ph, "offsets": off}
    for interp in (0, 1):
        tot = np.zeros(vs, np.uint64)
        for f in range(len(off) - 1):
            hl = np.ascontiguousarray(ph[off[f]:off[f + 1]])
            tmp = np.zeros(10000 * vs, np.uint64)
            P = np.array([len(hl), vs, sh.max_q, sh.dq_per_step, 100.0, 10000, interp], np.float64)
            ref.iacref_AutoCorr_sparseHL_AAV(p(hl), p(P), p(tmp), len(hl))
            tot += tmp.reshape(10000, vs).sum(axis=0, dtype=np.uint64)
        out[f"ac1d_sparse_{interp}"] = tot
    np.savez_compressed(os.path.join(HERE, "ac1d_sparse.npz"), **out)

    # ---- SimulateCrystal ----------------------------------------------------
    pm = W.flat_pixel_map(20, 24, pitch=2e-3, dist=0.1) * np.float32(1e10)
    LV = np.diag([4.0, 4.0, 4.0]).reshape(-1)
    atoms = np.zeros(3 * 12)
    o.lib().iaco_crystal_lattice(p(LV), (C.c_uint32 * 3)(2, 2, 3), p(np.zeros(3)), 1, p(atoms))
    em = np.zeros((12, 4), np.float32)
    em[:, :3] = atoms.reshape(-1, 3)
    em[:, 3] = rng.uniform(0, 2 * np.pi, 12)
    out = {"pixel_map": pm.astype(np.float32), "emitters": em}
    for susa in (0, 1):
        us = 2e7 / (2 * susa + 1)
        P = np.array([12, 1, susa, us, 0, 0, 0, us, 0, 1.55], np.float64)
        r = np.zeros(pm.size // 3, np.float32)
        ref.iacref_SimulateCrystal(p(pm), p(em), p(P), p(r), pm.size // 3)
        out[f"sim_params_{susa}"] = P
        out[f"sim_{susa}"] = r
    np.savez_compressed(os.path.join(HERE, "simulate.npz"), **out)
    print("fixtures written:", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
