"""The oracle's restatement of the sparse pair path against the reference's own
kernel.cl compiled for the CPU (oracle/_ref), and the reference's invariants."""
import ctypes as C
import itertools

import numpy as np
import pytest

from helpers import random_frames, small_detector

MODES = [(d, i1, i2) for d in (0, 1) for i1 in (0, 1) for i2 in (0, 1) if d or i1 == 0]


def _ref_halfmesh(ref, oracle, hl, R, shape, dmap, i1, i2, mult=1000.0):
    S = shape.size_ab
    half = np.zeros(oracle.half_words(S), np.uint64)
    P = oracle.sparse_params_array(shape, len(hl), dmap, i1, i2, mult)
    if len(hl):
        ref.iacref_Autocor_sparseHL(oracle.p(hl), oracle.p(P), oracle.p(R), oracle.p(half), len(hl))
    return half


def _oracle_halfmesh(oracle, hl, R, shape, dmap, i1, i2, mult=1000.0):
    S = shape.size_ab
    half = np.zeros(oracle.half_words(S), np.uint64)
    P = oracle.sparse_params_array(shape, len(hl), dmap, i1, i2, mult)
    oob = oracle.lib().iaco_sparse_ac_halfmesh(oracle.p(hl), len(hl), oracle.p(P), oracle.p(R),
                                               oracle.p(half))
    return half, oob


@pytest.mark.parametrize("dmap,i1,i2", MODES)
def test_halfmesh_matches_reference_kernel(oracle_lib, ref_lib, rng, dmap, i1, i2):
    from incohautocorrelate_b200 import workloads as W
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    sizes = [0, 1, 2, 7, 40, 120]
    ph, off = random_frames(km, sizes, rng, integer=(i1 == 0 and i2 == 0))
    rots = W.haar_rotations(len(sizes), seed=3)
    for f in range(len(sizes)):
        hl = np.ascontiguousarray(ph[off[f]:off[f + 1]])
        R = np.ascontiguousarray(rots[f])
        want = _ref_halfmesh(ref_lib, oracle_lib, hl, R, shape, dmap, i1, i2)
        got, oob = _oracle_halfmesh(oracle_lib, hl, R, shape, dmap, i1, i2)
        assert oob == 0
        np.testing.assert_array_equal(got, want)


def test_cpu_and_device_routes_agree_for_nearest(oracle_lib, rng):
    """IAC/Detector.cpp:1025-1050 vs :1053-1170: for photon counts the CPU
    route (per-pair FloatToInt, +q and -q) and the device route (half mesh,
    per-frame fold) give the same mesh."""
    from incohautocorrelate_b200 import workloads as W
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    ph, off = random_frames(km, [3, 50, 90, 1, 0, 140], rng)
    rot = W.haar_rotations(len(off) - 1, seed=5)
    cpu, o1 = oracle_lib.sparse_batch(ph, off, rot, shape, cpu_gpu=0)
    dev, o2 = oracle_lib.sparse_batch(ph, off, rot, shape, cpu_gpu=1)
    assert o1 == 0 and o2 == 0
    np.testing.assert_array_equal(cpu, dev)


def test_point_symmetry_and_sum_rule(oracle_lib, rng):
    """M[C+v] = M[C-v]; sum = 1000 * sum over ordered pairs within MaxQ of n_i n_j
    (every pair lies within MaxQ on this detector at QZoom 1)."""
    from incohautocorrelate_b200 import workloads as W
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    ph, off = random_frames(km, [30, 80], rng)
    rot = W.haar_rotations(2, seed=9)
    full, _ = oracle_lib.sparse_batch(ph, off, rot, shape)
    S = shape.size_ab
    m = full.reshape(S, S, S)
    np.testing.assert_array_equal(m, m[::-1, ::-1, ::-1])
    total = 0
    for f in range(2):
        w = ph[off[f]:off[f + 1], 3].astype(np.float64)
        k = ph[off[f]:off[f + 1], :3].astype(np.float64)
        d = np.linalg.norm(k[:, None, :] - k[None, :, :], axis=-1)
        inside = d <= shape.max_q * (1 + 1e-6)
        total += int(round((np.outer(w, w) * inside).sum())) * 1000
    assert int(full.sum()) == total


def test_fold_float_to_int_identity_bound(oracle_lib):
    """The per-frame fold FloatToInt(H / 1000) (IAC/Detector.cpp:1156-1158)
    returns H exactly while H stays below ~1.05e7; beyond that the
    reference's float Step 0.001f makes it drop units.  The batched device
    path folds once per batch, so it reproduces the reference wherever a frame
    adds less than that bound to one voxel."""
    S = 5
    half = np.zeros(oracle_lib.half_words(S), np.uint64)
    vals = np.array([1000, 123456000, 10_000_000, 10_600_000, 50_000_000], np.uint64)
    half[:len(vals)] = vals
    full = np.zeros(S ** 3, np.uint64)
    oracle_lib.lib().iaco_fold_halfmesh(oracle_lib.p(half), S, 1000.0, 0.001, 0.0,
                                        oracle_lib.p(full))
    C0 = (S - 1) // 2
    got = full.reshape(S, S, S)[C0, 0, :len(vals)]
    assert got[0] == 1000 and got[2] == 10_000_000
    assert got[3] < 10_600_000 and got[4] < 50_000_000  # reference quirk beyond the bound


def test_even_mesh_rejected(oracle_lib):
    with pytest.raises(ValueError):
        oracle_lib.big_mesh_shape([0.1, 0.1, 0.01], 64)


def test_out_of_mesh_counted_not_written(oracle_lib, rng):
    _, km, mq = small_detector()
    shape = oracle_lib.big_mesh_shape(mq, 31)
    ph, off = random_frames(km, [60], rng)
    R = np.array([3, 0, 0, 0, 3, 0, 0, 0, 3], np.float32)  # not orthonormal
    half, oob = _oracle_halfmesh(oracle_lib, ph, R, shape, 1, 0, 0)
    assert oob > 0
