"""ctypes binding of the test oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker, never as the measured or
shipped path.

* ``lib()`` -- liboracle.so, the C restatement in iac_oracle.c.
* ``ref()`` -- _ref/libiacref.so, the reference's own IAC/kernel.cl compiled for
  the CPU (built from the reference checkout by the Makefile; None if absent).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF = os.path.join(HERE, "_ref", "libiacref.so")

_lib = None
_ref = None
VP = C.c_void_p
U64 = C.c_uint64
U32 = C.c_uint32
F = C.c_float
D = C.c_double


class MeshShape(C.Structure):
    _fields_ = [("k_a", U32), ("k_b", U32), ("k_c", U32), ("size_ab", U32), ("size_c", U32),
                ("center", U32 * 3), ("dq_per_voxel", F), ("voxel_per_dq", U32), ("max_q", F)]


class AC1DShape(C.Structure):
    _fields_ = [("size", U32), ("max_q", F), ("dq_per_step", F)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _decl(lib):
    def fn(name, args, res=None):
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    P = C.POINTER
    fn("iaco_calc_kmap", [VP, U64, VP, P(F)])
    fn("iaco_generate_pixel_map", [C.c_int, C.c_int, F, P(F), P(F), P(F), VP])
    fn("iaco_big_mesh_shape", [P(F), C.c_int, F, P(MeshShape)], C.c_int)
    fn("iaco_small_cq_mesh_shape", [P(F), C.c_int, F, P(MeshShape)], C.c_int)
    fn("iaco_ac1d_shape_init", [P(F), U32, F, P(AC1DShape)])
    fn("iaco_discretize_to_photons", [VP, U64, F, F])
    fn("iaco_sparse_hitlist", [VP, VP, U64, F, F, C.c_int, VP], U64)
    fn("iaco_average_frames", [VP, U64, U32, VP, F, F, VP, VP, VP, VP])
    fn("iaco_average_finish", [VP, VP, U64, U32, VP])
    fn("iaco_sparse_ac_halfmesh", [VP, U32, VP, VP, VP], U64)
    fn("iaco_fold_halfmesh", [VP, U32, D, F, F, VP])
    fn("iaco_sparse_ac_cpu_route", [VP, U32, VP, P(MeshShape), C.c_int, C.c_int, C.c_int, F, F,
                                    VP], U64)
    fn("iaco_autocorrelate_sparse_list", [VP, U32, U64, VP, P(MeshShape), C.c_int, C.c_int,
                                          C.c_int, F, F, C.c_int, VP, VP, P(U64)], C.c_int)
    fn("iaco_sparse_ac_batch", [VP, VP, U32, VP, P(MeshShape), C.c_int, C.c_int, C.c_int, F, F,
                                C.c_int, U64, VP], U64)
    fn("iaco_cq_small_multiplicator", [VP, U64], D)
    fn("iaco_cq_small", [VP, VP, U64, P(MeshShape), C.c_int, D, U64, U64, VP], U64)
    fn("iaco_cq_merge_weights", [VP, VP, U32, VP, U64, VP, P(D)])
    fn("iaco_cq_merge", [VP, VP, U32, P(MeshShape), C.c_int, D, U64, U64, VP], U64)
    fn("iaco_ac1d_cq_multiplicator", [VP, U64], D)
    fn("iaco_ac1d_cq", [VP, VP, U64, P(AC1DShape), C.c_int, D, U64, U64, VP], U64)
    fn("iaco_ac1d_vecsize", [F, F], U32)
    fn("iaco_ac1d_sparse_frame", [VP, U32, F, F, C.c_int, D, VP])
    fn("iaco_ac1d_sparse_frame_cpu_route", [VP, U32, F, F, C.c_int, VP])
    fn("iaco_ac1d_uw_frames", [VP, VP, U32, U64, F, F, U32, C.c_int, C.c_int, VP])
    fn("iaco_simulate_crystal", [VP, U64, VP, U32, VP, C.c_int, VP])
    fn("iaco_simulate_crystal_f64", [VP, U64, VP, U32, VP, C.c_int, VP])
    fn("iaco_philox4x32_10", [P(U32), P(U32), P(U32)])
    fn("iaco_uniform_double", [U64, U64, U64, U32], D)
    fn("iaco_poisson", [D, U64, U64, U64], U32)
    fn("iaco_poisson_array", [VP, U64, U64, U64, VP])
    fn("iaco_crystal_lattice", [VP, P(U32), VP, U32, VP])
    fn("iaco_rotation_axis_angle", [D, P(D), P(F)])
    fn("iaco_invert3", [P(F), P(F)])
    fn("iaco_merge_ac_and_cq", [VP, VP, U64, F, F, VP])
    return lib


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = _decl(C.CDLL(LIB))
    return _lib


def ref():
    """The reference's kernel.cl compiled for the CPU, or None if not built."""
    global _ref
    if _ref is None and os.path.exists(REF):
        r = C.CDLL(REF)
        for name, args in [
            ("iacref_AutoCorr_CQ_small", [VP, VP, VP, VP, U64]),
            ("iacref_AutoCorr_CQ_small_rows", [VP, VP, VP, VP, U64, U64]),
            ("iacref_Merge_CQ", [VP, VP, VP, VP, U64]),
            ("iacref_Autocor_sparseHL", [VP, VP, VP, VP, U64]),
            ("iacref_AutoCorr_CQ_AV", [VP, VP, VP, VP, U64]),
            ("iacref_AutoCorr_CQ_AV_rows", [VP, VP, VP, VP, U64, U64]),
            ("iacref_SimulateCrystal", [VP, VP, VP, VP, U64]),
            ("iacref_AutoCorr_sparseHL_AAV", [VP, VP, VP, U64]),
        ]:
            f = getattr(r, name)
            f.argtypes = args
            f.restype = None
        _ref = r
    return _ref


def p(a):
    return a.ctypes.data_as(VP)


def f3(v):
    return (F * 3)(*[float(x) for x in v])


# ---------------------------------------------------------------------------
# numpy-level helpers
# ---------------------------------------------------------------------------

def calc_kmap(pm: np.ndarray):
    pm = np.ascontiguousarray(pm, np.float32)
    n = pm.size // 3
    km = np.empty_like(pm)
    mq = (F * 3)()
    lib().iaco_calc_kmap(p(pm), n, p(km), mq)
    return km, [mq[0], mq[1], mq[2]]


def big_mesh_shape(max_q, edge, q_zoom=1.0) -> MeshShape:
    s = MeshShape()
    if lib().iaco_big_mesh_shape(f3(max_q), int(edge), float(q_zoom), C.byref(s)) != 0:
        raise ValueError("Meshsize must be odd for each dimension")
    return s


def small_cq_mesh_shape(max_q, perp, q_zoom=1.0) -> MeshShape:
    s = MeshShape()
    if lib().iaco_small_cq_mesh_shape(f3(max_q), int(perp), float(q_zoom), C.byref(s)) != 0:
        raise ValueError("Meshsize must be odd for each dimension")
    return s


def ac1d_shape(max_q, size, q_zoom=1.0) -> AC1DShape:
    s = AC1DShape()
    lib().iaco_ac1d_shape_init(f3(max_q), int(size), float(q_zoom), C.byref(s))
    return s


def half_words(S):
    return S * S * ((S + 1) // 2)


def sparse_params_array(shape: MeshShape, n, dmap, i1, i2, mult=1000.0):
    """Params[9] of IAC/Detector.cpp:1060-1073."""
    return np.array([n, shape.voxel_per_dq, shape.size_ab, shape.size_c, shape.max_q,
                     float(dmap), mult, i1, i2], np.float64)


def sparse_batch(photons, offsets, rot, shape: MeshShape, i1=0, i2=0, dmap=1, step=0.001,
                 offset=0.0, cpu_gpu=1, det_pixels=1):
    """RunIAC's per-frame loop of Detector::AutoCorrelateSparseList; returns
    (full mesh uint64[S^3], skipped out-of-mesh writes)."""
    S = shape.size_ab
    full = np.zeros(S * S * S, np.uint64)
    ph = np.ascontiguousarray(photons, np.float32)
    off = np.ascontiguousarray(offsets, np.uint64)
    R = np.ascontiguousarray(rot, np.float32)
    oob = lib().iaco_sparse_ac_batch(p(ph), p(off), len(off) - 1, p(R), C.byref(shape), i1, i2,
                                     int(dmap), step, offset, int(cpu_gpu), int(det_pixels),
                                     p(full))
    return full, int(oob)
