"""ctypes binding of libiac_b200.so (the C ABI declared in include/iac_b200.h).

This is the thin Python view of the C ABI used by the tests and by bench.py.
It loads the in-tree shared library and fails loudly when it is missing:
there is no Python or CPU fallback for any kernel.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libiac_b200.so")

IAC_OK = 0
IAC_ERR_INVALID_ARG = 1
IAC_ERR_CUDA = 2
IAC_ERR_NO_MEMORY = 3
IAC_ERR_TIMEOUT = 4
IAC_ERR_OUT_OF_MESH = 5
IAC_ERR_UNSUPPORTED = 6

NEAREST = 0
LINEAR = 1

# AC1D sparse route (iac_ac1d_uw_batch)
AC1D_ROUTE_REFERENCE = -1
AC1D_ROUTE_HOST = 0
AC1D_ROUTE_DEVICE = 1


class IacError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"iac status {status}: {message}")
        self.status = status


class MeshShape(C.Structure):
    """ACMesh::MeshShape (IAC/ACMesh.h:21-29)."""
    _fields_ = [("k_a", C.c_uint32), ("k_b", C.c_uint32), ("k_c", C.c_uint32),
                ("size_ab", C.c_uint32), ("size_c", C.c_uint32),
                ("center", C.c_uint32 * 3), ("dq_per_voxel", C.c_float),
                ("voxel_per_dq", C.c_uint32), ("max_q", C.c_float)]

    def as_dict(self):
        return {"k": (self.k_a, self.k_b, self.k_c), "size_ab": self.size_ab,
                "size_c": self.size_c, "center": tuple(self.center),
                "dq_per_voxel": self.dq_per_voxel, "voxel_per_dq": self.voxel_per_dq,
                "max_q": self.max_q}


class AC1DShape(C.Structure):
    _fields_ = [("size", C.c_uint32), ("max_q", C.c_float), ("dq_per_step", C.c_float)]


class SparseParams(C.Structure):
    _fields_ = [("shape", MeshShape), ("interp_first", C.c_int32),
                ("interp_second", C.c_int32), ("double_map", C.c_int32),
                ("multiplicator", C.c_double)]


class SparseTuning(C.Structure):
    _fields_ = [("tile_pairs", C.c_uint32), ("block_threads", C.c_uint32),
                ("ctas_per_sm", C.c_uint32), ("cache_hints", C.c_uint32)]


class CrystalParams(C.Structure):
    _fields_ = [("incoherent", C.c_int32), ("fluorescence_yield", C.c_float),
                ("random_orientation", C.c_int32), ("isotropy", C.c_float)]


class SimParams(C.Structure):
    _fields_ = [("subsampling", C.c_int32), ("u_step", C.c_double * 3),
                ("v_step", C.c_double * 3), ("wavelength", C.c_double),
                ("intensity_squared", C.c_int32), ("accurate_sincos", C.c_int32)]


class PhotonParams(C.Structure):
    _fields_ = [("expected_photons", C.c_double), ("poisson", C.c_int32),
                ("adu_noise", C.c_float), ("value_per_photon", C.c_float)]


class AdamW(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float),
                ("eps", C.c_float), ("weight_decay", C.c_float)]


# Philox stream tags of csrc/rng.cuh
RNG_POISSON = 0x01 << 56
RNG_ROTATION = 0x02 << 56
RNG_PHASE = 0x03 << 56
RNG_YIELD = 0x04 << 56
RNG_NOISE = 0x05 << 56

_lib = None
_VP = C.c_void_p
_U64 = C.c_uint64
_U32 = C.c_uint32


def _declare(lib):
    def fn(name, args, res=C.c_int):
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
        return f

    fn("iac_ctx_create", [C.c_int, C.POINTER(_VP)])
    fn("iac_ctx_destroy", [_VP])
    fn("iac_ctx_check", [_VP, _VP, C.POINTER(_U64)])
    fn("iac_status_string", [C.c_int], C.c_char_p)
    fn("iac_last_error", [], C.c_char_p)
    fn("iac_abi_version", [], C.c_int)
    fn("iac_ctx_launch_count", [_VP], _U64)
    fn("iac_ctx_set_scratch_limit", [_VP, _U64])
    fn("iac_ctx_wait_flag", [_VP, _VP, _U32, _VP])
    fn("iac_calc_kmap", [_VP, _VP, _U64, _VP, C.POINTER(C.c_float), _VP])
    fn("iac_big_mesh_shape", [C.POINTER(C.c_float), C.c_int, C.c_float, C.POINTER(MeshShape)])
    fn("iac_small_cq_mesh_shape", [C.POINTER(C.c_float), C.c_int, C.c_float,
                                   C.POINTER(MeshShape)])
    fn("iac_ac1d_shape_init", [C.POINTER(C.c_float), _U32, C.c_float, C.POINTER(AC1DShape)])
    fn("iac_half_mesh_words", [_U32], _U64)
    fn("iac_full_mesh_words", [_U32], _U64)
    fn("iac_sparse_ac_batch", [_VP, _VP, _VP, _VP, _U32, C.POINTER(SparseParams), _VP, _VP])
    fn("iac_sparse_fold", [_VP, _VP, _U32, _VP, _VP])
    fn("iac_sparse_ac_batch_static", [_VP, _VP, _VP, _VP, _U32, C.POINTER(SparseParams), _VP, _VP])
    fn("iac_sparse_ac_frames_host", [_VP, _VP, _VP, _VP, _U32, C.POINTER(SparseParams), _VP])
    fn("iac_sparse_ac_frames_host_to_device", [_VP, _VP, _VP, _VP, _U32, C.POINTER(SparseParams), _VP, _VP])
    fn("iac_sparse_set_tuning", [_VP, C.POINTER(SparseTuning)])
    fn("iac_sparse_get_tuning", [_VP, _U32, C.POINTER(SparseTuning)])
    fn("iac_bench_scatter_add", [_VP, _VP, _U64, C.c_int, _U64, _U32, _VP])
    D = C.c_double
    fn("iac_cq_small_multiplicator", [_VP, _U64, C.POINTER(D)])
    fn("iac_cq_small", [_VP, _VP, _VP, _U64, _U32, C.POINTER(MeshShape), C.c_int, D, _VP, _VP])
    fn("iac_cq_small_part", [_VP, _VP, _VP, _U64, _U32, C.POINTER(MeshShape), C.c_int, D, _U32, _U32, _VP, _VP])
    fn("iac_cq_merge_weights", [_VP, _VP, _U32, _VP, _U64, _VP, C.POINTER(D)])
    fn("iac_cq_merge", [_VP, _VP, _VP, _U32, C.POINTER(MeshShape), C.c_int, D, _VP, _VP])
    fn("iac_ac1d_cq_multiplicator", [_VP, _U64, C.POINTER(D)])
    fn("iac_ac1d_cq", [_VP, _VP, _VP, _U64, C.POINTER(AC1DShape), C.c_int, D, _VP, _VP])
    fn("iac_ac1d_cq_part", [_VP, _VP, _VP, _U64, C.POINTER(AC1DShape), C.c_int, D, _U32, _U32, _VP, _VP])
    fn("iac_ac1d_vecsize", [C.c_float, C.c_float], _U32)
    fn("iac_cq_small_rows", [_VP, _VP, _VP, _U64, _VP, _U32, C.POINTER(MeshShape), C.c_int, D, _VP, _VP])
    fn("iac_ac1d_cq_rows", [_VP, _VP, _VP, _U64, _VP, _U32, C.POINTER(AC1DShape), C.c_int, D, _VP, _VP])
    fn("iac_ac1d_sparse_batch", [_VP, _VP, _VP, _U32, C.c_float, C.c_float, C.c_int, D, _VP, _VP])
    fn("iac_ac1d_uw_words", [C.POINTER(AC1DShape)], _U64)
    fn("iac_ac1d_uw_batch", [_VP, _VP, _VP, _U32, _U64, C.POINTER(AC1DShape), C.c_int, C.c_int, _VP, _VP])
    fn("iac_ac1d_uw_finish", [_VP, _VP, C.POINTER(AC1DShape), _VP, _VP])
    fn("iac_crystal_emitters", [_VP, _VP, _U32, _U32, _U32, C.POINTER(CrystalParams), _U64, _VP,
                                _VP, _VP, _VP, _VP])
    fn("iac_simulate_intensity", [_VP, _VP, _U64, _VP, _VP, _U32, _U32, _U32,
                                  C.POINTER(SimParams), _VP, _VP])
    fn("iac_simulate_photons", [_VP, _VP, _U64, _U32, _U64, C.POINTER(PhotonParams), _U64, _VP])
    fn("iac_sparsify_frames", [_VP, _VP, _VP, _VP, _U64, _U32, C.c_float, C.c_float, C.c_int,
                               _VP, _U64, _VP, C.POINTER(_U64), _VP])
    fn("iac_average_frames", [_VP, _VP, _U64, _U32, _VP, C.c_float, C.c_float, _VP, _VP, _VP, _VP, _VP])
    fn("iac_average_finish", [_VP, _VP, _VP, _U64, _U32, _VP, _VP])
    fn("iac_denoise_param_count", [], _U64)
    fn("iac_denoise_create", [_VP, _U32, _U32, _U32, _U32, C.c_int, C.POINTER(_VP)])
    fn("iac_denoise_destroy", [_VP], None)
    fn("iac_denoise_init_params", [_VP, _U64])
    fn("iac_denoise_set_params", [_VP, _VP])
    fn("iac_denoise_get_params", [_VP, _VP])
    fn("iac_denoise_get_grads", [_VP, _VP])
    fn("iac_denoise_grad_buffer", [_VP, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)])
    fn("iac_denoise_get_state", [_VP, _VP, _VP, C.POINTER(_U64)])
    fn("iac_denoise_set_state", [_VP, _VP, _VP, _VP, _U64])
    fn("iac_denoise_forward", [_VP, _VP, _U32, _U32, _U32, _U32, _VP, _VP])
    fn("iac_denoise_backward", [_VP, _VP, _VP, _VP, _U32, _U32, _U32, _U32, _VP,
                                C.POINTER(C.c_double), _VP])
    fn("iac_denoise_adamw_step", [_VP, C.POINTER(AdamW), _VP])
    fn("iac_denoise_train_steps", [_VP, _VP, _VP, _U32, _U32, _VP, _VP, _U32, _U32, _U32,
                                   C.POINTER(AdamW), _VP, _VP])
    fn("iac_denoise_conv3x3", [_VP, C.c_int, _VP, _U32, C.c_int, _VP, _U32, _VP, _VP, _U32, C.c_int,
                               _U32, _U32, _U32, _U32, _VP, _VP])
    fn("iac_denoise_wgrad3x3", [_VP, C.c_int, _VP, _U32, C.c_int, _VP, _U32, _VP, _U32, _U32, _U32,
                                _U32, _U32, _VP, _VP, _VP])
    fn("iac_denoise_mesh_input", [_VP, _VP, _U32, _U32, D, _VP, _VP, _VP])
    fn("iac_denoise_crop_patches", [_VP, _VP, _U32, _U32, _VP, _U32, _U32, _VP, _VP])
    return lib


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `make -C incohautocorrelate_b200` "
                "(or __graft_entry__.build()); there is no fallback implementation")
        _lib = _declare(C.CDLL(LIB_PATH))
    return _lib


def check(status: int):
    if status != IAC_OK:
        L = lib()
        raise IacError(status, (L.iac_last_error() or b"").decode() or
                       L.iac_status_string(status).decode())
    return status


def _f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


def big_mesh_shape(max_q, edge_size: int, q_zoom: float = 1.0) -> MeshShape:
    s = MeshShape()
    check(lib().iac_big_mesh_shape(_f3(max_q), int(edge_size), float(q_zoom), C.byref(s)))
    return s


def small_cq_mesh_shape(max_q, perp_size: int, q_zoom: float = 1.0) -> MeshShape:
    s = MeshShape()
    check(lib().iac_small_cq_mesh_shape(_f3(max_q), int(perp_size), float(q_zoom), C.byref(s)))
    return s


def ac1d_shape(max_q, size: int, q_zoom: float = 1.0) -> AC1DShape:
    s = AC1DShape()
    check(lib().iac_ac1d_shape_init(_f3(max_q), int(size), float(q_zoom), C.byref(s)))
    return s


def cq_small_multiplicator(h_intensity) -> float:
    m = C.c_double()
    check(lib().iac_cq_small_multiplicator(_ptr(h_intensity), int(h_intensity.size), C.byref(m)))
    return m.value


def ac1d_cq_multiplicator(h_intensity) -> float:
    m = C.c_double()
    check(lib().iac_ac1d_cq_multiplicator(_ptr(h_intensity), int(h_intensity.size), C.byref(m)))
    return m.value


def cq_merge_weights(h_rot9, h_mean_intensity, h_small_cq):
    """(rw10 table float32[n, 10], Multiplicator) of Detector::Merge_smallCofQ."""
    import numpy as np
    nf = int(len(h_mean_intensity))
    rw = np.zeros((nf, 10), np.float32)
    m = C.c_double()
    check(lib().iac_cq_merge_weights(_ptr(h_rot9), _ptr(h_mean_intensity), nf, _ptr(h_small_cq),
                                     int(h_small_cq.size), _ptr(rw), C.byref(m)))
    return rw, m.value


def ac1d_vecsize(max_q: float, dqdx: float) -> int:
    return int(lib().iac_ac1d_vecsize(float(max_q), float(dqdx)))


def ac1d_uw_words(shape: AC1DShape) -> int:
    """uint64 words of the accumulator of Context.ac1d_uw_batch."""
    return int(lib().iac_ac1d_uw_words(C.byref(shape)))


def half_mesh_words(S: int) -> int:
    return int(lib().iac_half_mesh_words(S))


def full_mesh_words(S: int) -> int:
    return int(lib().iac_full_mesh_words(S))


def sparse_params(shape: MeshShape, interp_first=NEAREST, interp_second=NEAREST,
                  double_map=True, multiplicator=1000.0) -> SparseParams:
    p = SparseParams()
    p.shape = shape
    p.interp_first = int(interp_first)
    p.interp_second = int(interp_second)
    p.double_map = int(bool(double_map))
    p.multiplicator = float(multiplicator)
    return p


def _ptr(x):
    """Device or host address of a torch tensor / numpy array / int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(type(x))


class Context:
    """An iac_ctx on one CUDA device."""

    def __init__(self, device: int = 0):
        self._h = _VP()
        check(lib().iac_ctx_create(int(device), C.byref(self._h)))
        self.device = device

    def close(self):
        if self._h:
            lib().iac_ctx_destroy(self._h)
            self._h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def launches(self) -> int:
        return int(lib().iac_ctx_launch_count(self._h))

    def set_scratch_limit(self, max_bytes: int):
        """Cap the device scratch the context may grow (0: no limit); larger
        requests fail with IAC_ERR_NO_MEMORY before allocating."""
        check(lib().iac_ctx_set_scratch_limit(self._h, int(max_bytes)))

    def wait_flag(self, d_flag, max_polls: int, stream=None):
        """One device thread waits (bounded) for *d_flag != 0; a wait that runs
        out makes the next check() raise IAC_ERR_TIMEOUT."""
        check(lib().iac_ctx_wait_flag(self._h, _ptr(d_flag), int(max_polls), _ptr(stream)))

    def check(self, stream=None) -> int:
        """Synchronise and return the number of skipped out-of-mesh writes."""
        oob = _U64(0)
        st = lib().iac_ctx_check(self._h, _ptr(stream), C.byref(oob))
        if st not in (IAC_OK, IAC_ERR_OUT_OF_MESH):
            check(st)
        return int(oob.value)

    def calc_kmap(self, d_pixel_map, npix, d_kmap, stream=None):
        mq = (C.c_float * 3)()
        check(lib().iac_calc_kmap(self._h, _ptr(d_pixel_map), int(npix), _ptr(d_kmap), mq,
                                  _ptr(stream)))
        return [mq[0], mq[1], mq[2]]

    def sparse_ac_batch(self, d_photons, d_offsets, d_rot, nframes, params, d_half, stream=None):
        check(lib().iac_sparse_ac_batch(self._h, _ptr(d_photons), _ptr(d_offsets), _ptr(d_rot),
                                        int(nframes), C.byref(params), _ptr(d_half),
                                        _ptr(stream)))

    def sparse_ac_batch_static(self, d_photons, d_offsets, d_rot, nframes, params, d_half,
                               stream=None):
        """iac_sparse_ac_batch_static: the batched pair correlator with its work queue in
        a fixed device array of the library (no device allocation at all)."""
        check(lib().iac_sparse_ac_batch_static(self._h, _ptr(d_photons), _ptr(d_offsets),
                                               _ptr(d_rot), int(nframes), C.byref(params),
                                               _ptr(d_half), _ptr(stream)))

    def sparse_fold(self, d_half, S, d_full, stream=None):
        check(lib().iac_sparse_fold(self._h, _ptr(d_half), int(S), _ptr(d_full), _ptr(stream)))

    def sparse_ac_frames_host(self, h_photons, h_offsets, h_rot, nframes, params, h_full):
        check(lib().iac_sparse_ac_frames_host(self._h, _ptr(h_photons), _ptr(h_offsets),
                                              _ptr(h_rot), int(nframes), C.byref(params),
                                              _ptr(h_full)))

    def sparse_ac_frames_host_to_device(self, h_photons, h_offsets, h_rot, nframes, params, d_half,
                                        stream=None):
        check(lib().iac_sparse_ac_frames_host_to_device(self._h, _ptr(h_photons), _ptr(h_offsets), _ptr(h_rot),
                                                        int(nframes), C.byref(params), _ptr(d_half),
                                                        _ptr(stream)))

    def set_sparse_tuning(self, tile_pairs=0, block_threads=0, ctas_per_sm=0, cache_hints=0):
        t = SparseTuning(int(tile_pairs), int(block_threads), int(ctas_per_sm), int(cache_hints))
        check(lib().iac_sparse_set_tuning(self._h, C.byref(t)))

    def sparse_tuning(self, size_ab: int = 0):
        t = SparseTuning()
        check(lib().iac_sparse_get_tuning(self._h, int(size_ab), C.byref(t)))
        return {"tile_pairs": t.tile_pairs, "block_threads": t.block_threads,
                "ctas_per_sm": t.ctas_per_sm, "cache_hints": t.cache_hints}

    def cq_small(self, d_I, d_kmap, npix, shape, interp, mult, d_mesh, stream=None, fast_size=0,
                 part=0, nparts=1):
        """iac_cq_small, or with nparts > 1 its share `part` (iac_cq_small_part)."""
        if nparts == 1 and part == 0:
            check(lib().iac_cq_small(self._h, _ptr(d_I), _ptr(d_kmap), int(npix), int(fast_size),
                                     C.byref(shape), int(interp), float(mult), _ptr(d_mesh),
                                     _ptr(stream)))
        else:
            check(lib().iac_cq_small_part(self._h, _ptr(d_I), _ptr(d_kmap), int(npix), int(fast_size),
                                          C.byref(shape), int(interp), float(mult), int(part), int(nparts),
                                          _ptr(d_mesh), _ptr(stream)))

    def cq_small_rows(self, d_I, d_kmap, npix, d_rows, nrows, shape, interp, mult, d_mesh, stream=None):
        check(lib().iac_cq_small_rows(self._h, _ptr(d_I), _ptr(d_kmap), int(npix), _ptr(d_rows), int(nrows),
                                      C.byref(shape), int(interp), float(mult), _ptr(d_mesh), _ptr(stream)))

    def ac1d_cq_rows(self, d_I, d_kmap, npix, d_rows, nrows, shape, interp, mult, d_hist, stream=None):
        check(lib().iac_ac1d_cq_rows(self._h, _ptr(d_I), _ptr(d_kmap), int(npix), _ptr(d_rows), int(nrows),
                                     C.byref(shape), int(interp), float(mult), _ptr(d_hist), _ptr(stream)))

    def cq_merge(self, d_small, d_rw, nframes, shape, interp, mult, d_big, stream=None):
        check(lib().iac_cq_merge(self._h, _ptr(d_small), _ptr(d_rw), int(nframes), C.byref(shape),
                                 int(interp), float(mult), _ptr(d_big), _ptr(stream)))

    def ac1d_cq(self, d_I, d_kmap, npix, shape, interp, mult, d_hist, stream=None, part=0, nparts=1):
        """iac_ac1d_cq, or with nparts > 1 its share `part` (iac_ac1d_cq_part)."""
        if nparts == 1 and part == 0:
            check(lib().iac_ac1d_cq(self._h, _ptr(d_I), _ptr(d_kmap), int(npix), C.byref(shape),
                                    int(interp), float(mult), _ptr(d_hist), _ptr(stream)))
        else:
            check(lib().iac_ac1d_cq_part(self._h, _ptr(d_I), _ptr(d_kmap), int(npix), C.byref(shape),
                                         int(interp), float(mult), int(part), int(nparts), _ptr(d_hist),
                                         _ptr(stream)))

    def ac1d_sparse_batch(self, d_photons, d_offsets, nframes, max_q, dqdx, interp, mult, d_hist,
                          stream=None):
        check(lib().iac_ac1d_sparse_batch(self._h, _ptr(d_photons), _ptr(d_offsets), int(nframes),
                                          float(max_q), float(dqdx), int(interp), float(mult),
                                          _ptr(d_hist), _ptr(stream)))

    def ac1d_uw_batch(self, d_photons, d_offsets, nframes, detector_pixels, shape, interp, d_acc,
                      route=AC1D_ROUTE_REFERENCE, stream=None):
        check(lib().iac_ac1d_uw_batch(self._h, _ptr(d_photons), _ptr(d_offsets), int(nframes),
                                      int(detector_pixels), C.byref(shape), int(interp), int(route),
                                      _ptr(d_acc), _ptr(stream)))

    def ac1d_uw_finish(self, d_acc, shape, d_ac_uw, stream=None):
        check(lib().iac_ac1d_uw_finish(self._h, _ptr(d_acc), C.byref(shape), _ptr(d_ac_uw), _ptr(stream)))

    def crystal_emitters(self, d_atoms, natoms, nframes, nmodes, cparams, seed, d_em, d_count,
                         d_rot_event, d_rot_crystal=None, stream=None):
        check(lib().iac_crystal_emitters(self._h, _ptr(d_atoms), int(natoms), int(nframes),
                                         int(nmodes), C.byref(cparams), int(seed), _ptr(d_em),
                                         _ptr(d_count), _ptr(d_rot_event), _ptr(d_rot_crystal),
                                         _ptr(stream)))

    def simulate_intensity(self, d_pm, npix, d_em, d_count, natoms, nmodes, nframes, sparams,
                           d_out, stream=None):
        check(lib().iac_simulate_intensity(self._h, _ptr(d_pm), int(npix), _ptr(d_em),
                                           _ptr(d_count), int(natoms), int(nmodes), int(nframes),
                                           C.byref(sparams), _ptr(d_out), _ptr(stream)))

    def simulate_photons(self, d_I, npix, nframes, first_frame, pparams, seed, stream=None):
        check(lib().iac_simulate_photons(self._h, _ptr(d_I), int(npix), int(nframes),
                                         int(first_frame), C.byref(pparams), int(seed),
                                         _ptr(stream)))

    def sparsify_frames(self, d_I, d_mask, d_kmap, npix, nframes, threshold, step, photonize,
                        d_photons, capacity, d_offsets, stream=None, want_total=True):
        tot = _U64(0)
        check(lib().iac_sparsify_frames(self._h, _ptr(d_I), _ptr(d_mask), _ptr(d_kmap), int(npix),
                                        int(nframes), float(threshold), float(step),
                                        int(photonize), _ptr(d_photons), int(capacity),
                                        _ptr(d_offsets), C.byref(tot) if want_total else None,
                                        _ptr(stream)))
        return int(tot.value)

    def average_frames(self, d_frames, npix, nframes, d_mask, threshold, step, d_sum, d_discr,
                       d_mean, d_photon_sum=None, stream=None):
        check(lib().iac_average_frames(self._h, _ptr(d_frames), int(npix), int(nframes), _ptr(d_mask),
                                       float(threshold), float(step), _ptr(d_sum), _ptr(d_discr),
                                       _ptr(d_mean), _ptr(d_photon_sum), _ptr(stream)))

    def average_finish(self, d_sum, d_discr, npix, nframes_total, d_intensity, stream=None):
        check(lib().iac_average_finish(self._h, _ptr(d_sum), _ptr(d_discr), int(npix), int(nframes_total),
                                       _ptr(d_intensity), _ptr(stream)))

    def bench_scatter_add(self, d_buf, words, word_bits, updates, seed=1, stream=None):
        check(lib().iac_bench_scatter_add(self._h, _ptr(d_buf), int(words), int(word_bits),
                                          int(updates), int(seed), _ptr(stream)))


# --------------------------------------------------------------------------
# mesh denoiser
# --------------------------------------------------------------------------
TCGEN05 = 0          # tcgen05 + TMEM over padded-row slabs (default)
MMA_SYNC = 1
TCGEN05_PER_TAP = 2


def denoise_param_count() -> int:
    return int(lib().iac_denoise_param_count())


class Denoiser:
    """Owns an iac_denoiser workspace (a 3-level 3D U-Net) on `ctx`'s device."""

    def __init__(self, ctx, max_batch, D, H, W, backend=TCGEN05):
        self.ctx = ctx
        h = _VP()
        check(lib().iac_denoise_create(ctx._h, int(max_batch), int(D), int(H), int(W), int(backend),
                                       C.byref(h)))
        self._h = h
        self.nparams = denoise_param_count()

    def close(self):
        if self._h:
            lib().iac_denoise_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_params(self, seed=0):
        check(lib().iac_denoise_init_params(self._h, int(seed)))

    def set_params(self, params):
        import numpy as np
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == self.nparams
        check(lib().iac_denoise_set_params(self._h, p.ctypes.data))

    def get_params(self):
        import numpy as np
        p = np.zeros(self.nparams, np.float32)
        check(lib().iac_denoise_get_params(self._h, p.ctypes.data))
        return p

    def get_grads(self):
        import numpy as np
        g = np.zeros(self.nparams, np.float32)
        check(lib().iac_denoise_get_grads(self._h, g.ctypes.data))
        return g

    def grad_tensor(self):
        """The device gradient vector as a float32 torch tensor sharing its
        memory (iac_denoise_grad_buffer): written by backward, read by
        adamw_step; a data-parallel step all-reduces it in place."""
        import torch
        p, n = C.c_void_p(), C.c_uint64()
        check(lib().iac_denoise_grad_buffer(self._h, C.byref(p), C.byref(n)))

        class _View:
            __cuda_array_interface__ = {"shape": (int(n.value),), "typestr": "<f4",
                                        "data": (int(p.value), False), "version": 2}
        return torch.as_tensor(_View(), device="cuda")

    def get_state(self):
        """(parameters, AdamW first moments, second moments, optimizer steps)."""
        import numpy as np
        m = np.zeros(self.nparams, np.float32)
        v = np.zeros(self.nparams, np.float32)
        step = _U64(0)
        check(lib().iac_denoise_get_state(self._h, m.ctypes.data, v.ctypes.data, C.byref(step)))
        return self.get_params(), m, v, int(step.value)

    def set_state(self, params, m, v, step: int):
        """Restore parameters, moments and step count together (a resumed run)."""
        import numpy as np
        arrs = [np.ascontiguousarray(a, np.float32) for a in (params, m, v)]
        for a in arrs:
            if a.size != self.nparams:
                raise ValueError(f"state arrays need {self.nparams} values, got {a.size}")
        check(lib().iac_denoise_set_state(self._h, arrs[0].ctypes.data, arrs[1].ctypes.data,
                                          arrs[2].ctypes.data, int(step)))

    def forward(self, d_in, nb, D, H, W, d_out, stream=None):
        check(lib().iac_denoise_forward(self._h, _ptr(d_in), int(nb), int(D), int(H), int(W),
                                        _ptr(d_out), _ptr(stream)))

    def backward(self, d_in, d_target, nb, D, H, W, d_weight=None, d_out=None, stream=None,
                 want_loss=True):
        loss = C.c_double(0.0)
        check(lib().iac_denoise_backward(self._h, _ptr(d_in), _ptr(d_target), _ptr(d_weight),
                                         int(nb), int(D), int(H), int(W), _ptr(d_out),
                                         C.byref(loss) if want_loss else None, _ptr(stream)))
        return loss.value if want_loss else None

    def adamw_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=1e-4, stream=None):
        opt = AdamW(lr, beta1, beta2, eps, weight_decay)
        check(lib().iac_denoise_adamw_step(self._h, C.byref(opt), _ptr(stream)))

    def train_steps(self, d_in_meshes, d_tgt_meshes, nmeshes, E, d_plans, d_lrs, nsteps, nb, P,
                    d_losses=None, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=1e-4, stream=None):
        """nsteps steps replayed from one CUDA graph (plans [nsteps][nb][5] int32, lrs
        [nsteps] float32 on the device)."""
        opt = AdamW(0.0, beta1, beta2, eps, weight_decay)
        check(lib().iac_denoise_train_steps(self._h, _ptr(d_in_meshes), _ptr(d_tgt_meshes), int(nmeshes),
                                            int(E), _ptr(d_plans), _ptr(d_lrs), int(nsteps), int(nb),
                                            int(P), C.byref(opt), _ptr(d_losses), _ptr(stream)))


def denoise_mesh_input(ctx, d_full, S, E, scale, d_f32=None, d_bf16=None, stream=None):
    check(lib().iac_denoise_mesh_input(ctx._h, _ptr(d_full), int(S), int(E), float(scale),
                                       _ptr(d_f32), _ptr(d_bf16), _ptr(stream)))


def denoise_crop_patches(ctx, d_meshes, nmeshes, E, d_plan, nb, P, d_out, stream=None):
    check(lib().iac_denoise_crop_patches(ctx._h, _ptr(d_meshes), int(nmeshes), int(E), _ptr(d_plan),
                                         int(nb), int(P), _ptr(d_out), _ptr(stream)))


def denoise_conv3x3(ctx, backend, d_src0, c0, up0, d_src1, c1, d_wtile, d_bias, cout, relu, nb, D, H,
                    W, d_y, stream=None):
    check(lib().iac_denoise_conv3x3(ctx._h, int(backend), _ptr(d_src0), int(c0), int(up0),
                                    _ptr(d_src1), int(c1), _ptr(d_wtile), _ptr(d_bias), int(cout),
                                    int(relu), int(nb), int(D), int(H), int(W), _ptr(d_y),
                                    _ptr(stream)))


def denoise_wgrad3x3(ctx, d_src0, c0, up0, d_src1, c1, d_grad, cout, nb, D, H, W, d_dw, d_db=None,
                     stream=None, slabs=1):
    check(lib().iac_denoise_wgrad3x3(ctx._h, int(slabs), _ptr(d_src0), int(c0), int(up0), _ptr(d_src1),
                                     int(c1),
                                     _ptr(d_grad), int(cout), int(nb), int(D), int(H), int(W),
                                     _ptr(d_dw), _ptr(d_db), _ptr(stream)))


def conv_weight_tiles(w):
    """W[cout][27][cin] (any float array) -> bf16-ready tile order [27][cin/8][cout][8]."""
    import numpy as np
    cout, taps, cin = w.shape
    return np.ascontiguousarray(w.reshape(cout, taps, cin // 8, 8).transpose(1, 2, 0, 3))


def dgrad_weight_tiles(w):
    """Tiles of the data-gradient layer: Wd(tap)[ci][co] = W[co][26 - tap][ci], as
    [27][cout/8][cin][8]."""
    import numpy as np
    cout, taps, cin = w.shape
    wt = w[:, ::-1, :].transpose(2, 1, 0)  # [cin][tap'][cout]
    return conv_weight_tiles(np.ascontiguousarray(wt))
