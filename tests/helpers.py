"""Small seeded inputs shared by the tests."""
import ctypes as C

import numpy as np

from incohautocorrelate_b200 import workloads as W


def small_detector(ny=32, nx=40, pitch=6e-4, dist=0.10):
    """A coarse flat detector whose pairs spread over the whole mesh."""
    pm = W.flat_pixel_map(ny, nx, pitch=pitch, dist=dist)
    km, mq = W.kmap_numpy(pm)
    return pm, km, mq


def random_frames(kmap, sizes, rng, max_count=3, integer=True):
    """One frame per entry of `sizes` (photon count), distinct pixels in pixel
    order, counts in [1, max_count] (or real values when integer=False)."""
    npix = kmap.size // 3
    k3 = kmap.reshape(-1, 3)
    photons, offs = [], [0]
    for n in sizes:
        n = min(int(n), npix)
        pix = np.sort(rng.choice(npix, n, replace=False))
        ph = np.empty((n, 4), np.float32)
        ph[:, :3] = k3[pix]
        if integer:
            ph[:, 3] = rng.integers(1, max_count + 1, n)
        else:
            ph[:, 3] = rng.uniform(0.05, max_count, n).astype(np.float32)
        photons.append(ph)
        offs.append(offs[-1] + n)
    photons = np.concatenate(photons) if photons else np.zeros((0, 4), np.float32)
    return np.ascontiguousarray(photons, np.float32), np.array(offs, np.uint64)


def mesh_shape_dict(s):
    return dict(k=(s.k_a, s.k_b, s.k_c), size_ab=s.size_ab, size_c=s.size_c,
                center=tuple(s.center), dq=s.dq_per_voxel, vpdq=s.voxel_per_dq, max_q=s.max_q)


def to_capi_shape(s):
    from incohautocorrelate_b200 import capi
    o = capi.MeshShape()
    for f, _ in capi.MeshShape._fields_:
        if f == "center":
            o.center = (C.c_uint32 * 3)(*s.center)
        else:
            setattr(o, f, getattr(s, f))
    return o
