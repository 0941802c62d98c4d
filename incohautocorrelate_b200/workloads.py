"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No public dataset exists for this path; every input here is generated from a
seed (numpy PCG64) and carries the geometry, sizes and value distributions of
the configuration it stands in for:

* ``small``      -- flat 128x128 detector, 75 um pitch at 0.10 m, 2 000 frames,
                    per-pixel photon counts ~ Poisson(0.01), identity orientation,
                    65^3 mesh (MeshSize 63).
* ``rotated``    -- 1024x512 detector (two 512x512 panels, 2 mm gap), 5 % of
                    pixels masked, 100 000 frames with photon count
                    ~ Poisson(lambda_f), lambda_f log-normal (median 80,
                    sigma 0.8), uniform-random SO(3) orientation, 201^3 mesh.
* ``dense``      -- 1024x1024 mean-intensity map I(r) = 1/(1+(r/300 px)^2) *
                    (1 + 0.02 N(0,1)), 5 % masked.
* ``simulator``  -- 512x512 detector, 5x5x8 simple-cubic crystal (a = 4 A),
                    lambda = 1.55 A.

Pixel maps follow the reference layout [n_y][n_x][3] with x fastest
(IAC/Detector.h:13-16).
"""
from __future__ import annotations

import math

import numpy as np

PITCH = 75e-6
DISTANCE = 0.10
WAVELENGTH_A = 1.55


def flat_pixel_map(ny: int, nx: int, pitch: float = PITCH, dist: float = DISTANCE,
                   gap_x: float = 0.0, gap_after: int | None = None) -> np.ndarray:
    """Pixel centres of a flat detector normal to the beam, centred on it.

    A gap of ``gap_x`` metres is inserted after column ``gap_after`` (two
    panels side by side)."""
    x = (np.arange(nx) - (nx - 1) / 2.0) * pitch
    if gap_x and gap_after is not None:
        x = x + np.where(np.arange(nx) >= gap_after, gap_x / 2.0, -gap_x / 2.0)
    y = (np.arange(ny) - (ny - 1) / 2.0) * pitch
    pm = np.empty((ny, nx, 3), np.float64)
    pm[..., 0] = x[None, :]
    pm[..., 1] = y[:, None]
    pm[..., 2] = dist
    return pm.astype(np.float32).reshape(-1)


def kmap_numpy(pm: np.ndarray):
    """Detector::Calc_kMap in float32 numpy (IAC/Detector.cpp:310-361)."""
    p = pm.reshape(-1, 3).astype(np.float32)
    r = np.sqrt((p[:, 0] * p[:, 0] + p[:, 1] * p[:, 1]) + p[:, 2] * p[:, 2]).astype(np.float32)
    k = (p / r[:, None]).astype(np.float32)
    mq = np.abs(k.max(axis=0) - k.min(axis=0)).astype(np.float32)
    return k.reshape(-1), [float(v) for v in mq]


def random_mask(npix: int, frac: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    m = np.ones(npix, np.int32)
    m[rng.choice(npix, int(round(frac * npix)), replace=False)] = 0
    return m


def haar_rotations(n: int, seed: int) -> np.ndarray:
    """Uniform SO(3) rotations from normalised Gaussian quaternions, row-major
    float32 [n, 9] (HitEvent::RotMatrix convention, IAC/Settings.h:107)."""
    rng = np.random.default_rng(seed)
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((n, 9))
    R[:, 0] = 1 - 2 * (y * y + z * z)
    R[:, 1] = 2 * (x * y - z * w)
    R[:, 2] = 2 * (x * z + y * w)
    R[:, 3] = 2 * (x * y + z * w)
    R[:, 4] = 1 - 2 * (x * x + z * z)
    R[:, 5] = 2 * (y * z - x * w)
    R[:, 6] = 2 * (x * z - y * w)
    R[:, 7] = 2 * (y * z + x * w)
    R[:, 8] = 1 - 2 * (x * x + y * y)
    return R.astype(np.float32)


def identity_rotations(n: int) -> np.ndarray:
    return np.tile(np.eye(3, dtype=np.float32).reshape(1, 9), (n, 1))


def _photon_lists(kmap: np.ndarray, frame: np.ndarray, pixel: np.ndarray, count: np.ndarray,
                  nframes: int):
    """(frame, pixel, count) sorted by frame then pixel -> float4 list + offsets."""
    k3 = kmap.reshape(-1, 3)
    ph = np.empty((len(pixel), 4), np.float32)
    ph[:, :3] = k3[pixel]
    ph[:, 3] = count.astype(np.float32)
    off = np.searchsorted(frame, np.arange(nframes + 1)).astype(np.uint64)
    return ph, off


def poisson_pixel_frames(kmap: np.ndarray, nframes: int, mean: float, seed: int,
                         mask: np.ndarray | None = None):
    """Per-pixel counts ~ Poisson(mean) in every frame; the sparse list keeps
    pixels with a count > 0 in pixel order, value = count (photonised)."""
    npix = kmap.size // 3
    rng = np.random.default_rng(seed)
    frames, pixels, counts = [], [], []
    block = max(1, (1 << 24) // npix)
    for f0 in range(0, nframes, block):
        f1 = min(nframes, f0 + block)
        c = rng.poisson(mean, size=(f1 - f0, npix))
        if mask is not None:
            c = c * mask[None, :]
        fi, pi = np.nonzero(c)
        frames.append(fi + f0)
        pixels.append(pi)
        counts.append(c[fi, pi])
    frame = np.concatenate(frames)
    pixel = np.concatenate(pixels)
    count = np.concatenate(counts)
    return _photon_lists(kmap, frame, pixel, count, nframes)


def lognormal_photon_frames(kmap: np.ndarray, nframes: int, median: float, sigma: float,
                            seed: int, mask: np.ndarray | None = None):
    """Photon count per frame ~ Poisson(lambda_f), lambda_f ~ LogNormal(ln median,
    sigma); every photon lands on a uniform-random unmasked pixel and photons
    on one pixel add up to its count."""
    npix = kmap.size // 3
    rng = np.random.default_rng(seed)
    lam = rng.lognormal(math.log(median), sigma, nframes)
    nph = rng.poisson(lam)
    good = np.nonzero(mask)[0] if mask is not None else np.arange(npix)
    total = int(nph.sum())
    pix = good[rng.integers(0, len(good), total)]
    fr = np.repeat(np.arange(nframes, dtype=np.int64), nph)
    key = fr * npix + pix
    uk, cnt = np.unique(key, return_counts=True)
    frame = uk // npix
    pixel = (uk - frame * npix).astype(np.int64)
    return _photon_lists(kmap, frame, pixel, cnt, nframes)


def pair_count(offsets: np.ndarray) -> int:
    """Distinct + self photon pairs n(n+1)/2 summed over frames."""
    n = np.diff(offsets.astype(np.int64))
    return int((n * (n + 1) // 2).sum())


def radial_mean_intensity(ny: int, nx: int, r0_px: float, noise: float, mask_frac: float,
                          seed: int) -> np.ndarray:
    """I(r) = 1/(1+(r/r0)^2) * (1 + noise N(0,1)), masked pixels set to 0."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:ny, 0:nx]
    r = np.hypot(xx - (nx - 1) / 2.0, yy - (ny - 1) / 2.0)
    I = 1.0 / (1.0 + (r / r0_px) ** 2) * (1.0 + noise * rng.standard_normal((ny, nx)))
    I = np.clip(I, 0, None).reshape(-1)
    m = random_mask(ny * nx, mask_frac, seed + 1)
    return (I * m).astype(np.float32)


# ---------------------------------------------------------------------------
# named configurations
# ---------------------------------------------------------------------------

def small_config(nframes: int = 2000, seed: int = 1):
    pm = flat_pixel_map(128, 128)
    kmap, mq = kmap_numpy(pm)
    ph, off = poisson_pixel_frames(kmap, nframes, 0.01, seed)
    rot = identity_rotations(nframes)
    return dict(pixel_map=pm, kmap=kmap, max_q=mq, photons=ph, offsets=off, rot=rot,
                mesh_size=63, npix=128 * 128)


def rotated_detector():
    pm = flat_pixel_map(512, 1024, gap_x=2e-3, gap_after=512)
    kmap, mq = kmap_numpy(pm)
    mask = random_mask(512 * 1024, 0.05, seed=7)
    return pm, kmap, mq, mask


def rotated_config(nframes: int = 100_000, seed: int = 2):
    pm, kmap, mq, mask = rotated_detector()
    ph, off = lognormal_photon_frames(kmap, nframes, 80.0, 0.8, seed, mask)
    rot = haar_rotations(nframes, seed + 1000)
    return dict(pixel_map=pm, kmap=kmap, max_q=mq, mask=mask, photons=ph, offsets=off,
                rot=rot, mesh_size=199, npix=512 * 1024)
