"""Seeded synthetic DTMs and the unit flow field ``uv`` the tracer consumes.

The reference is run on lidar DTMs read with GDAL; the workloads here use
seeded synthetic terrain of the same shapes instead (no dataset ships with this
repository).  ``uv_from_dtm`` follows the reference's simple (unconditioned)
preprocessing path: ``np.gradient`` / pixel size (preprocess.py:51-62), flow =
minus the gradient (:105-118), unit-normalised with zero or non-finite speeds
set to 1 (:120-149), edge-padded (:64-79, 594-596), and the DTM mask padded
with masked pixels (geodata.py:252-273); NaN flow pixels are masked and zeroed
(preprocess.py:602-621).

Terrain recipes (all arrays are indexed [x, y], x-major like the reference):

* ``hills_dtm``  512^2 @ 1 m: planar tilt 0.05 + 12 Gaussian hills
  (5-40 m, sigma 20-80 px) + fBm (Hurst 0.7, rms 0.5 m), sinks filled.
* ``incised_dtm``  2048^2 @ 2 m: fBm (Hurst 0.75, rms 30 m) + 400 random-walk
  incisions 1-8 m deep.
* ``fan_dtm``  8192^2 @ 1 m: fBm mountains + planar alluvial cone (slope
  0.03, radial ridges +-0.3 m) + 5000 unfilled pits 0.05-0.5 m deep.
* ``tile_dtm``  the hills relief without sink filling, any size (batched tiles).
"""
from __future__ import annotations

import heapq

import numpy as np


def fbm(nx, ny, hurst, rms, rng):
    """Isotropic fractional Brownian surface by spectral synthesis, zero mean, given rms."""
    kx = np.fft.fftfreq(nx)[:, None]
    ky = np.fft.rfftfreq(ny)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (-(hurst + 1.0))
    amp[0, 0] = 0.0
    phase = rng.uniform(0.0, 2.0 * np.pi, size=amp.shape)
    spec = amp * np.exp(1j * phase)
    z = np.fft.irfft2(spec, s=(nx, ny))
    z -= z.mean()
    s = z.std()
    if s > 0:
        z *= rms / s
    return z


def gaussian_hills(nx, ny, n, amp_range, sigma_range, rng, truncate=None):
    """Sum of n Gaussian hills; with ``truncate`` (in sigmas) each hill is
    evaluated only within that radius (for large grids; the same draws)."""
    x = np.arange(nx, dtype=np.float64)[:, None]
    y = np.arange(ny, dtype=np.float64)[None, :]
    z = np.zeros((nx, ny))
    for _ in range(n):
        a = rng.uniform(*amp_range)
        s = rng.uniform(*sigma_range)
        cx, cy = rng.uniform(0, nx), rng.uniform(0, ny)
        if truncate is None:
            z += a * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * s * s))
        else:
            r = truncate * s
            x0, x1 = max(0, int(cx - r)), min(nx, int(cx + r) + 1)
            y0, y1 = max(0, int(cy - r)), min(ny, int(cy + r) + 1)
            if x0 < x1 and y0 < y1:
                xs, ys = x[x0:x1], y[:, y0:y1]
                z[x0:x1, y0:y1] += a * np.exp(-((xs - cx) ** 2 + (ys - cy) ** 2) / (2.0 * s * s))
    return z


def fill_sinks(dtm, eps=1e-3):
    """Priority-flood sink filling with a small eps gradient across filled areas
    (outflow through the grid border)."""
    z = dtm.astype(np.float64).copy()
    nx, ny = z.shape
    done = np.zeros_like(z, dtype=bool)
    heap = []
    for x in range(nx):
        for y in (0, ny - 1):
            if not done[x, y]:
                done[x, y] = True
                heapq.heappush(heap, (z[x, y], x, y))
    for y in range(ny):
        for x in (0, nx - 1):
            if not done[x, y]:
                done[x, y] = True
                heapq.heappush(heap, (z[x, y], x, y))
    nbrs = [(-1, -1), (-1, 0), (-1, 1), (0, -1), (0, 1), (1, -1), (1, 0), (1, 1)]
    while heap:
        h, x, y = heapq.heappop(heap)
        for dx, dy in nbrs:
            u, v = x + dx, y + dy
            if 0 <= u < nx and 0 <= v < ny and not done[u, v]:
                done[u, v] = True
                if z[u, v] <= h:
                    z[u, v] = h + eps
                heapq.heappush(heap, (z[u, v], u, v))
    return z


def hills_dtm(n=512, seed=1, fill=True):
    rng = np.random.default_rng(seed)
    x = np.arange(n, dtype=np.float64)[:, None]
    z = 0.05 * x + np.zeros((1, n))
    z = z + gaussian_hills(n, n, 12, (5.0, 40.0), (20.0, 80.0), rng)
    z = z + fbm(n, n, 0.7, 0.5, rng)
    if fill:
        z = fill_sinks(z, eps=1e-3)
    return z.astype(np.float32)


def tile_dtm(nx, ny, seed, hill_truncate=None):
    """The hills relief (tilt + hills + fBm) without sink filling, any size (batched tiles)."""
    rng = np.random.default_rng(seed)
    x = np.arange(nx, dtype=np.float64)[:, None]
    z = 0.05 * x + np.zeros((1, ny))
    n_hills = max(1, int(round(12 * nx * ny / 512.0 ** 2)))
    z = z + gaussian_hills(nx, ny, n_hills, (5.0, 40.0), (20.0, 80.0), rng, hill_truncate)
    z = z + fbm(nx, ny, 0.7, 0.5, rng)
    return z.astype(np.float32)


def incised_dtm(n=2048, seed=2, n_incisions=400):
    rng = np.random.default_rng(seed)
    z = fbm(n, n, 0.75, 30.0, rng)
    depth_map = np.zeros_like(z)
    steps = max(64, n // 8)
    for _ in range(n_incisions):
        depth = rng.uniform(1.0, 8.0)
        px, py = rng.uniform(0, n), rng.uniform(0, n)
        ang = rng.uniform(0, 2 * np.pi)
        xs = np.empty(steps)
        ys = np.empty(steps)
        for s in range(steps):
            ang += rng.normal(0.0, 0.3)
            px = min(max(px + np.cos(ang), 0.0), n - 1.0)
            py = min(max(py + np.sin(ang), 0.0), n - 1.0)
            xs[s], ys[s] = px, py
        ix = np.clip(np.round(xs).astype(int), 0, n - 1)
        iy = np.clip(np.round(ys).astype(int), 0, n - 1)
        for ox in (-1, 0, 1):
            for oy in (-1, 0, 1):
                w = depth * (1.0 if ox == 0 and oy == 0 else 0.5)
                jx = np.clip(ix + ox, 0, n - 1)
                jy = np.clip(iy + oy, 0, n - 1)
                depth_map[jx, jy] = np.maximum(depth_map[jx, jy], w)
    return (z - depth_map).astype(np.float32)


def fan_dtm(n=8192, seed=5, n_pits=5000):
    rng = np.random.default_rng(seed)
    z = fbm(n, n, 0.8, 40.0, rng).astype(np.float32)
    x = np.arange(n, dtype=np.float32)[:, None]
    y = np.arange(n, dtype=np.float32)[None, :]
    cx, cy = 0.5 * n, 0.0
    r = np.sqrt((x - cx) ** 2 + (y - cy) ** 2)
    theta = np.arctan2(y - cy, x - cx)
    fan = (-0.03 * r + 0.3 * np.sin(24.0 * theta)).astype(np.float32)
    w = np.clip(1.0 - r / (0.6 * n), 0.0, 1.0).astype(np.float32)
    z = (1.0 - w) * z + w * fan + 0.03 * (n * 0.6)
    del r, theta, fan, w
    px = rng.integers(2, n - 2, size=n_pits)
    py = rng.integers(2, n - 2, size=n_pits)
    d = rng.uniform(0.05, 0.5, size=n_pits).astype(np.float32)
    for ox in (-1, 0, 1):
        for oy in (-1, 0, 1):
            f = 1.0 if (ox == 0 and oy == 0) else 0.5
            z[px + ox, py + oy] -= f * d
    return z.astype(np.float32)


def uv_from_dtm(dtm, pixel_size=1.0, pad=2):
    """Unit flow field, padded mask and uv as the reference's preprocess builds them.

    Returns ``(uv_array [nxp,nyp,2] float32, mask_array [nxp,nyp] bool)``.
    """
    roi = dtm.astype(np.float32)
    gx = np.gradient(roi, axis=0) / pixel_size
    gy = np.gradient(roi, axis=1) / pixel_size
    u, v = -gx.copy(), -gy.copy()
    speed = np.hypot(u, v)
    speed[(~np.isfinite(speed)) | (speed == 0.0)] = 1.0
    u, v = u / speed, v / speed
    uv = np.stack((np.pad(u, (int(pad), int(pad)), "edge"),
                   np.pad(v, (int(pad), int(pad)), "edge")), axis=2).astype(np.float32)
    mask = np.zeros_like(roi, dtype=bool)
    mask[np.isnan(roi)] = True
    mask = np.pad(mask, (int(pad), int(pad)), "constant", constant_values=(True, True))
    bad = np.isnan(uv[:, :, 0]) | np.isnan(uv[:, :, 1])
    mask |= bad
    uv[bad] = [0.0, 0.0]
    return np.ascontiguousarray(uv), mask
