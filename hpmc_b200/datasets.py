"""Seeded synthetic volumes of the benchmark workloads (no external datasets).

Every field is computed in float64 with numpy from a fixed seed and cast once
to its storage type, so the GPU and the CPU oracle see the same array.

  metaballs_64    float32 64^3 on [0,1]^3 (x_i = i/63): sum of 8 metaballs
                  r^2/|x-c|^2, c ~ U[0.2,0.8]^3, r ~ U[0.05,0.15]; iso 1.0
  noise_u8_256    uint8 256^3: i.i.d. U[0,1) smoothed by a periodic Gaussian
                  (sigma = 3 voxels, applied in Fourier space), affinely
                  rescaled to [0,255] and rounded; iso 128 (many ties)
  cayley_512      float32 512^3 on [-1,1]^3: 16xyz + 4(x^2+y^2+z^2) - 1
                  + N(0, 1e-3); iso 0
  batch_64        64 float32 volumes, edge log-uniform in [32,192] rounded to
                  a multiple of 4, 4-32 metaballs each (centres/radii as
                  metaballs_64), iso U[0.8,1.5] per volume
  spheres_128     float32 128^3 on [0,1]^3: signed distance of the union of
                  16 spheres, c ~ U[0.2,0.8]^3, r ~ U[0.05,0.12]; iso 0
"""
from __future__ import annotations

import numpy as np


def _grid(n: int, lo: float, hi: float) -> np.ndarray:
    return lo + (hi - lo) * np.arange(n, dtype=np.float64) / (n - 1)


def metaballs(n: int, centers: np.ndarray, radii: np.ndarray, shape=None) -> np.ndarray:
    """sum_i r_i^2/|x-c_i|^2 on [0,1]^3 with x_i = i/(n-1); returns (z, y, x) float32."""
    nx, ny, nz = shape if shape is not None else (n, n, n)
    xs, ys, zs = _grid(nx, 0, 1), _grid(ny, 0, 1), _grid(nz, 0, 1)
    out = np.zeros((nz, ny, nx), np.float64)
    for c, r in zip(centers, radii):
        dz = (zs - c[2])[:, None, None] ** 2
        dy = (ys - c[1])[None, :, None] ** 2
        dx = (xs - c[0])[None, None, :] ** 2
        with np.errstate(divide="ignore"):
            out += (r * r) / (dx + dy + dz)
    return out.astype(np.float32)


def metaballs_64(seed: int = 0, n: int = 64):
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.2, 0.8, size=(8, 3))
    r = rng.uniform(0.05, 0.15, size=8)
    return metaballs(n, c, r), 1.0


def noise_u8(n: int = 256, seed: int = 1, sigma: float = 3.0):
    rng = np.random.default_rng(seed)
    u = rng.random((n, n, n))
    k = np.fft.fftfreq(n)
    g = np.exp(-2.0 * (np.pi * sigma) ** 2 * k * k)  # Fourier transform of the Gaussian
    U = np.fft.rfftn(u)
    U *= g[:, None, None] * g[None, :, None] * g[None, None, : n // 2 + 1]
    s = np.fft.irfftn(U, s=u.shape, axes=(0, 1, 2))
    lo, hi = s.min(), s.max()
    v = np.rint((s - lo) * (255.0 / (hi - lo)))
    return v.astype(np.uint8), 128.0


def cayley(n: int = 512, seed: int = 2, noise: float = 1e-3, slices: int | None = None):
    """16xyz + 4(x^2+y^2+z^2) - 1 + N(0, noise) on [-1,1]^3, (z, y, x) float32.
    `slices` keeps only the first slices (bit-identical to cayley(n)[:slices]:
    the noise is drawn slice by slice)."""
    rng = np.random.default_rng(seed)
    xs = _grid(n, -1, 1)
    nz = n if slices is None else int(slices)
    out = np.empty((nz, n, n), np.float32)
    x = xs[None, :]
    y = xs[:, None]
    for k in range(nz):
        z = xs[k]
        f = 16.0 * x * y * z + 4.0 * (x * x + y * y + z * z) - 1.0
        f = f + rng.normal(0.0, noise, size=(n, n))
        out[k] = f.astype(np.float32)
    return out, 0.0


def spheres_sdf(n: int = 128, seed: int = 4, count: int = 16):
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.2, 0.8, size=(count, 3))
    r = rng.uniform(0.05, 0.12, size=count)
    xs = _grid(n, 0, 1)
    out = np.full((n, n, n), np.inf)
    for ci, ri in zip(c, r):
        d = np.sqrt((xs[None, None, :] - ci[0]) ** 2 + (xs[None, :, None] - ci[1]) ** 2 +
                    (xs[:, None, None] - ci[2]) ** 2) - ri
        out = np.minimum(out, d)
    return out.astype(np.float32), 0.0


def batch_64(seed: int = 3, count: int = 64):
    """List of (field (z,y,x) float32, iso) with uneven cubic sizes."""
    rng = np.random.default_rng(seed)
    vols = []
    for _ in range(count):
        e = float(np.exp(rng.uniform(np.log(32.0), np.log(192.0))))
        n = int(max(32, min(192, 4 * round(e / 4.0))))
        m = int(rng.integers(4, 33))
        c = rng.uniform(0.2, 0.8, size=(m, 3))
        r = rng.uniform(0.05, 0.15, size=m)
        iso = float(rng.uniform(0.8, 1.5))
        vols.append((metaballs(n, c, r), iso))
    return vols
