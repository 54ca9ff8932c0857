"""Seeded synthetic inputs for the benchmark workloads (host NumPy, float32).

The reference benchmarks on no public dataset; these generators stand in for
its PSF model and phantoms with the workload shapes and value ranges:

  * ``widefield_psf``: scalar widefield PSF of a circular pupil of radius
    NA / lambda with an anti-aliased edge, defocus phase exp(2 pi i kz z) over
    FFT-ordered z planes, optional depth-induced index-mismatch phase and
    Zernike spherical / horizontal-coma terms; |2-D inverse FFT|^2 per plane,
    normalised to unit sum, corner origin (the convention of deconlib's
    psf/widefield.py:18-73 pupil_to_psf).
  * ``beads``, ``shells``, ``filaments``: the phantoms of the workloads
    (seeded point beads, hollow shells, Gaussian-section polylines).
  * ``poisson_observation``: scale to a peak photon count, add background,
    Poisson noise.
"""

from __future__ import annotations

import math
from typing import Optional, Sequence, Tuple

import numpy as np


def fft_coords(n: int, spacing: float) -> np.ndarray:
    """0, d, 2d, ..., -2d, -d (FFT order)."""
    return np.fft.fftfreq(n) * n * spacing


def widefield_psf(shape: Tuple[int, int, int], dz: float, dxy: float, wavelength: float = 0.525,
                  na: float = 1.4, ni: float = 1.515, ns: float = 1.334, depth: float = 0.0,
                  spherical: float = 0.0, coma_x: float = 0.0) -> np.ndarray:
    nz, ny, nx = shape
    ky = np.fft.fftfreq(ny, d=dxy)[:, None]
    kx = np.fft.fftfreq(nx, d=dxy)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    kmax = na / wavelength
    # anti-aliased support: linear ramp over one frequency-grid step
    dk = 1.0 / (max(ny, nx) * dxy)
    weight = np.clip((kmax - k) / dk + 0.5, 0.0, 1.0)
    kn = ni / wavelength
    kz = np.sqrt(np.maximum(kn * kn - k * k, 0.0))
    rho = np.clip(k / kmax, 0.0, 1.0)
    theta = np.arctan2(ky, kx)
    phase = np.zeros_like(k)
    if spherical:
        phase += spherical * math.sqrt(5.0) * (6 * rho ** 4 - 6 * rho ** 2 + 1)
    if coma_x:
        phase += coma_x * math.sqrt(8.0) * (3 * rho ** 3 - 2 * rho) * np.cos(theta)
    if depth:
        ks = ns / wavelength
        kzs = np.sqrt(np.maximum(ks * ks - k * k, 0.0))
        phase += 2 * np.pi * depth * (kzs - kz)
    pupil = weight * np.exp(1j * phase)
    z = fft_coords(nz, dz)
    psf = np.empty(shape, np.float64)
    for i, zi in enumerate(z):
        a = np.fft.ifft2(pupil * np.exp(2j * np.pi * kz * zi))
        psf[i] = (a * np.conj(a)).real
    psf /= psf.sum()
    return psf.astype(np.float32)


def beads(shape, n: int, rng: np.random.Generator, out: Optional[np.ndarray] = None) -> np.ndarray:
    t = np.zeros(shape, np.float32) if out is None else out
    idx = tuple(rng.integers(0, s, n) for s in shape)
    np.add.at(t, idx, rng.uniform(0.5, 1.0, n).astype(np.float32))
    return t


def shells(shape, spacing, n: int, rng: np.random.Generator, out=None, r_range=(0.6, 2.0),
           margin: float = 2.0) -> np.ndarray:
    """Hollow spheres one lateral voxel thick; radius in physical units."""
    t = np.zeros(shape, np.float32) if out is None else out
    dz, dy, dx = spacing
    ext = [s * d for s, d in zip(shape, spacing)]
    for _ in range(n):
        c = [rng.uniform(min(margin, e / 2), max(e - margin, e / 2)) for e in ext]
        r = rng.uniform(*r_range)
        lo = [max(0, int((ci - r - 2 * d) / d)) for ci, d in zip(c, spacing)]
        hi = [min(s, int((ci + r + 2 * d) / d) + 1) for ci, d, s in zip(c, spacing, shape)]
        zz, yy, xx = np.meshgrid(*[np.arange(a, b) for a, b in zip(lo, hi)], indexing="ij")
        d = np.sqrt(((zz * dz - c[0])) ** 2 + ((yy * dy - c[1])) ** 2 + ((xx * dx - c[2])) ** 2)
        m = np.abs(d - r) <= 0.5 * dy
        t[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]][m] = 1.0
    return t


def filaments(shape, n: int, rng: np.random.Generator, segments: int = 4,
              sigma: float = 1.0) -> np.ndarray:
    """Random 3-D polylines with a Gaussian cross-section (sigma in voxels)."""
    from scipy.ndimage import gaussian_filter

    t = np.zeros(shape, np.float32)
    sh = np.array(shape, np.float64)
    for _ in range(n):
        v = rng.uniform(0, 1, (segments + 1, 3)) * (sh - 1)
        for a, b in zip(v[:-1], v[1:]):
            npts = int(np.ceil(np.linalg.norm(b - a) * 2)) + 1
            p = a[None] + (b - a)[None] * np.linspace(0, 1, npts)[:, None]
            q = np.clip(np.rint(p).astype(np.int64), 0, sh.astype(np.int64) - 1)
            np.add.at(t, (q[:, 0], q[:, 1], q[:, 2]), 0.5)
    t = gaussian_filter(t, sigma).astype(np.float32)
    m = t.max()
    return t / m if m > 0 else t


def poisson_observation(blurred: np.ndarray, peak: float, background: float,
                        rng: np.random.Generator) -> np.ndarray:
    b = np.asarray(blurred, np.float64)
    b = np.maximum(b, 0.0) / max(b.max(), 1e-30) * peak + background
    return rng.poisson(b).astype(np.float32)


def rl_workload(shape=(64, 128, 128), spacing=(0.1, 0.085, 0.085), seed=0):
    """Beads + shells widefield RL input (NA 1.4, 525 nm, 1000 peak photons, background 10)."""
    rng = np.random.default_rng(seed)
    psf = widefield_psf(shape, spacing[0], spacing[1])
    truth = beads(shape, 200, rng)
    shells(shape, spacing, 5, rng, out=truth)
    return psf, truth


def pdhg_workload(shape=(128, 256, 256), spacing=(0.05, 0.0425, 0.0425), seed=2):
    """Filament network + beads, PSF with depth 10 um mismatch, spherical 0.5 and coma -0.2 rad."""
    rng = np.random.default_rng(seed)
    psf = widefield_psf(shape, spacing[0], spacing[1], depth=10.0, spherical=0.5, coma_x=-0.2)
    truth = filaments(shape, 200, rng)
    beads(shape, 200, rng, out=truth)
    return psf, truth
