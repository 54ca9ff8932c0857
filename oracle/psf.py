"""CPU oracle for widefield PSF synthesis.

TEST INFRASTRUCTURE ONLY.  The checker that ``decon_pupil_to_psf`` is compared
against; only ``tests/`` may import it.

Float64 NumPy restatements of deconlib's widefield PSF model:

  * ``pupil_to_psf`` (psf/widefield.py:18-73): defocus the pupil by
    exp(2 pi i kz z) for every z, inverse 2-D FFT of each plane (DC at the
    corner), intensity |.|^2, and an optional unit-sum normalisation;
  * ``make_geometry`` (psf/optics.py:96-225): FFT-ordered frequency grid,
    binary NA mask, the anti-aliased support weight (fraction of an
    oversample x oversample sub-grid inside the NA disc, optionally smoothed
    by a wrapped Gaussian), rho, phi, sin / cos theta and kz;
  * ``make_pupil`` / aplanatic apodization (psf/pupil.py:17-97);
  * ``index_mismatch`` (psf/aberrations/geometric.py:38-58, Gibson-Lanni
    phase) and ``zernike_phase_factor`` (psf/aberrations/zernike.py:92-115
    with utils/zernike.py's OSA/ANSI orthonormal polynomials).

Parity pin: ``tests/test_oracle_golden.py::test_pupil_to_psf`` checks
``pupil_to_psf`` against ``tests/golden/golden_psf.npz``, written by the
reference's own code (``tests/golden/make_golden.py``), and
``tests/test_psf_nlcg_cpu.py::test_pupil_restatement_matches_reference_pupils``
rebuilds the four reference pupils and kz grids of that file.
"""

from __future__ import annotations

import math
from math import factorial

import numpy as np


def pupil_to_psf(pupil, kz, z, normalize: bool = True) -> np.ndarray:
    """psf[z] = |ifft2(pupil * exp(2 pi i kz z))|^2 (psf/widefield.py:53-73)."""
    z = np.atleast_1d(np.asarray(z, np.float64))
    pupil = np.asarray(pupil, np.complex128)
    kz = np.asarray(kz, np.float64)
    out = np.empty((len(z),) + pupil.shape, np.float64)
    for i, zi in enumerate(z):
        a = np.fft.ifft2(pupil * np.exp(2j * np.pi * kz * zi))
        out[i] = a.real * a.real + a.imag * a.imag
    if normalize:
        total = out.sum()
        if total > 0:
            out /= total
    return out


def make_geometry(shape, spacing, wavelength, na, ni, oversample=8, boundary_smoothing_sigma=0.0):
    """Frequency-space geometry of psf/optics.py:96-225 as a dict of arrays."""
    ny, nx = shape
    dy, dx = (float(spacing), float(spacing)) if np.isscalar(spacing) else spacing
    kx, ky = np.meshgrid(np.fft.fftfreq(nx, dx), np.fft.fftfreq(ny, dy), indexing="xy")
    kr = np.sqrt(kx ** 2 + ky ** 2)
    k_cut = na / wavelength
    mask = kr <= k_cut
    dkx, dky = 1.0 / (nx * dx), 1.0 / (ny * dy)
    if oversample == 1:
        sw = mask.astype(np.float64)
    else:
        sub = (np.arange(oversample) + 0.5) / oversample - 0.5
        sw = np.zeros_like(kr)
        for jx in range(oversample):
            kxs = kx + sub[jx] * dkx
            kxs_sq = kxs * kxs
            for jy in range(oversample):
                kys = ky + sub[jy] * dky
                sw += (kxs_sq + kys * kys <= k_cut ** 2)
        sw /= oversample * oversample
    if boundary_smoothing_sigma > 0:
        from scipy.ndimage import gaussian_filter

        sw = np.clip(gaussian_filter(sw, sigma=boundary_smoothing_sigma, mode="wrap"), 0.0, 1.0)
    rho = np.zeros_like(kr)
    rho[mask] = kr[mask] / k_cut
    phi = np.arctan2(ky, kx)
    sin_t = np.clip(wavelength * kr / ni, 0.0, 1.0)
    cos_t = np.sqrt(1.0 - sin_t ** 2)
    kz = np.sqrt(np.maximum(0.0, (ni / wavelength) ** 2 - kr ** 2))
    return dict(kx=kx, ky=ky, kz=kz, rho=rho, phi=phi, mask=mask, support_weight=sw,
                cos_theta=cos_t, sin_theta=sin_t)


def make_pupil(geom, apodize=False):
    """support_weight as complex, optionally x 1/sqrt(cos theta) inside the
    NA mask (psf/pupil.py:17-97)."""
    pupil = geom["support_weight"].astype(np.complex128)
    if apodize:
        cos_t = np.maximum(geom["cos_theta"], np.finfo(np.float64).eps)
        pupil = pupil * ((1.0 / np.sqrt(cos_t)) * geom["mask"].astype(np.float64))
    return pupil


def index_mismatch(geom, depth, wavelength, ni, ns):
    """exp(i 2 pi depth (ns cos t2 - ni cos t1) / lambda), Snell's law for t2
    (psf/aberrations/geometric.py:38-58)."""
    sin_t2 = np.clip((ni / ns) * geom["sin_theta"], 0.0, 1.0)
    cos_t2 = np.sqrt(1.0 - sin_t2 ** 2)
    opd = depth * (ns * cos_t2 - ni * geom["cos_theta"])
    return np.exp(1j * (2.0 * np.pi * opd / wavelength))


def ansi_to_nm(j):
    n = int(math.ceil((-3 + math.sqrt(9 + 8 * j)) / 2))
    return n, 2 * j - n * (n + 2)


def zernike(j, rho, phi):
    """Orthonormal OSA/ANSI Zernike Z_j (utils/zernike.py)."""
    n, m = ansi_to_nm(j)
    am = abs(m)
    norm = np.sqrt(2.0 * (n + 1) / (1.0 + float(m == 0)))
    r = np.zeros_like(rho)
    for k in range((n - am) // 2 + 1):
        c = (-1) ** k * factorial(n - k) / (
            factorial(k) * factorial((n + am) // 2 - k) * factorial((n - am) // 2 - k))
        r += c * np.power(rho, n - 2 * k)
    return norm * r * np.cos(m * phi) if m >= 0 else -norm * r * np.sin(am * phi)


def zernike_phase_factor(geom, coefficients):
    """exp(i mask * sum_j c_j Z_j(rho, phi)) (psf/aberrations/zernike.py:92-115)."""
    phase = np.zeros_like(geom["rho"])
    for j, c in coefficients.items():
        if c != 0:
            phase += c * zernike(int(j), geom["rho"], geom["phi"])
    return np.exp(1j * (phase * geom["mask"]))
