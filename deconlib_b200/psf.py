"""Widefield PSF model on the device.

Mirrors deconlib's ``deconlib.psf`` names used to build a job's PSF:

  * ``Optics`` (psf/optics.py:10-54): wavelength, NA, ni, ns, with the same
    validation and ``k_cutoff`` / ``k_immersion``;
  * ``make_geometry`` / ``Geometry`` (psf/optics.py:57-225): the FFT-ordered
    frequency grid, NA mask, anti-aliased support weight, rho, phi, sin / cos
    theta and kz, as FP64 CUDA tensors (``mask`` bool);
  * ``make_pupil`` (psf/pupil.py:17-45) with optional aplanatic apodization;
  * ``IndexMismatch``, ``Defocus`` (psf/aberrations/geometric.py:11-96),
    ``ZernikeMode``, ``ZernikeAberration`` (psf/aberrations/zernike.py:15-130)
    and ``apply_aberrations`` (psf/aberrations/base.py:37-62);
  * ``pupil_to_psf`` (psf/widefield.py:18-73): PSF(z) = |IFFT2(pupil *
    exp(2 pi i kz z))|^2 of shape (nz, ny, nx), unit sum when normalised.

Every array operation runs in ``libdecon_b200.so``: the geometry in one FP64
kernel, each aberration as an in-place phase kernel on the pupil, and the PSF
in ``decon_pupil_to_psf`` (the FP64 defocus phase fused into the y FFT, the x
FFT fused with the intensity and the Parseval normalisation).  The result is
a CUDA float32 tensor, ready to become a convolution kernel without a host
round trip.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from enum import IntEnum
from typing import Dict, Tuple, Union

import numpy as np
import torch

from . import _lib
from .deconvolution._device import empty, stream

__all__ = ["Optics", "Geometry", "make_geometry", "make_pupil", "Aberration", "IndexMismatch",
           "Defocus", "ZernikeMode", "ZernikeAberration", "apply_aberrations", "pupil_to_psf"]


@dataclass(frozen=True)
class Optics:
    """Immutable optical parameters (um); ns defaults to ni (psf/optics.py:10-54)."""

    wavelength: float
    na: float
    ni: float
    ns: float = None

    def __post_init__(self) -> None:
        if self.ns is None:
            object.__setattr__(self, "ns", self.ni)
        if self.na > self.ni:
            raise ValueError(f"NA ({self.na}) cannot exceed immersion refractive index ({self.ni})")
        if self.wavelength <= 0:
            raise ValueError(f"Wavelength must be positive, got {self.wavelength}")

    @property
    def k_cutoff(self) -> float:
        return self.na / self.wavelength

    @property
    def k_immersion(self) -> float:
        return self.ni / self.wavelength


@dataclass(frozen=True)
class Geometry:
    """Frequency-space geometry (psf/optics.py:57-93); FP64 CUDA tensors of
    shape (ny, nx), ``mask`` bool."""

    kx: torch.Tensor
    ky: torch.Tensor
    kz: torch.Tensor
    rho: torch.Tensor
    phi: torch.Tensor
    mask: torch.Tensor
    support_weight: torch.Tensor
    cos_theta: torch.Tensor
    sin_theta: torch.Tensor

    @property
    def shape(self) -> Tuple[int, int]:
        return tuple(self.mask.shape)


def _dptr(t: torch.Tensor) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def make_geometry(shape: Tuple[int, int], spacing: Union[float, Tuple[float, float]], optics: Optics,
                  oversample: int = 8, boundary_smoothing_sigma: float = 0.0) -> Geometry:
    """make_geometry of psf/optics.py:96-225 on the device."""
    _lib.require_cuda()
    ny, nx = (int(s) for s in shape)
    if isinstance(spacing, (int, float)):
        dy = dx = float(spacing)
    else:
        dy, dx = (float(s) for s in spacing)
    if dy <= 0 or dx <= 0:
        raise ValueError(f"Spacing must be positive, got ({dy}, {dx})")
    if oversample < 1:
        raise ValueError(f"oversample must be >= 1, got {oversample}")
    if boundary_smoothing_sigma < 0:
        raise ValueError(
            f"boundary_smoothing_sigma must be >= 0, got {boundary_smoothing_sigma}")
    f = lambda: torch.empty((ny, nx), dtype=torch.float64, device="cuda")  # noqa: E731
    kx, ky, kz, rho, phi, sw, ct, st = (f() for _ in range(8))
    mask = torch.empty((ny, nx), dtype=torch.uint8, device="cuda")
    scratch = f() if boundary_smoothing_sigma > 0 else None
    _lib.call("decon_psf_geometry", ny, nx, dy, dx, float(optics.wavelength), float(optics.na),
              float(optics.ni), int(oversample), float(boundary_smoothing_sigma), _dptr(kx),
              _dptr(ky), _dptr(kz), _dptr(rho), _dptr(phi), _dptr(mask), _dptr(sw), _dptr(ct),
              _dptr(st), _dptr(scratch) if scratch is not None else None, stream())
    return Geometry(kx=kx, ky=ky, kz=kz, rho=rho, phi=phi, mask=mask.view(torch.bool),
                    support_weight=sw, cos_theta=ct, sin_theta=st)


def make_pupil(geom: Geometry, apodize: bool = False) -> torch.Tensor:
    """Complex128 pupil = support weight (x aplanatic 1/sqrt(cos theta) inside
    the NA when ``apodize``) (psf/pupil.py:17-97)."""
    out = torch.empty(geom.shape, dtype=torch.complex128, device="cuda")
    _lib.call("decon_psf_pupil", _dptr(geom.support_weight), _dptr(geom.cos_theta),
              _dptr(geom.mask), out.numel(), int(bool(apodize)), _dptr(out), stream())
    return out


class Aberration:
    """Base of the pupil aberrations: ``__call__(geom, optics)`` returns the
    complex factor; ``apply_(pupil, geom, optics)`` multiplies a complex128
    CUDA pupil by it in place (psf/aberrations/base.py:11-34)."""

    def apply_(self, pupil: torch.Tensor, geom: Geometry, optics: Optics) -> torch.Tensor:
        raise NotImplementedError

    def __call__(self, geom: Geometry, optics: Optics) -> torch.Tensor:
        one = torch.ones(geom.shape, dtype=torch.complex128, device="cuda")
        return self.apply_(one, geom, optics)


class IndexMismatch(Aberration):
    """Gibson-Lanni depth aberration (psf/aberrations/geometric.py:11-62)."""

    def __init__(self, depth: float):
        self.depth = depth

    def apply_(self, pupil, geom, optics):
        _lib.call("decon_psf_index_mismatch", _dptr(geom.sin_theta), _dptr(geom.cos_theta),
                  pupil.numel(), float(optics.wavelength), float(optics.ni), float(optics.ns),
                  float(self.depth), _dptr(pupil), stream())
        return pupil

    def __repr__(self) -> str:
        return f"IndexMismatch(depth={self.depth})"


class Defocus(Aberration):
    """exp(2 pi i kz z) (psf/aberrations/geometric.py:65-96)."""

    def __init__(self, z: float):
        self.z = z

    def apply_(self, pupil, geom, optics):
        _lib.call("decon_psf_defocus", _dptr(geom.kz), pupil.numel(), float(self.z), _dptr(pupil),
                  stream())
        return pupil

    def __repr__(self) -> str:
        return f"Defocus(z={self.z})"


class ZernikeMode(IntEnum):
    """OSA/ANSI Zernike indices (psf/aberrations/zernike.py:15-51)."""

    PISTON = 0
    TILT_Y = 1
    TILT_X = 2
    ASTIG_OBLIQUE = 3
    DEFOCUS = 4
    ASTIG_VERTICAL = 5
    TREFOIL_Y = 6
    COMA_Y = 7
    COMA_X = 8
    TREFOIL_X = 9
    QUADRAFOIL_Y = 10
    ASTIG2_OBLIQUE = 11
    SPHERICAL = 12
    ASTIG2_VERTICAL = 13
    QUADRAFOIL_X = 14


class ZernikeAberration(Aberration):
    """exp(i mask sum_j c_j Z_j(rho, phi)), orthonormal OSA/ANSI Zernike
    polynomials, coefficients in radians (psf/aberrations/zernike.py:54-130)."""

    def __init__(self, coefficients: Union[Dict[Union[ZernikeMode, int], float], np.ndarray]):
        if isinstance(coefficients, dict):
            self._coefficients = dict(coefficients)
            self._array_form = None
        else:
            self._coefficients = None
            self._array_form = np.asarray(coefficients)

    def _terms(self):
        if self._coefficients is not None:
            items = [(int(j), float(c)) for j, c in self._coefficients.items()]
        else:
            items = [(j, float(c)) for j, c in enumerate(self._array_form)]
        return [(j, c) for j, c in items if c != 0]

    def apply_(self, pupil, geom, optics):
        terms = self._terms()
        js = (C.c_int * max(len(terms), 1))(*[j for j, _ in terms])
        cs = (C.c_double * max(len(terms), 1))(*[c for _, c in terms])
        _lib.call("decon_psf_zernike", _dptr(geom.rho), _dptr(geom.phi), _dptr(geom.mask),
                  pupil.numel(), len(terms), js, cs, _dptr(pupil), stream())
        return pupil

    def __repr__(self) -> str:
        if self._coefficients is not None:
            items = ", ".join(
                f"{ZernikeMode(k).name if isinstance(k, int) and k <= 14 else k}: {v:.3f}"
                for k, v in self._coefficients.items() if v != 0)
            return f"ZernikeAberration({{{items}}})"
        return f"ZernikeAberration(array with {np.count_nonzero(self._array_form)} nonzero terms)"


def apply_aberrations(pupil, geom: Geometry, optics: Optics, aberrations) -> torch.Tensor:
    """pupil * a_1(geom, optics) * a_2(geom, optics) ... in list order
    (psf/aberrations/base.py:37-62), on a copy of the pupil."""
    if isinstance(pupil, torch.Tensor):
        p = pupil.to(device="cuda", dtype=torch.complex128).clone()
    else:
        p = torch.from_numpy(np.ascontiguousarray(np.asarray(pupil, np.complex128))).to("cuda")
    for ab in aberrations:
        if isinstance(ab, Aberration):
            ab.apply_(p, geom, optics)
        else:  # any callable returning a factor of the pupil's shape
            f = ab(geom, optics)
            f = f if isinstance(f, torch.Tensor) else torch.from_numpy(np.asarray(f, np.complex128))
            p.mul_(f.to(device="cuda", dtype=torch.complex128))
    return p


def _kz(geom) -> np.ndarray:
    k = getattr(geom, "kz", geom)
    if isinstance(k, torch.Tensor):
        return k
    return np.asarray(k, np.float64)


def pupil_to_psf(pupil, geom, z, normalize: bool = True) -> torch.Tensor:
    """PSF of shape (nz, ny, nx), DC (the in-focus peak) at the corner of each
    plane.  ``geom`` is a ``Geometry`` (device or the reference's), or a ``kz``
    array of the pupil's shape.  Plane sizes factor into 2, 3, 5 and 7 and are
    at most 8192 points per axis."""
    _lib.require_cuda()
    if isinstance(pupil, torch.Tensor):
        p = pupil.to(device="cuda", dtype=torch.complex64).contiguous()
    else:
        p = torch.from_numpy(np.ascontiguousarray(np.asarray(pupil, np.complex64))).to("cuda")
    if p.ndim != 2:
        raise ValueError(f"pupil must be 2-D (ny, nx), got shape {tuple(p.shape)}")
    kz = _kz(geom)
    if tuple(kz.shape) != tuple(p.shape):
        raise ValueError(f"kz shape {tuple(kz.shape)} does not match the pupil's {tuple(p.shape)}")
    zz = np.atleast_1d(np.asarray(z, np.float64))
    if zz.ndim != 1 or zz.size == 0:
        raise ValueError("z must be a scalar or a non-empty 1-D array")
    ny, nx = p.shape
    if isinstance(kz, torch.Tensor):
        kz_d = kz.to(device="cuda", dtype=torch.float64).contiguous()
    else:
        kz_d = torch.from_numpy(np.ascontiguousarray(kz)).to("cuda")
    z_d = torch.from_numpy(np.ascontiguousarray(zz)).to("cuda")
    out = empty((len(zz), ny, nx))
    _lib.call("decon_pupil_to_psf", p.data_ptr(), kz_d.data_ptr(), z_d.data_ptr(), len(zz), ny, nx,
              int(bool(normalize)), out.data_ptr(), stream())
    return out
