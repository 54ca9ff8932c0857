"""Widefield PSF synthesis on the device.

``pupil_to_psf`` mirrors deconlib's ``pupil_to_psf`` (psf/widefield.py:18-73):
same arguments (complex pupil (ny, nx) with DC at the corner, a geometry
holding ``kz``, axial positions ``z`` in um, ``normalize``) and the same
result, PSF(z) = |IFFT2(pupil * exp(2 pi i kz z))|^2 of shape (nz, ny, nx),
unit sum when normalised.  The work runs in ``decon_pupil_to_psf``: two FFT
passes (the FP64 defocus phase fused into the y transform; the x transform
fused with the intensity and the final scale) and an FP64 pupil energy that
gives the unit-sum total by Parseval.  The result is a CUDA float32 tensor,
ready to become a convolution kernel without a host round trip.

The pupil itself (make_geometry / make_pupil / aberrations) is a small 2-D
host computation and stays with the caller.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .deconvolution._device import empty, stream

__all__ = ["pupil_to_psf"]


def _kz(geom) -> np.ndarray:
    return np.asarray(getattr(geom, "kz", geom), np.float64)


def pupil_to_psf(pupil, geom, z, normalize: bool = True) -> torch.Tensor:
    """PSF of shape (nz, ny, nx), DC (the in-focus peak) at the corner of each
    plane.  ``geom`` is any object with a ``kz`` array of the pupil's shape
    (the reference's ``Geometry``), or that array itself.  Plane sizes factor
    into 2, 3, 5 and 7 and are at most 8192 points per axis."""
    _lib.require_cuda()
    if isinstance(pupil, torch.Tensor):
        p = pupil.to(device="cuda", dtype=torch.complex64).contiguous()
    else:
        p = torch.from_numpy(np.ascontiguousarray(np.asarray(pupil, np.complex64))).to("cuda")
    if p.ndim != 2:
        raise ValueError(f"pupil must be 2-D (ny, nx), got shape {tuple(p.shape)}")
    kz = _kz(geom)
    if kz.shape != tuple(p.shape):
        raise ValueError(f"kz shape {kz.shape} does not match the pupil's {tuple(p.shape)}")
    zz = np.atleast_1d(np.asarray(z, np.float64))
    if zz.ndim != 1 or zz.size == 0:
        raise ValueError("z must be a scalar or a non-empty 1-D array")
    ny, nx = p.shape
    kz_d = torch.from_numpy(np.ascontiguousarray(kz)).to("cuda")
    z_d = torch.from_numpy(np.ascontiguousarray(zz)).to("cuda")
    out = empty((len(zz), ny, nx))
    _lib.call("decon_pupil_to_psf", p.data_ptr(), kz_d.data_ptr(), z_d.data_ptr(), len(zz), ny, nx,
              int(bool(normalize)), out.data_ptr(), stream())
    return out
