"""CPU oracle for widefield PSF synthesis.

TEST INFRASTRUCTURE ONLY.  The checker that ``decon_pupil_to_psf`` is compared
against; only ``tests/`` may import it.

A float64 NumPy restatement of deconlib's ``pupil_to_psf``
(psf/widefield.py:18-73): defocus the pupil by exp(2 pi i kz z) for every z,
inverse 2-D FFT of each plane (DC at the corner), intensity |.|^2, and an
optional unit-sum normalisation.

Parity pin: ``tests/test_oracle_golden.py::test_pupil_to_psf`` checks it
against ``tests/golden/golden_psf.npz``, written by the reference's own
``pupil_to_psf`` (``tests/golden/make_golden.py``).
"""

from __future__ import annotations

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
