"""On-device PSF synthesis (``decon_pupil_to_psf``) against the reference's
``pupil_to_psf`` (psf/widefield.py:18-73).

Tolerance: relative L2 <= 1e-5 against the reference's float64 PSF.  The
device evaluates the defocus phase in FP64 and the FFTs in FP32 (error
~1e-7 per transform); the pupil enters as complex64."""

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def psfmod():
    from deconlib_b200 import psf

    return psf


def _pupil(ny, nx, dxy, seed, na=1.4, wl=0.525, ni=1.515):
    """Anti-aliased NA disc with a seeded smooth phase, and its kz grid."""
    ky = np.fft.fftfreq(ny, dxy)[:, None]
    kx = np.fft.fftfreq(nx, dxy)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    kmax = na / wl
    w = np.clip((kmax - k) * max(ny, nx) * dxy + 0.5, 0.0, 1.0)
    kz = np.sqrt(np.maximum((ni / wl) ** 2 - k * k, 0.0))
    rho = np.clip(k / kmax, 0, 1)
    c = np.random.default_rng(seed).normal(size=3)
    phase = c[0] * (6 * rho ** 4 - 6 * rho ** 2 + 1) + c[1] * rho ** 2 + c[2] * rho ** 3 * np.cos(
        np.arctan2(ky, kx))
    return w * np.exp(1j * phase), kz


@pytest.mark.parametrize("case", range(4))
def test_golden(psfmod, case):
    g = np.load(os.path.join(HERE, "golden", "golden_psf.npz"))
    out = psfmod.pupil_to_psf(g[f"psf{case}_pupil"], g[f"psf{case}_kz"], g[f"psf{case}_z"],
                              normalize=bool(g[f"psf{case}_normalize"]))
    ref = g[f"psf{case}_psf"].astype(np.float64)
    assert tuple(out.shape) == ref.shape
    e = rel(out, ref)
    print(f"pupil_to_psf golden {ref.shape}: rel-L2 {e:.2e}")
    assert e < 1e-5


# (40, 1024, 1024) spans two chunks of planes; 8192 is the longest axis
@pytest.mark.parametrize("shape", [(33, 512, 768), (40, 1024, 1024), (3, 2048, 1470), (2, 8192, 40)])
def test_against_oracle(psfmod, shape):
    from oracle import psf as P

    nz, ny, nx = shape
    pupil, kz = _pupil(ny, nx, 0.06, seed=nz)
    z = np.fft.fftfreq(nz) * nz * 0.12
    for norm in (True, False):
        out = psfmod.pupil_to_psf(pupil, kz, z, normalize=norm)
        ref = P.pupil_to_psf(pupil.astype(np.complex64), kz, z, norm)
        e = rel(out, ref)
        print(f"pupil_to_psf {shape} normalize={norm}: rel-L2 {e:.2e}")
        assert e < 1e-5
        if norm:
            assert abs(out.double().sum().item() - 1.0) < 1e-5


def test_geometry_object_torch_pupil_and_scalar_z(psfmod):
    from oracle import psf as P

    pupil, kz = _pupil(64, 96, 0.08, seed=5)

    class Geom:
        pass

    geom = Geom()
    geom.kz = kz
    out = psfmod.pupil_to_psf(torch.from_numpy(pupil.astype(np.complex64)), geom, 0.3)
    assert tuple(out.shape) == (1, 64, 96)
    assert rel(out, P.pupil_to_psf(pupil.astype(np.complex64), kz, 0.3)) < 1e-5


def test_psf_feeds_the_convolver(psfmod):
    """A device PSF becomes a LinearFFTConvolver kernel without leaving HBM."""
    import deconlib_b200.deconvolution as D

    pupil, kz = _pupil(64, 64, 0.085, seed=9)
    z = np.fft.fftfreq(32) * 32 * 0.1
    psf_d = psfmod.pupil_to_psf(pupil, kz, z)
    psf_h = psf_d.cpu().numpy()
    x = np.random.default_rng(0).random((32, 64, 64)).astype(np.float32)
    a = D.LinearFFTConvolver(psf_d, (32, 64, 64)).forward(x)
    b = D.LinearFFTConvolver(psf_h, (32, 64, 64)).forward(x)
    torch.testing.assert_close(a, b, rtol=0, atol=0)


def test_errors(psfmod):
    from deconlib_b200._lib import DeconError

    pupil, kz = _pupil(44, 44, 0.08, seed=1)
    with pytest.raises(DeconError, match="2, 3, 5 and 7"):
        psfmod.pupil_to_psf(pupil, kz, [0.0])
    pupil, kz = _pupil(32, 32, 0.08, seed=1)
    with pytest.raises(ValueError):
        psfmod.pupil_to_psf(pupil, kz[:, :16], [0.0])
    with pytest.raises(ValueError):
        psfmod.pupil_to_psf(pupil, kz, np.zeros(0))
    with pytest.raises(DeconError, match="8192"):
        p2, k2 = _pupil(8, 16384, 0.08, seed=1)
        psfmod.pupil_to_psf(p2, k2, [0.0])
