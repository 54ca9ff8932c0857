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


# ---- pupil model on the device (make_geometry / make_pupil / aberrations) ----

PUPIL_CASES = [((64, 64), 0.085, False, False), ((36, 50), 0.1, False, True),
               ((120, 256), 0.065, True, True), ((48, 63), 0.09, True, False)]


@pytest.mark.parametrize("i", range(4))
def test_device_pupil_matches_reference_pupils(i):
    # The four pupils and kz grids of golden_psf.npz, written by the reference
    # (tests/golden/make_golden.py::_run_psf: 525 nm, NA 1.4, ni 1.515, ns
    # 1.334; aberrated: IndexMismatch(6) then Zernike {SPHERICAL 0.4, COMA_X
    # 0.3}): kz bit for bit, the pupil to 1e-12 (FP64 transcendental ulps),
    # and the PSF synthesised from the device pupil to the reference's PSF.
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from deconlib_b200 import psf as P

    g = np.load(os.path.join(HERE, "golden", "golden_psf.npz"))
    shape, dxy, apod, aberr = PUPIL_CASES[i]
    optics = P.Optics(wavelength=0.525, na=1.4, ni=1.515, ns=1.334)
    geom = P.make_geometry(shape, dxy, optics)
    pupil = P.make_pupil(geom, apodize=apod)
    if aberr:
        pupil = P.apply_aberrations(pupil, geom, optics, [
            P.IndexMismatch(depth=6.0),
            P.ZernikeAberration({P.ZernikeMode.SPHERICAL: 0.4, P.ZernikeMode.COMA_X: 0.3})])
    np.testing.assert_array_equal(geom.kz.cpu().numpy(), g[f"psf{i}_kz"])
    assert np.abs(pupil.cpu().numpy() - g[f"psf{i}_pupil"]).max() <= 1e-12
    psf = P.pupil_to_psf(pupil, geom, g[f"psf{i}_z"], normalize=bool(g[f"psf{i}_normalize"]))
    ref = g[f"psf{i}_psf"].astype(np.float64)
    assert np.linalg.norm(psf.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-5


def test_device_geometry_vs_oracle_all_fields():
    # every Geometry field against the FP64 oracle restatement at the
    # benchmark's pupil size, anisotropic spacing, oversample 1 / 4 / 8 and the
    # wrapped Gaussian boundary smoothing; Defocus and the factor form of an
    # aberration (aberration(geom, optics)) as well
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from deconlib_b200 import psf as P
    from oracle import psf as opsf

    optics = P.Optics(wavelength=0.6, na=1.2, ni=1.33, ns=1.33)
    for shape, spacing, over, sigma in [((256, 256), 0.0425, 8, 0.0), ((90, 128), (0.07, 0.05), 4, 0.0),
                                        ((64, 80), 0.1, 1, 0.0), ((128, 128), 0.08, 8, 1.5)]:
        geom = P.make_geometry(shape, spacing, optics, oversample=over,
                               boundary_smoothing_sigma=sigma)
        ref = opsf.make_geometry(shape, spacing, 0.6, 1.2, 1.33, oversample=over,
                                 boundary_smoothing_sigma=sigma)
        for name in ("kx", "ky", "kz", "rho", "cos_theta", "sin_theta"):
            np.testing.assert_array_equal(getattr(geom, name).cpu().numpy(), ref[name], err_msg=name)
        np.testing.assert_array_equal(geom.mask.cpu().numpy(), ref["mask"])
        assert np.abs(geom.phi.cpu().numpy() - ref["phi"]).max() <= 1e-14
        tol = 0.0 if sigma == 0 else 1e-14
        assert np.abs(geom.support_weight.cpu().numpy() - ref["support_weight"]).max() <= tol
    geom = P.make_geometry((96, 96), 0.08, optics)
    ref = opsf.make_geometry((96, 96), 0.08, 0.6, 1.2, 1.33)
    f = P.Defocus(0.7)(geom, optics).cpu().numpy()
    assert np.abs(f - np.exp(1j * (2.0 * np.pi * ref["kz"] * 0.7))).max() <= 1e-12
    z = P.ZernikeAberration(np.array([0, 0.1, 0, 0.2, 0.3, 0, 0, -0.1, 0, 0, 0, 0, 0.25]))
    want = opsf.zernike_phase_factor(ref, {1: 0.1, 3: 0.2, 4: 0.3, 7: -0.1, 12: 0.25})
    assert np.abs(z(geom, optics).cpu().numpy() - want).max() <= 1e-12
    with pytest.raises(ValueError):
        P.Optics(wavelength=0.5, na=1.6, ni=1.5)
    with pytest.raises(ValueError):
        P.make_geometry((8, 8), -1.0, optics)
