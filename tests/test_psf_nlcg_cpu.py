"""CPU checks of the identities the device PSF and NLCG paths rely on,
evaluated with the oracle (no GPU)."""

import numpy as np
import pytest

from oracle import nlcg, ops
from oracle import psf as opsf


def _pupil(ny, nx, seed):
    rng = np.random.default_rng(seed)
    ky = np.fft.fftfreq(ny, 0.07)[:, None]
    kx = np.fft.fftfreq(nx, 0.07)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    w = np.clip((1.3 / 0.525 - k) * max(ny, nx) * 0.07 + 0.5, 0.0, 1.0)
    pupil = w * np.exp(1j * rng.normal(size=3) @ np.array([k, k * k, k ** 3]).reshape(3, -1)).reshape(ny, nx)
    kz = np.sqrt(np.maximum((1.515 / 0.525) ** 2 - k * k, 0.0))
    return pupil, kz


@pytest.mark.parametrize("shape", [(5, 24, 40), (1, 36, 50), (9, 64, 63)])
def test_psf_total_is_parseval(shape):
    """decon_pupil_to_psf normalises with nz * ny * nx * sum|P|^2 instead of
    summing the PSF: |exp(i phi)| = 1 and Parseval make every unnormalised
    plane sum to ny nx sum|P|^2 (numpy's ifft2 scaling divides by (ny nx)^2)."""
    nz, ny, nx = shape
    pupil, kz = _pupil(ny, nx, nz)
    z = np.fft.fftfreq(nz) * nz * 0.15
    raw = opsf.pupil_to_psf(pupil, kz, z, normalize=False)
    energy = np.sum(np.abs(pupil) ** 2)
    np.testing.assert_allclose(raw.sum(axis=(1, 2)), energy / (ny * nx), rtol=1e-12)
    norm = opsf.pupil_to_psf(pupil, kz, z, normalize=True)
    np.testing.assert_allclose(norm, raw * (ny * nx) / (nz * energy), rtol=1e-12)
    assert abs(norm.sum() - 1.0) < 1e-12


def test_psf_zero_pupil_is_left_unnormalised():
    pupil = np.zeros((8, 8), complex)
    out = opsf.pupil_to_psf(pupil, np.zeros((8, 8)), [0.0, 0.1])
    assert out.shape == (2, 8, 8) and not out.any()


def _problem(seed=0):
    rng = np.random.default_rng(seed)
    shape = (8, 16, 16)
    psf = rng.random((5, 7, 7)) ** 3
    truth = rng.random(shape) ** 4 * 50
    conv = ops.LinearFFTConvolver(psf, shape, dtype=np.float64)
    obs = rng.poisson(conv.forward(truth) + 5.0).astype(np.float64)
    return conv, obs


def test_nlcg_step_failure_branch():
    """newton_iters=0 leaves lambda = 0: the first step cannot lower phi and
    d is r, so the solve stops at once as converged (nlcg_mlx.py:476-479)."""
    conv, obs = _problem()
    r = nlcg.nlcg_with_operator(obs, conv, num_iter=6, background=5.0, newton_iters=0,
                                dtype=np.float64)
    assert r["iterations"] == 1 and r["converged"] and len(r["loss_history"]) == 1


def test_nlcg_regulariser_sums_are_polynomials_in_lambda():
    """The device Newton step evaluates the regulariser's terms from the Gram
    matrix of C f, C(sd), C(dd); by linearity they equal the sums over
    u = C f(lam) = Cf + 2 lam C(sd) + lam^2 C(dd)."""
    rng = np.random.default_rng(4)
    H = ops.Hessian3D(0.8, np.float64)
    f, sd, dd = (rng.random((6, 10, 12)) for _ in range(3))
    A, B, Cc = H.forward(f), H.forward(sd), H.forward(dd)
    G = [np.sum(A * A), np.sum(A * B), np.sum(A * Cc), np.sum(B * B), np.sum(B * Cc), np.sum(Cc * Cc)]
    for lam in (0.0, 0.3, -1.7):
        u = A + 2 * lam * B + lam * lam * Cc
        bl = B + lam * Cc
        np.testing.assert_allclose(np.sum(u * bl), G[1] + lam * (G[2] + 2 * G[3]) + 3 * lam ** 2 * G[4]
                                   + lam ** 3 * G[5], rtol=1e-10)
        np.testing.assert_allclose(np.sum(bl * bl), G[3] + 2 * lam * G[4] + lam ** 2 * G[5], rtol=1e-10)
        np.testing.assert_allclose(np.sum(u * Cc), G[2] + 2 * lam * G[4] + lam ** 2 * G[5], rtol=1e-10)


def test_nlcg_objective_decreases_monotonically():
    conv, obs = _problem(1)
    phis = []
    nlcg.nlcg_with_operator(obs, conv, num_iter=8, background=5.0, min_iter=100, dtype=np.float64,
                            callback=lambda k, f: phis.append(
                                nlcg.nlcg_objective(np.sqrt(f), conv, obs, 5.0, dtype=np.float64)))
    assert len(phis) == 8 and all(b < a for a, b in zip(phis, phis[1:]))


def test_pupil_restatement_matches_reference_pupils():
    """The oracle's make_geometry / make_pupil / IndexMismatch / Zernike
    rebuild the four pupils and kz grids the reference wrote into
    golden_psf.npz (tests/golden/make_golden.py::_run_psf: 525 nm, NA 1.4,
    ni 1.515, ns 1.334; aberrated cases IndexMismatch(6) then Zernike
    {SPHERICAL: 0.4, COMA_X: 0.3})."""
    import os

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_psf.npz"))
    cases = [((64, 64), 0.085, False, False), ((36, 50), 0.1, False, True),
             ((120, 256), 0.065, True, True), ((48, 63), 0.09, True, False)]
    for i, (shape, dxy, apod, aberr) in enumerate(cases):
        geom = opsf.make_geometry(shape, dxy, 0.525, 1.4, 1.515)
        pupil = opsf.make_pupil(geom, apodize=apod)
        if aberr:
            pupil = pupil * opsf.index_mismatch(geom, 6.0, 0.525, 1.515, 1.334)
            pupil = pupil * opsf.zernike_phase_factor(geom, {12: 0.4, 8: 0.3})
        ref = g[f"psf{i}_pupil"]
        np.testing.assert_array_equal(geom["kz"], g[f"psf{i}_kz"])
        assert np.abs(pupil - ref).max() <= 1e-12
