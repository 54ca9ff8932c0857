"""GPU parity at the benchmark configurations, against the FP32 and FP64 oracle.

These are the sizes whose kernels the smaller parity cases do not reach:

  * ``LinearFFTConvolver`` on a 128x256x256 signal (canvas 256x512x512): the
    two-CTA axial kernel of length 256, the 512-point Y passes with the
    half-zero split and the X passes of packed length 256 (Fx = 512).
    Tolerance: 1e-6 relative L2 against the FP64 oracle (the FP32 transforms
    round at ~1e-7 per pass).
  * ``solve_pdhg_mlx`` on the headline workload (object 128x256x256, data
    64x128x128, sampling 2, Hessian L1, alpha 1e-3, background 5), 20
    iterations.  Tolerance: max(1e-4, 2 x the FP32-vs-FP64 oracle spread) on
    x, and the same rule (at least 1e-4) on the tau / sigma / loss histories,
    because the device computes step sizes and sums in FP64 while the FP32
    reference rounds them to float32 (deconlib/deconvolution/pdhg_mlx.py:717-900).
  * ``richardson_lucy_with_operator`` on the RL workload (64x128x128 beads and
    shells, canvas 128x256x256, background 10), the full 50 iterations.
    Tolerance: max(1e-5, 2 x the FP32-vs-FP64 oracle spread) on x, 1e-6 on the
    prediction relative to the FP64 oracle's, loss history rtol 1e-5
    (deconlib/deconvolution/rl_mlx.py:117-175).

Inputs are the seeded synthetic workloads of the benchmark, observed through
the FP64 oracle (no device code is involved in making them).  The oracle runs
its FFTs with every host thread (scipy.fft workers).
"""

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

OBJ = (128, 256, 256)
DATA = (64, 128, 128)
SPACING_PD = (0.05, 0.0425, 0.0425)
RL_SHAPE = (64, 128, 128)
SPACING_RL = (0.1, 0.085, 0.085)


def rel(a, b):
    a = np.asarray(a.detach().cpu().numpy() if hasattr(a, "detach") else a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def D():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import deconlib_b200.deconvolution as d

    return d


@pytest.fixture(scope="module")
def oracle():
    from oracle import ops, solvers

    ops.set_fft_workers(os.cpu_count() or 1)
    yield ops, solvers
    ops.set_fft_workers(1)


@pytest.fixture(scope="module")
def pdhg_case(oracle):
    from deconlib_b200 import synth

    ops, _ = oracle
    psf, truth = synth.pdhg_workload(OBJ, SPACING_PD, seed=2)
    fwd = ops.compose(ops.FractionalAreaDownsample(2.0, in_shape=OBJ, dtype=np.float64),
                      ops.LinearFFTConvolver(psf, OBJ, dtype=np.float64))
    obs = synth.poisson_observation(fwd.forward(truth.astype(np.float64)), 500.0, 5.0,
                                    np.random.default_rng(3))
    assert obs.shape == DATA
    return psf, truth, obs


def test_conv_headline_canvas_vs_fp64_oracle(D, oracle, pdhg_case):
    ops, _ = oracle
    psf, truth, _ = pdhg_case
    c = D.LinearFFTConvolver(psf, OBJ)
    assert c.fft_shape == (256, 512, 512)
    o = ops.LinearFFTConvolver(psf, OBJ, dtype=np.float64)
    rng = np.random.default_rng(5)
    x = (truth + 0.1 * rng.random(OBJ, dtype=np.float32)).astype(np.float32)
    ef = rel(c.forward(x), o.forward(x.astype(np.float64)))
    ea = rel(c.adjoint(x), o.adjoint(x.astype(np.float64)))
    print(f"\nconv 128x256x256 (canvas 256x512x512) vs FP64 oracle: forward {ef:.2e}, "
          f"adjoint {ea:.2e}")
    assert ef < 1e-6 and ea < 1e-6
    assert abs(c.operator_norm_sq - o.operator_norm_sq) <= 1e-6 * o.operator_norm_sq
    from deconlib_b200 import _lib

    _lib.call("decon_device_status", _lib.stream_ptr())


def test_pdhg_headline_vs_oracle(D, oracle, pdhg_case):
    _, solvers = oracle
    psf, _, obs = pdhg_case
    kw = dict(alpha=1e-3, regularization="hessian", sampling_factors=2.0, spacing=SPACING_PD,
              background=5.0, num_iter=20, eval_interval=10)
    r = D.solve_pdhg_mlx(obs, psf, **kw)
    r32 = solvers.solve_pdhg_mlx(obs, psf, dtype=np.float32, **kw)
    r64 = solvers.solve_pdhg_mlx(obs, psf, dtype=np.float64, **kw)
    spread = rel(r32["restored"], r64["restored"])
    tol = max(1e-4, 2 * spread)
    e64 = rel(r.restored, r64["restored"])
    e32 = rel(r.restored, r32["restored"])
    print(f"\nPDHG headline, 20 it.: vs FP64 {e64:.2e}, vs FP32 {e32:.2e}, "
          f"FP32-FP64 spread {spread:.2e}, tolerance {tol:.2e}")
    assert r.iterations == r64["iterations"] == 20
    assert e64 < tol and e32 < tol
    np.testing.assert_allclose(r.tau_history, r64["tau_history"], rtol=tol)
    np.testing.assert_allclose(r.sigma_history, r64["sigma_history"], rtol=tol)
    np.testing.assert_allclose(r.loss_history, r64["loss_history"], rtol=tol)
    assert len(r.loss_history) == 2


def test_rl_workload_50_iterations_vs_oracle(D, oracle):
    from deconlib_b200 import synth

    ops, solvers = oracle
    psf, truth = synth.rl_workload(RL_SHAPE, SPACING_RL, seed=0)
    o64 = ops.LinearFFTConvolver(psf, RL_SHAPE, dtype=np.float64)
    obs = synth.poisson_observation(o64.forward(truth.astype(np.float64)), 1000.0, 10.0,
                                    np.random.default_rng(1))
    c = D.LinearFFTConvolver(psf, RL_SHAPE)
    assert c.fft_shape == (128, 256, 256)
    r = D.richardson_lucy_with_operator(obs, c, num_iter=50, background=10.0)
    r32 = solvers.richardson_lucy_with_operator(
        obs, ops.LinearFFTConvolver(psf, RL_SHAPE, dtype=np.float32), num_iter=50,
        background=10.0, dtype=np.float32)
    r64 = solvers.richardson_lucy_with_operator(obs, o64, num_iter=50, background=10.0,
                                                dtype=np.float64)
    spread = rel(r32["restored"], r64["restored"])
    tol = max(1e-5, 2 * spread)
    e64 = rel(r.restored, r64["restored"])
    ep = rel(r.pred, r64["pred"])
    print(f"\nRL 64x128x128, 50 it.: x vs FP64 {e64:.2e} (FP32-FP64 spread {spread:.2e}, "
          f"tolerance {tol:.2e}); prediction {ep:.2e}")
    assert r.iterations == 50
    assert e64 < tol
    assert ep < 1e-6
    np.testing.assert_allclose(r.loss_history, r64["loss_history"], rtol=1e-5)
