"""Mixed precision: the OTF stored as FP16 complex with a power-of-two scale
per kz plane, read by the pipelined axial pass.

The FP16 mantissa (11 bits) bounds the relative error of each OTF value by
2^-12 after rounding (per-plane power-of-two scales keep every plane's
largest value near the top of the FP16 range); a convolution output is a sum
over many such products, so its relative L2 error against the FP32 path is
~1e-4 (measured 7-9e-5 at 64x128x128 and 128x256x256).  RL multiplies
these errors into its iterate: against the FP64 oracle the mixed form
measured 8.2e-5 / 8.5e-5 / 1.3e-4 at iterations 10 / 50 / 200 (the FP32 form
6.8e-7 / 3.1e-6 / 1.2e-5).  Tolerances here: 2e-3 for one convolution,
3e-4 for 20 RL iterations against the FP64 oracle (3x the measured error;
a 1e-4 bound would need about two more mantissa bits than FP16 stores).
Every result states its error."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    b = b.detach().cpu().numpy() if hasattr(b, "detach") else np.asarray(b)
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def D():
    import deconlib_b200.deconvolution as D

    return D


@pytest.mark.parametrize("shape", [(64, 128, 128), (128, 256, 256)])
def test_mixed_convolution_close_to_fp32(D, shape):
    from deconlib_b200 import synth

    rng = np.random.default_rng(1)
    psf = synth.widefield_psf(shape, 0.1, 0.085)
    x = rng.random(shape).astype(np.float32)
    c32 = D.LinearFFTConvolver(psf, shape)
    c16 = D.LinearFFTConvolver(psf, shape, precision="mixed")
    f32, f16 = c32.forward(x), c16.forward(x)
    a32, a16 = c32.adjoint(x), c16.adjoint(x)
    e_f, e_a = rel(f16, f32), rel(a16, a32)
    print(f"mixed conv {shape}: forward rel-L2 {e_f:.2e}, adjoint {e_a:.2e}")
    assert 0 < e_f < 2e-3 and 0 < e_a < 2e-3
    # back to FP32 restores the FP32 results exactly
    c16.set_precision("fp32")
    np.testing.assert_array_equal(c16.forward(x).cpu().numpy(), f32.cpu().numpy())


def test_mixed_precision_needs_the_pipelined_axial_pass(D):
    rng = np.random.default_rng(2)
    k = rng.random((5, 9, 9)).astype(np.float32)
    c = D.LinearFFTConvolver(k, (20, 40, 40), fft_shape=(30, 48, 48))
    with pytest.raises(RuntimeError, match="pipelined axial pass"):
        c.set_precision("mixed")
    with pytest.raises(ValueError):
        c.set_precision("fp8")


def test_mixed_rl_against_fp64_oracle(D):
    from deconlib_b200 import synth

    shape = (64, 128, 128)
    rng = np.random.default_rng(3)
    psf = synth.widefield_psf(shape, 0.1, 0.085)
    truth = synth.beads(shape, 200, rng) + 0.02
    blur = D.LinearFFTConvolver(psf, shape).forward(truth).cpu().numpy()
    obs = synth.poisson_observation(blur, 1000.0, 10.0, rng)
    n = 20
    r32 = D.richardson_lucy_with_operator(obs, D.LinearFFTConvolver(psf, shape), num_iter=n,
                                          background=10.0).restored
    r16 = D.richardson_lucy_with_operator(obs, D.LinearFFTConvolver(psf, shape, precision="mixed"),
                                          num_iter=n, background=10.0).restored
    from oracle import ops as O
    from oracle import solvers as S

    O.set_fft_workers(8)
    op64 = O.LinearFFTConvolver(psf.astype(np.float64), shape, dtype=np.float64)
    ref = S.richardson_lucy_with_operator(obs, op64, num_iter=n, background=10.0,
                                          dtype=np.float64)["restored"]
    e32, e16 = rel(r32, ref), rel(r16, ref)
    print(f"RL {shape} x{n}: FP32 rel-L2 vs FP64 oracle {e32:.2e}, mixed {e16:.2e}")
    assert e32 < 1e-4
    assert e16 < 3e-4


def test_mixed_lean_axial_pass_bit_identical_to_register_form(D, monkeypatch):
    """Axial length 256: the lean two-CTA kernel stages each FP16 OTF tile by
    TMA into shared memory, the one-CTA form (DECON_PIPE_LEAN=0) loads it into
    registers; the products and transforms are the same, so are the bits."""
    from deconlib_b200 import synth

    shape = (64, 128, 128)
    rng = np.random.default_rng(4)
    psf = synth.widefield_psf(shape, 0.1, 0.085)
    x = rng.random(shape).astype(np.float32)
    c = D.LinearFFTConvolver(psf, shape, fft_shape=(256, 256, 256), precision="mixed")
    f_lean, a_lean = c.forward(x).cpu().numpy(), c.adjoint(x).cpu().numpy()
    monkeypatch.setenv("DECON_PIPE_LEAN", "0")
    f_reg, a_reg = c.forward(x).cpu().numpy(), c.adjoint(x).cpu().numpy()
    np.testing.assert_array_equal(f_lean, f_reg)
    np.testing.assert_array_equal(a_lean, a_reg)
    c32 = D.LinearFFTConvolver(psf, shape, fft_shape=(256, 256, 256))
    e = rel(f_lean, c32.forward(x))
    print(f"mixed lean axial pass vs FP32: {e:.2e}")
    assert 0 < e < 2e-3
