"""GPU parity: the CUDA path (through libdecon_b200's C ABI) against the
golden vectors of the reference and against the CPU oracle.

Tolerances (relative L2 unless stated):
  * operators (conv, resampling, stencils): 2e-6 vs the float32 reference
    (both are float32 evaluations of the same formulas; only FFT rounding
    differs) and 1e-6 against the float64 oracle for the convolution;
  * Pad / Crop: bit-exact;
  * Richardson-Lucy trajectories: 1e-5 after 8-12 iterations;
  * PDHG trajectories: max(1e-4, 2 x the float32-vs-float64 reference spread),
    because the GPU computes step sizes and reductions in FP64 while the
    float32 reference rounds them to float32 (the stated tolerance rule).
"""

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def g32():
    return np.load(os.path.join(HERE, "golden", "golden_fp32.npz"))


@pytest.fixture(scope="module")
def g64():
    return np.load(os.path.join(HERE, "golden", "golden_fp64.npz"))


@pytest.fixture(scope="module")
def D():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import deconlib_b200.deconvolution as d

    return d


def rel(a, b):
    a = np.asarray(a.detach().cpu().numpy() if hasattr(a, "detach") else a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def cpu(t):
    return t.detach().cpu().numpy()


def test_conv_forward_adjoint(D, g32, g64):
    c = D.LinearFFTConvolver(g32["psf16"], (16, 32, 32))
    assert c.fft_shape == tuple(g32["conv_fft_shape"])
    assert abs(c.operator_norm_sq - float(g32["conv_norm"])) < 1e-5
    x = g32["conv_x"]
    assert rel(c.forward(x), g32["conv_fwd"]) < 2e-6
    assert rel(c.adjoint(x), g32["conv_adj"]) < 2e-6
    assert rel(c.forward(x), g64["conv_fwd"]) < 1e-6
    assert rel(c.adjoint(x), g64["conv_adj"]) < 1e-6


def test_conv_odd_and_explicit_canvas(D, g32, g64):
    co = D.LinearFFTConvolver(g32["kodd"], (9, 11, 13))
    assert co.fft_shape == tuple(g32["convodd_fft_shape"])
    xo = g32["convodd_x"]
    assert rel(co.forward(xo), g64["convodd_fwd"]) < 1e-6
    assert rel(co.adjoint(xo), g64["convodd_adj"]) < 1e-6
    assert abs(co.operator_norm_sq - float(g64["convodd_norm"])) < 1e-6 * float(g64["convodd_norm"])
    cx = D.LinearFFTConvolver(g32["kodd"], (9, 11, 13), normalize=False, fft_shape=(15, 18, 25))
    assert rel(cx.forward(xo), g64["convx_fwd"]) < 1e-6
    assert rel(cx.adjoint(xo), g64["convx_adj"]) < 1e-6


def test_conv_2d(D, g64):
    c = D.LinearFFTConvolver(g64["k2d"].astype(np.float32), (20, 30))
    x = g64["conv2d_x"].astype(np.float32)
    assert rel(c.forward(x), g64["conv2d_fwd"]) < 1e-6
    assert rel(c.adjoint(x), g64["conv2d_adj"]) < 1e-6


def test_otf_matches_oracle(D, g32):
    from oracle import ops

    c = D.LinearFFTConvolver(g32["psf16"], (16, 32, 32))
    o = ops.LinearFFTConvolver(g32["psf16"], (16, 32, 32), dtype=np.float64)
    err = np.linalg.norm(cpu(c.otf) - o.otf) / np.linalg.norm(o.otf)
    assert err < 1e-6


@pytest.mark.parametrize("shape,kshape", [((64, 128, 128), (64, 128, 128)),
                                          ((40, 96, 72), (17, 33, 25)),
                                          ((30, 50, 45), (9, 15, 12))])
def test_conv_sizes_vs_fp64_oracle(D, shape, kshape):
    from oracle import ops

    rng = np.random.default_rng(sum(shape))
    k = rng.random(kshape).astype(np.float32)
    x = rng.random(shape).astype(np.float32)
    c = D.LinearFFTConvolver(k, shape)
    o = ops.LinearFFTConvolver(k, shape, dtype=np.float64)
    assert rel(c.forward(x), o.forward(x.astype(np.float64))) < 2e-6
    assert rel(c.adjoint(x), o.adjoint(x.astype(np.float64))) < 2e-6


@pytest.mark.parametrize("fft", [(80, 96, 160), (160, 192, 192), (240, 320, 320), (384, 480, 384),
                                 (64, 640, 480), (64, 768, 640), (64, 960, 768), (64, 64, 960),
                                 (64, 64, 1280), (64, 64, 1536), (64, 64, 1920)])
def test_static_length_canvases_vs_fp64_oracle(D, fft):
    """Every compile-time FFT length of 2^a x {3, 5, 15} in the strided
    passes (z, y) and in the X passes (packed length Fx / 2)."""
    from oracle import ops

    shape, kshape = (16, 24, 32), (7, 9, 11)
    rng = np.random.default_rng(sum(fft))
    k = rng.random(kshape).astype(np.float32)
    x = rng.random(shape).astype(np.float32)
    c = D.LinearFFTConvolver(k, shape, fft_shape=fft)
    o = ops.LinearFFTConvolver(k, shape, fft_shape=fft, dtype=np.float64)
    ef = rel(c.forward(x), o.forward(x.astype(np.float64)))
    ea = rel(c.adjoint(x), o.adjoint(x.astype(np.float64)))
    assert ef < 2e-6 and ea < 2e-6, (ef, ea)


def test_static_fft_shape_rule(D):
    assert D.static_fft_shape((76, 362, 244), (76, 362, 244)) == (256, 768, 512)
    assert D.static_fft_shape((128, 256, 256), (128, 256, 256)) == (256, 512, 512)
    # small axes keep the 5-smooth length when the static one is > 4/3 of it
    assert D.static_fft_shape((16, 32, 32), (16, 32, 32)) == (32, 64, 64)
    c = D.LinearFFTConvolver(np.ones((5, 5, 5), np.float32), (60, 70, 90),
                             fft_shape=D.static_fft_shape((60, 70, 90), (5, 5, 5)))
    assert c.fft_shape == (64, 80, 128)


def test_conv_adjoint_identity(D):
    # <A x, y> == <x, A^T y>  (tests/test_composition.py:66-73, rtol 1e-4)
    rng = np.random.default_rng(3)
    k = rng.random((7, 9, 11)).astype(np.float32)
    c = D.LinearFFTConvolver(k, (20, 24, 28))
    x = rng.random((20, 24, 28)).astype(np.float32)
    y = rng.random((20, 24, 28)).astype(np.float32)
    lhs = float(np.sum(cpu(c.forward(x)).astype(np.float64) * y))
    rhs = float(np.sum(x.astype(np.float64) * cpu(c.adjoint(y))))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)


def test_pad_crop_exact(D, g32):
    x = g32["pad_x"]
    np.testing.assert_array_equal(cpu(D.Pad(((1, 2), (0, 3), (4, 0))).forward(x)), g32["pad_fwd"])
    c = D.Crop((9, 10, 11), (5, 6, 7))
    np.testing.assert_array_equal(cpu(c.forward(x)), g32["crop_fwd"])
    np.testing.assert_array_equal(cpu(c.adjoint(g32["crop_y"])), g32["crop_adj"])
    c2 = D.Crop((9, 10, 11), (5, 6, 7), start=(4, 0, 3))
    np.testing.assert_array_equal(cpu(c2.forward(x)), g32["crop2_fwd"])
    np.testing.assert_array_equal(cpu(c2.adjoint(g32["crop_y"])), g32["crop2_adj"])
    p = D.Pad(((1, 2), (0, 3), (4, 0)))
    np.testing.assert_array_equal(cpu(p.adjoint(p.forward(x))), x)


def test_resampling(D, g32):
    x, y = g32["rs_x"], g32["rs_y"]
    d2 = D.FractionalAreaDownsample(2.0, in_shape=(12, 20, 18))
    assert rel(d2.forward(x), g32["down2_fwd"]) < 2e-7
    assert rel(d2.adjoint(y), g32["down2_adj"]) < 2e-7
    d15 = D.FractionalAreaDownsample((1.5, 1.25, 2.5), in_shape=(12, 20, 18))
    assert rel(d15.forward(x), g32["down15_fwd"]) < 2e-7
    assert rel(d15.adjoint(g32["down15_y"]), g32["down15_adj"]) < 2e-7
    assert rel(D.FractionalAreaDownsample(2.0).forward(x), g32["down2np_fwd"]) < 2e-7
    up = D.FractionalAreaUpsample(2.0)
    assert rel(up.forward(y), g32["up2_fwd"]) < 2e-7
    assert rel(up.adjoint(x), g32["up2_adj"]) < 2e-7
    up3 = D.FractionalAreaUpsample((1.5, 2.0, 3.0))
    assert rel(up3.forward(y), g32["up3_fwd"]) < 2e-7
    assert rel(D.FractionalAreaDownsample(3.0).forward(g32["rs2d_x"]), g32["down2d_fwd"]) < 2e-7
    assert rel(D.FractionalAreaDownsample(2.5).forward(g32["rs1d_x"]), g32["down1d_fwd"]) < 2e-7


def test_stencils(D, g32):
    x, y = g32["hess_x"], g32["hess_y"]
    h = D.Hessian3D(0.7)
    assert rel(h.forward(x), g32["hess_fwd"]) < 2e-7
    assert rel(h.adjoint(y), g32["hess_adj"]) < 2e-7
    gr = D.Gradient3D(0.7)
    assert rel(gr.forward(x), g32["grad_fwd"]) < 2e-7
    assert rel(gr.adjoint(y[:3]), g32["grad_adj"]) < 2e-7


def test_prox(D, g32):
    y, d = g32["prox_y"], g32["prox_d"]
    assert rel(D.prox_poisson_dual(y, 0.3, d, 2.0), g32["prox_poisson"]) < 1e-6
    assert rel(D.prox_gaussian_dual(y, 0.3, d, 2.0), g32["prox_gauss"]) < 1e-6
    np.testing.assert_array_equal(cpu(D.prox_l1_dual(y, 0.5)), g32["prox_l1"])
    assert rel(D.prox_l1_2_dual(g32["prox_l12_y"], 0.5), g32["prox_l12"]) < 1e-6


def test_rl_fused(D, g32, g64):
    c = D.LinearFFTConvolver(g32["psf16"], (16, 32, 32))
    r = D.richardson_lucy_with_operator(g32["rl_obs"], c, num_iter=12, background=10.0,
                                        eval_interval=5)
    assert r.iterations == int(g32["rl_iters"])
    assert rel(r.restored, g32["rl_x"]) < 1e-5
    assert rel(r.restored, g64["rl_x"]) < 1e-5
    assert rel(r.pred, g64["rl_pred"]) < 1e-6
    np.testing.assert_allclose(r.loss_history, g64["rl_loss"], rtol=1e-5)


def test_rl_composed_crop(D, g32, g64):
    c = D.LinearFFTConvolver(g32["psf16"], (16, 32, 32))
    op = D.compose(D.Crop((16, 32, 32), (12, 26, 28), start=(2, 3, 2)), c)
    r = D.richardson_lucy_with_operator(g32["rlc_obs"], op, num_iter=8, background=10.0,
                                        eval_interval=3)
    assert rel(r.restored, g64["rlc_x"]) < 1e-5
    assert rel(r.pred, g64["rlc_pred"]) < 1e-6
    np.testing.assert_allclose(r.loss_history, g64["rlc_loss"], rtol=1e-5)


def test_rl_callback_stops(D, g32):
    c = D.LinearFFTConvolver(g32["psf16"], (16, 32, 32))
    seen = []
    r = D.richardson_lucy_with_operator(g32["rl_obs"], c, num_iter=12, background=10.0,
                                        callback=lambda k, x: seen.append(k) or k == 4)
    assert r.iterations == 5 and seen == [0, 1, 2, 3, 4]


PD_CASES = {
    "pd_h_l1": dict(regularization="hessian", norm="L1"),
    "pd_h_l12": dict(regularization="hessian", norm="L1_2"),
    "pd_g_l1": dict(regularization="gradient", norm="L1"),
    "pd_i_l1": dict(regularization="identity", norm="L1"),
    "pd_h_gauss": dict(regularization="hessian", norm="L1", loss_type="gaussian"),
}


def _pd_tol(g32, g64, name):
    spread = rel(g32[name + "_x"], g64[name + "_x"])
    return max(1e-4, 2 * spread)


@pytest.mark.parametrize("name", list(PD_CASES))
def test_pdhg_sampling(D, g32, g64, name):
    r = D.solve_pdhg_mlx(g32["pd_obs"], g32["psf_hr"], alpha=1e-3, sampling_factors=2.0,
                         spacing=(0.05, 0.0425, 0.0425), background=5.0, num_iter=30,
                         eval_interval=10, **PD_CASES[name])
    t = _pd_tol(g32, g64, name)
    assert r.iterations == int(g64[name + "_iters"])
    assert rel(r.restored, g64[name + "_x"]) < t
    np.testing.assert_allclose(r.tau_history, g64[name + "_tau"], rtol=max(t, 1e-4))
    np.testing.assert_allclose(r.sigma_history, g64[name + "_sigma"], rtol=max(t, 1e-4))
    np.testing.assert_allclose(r.loss_history, g64[name + "_loss"], rtol=1e-4)


def test_pdhg_convergence_bin_plain_operator(D, g32, g64):
    r = D.solve_pdhg_mlx(g32["pd_obs"], g32["psf_hr"], alpha=5.0, sampling_factors=2.0,
                         background=5.0, num_iter=60, tol=5e-2, min_iter=3, patience=2)
    assert r.iterations == int(g64["pd_conv_iters"])
    assert r.converged == bool(g64["pd_conv_converged"])
    assert rel(r.restored, g64["pd_conv_x"]) < 1e-4
    r = D.solve_pdhg_mlx(g32["pd_obs"], g32["psf_hr"], alpha=1e-3, bin_factors=2,
                         background=5.0, num_iter=15)
    assert rel(r.restored, g64["pd_bin_x"]) < 1e-4
    r = D.solve_pdhg_mlx(g32["rl_obs"], g32["psf16"], alpha=1e-3, background=10.0, num_iter=15,
                         spacing=(0.1, 0.085, 0.085))
    assert rel(r.restored, g64["pd_plain_x"]) < 1e-4
    np.testing.assert_allclose(r.loss_history, g64["pd_plain_loss"], rtol=1e-4)
    op = D.LinearFFTConvolver(g32["psf16"], (16, 32, 32))
    seen = []
    r = D.solve_pdhg_with_operator(g32["rl_obs"], op, alpha=1e-3, regularization="hessian",
                                   background=10.0, num_iter=15,
                                   callback=lambda k, x, loss: seen.append(loss))
    assert rel(r.restored, g64["pdo_x"]) < 1e-4
    np.testing.assert_allclose(r.tau_history, g64["pdo_tau"], rtol=1e-4)
    np.testing.assert_allclose(r.loss_history, g64["pdo_loss"], rtol=1e-4)
    assert len(seen) == 15


@pytest.mark.parametrize("shape,fft", [((64, 128, 128), (128, 256, 256)),
                                       ((128, 256, 256), (256, 512, 512)),
                                       ((20, 60, 40), (64, 128, 128)),
                                       ((30, 100, 90), (64, 256, 256)),
                                       ((8, 24, 500), (16, 64, 1024))])
def test_column_pass_variants_agree(D, monkeypatch, shape, fft):
    # The pipelined column kernel (R x R Stockham, half-zero split for 128 /
    # 512), the one-tile TMA kernel (DECON_NO_PIPE) and the plain-load kernel
    # (DECON_NO_TMA) compute the same transforms with different factorings;
    # so does the fused Y / axial pass (opt-in, DECON_YZ=1);
    # DECON_PIPE_LEAN selects the two-CTA axial kernel (twiddles in shared
    # memory, one ring slot) or the one-CTA kernel (same arithmetic).
    rng = np.random.default_rng(11)
    kshape = tuple(f - n + 1 for n, f in zip(shape, fft))
    k = rng.random(kshape).astype(np.float32)
    x = rng.random(shape).astype(np.float32)
    outs = []
    # DECON_YZ=1 selects the fused Y / axial pass where the canvas allows it
    # (tests/test_gpu_yz.py); the others choose among the separate passes
    keys = ("DECON_NO_PIPE", "DECON_NO_TMA", "DECON_PIPE_LEAN", "DECON_YZ")
    for env in ({}, {"DECON_YZ": "1"}, {"DECON_NO_PIPE": "1"}, {"DECON_NO_TMA": "1"},
                {"DECON_PIPE_LEAN": "0"}, {"DECON_PIPE_LEAN": "1"}):
        for key in keys:
            monkeypatch.delenv(key, raising=False)
        for key, val in env.items():
            monkeypatch.setenv(key, val)
        c = D.LinearFFTConvolver(k, shape, fft_shape=fft)
        outs.append((cpu(c.forward(x)), cpu(c.adjoint(x))))
    for key in keys:
        monkeypatch.delenv(key, raising=False)
    for f, a in outs[1:]:
        assert rel(f, outs[0][0]) < 1e-6
        assert rel(a, outs[0][1]) < 1e-6
    from deconlib_b200 import _lib
    _lib.call("decon_device_status", _lib.stream_ptr())


@pytest.mark.parametrize("norm", ["L1", "L1_2"])
def test_pdhg_fused_hessian_matches_operator_path(D, g32, norm):
    # The fused Hessian kernels evaluate the same float32 stencils as
    # Hessian3D.forward / adjoint; only the FP64 summation order of
    # ||L dx||^2 differs, so the trajectories agree to rounding.
    from deconlib_b200.deconvolution.pdhg import (HessianRegularizer, PDHGRunner,
                                                   _compute_spacing_ratio)
    from deconlib_b200.deconvolution._device import to_device

    data = to_device(g32["pd_obs"])
    conv = D.LinearFFTConvolver(g32["psf_hr"], (16, 32, 32))
    A = D.compose(D.FractionalAreaDownsample(2.0), conv)
    reg = HessianRegularizer(3, _compute_spacing_ratio((0.05, 0.0425, 0.0425), 3), norm)
    out = []
    for fused in (True, False):
        x0 = D.prox_nonneg(A.adjoint(data))
        run = PDHGRunner(data, A, reg, x0, 1e-3, "poisson", 30, 5.0, 0.99, 0.5, 10, 1e-5, 20, 5,
                         fused=fused)
        assert run.fused == fused
        out.append(run.run().result())
    assert rel(out[0][0], cpu(out[1][0])) < 1e-6
    np.testing.assert_allclose(out[0][3], out[1][3], rtol=1e-6)
    np.testing.assert_allclose(out[0][5], out[1][5], rtol=1e-6)


def test_kernel_shared_memory_opt_in_never_shrinks(D):
    # The runtime-radix X-pass kernel serves every non-power-of-two length with
    # a dynamic shared-memory size that depends on the length: a plan that
    # needs less (Fx = 400, 51 KB) used after one that needs more (Fx = 480,
    # 61 KB) must not lower the kernel's opt-in under the larger plan.
    rng = np.random.default_rng(4)
    k = rng.random((3, 5, 100)).astype(np.float32)
    x = rng.random((4, 8, 200)).astype(np.float32)
    big = D.LinearFFTConvolver(k, (4, 8, 200), fft_shape=(8, 16, 480))
    small = D.LinearFFTConvolver(k, (4, 8, 200), fft_shape=(8, 16, 400))
    a = cpu(big.forward(x))
    b = cpu(small.forward(x))
    c = cpu(big.forward(x))
    assert rel(b, a) < 1e-5
    np.testing.assert_array_equal(a, c)


@pytest.mark.parametrize("fx", [1024, 2048])
def test_long_x_axis_matches_fp64_fft(D, fx):
    # X passes of packed length 512 and 1024 (compile-time lines per CTA)
    rng = np.random.default_rng(12)
    n, k = (6, 20, fx // 2), (3, 5, fx // 4)
    x = rng.random(n)
    ker = rng.random(k)
    f = (8, 24, fx)
    ref_f = np.fft.irfftn(np.fft.rfftn(x, f) * np.fft.rfftn(
        np.asarray(D.pad_corner_origin_kernel(ker / ker.sum(), f)), f), f)[:n[0], :n[1], :n[2]]
    c = D.LinearFFTConvolver(ker.astype(np.float32), n, fft_shape=f)
    got = cpu(c.forward(x.astype(np.float32)))
    assert rel(got, ref_f) < 2e-6


def test_axial_pass_bit_identical_under_concurrent_streams(D):
    # Convolutions whose axial pass runs the two-CTA pipelined kernel (Fz =
    # 256), queued on four streams at once so that their CTAs share SMs, must
    # give exactly the single-stream result: the kernel's TMA refill of its
    # OTF buffer is ordered after every thread's reads by a proxy fence.
    rng = np.random.default_rng(21)
    shape = (128, 160, 96)
    psf = rng.random(shape).astype(np.float32)
    xs = [torch.from_numpy(rng.random(shape, dtype=np.float32)).cuda() for _ in range(4)]
    convs = [D.LinearFFTConvolver(psf, shape) for _ in range(4)]
    assert convs[0].fft_shape[0] == 256
    ref = [(c.forward(x), c.adjoint(x)) for c, x in zip(convs, xs)]
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream() for _ in range(4)]
    for _ in range(6):
        outs = []
        for st, c, x in zip(streams, convs, xs):
            st.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(st):
                outs.append([(c.forward(x), c.adjoint(x)) for _ in range(3)])
        torch.cuda.synchronize()
        for (f0, a0), reps in zip(ref, outs):
            for f, a in reps:
                assert torch.equal(f, f0) and torch.equal(a, a0)


@pytest.mark.parametrize("shape", [(16, 32, 32), (9, 15, 21), (20, 30), (48,)])
def test_circular_fft_convolver_vs_fp64_oracle(D, shape):
    # FFTConvolver: circular convolution by the resident OTF of the whole
    # kernel (deconlib/deconvolution/linops_mlx.py:384-432): OTF, norm,
    # forward and adjoint (conj OTF) against the FP64 oracle.
    from oracle import ops

    rng = np.random.default_rng(len(shape) * 100 + shape[-1])
    k = (rng.random(shape, dtype=np.float32) ** 3).astype(np.float32)
    x = rng.random(shape, dtype=np.float32)
    c = D.FFTConvolver(k)
    o = ops.FFTConvolver(k, dtype=np.float64)
    assert c.in_shape == c.out_shape == tuple(shape)
    assert rel(c.forward(x), o.forward(x.astype(np.float64))) < 1e-6
    assert rel(c.adjoint(x), o.adjoint(x.astype(np.float64))) < 1e-6
    assert rel(c(x), o.forward(x.astype(np.float64))) < 1e-6
    def crel(a, b):
        a = a.detach().cpu().numpy().astype(np.complex128)
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    assert crel(c.otf, o.otf) < 1e-6
    assert crel(c.otf_conj, np.conj(o.otf)) < 1e-6
    assert abs(c.operator_norm_sq - o.operator_norm_sq) <= 1e-6 * o.operator_norm_sq
    cu = D.FFTConvolver(k, normalize=False)
    ou = ops.FFTConvolver(k, normalize=False, dtype=np.float64)
    assert rel(cu.forward(x), ou.forward(x.astype(np.float64))) < 1e-6


def test_as_numpy_op_pairs(D, g32, g64):
    # as_numpy_op (deconlib/deconvolution/composition.py:140-159): NumPy in,
    # NumPy out in native shape, for one of this package's compositions and
    # for a pure-NumPy operator (tried with the array first, as the reference).
    c = D.LinearFFTConvolver(g32["psf16"], (16, 32, 32))
    op = D.compose(D.Crop((16, 32, 32), (12, 26, 28), start=(2, 3, 2)), c)
    R, Rt = D.as_numpy_op(op)
    x = g32["conv_x"]
    fx = R(x)
    assert isinstance(fx, np.ndarray) and fx.shape == (12, 26, 28) and fx.dtype == np.float32
    np.testing.assert_array_equal(fx, cpu(op.forward(x)))
    y = np.random.default_rng(2).random((12, 26, 28), dtype=np.float32)
    aty = Rt(y)
    assert isinstance(aty, np.ndarray) and aty.shape == (16, 32, 32)
    np.testing.assert_array_equal(aty, cpu(op.adjoint(y)))
    lhs = float(np.sum(fx.astype(np.float64) * y))
    rhs = float(np.sum(x.astype(np.float64) * aty))
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
    R2, Rt2 = D.as_numpy_op(c)
    assert rel(R2(x), g64["conv_fwd"]) < 1e-6

    class NumpyScale:
        def forward(self, v):
            assert isinstance(v, np.ndarray)
            return 2.0 * v

        def adjoint(self, v):
            assert isinstance(v, np.ndarray)
            return 2.0 * v

    Rn, Rtn = D.as_numpy_op(NumpyScale())
    np.testing.assert_array_equal(Rn(x), 2.0 * x)
    np.testing.assert_array_equal(Rtn(x), 2.0 * x)
