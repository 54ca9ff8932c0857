"""Pin the CPU oracle against golden vectors made by the reference's own source.

The fixtures come from ``tests/golden/make_golden.py`` (deconlib 0.4.0 run
through a NumPy stand-in for ``mlx.core``), once in float32 and once in
float64.  The oracle replays every case in the same precision.  Operators must
agree to a few float32 ulps (float64: ~1e-12); solver trajectories to the
tolerances written beside each check.
"""

import os

import numpy as np
import pytest

from oracle import ops, solvers

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module", params=["fp32", "fp64"])
def gold(request):
    g = np.load(os.path.join(HERE, "golden", f"golden_{request.param}.npz"))
    dt = np.float32 if request.param == "fp32" else np.float64
    return g, dt


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def tol(dt, f32, f64=1e-11):
    return f32 if dt == np.float32 else f64


def test_fft_sizing(gold):
    g, _ = gold
    assert [ops.next_smooth_number(int(s)) for s in g["smooth_in"]] == list(g["smooth_out"])
    assert ops.fast_padded_shape((101, 589, 549), (101, 256, 256)) == tuple(g["fps_a"])
    assert ops.fast_padded_shape((101, 589, 549), (101, 256, 256), (0, None, None)) == tuple(g["fps_b"])
    assert ops.fast_padded_shape((34, 311, 311), (101, 160, 160), (0, None, None)) == tuple(g["fps_c"])


def test_pad_crop(gold):
    g, dt = gold
    x = g["pad_x"].astype(dt)
    np.testing.assert_array_equal(ops.Pad(((1, 2), (0, 3), (4, 0))).forward(x), g["pad_fwd"])
    c = ops.Crop((9, 10, 11), (5, 6, 7))
    np.testing.assert_array_equal(c.forward(x), g["crop_fwd"])
    np.testing.assert_array_equal(c.adjoint(g["crop_y"].astype(dt)), g["crop_adj"])
    c2 = ops.Crop((9, 10, 11), (5, 6, 7), start=(4, 0, 3))
    np.testing.assert_array_equal(c2.forward(x), g["crop2_fwd"])
    np.testing.assert_array_equal(c2.adjoint(g["crop_y"].astype(dt)), g["crop2_adj"])


def test_resampling(gold):
    g, dt = gold
    x, y = g["rs_x"].astype(dt), g["rs_y"].astype(dt)
    t = tol(dt, 2e-7, 1e-7)  # weights are float32 tables in both precisions
    d2 = ops.FractionalAreaDownsample(2.0, in_shape=(12, 20, 18), dtype=dt)
    assert rel(d2.forward(x), g["down2_fwd"]) < t
    assert rel(d2.adjoint(y), g["down2_adj"]) < t
    d15 = ops.FractionalAreaDownsample((1.5, 1.25, 2.5), in_shape=(12, 20, 18), dtype=dt)
    assert d15.out_shape == tuple(g["down15_shape"])
    assert rel(d15.forward(x), g["down15_fwd"]) < t
    assert rel(d15.adjoint(g["down15_y"].astype(dt)), g["down15_adj"]) < t
    assert rel(ops.FractionalAreaDownsample(2.0, dtype=dt).forward(x), g["down2np_fwd"]) < t
    up = ops.FractionalAreaUpsample(2.0, dtype=dt)
    assert rel(up.forward(y), g["up2_fwd"]) < t
    assert rel(up.adjoint(x), g["up2_adj"]) < t
    up3 = ops.FractionalAreaUpsample((1.5, 2.0, 3.0), dtype=dt)
    assert up3.forward(y).shape == tuple(g["up3_shape"])
    assert rel(up3.forward(y), g["up3_fwd"]) < t
    assert rel(ops.FractionalAreaDownsample(3.0, dtype=dt).forward(g["rs2d_x"].astype(dt)), g["down2d_fwd"]) < t
    assert rel(ops.FractionalAreaDownsample(2.5, dtype=dt).forward(g["rs1d_x"].astype(dt)), g["down1d_fwd"]) < t


def test_linear_fft_convolver(gold):
    g, dt = gold
    t = tol(dt, 1e-6)
    c = ops.LinearFFTConvolver(g["psf16"], (16, 32, 32), dtype=dt)
    assert c.fft_shape == tuple(g["conv_fft_shape"])
    assert abs(c.operator_norm_sq - float(g["conv_norm"])) < tol(dt, 1e-6)
    x = g["conv_x"].astype(dt)
    assert rel(c.forward(x), g["conv_fwd"]) < t
    assert rel(c.adjoint(x), g["conv_adj"]) < t
    co = ops.LinearFFTConvolver(g["kodd"], (9, 11, 13), dtype=dt)
    assert co.fft_shape == tuple(g["convodd_fft_shape"])
    xo = g["convodd_x"].astype(dt)
    assert rel(co.forward(xo), g["convodd_fwd"]) < t
    assert rel(co.adjoint(xo), g["convodd_adj"]) < t
    cx = ops.LinearFFTConvolver(g["kodd"], (9, 11, 13), normalize=False, fft_shape=(15, 18, 25), dtype=dt)
    assert rel(cx.forward(xo), g["convx_fwd"]) < t
    assert rel(cx.adjoint(xo), g["convx_adj"]) < t
    c2 = ops.LinearFFTConvolver(g["k2d"], (20, 30), dtype=dt)
    assert rel(c2.forward(g["conv2d_x"].astype(dt)), g["conv2d_fwd"]) < t
    assert rel(c2.adjoint(g["conv2d_x"].astype(dt)), g["conv2d_adj"]) < t


def test_hessian_gradient(gold):
    g, dt = gold
    t = tol(dt, 1e-6)
    x, y = g["hess_x"].astype(dt), g["hess_y"].astype(dt)
    h = ops.Hessian3D(0.7, dt)
    assert rel(h.forward(x), g["hess_fwd"]) < t
    assert rel(h.adjoint(y), g["hess_adj"]) < t
    gr = ops.Gradient3D(0.7, dt)
    assert rel(gr.forward(x), g["grad_fwd"]) < t
    assert rel(gr.adjoint(y[:3]), g["grad_adj"]) < t


def test_prox(gold):
    g, dt = gold
    y, d = g["prox_y"].astype(dt), g["prox_d"].astype(dt)
    t = tol(dt, 1e-6)
    assert rel(solvers.prox_poisson_dual(y, 0.3, d, 2.0), g["prox_poisson"]) < t
    assert rel(solvers.prox_gaussian_dual(y, 0.3, d, 2.0), g["prox_gauss"]) < t
    np.testing.assert_array_equal(solvers.prox_l1_dual(y, 0.5), g["prox_l1"])
    assert rel(solvers.prox_l1_2_dual(g["prox_l12_y"].astype(dt), 0.5), g["prox_l12"]) < t


def test_rl(gold):
    g, dt = gold
    c = ops.LinearFFTConvolver(g["psf16"], (16, 32, 32), dtype=dt)
    r = solvers.richardson_lucy_with_operator(g["rl_obs"], c, num_iter=12, background=10.0,
                                              eval_interval=5, dtype=dt)
    assert r["iterations"] == int(g["rl_iters"])
    assert rel(r["restored"], g["rl_x"]) < tol(dt, 2e-5, 1e-10)
    assert rel(r["pred"], g["rl_pred"]) < tol(dt, 2e-6, 1e-11)
    np.testing.assert_allclose(r["loss_history"], g["rl_loss"], rtol=tol(dt, 1e-4, 1e-10))
    op = ops.compose(ops.Crop((16, 32, 32), (12, 26, 28), start=(2, 3, 2)), c)
    rc = solvers.richardson_lucy_with_operator(g["rlc_obs"], op, num_iter=8, background=10.0,
                                               eval_interval=3, dtype=dt)
    assert rel(rc["restored"], g["rlc_x"]) < tol(dt, 2e-5, 1e-10)
    assert rel(rc["pred"], g["rlc_pred"]) < tol(dt, 2e-6, 1e-11)
    np.testing.assert_allclose(rc["loss_history"], g["rlc_loss"], rtol=tol(dt, 1e-4, 1e-10))


PD_CASES = {
    "pd_h_l1": dict(regularization="hessian", norm="L1"),
    "pd_h_l12": dict(regularization="hessian", norm="L1_2"),
    "pd_g_l1": dict(regularization="gradient", norm="L1"),
    "pd_i_l1": dict(regularization="identity", norm="L1"),
    "pd_h_gauss": dict(regularization="hessian", norm="L1", loss_type="gaussian"),
}


@pytest.mark.parametrize("name", list(PD_CASES))
def test_pdhg_sampling(gold, name):
    g, dt = gold
    r = solvers.solve_pdhg_mlx(g["pd_obs"], g["psf_hr"], alpha=1e-3, sampling_factors=2.0,
                               spacing=(0.05, 0.0425, 0.0425), background=5.0, num_iter=30,
                               eval_interval=10, dtype=dt, **PD_CASES[name])
    assert r["iterations"] == int(g[name + "_iters"])
    assert rel(r["restored"], g[name + "_x"]) < tol(dt, 1e-4, 1e-9)
    np.testing.assert_allclose(r["tau_history"], g[name + "_tau"], rtol=tol(dt, 1e-4, 1e-9))
    np.testing.assert_allclose(r["sigma_history"], g[name + "_sigma"], rtol=tol(dt, 1e-4, 1e-9))
    np.testing.assert_allclose(r["loss_history"], g[name + "_loss"], rtol=tol(dt, 1e-4, 1e-9))


def test_pdhg_convergence_bin_plain_operator(gold):
    g, dt = gold
    r = solvers.solve_pdhg_mlx(g["pd_obs"], g["psf_hr"], alpha=5.0, sampling_factors=2.0,
                               background=5.0, num_iter=60, tol=5e-2, min_iter=3, patience=2,
                               dtype=dt)
    assert r["iterations"] == int(g["pd_conv_iters"])
    assert r["converged"] == bool(g["pd_conv_converged"])
    assert rel(r["restored"], g["pd_conv_x"]) < tol(dt, 1e-4, 1e-9)
    np.testing.assert_allclose(r["tau_history"], g["pd_conv_tau"], rtol=tol(dt, 1e-4, 1e-9))
    r = solvers.solve_pdhg_mlx(g["pd_obs"], g["psf_hr"], alpha=1e-3, bin_factors=2,
                               background=5.0, num_iter=15, dtype=dt)
    assert rel(r["restored"], g["pd_bin_x"]) < tol(dt, 1e-4, 1e-9)
    np.testing.assert_allclose(r["tau_history"], g["pd_bin_tau"], rtol=tol(dt, 1e-4, 1e-9))
    r = solvers.solve_pdhg_mlx(g["rl_obs"], g["psf16"], alpha=1e-3, background=10.0,
                               num_iter=15, spacing=(0.1, 0.085, 0.085), dtype=dt)
    assert rel(r["restored"], g["pd_plain_x"]) < tol(dt, 1e-4, 1e-9)
    np.testing.assert_allclose(r["tau_history"], g["pd_plain_tau"], rtol=tol(dt, 1e-4, 1e-9))
    np.testing.assert_allclose(r["loss_history"], g["pd_plain_loss"], rtol=tol(dt, 1e-4, 1e-9))
    op = ops.LinearFFTConvolver(g["psf16"], (16, 32, 32), dtype=dt)
    seen = []
    r = solvers.solve_pdhg_with_operator(g["rl_obs"], op, alpha=1e-3, regularization="hessian",
                                         background=10.0, num_iter=15, dtype=dt,
                                         callback=lambda k, x, loss: seen.append(loss))
    assert rel(r["restored"], g["pdo_x"]) < tol(dt, 1e-4, 1e-9)
    np.testing.assert_allclose(r["tau_history"], g["pdo_tau"], rtol=tol(dt, 1e-4, 1e-9))
    np.testing.assert_allclose(r["sigma_history"], g["pdo_sigma"], rtol=tol(dt, 1e-4, 1e-9))
    np.testing.assert_allclose(r["loss_history"], g["pdo_loss"], rtol=tol(dt, 1e-4, 1e-9))
    assert len(seen) == 15


def test_pupil_to_psf():
    """oracle/psf.py against the reference's pupil_to_psf on four pupils
    (plain, aberrated, apodised; 7-smooth and power-of-two planes; with and
    without normalisation).  Fixtures are float32: agreement to ~3e-8."""
    from oracle import psf as P

    g = np.load(os.path.join(HERE, "golden", "golden_psf.npz"))
    for i in range(int(g["psf_cases"])):
        r = P.pupil_to_psf(g[f"psf{i}_pupil"], g[f"psf{i}_kz"], g[f"psf{i}_z"],
                           bool(g[f"psf{i}_normalize"]))
        assert rel(r, g[f"psf{i}_psf"]) < 1e-7, i


@pytest.fixture(scope="module", params=["fp32", "fp64"])
def nl_gold(request):
    g = np.load(os.path.join(HERE, "golden", f"golden_nlcg_{request.param}.npz"))
    dt = np.float32 if request.param == "fp32" else np.float64
    return g, dt


def _nl_ops(g, dt):
    shape = (16, 32, 32)
    conv = ops.LinearFFTConvolver(g["psf"], shape, dtype=dt)
    return dict(
        conv=conv,
        crop=ops.compose(ops.Crop(shape, (12, 26, 28), start=(2, 3, 2)), conv),
        down=ops.compose(ops.FractionalAreaDownsample(2.0, in_shape=shape, dtype=dt), conv),
    )


NL_CASES = {  # name: (observation key, operator, keyword arguments)
    "plain": ("obs", "conv", dict(num_iter=15, background=10.0, eval_interval=4, min_iter=100)),
    "stop": ("obs", "conv", dict(num_iter=40, background=10.0, slack=6.0, min_iter=3)),
    "hess": ("obs", "conv", dict(num_iter=12, background=10.0, reg="hess", reg_weight=1e-3, tol=1e-4,
                                 min_iter=5, eval_interval=3)),
    "tol": ("obs", "conv", dict(num_iter=40, background=10.0, reg="hess", reg_weight=1e-3, tol=3e-2,
                                min_iter=5)),
    "grad": ("obs", "conv", dict(num_iter=10, background=10.0, reg="grad", reg_weight=2e-3,
                                 restart_interval=4, min_iter=100, eval_interval=2)),
    "init": ("obs", "conv", dict(num_iter=6, background=10.0, init="mean", min_iter=100,
                                 newton_iters=2)),
    "crop": ("obs_c", "crop", dict(num_iter=8, background=10.0, min_iter=100)),
    "down": ("obs_d", "down", dict(num_iter=8, background=5.0, min_iter=100, reg="hess05",
                                   reg_weight=1e-3)),
}


def nl_kwargs(g, dt, kw):
    kw = dict(kw)
    reg = kw.pop("reg", None)
    if reg == "hess":
        kw["regularizer"] = ops.Hessian3D(1.0, dt)
    elif reg == "hess05":
        kw["regularizer"] = ops.Hessian3D(0.5, dt)
    elif reg == "grad":
        kw["regularizer"] = ops.Gradient3D(0.85, dt)
    if kw.get("init") == "mean":
        kw["init"] = np.full((16, 32, 32), float(g["obs"].mean()), np.float32)
    return kw


@pytest.mark.parametrize("name", list(NL_CASES))
def test_nlcg(nl_gold, name):
    """oracle/nlcg.py against the reference's nlcg_with_operator: the same
    iteration count, stop decision and loss history; iterates to float32
    round-off (the trajectory amplifies it over the iterations) or ~1e-9 in
    float64."""
    from oracle import nlcg

    g, dt = nl_gold
    obs_key, op_key, kw = NL_CASES[name]
    r = nlcg.nlcg_with_operator(g[obs_key], _nl_ops(g, dt)[op_key], dtype=dt, **nl_kwargs(g, dt, kw))
    assert r["iterations"] == int(g[name + "_iters"])
    assert r["converged"] == bool(g[name + "_converged"])
    assert rel(r["restored"], g[name + "_x"]) < tol(dt, 2e-4, 1e-9)
    assert rel(r["pred"], g[name + "_pred"]) < tol(dt, 2e-5, 1e-10)
    np.testing.assert_allclose(r["loss_history"], g[name + "_loss"], rtol=tol(dt, 1e-4, 1e-9))


def test_nlcg_helpers(nl_gold):
    from oracle import nlcg

    g, dt = nl_gold
    conv = _nl_ops(g, dt)["conv"]
    s, d, y = g["h_s"].astype(dt), g["h_d"].astype(dt), g["obs"].astype(dt)
    for tag, reg, beta in (("n", None, 0.0), ("r", ops.Hessian3D(1.0, dt), 1e-3)):
        assert nlcg.nlcg_objective(s, conv, y, 10.0, reg, beta, dtype=dt) == pytest.approx(
            float(g[f"h{tag}_obj"]), rel=tol(dt, 1e-6, 1e-12))
        grad, aux = nlcg.nlcg_gradient(s, conv, y, 10.0, reg, beta, dtype=dt)
        assert rel(grad, g[f"h{tag}_grad"]) < tol(dt, 1e-5, 1e-11)
        q = nlcg.nlcg_hessian_quadform(s, d, conv, y, 10.0, reg, beta, aux=aux, dtype=dt)
        assert q == pytest.approx(float(g[f"h{tag}_quad"]), rel=tol(dt, 1e-5, 1e-11))
        lam, m_lam = nlcg.nlcg_step_length(s, d, s * s, aux[0], conv, y, 10.0, reg, beta, dtype=dt)
        assert lam == pytest.approx(float(g[f"h{tag}_lam"]), rel=tol(dt, 1e-4, 1e-10))
        assert rel(m_lam, g[f"h{tag}_mlam"]) < tol(dt, 1e-6, 1e-12)
    v = nlcg.i_divergence_between(g["h_f1"].astype(dt), g["h_f2"].astype(dt))
    assert v == pytest.approx(float(g["h_idiv"]), rel=tol(dt, 1e-5, 1e-12))
