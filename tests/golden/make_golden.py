"""Generate golden fixtures by running deconlib's own source on the CPU.

Run from the repository root, in the container that holds the reference:

    python tests/golden/make_golden.py --reference PATH

The reference imports ``mlx.core``; ``tests/golden/mlx_standin`` supplies a
NumPy stand-in for the names it calls.  The script runs itself twice in
subprocesses, once in float32 and once with ``DECON_STANDIN_FP64=1``, and
writes ``tests/golden/golden_fp32.npz`` and ``golden_fp64.npz``; a third
subprocess runs the reference's NumPy ``pupil_to_psf`` into
``golden_psf.npz``.  The NLCG fixtures go to ``golden_nlcg_fp32.npz`` and
``golden_nlcg_fp64.npz``.  The
fixtures are small (volumes of at most 16x32x32) so the CPU oracle replays
them in seconds.  Nothing on the GPU side reads the reference at run time;
the fixtures are what travels.
"""

import argparse
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
STANDIN = os.path.join(HERE, "mlx_standin")


def _psf(shape, dz, dxy, na=1.4, ni=1.515, ns=1.334, wl=0.525, aberr=False):
    from deconlib.psf import Optics, make_geometry, make_pupil, pupil_to_psf
    from deconlib.utils import fft_coords

    optics = Optics(wavelength=wl, na=na, ni=ni, ns=ns)
    geom = make_geometry(shape[1:], dxy, optics)
    pupil = make_pupil(geom)
    if aberr:
        from deconlib.psf.aberrations import (IndexMismatch, ZernikeAberration, ZernikeMode,
                                             apply_aberrations)

        pupil = apply_aberrations(
            pupil, geom, optics,
            [IndexMismatch(depth=10.0),
             ZernikeAberration({ZernikeMode.SPHERICAL: 0.5, ZernikeMode.COMA_X: -0.2})],
        )
    z = fft_coords(shape[0], dz)
    return pupil_to_psf(pupil, geom, z).astype(np.float32)


def _beads(shape, n, seed):
    rng = np.random.default_rng(seed)
    t = np.zeros(shape, np.float64)
    idx = tuple(rng.integers(0, s, n) for s in shape)
    t[idx] += rng.uniform(0.5, 1.0, n)
    return t


def _run(out_path):
    import mlx.core as mx
    from deconlib.deconvolution import (
        Crop, FractionalAreaDownsample, FractionalAreaUpsample, Gradient3D, Hessian3D,
        LinearFFTConvolver, Pad, compose, richardson_lucy_with_operator,
        solve_pdhg_mlx, solve_pdhg_with_operator,
    )
    from deconlib.deconvolution.pdhg_mlx import (
        prox_l1_2_dual, prox_l1_dual, prox_poisson_dual, prox_gaussian_dual,
    )
    from deconlib.deconvolution.linops_mlx import fast_padded_shape

    g = {}
    rng = np.random.default_rng(1234)

    def arr(shape):
        return mx.array(rng.random(shape, dtype=np.float32))

    # --- FFT sizing -------------------------------------------------------
    sizes = [1, 2, 7, 11, 13, 17, 31, 97, 127, 255, 257, 511, 847, 1000, 1021]
    from deconlib.deconvolution.linops_mlx import _next_smooth_number
    g["smooth_in"] = np.array(sizes)
    g["smooth_out"] = np.array([_next_smooth_number(s) for s in sizes])
    g["fps_a"] = np.array(fast_padded_shape((101, 589, 549), (101, 256, 256)))
    g["fps_b"] = np.array(fast_padded_shape((101, 589, 549), (101, 256, 256), min_pad=(0, None, None)))
    g["fps_c"] = np.array(fast_padded_shape((34, 311, 311), (101, 160, 160), min_pad=(0, None, None)))

    # --- Pad / Crop -------------------------------------------------------
    x = arr((9, 10, 11))
    g["pad_x"] = np.array(x)
    g["pad_fwd"] = np.array(Pad(((1, 2), (0, 3), (4, 0))).forward(x))
    c = Crop((9, 10, 11), (5, 6, 7))
    g["crop_fwd"] = np.array(c.forward(x))
    y = arr((5, 6, 7))
    g["crop_y"] = np.array(y)
    g["crop_adj"] = np.array(c.adjoint(y))
    c2 = Crop((9, 10, 11), (5, 6, 7), start=(4, 0, 3))
    g["crop2_fwd"] = np.array(c2.forward(x))
    g["crop2_adj"] = np.array(c2.adjoint(y))

    # --- Fractional-area resampling --------------------------------------
    xr = arr((12, 20, 18))
    g["rs_x"] = np.array(xr)
    d2 = FractionalAreaDownsample(2.0, in_shape=(12, 20, 18))
    g["down2_fwd"] = np.array(d2.forward(xr))
    yr = arr((6, 10, 9))
    g["rs_y"] = np.array(yr)
    g["down2_adj"] = np.array(d2.adjoint(yr))
    d15 = FractionalAreaDownsample((1.5, 1.25, 2.5), in_shape=(12, 20, 18))
    g["down15_fwd"] = np.array(d15.forward(xr))
    g["down15_shape"] = np.array(d15.out_shape)
    y15 = arr(d15.out_shape)
    g["down15_y"] = np.array(y15)
    g["down15_adj"] = np.array(d15.adjoint(y15))
    dnp = FractionalAreaDownsample(2.0)  # no in_shape: shape-agnostic path
    g["down2np_fwd"] = np.array(dnp.forward(xr))
    up = FractionalAreaUpsample(2.0)
    g["up2_fwd"] = np.array(up.forward(yr))
    g["up2_adj"] = np.array(up.adjoint(xr))
    up3 = FractionalAreaUpsample((1.5, 2.0, 3.0))
    g["up3_fwd"] = np.array(up3.forward(yr))
    g["up3_shape"] = np.array(up3.forward(yr).shape)
    g["up3_adj"] = np.array(up3.adjoint(mx.array(rng.random(g["up3_shape"], dtype=np.float32))))
    # 2-D and 1-D forms
    x2 = arr((20, 30))
    g["rs2d_x"] = np.array(x2)
    g["down2d_fwd"] = np.array(FractionalAreaDownsample(3.0).forward(x2))
    x1 = arr((25,))
    g["rs1d_x"] = np.array(x1)
    g["down1d_fwd"] = np.array(FractionalAreaDownsample(2.5).forward(x1))

    # --- Linear FFT convolution ------------------------------------------
    psf = _psf((16, 32, 32), 0.1, 0.085)
    g["psf16"] = psf
    xc = arr((16, 32, 32))
    g["conv_x"] = np.array(xc)
    conv = LinearFFTConvolver(psf, (16, 32, 32))
    g["conv_fft_shape"] = np.array(conv.fft_shape)
    g["conv_norm"] = np.array(conv.operator_norm_sq)
    g["conv_fwd"] = np.array(conv.forward(xc))
    g["conv_adj"] = np.array(conv.adjoint(xc))
    # odd sizes and a kernel smaller than the signal
    k_odd = rng.random((5, 7, 9)).astype(np.float32)
    g["kodd"] = k_odd
    xo = arr((9, 11, 13))
    g["convodd_x"] = np.array(xo)
    co = LinearFFTConvolver(k_odd, (9, 11, 13))
    g["convodd_fft_shape"] = np.array(co.fft_shape)
    g["convodd_fwd"] = np.array(co.forward(xo))
    g["convodd_adj"] = np.array(co.adjoint(xo))
    g["convodd_norm"] = np.array(co.operator_norm_sq)
    # explicit fft_shape with an odd canvas and normalize=False
    cx = LinearFFTConvolver(k_odd, (9, 11, 13), normalize=False, fft_shape=(15, 18, 25))
    g["convx_fwd"] = np.array(cx.forward(xo))
    g["convx_adj"] = np.array(cx.adjoint(xo))
    # 2-D
    k2 = rng.random((7, 9)).astype(np.float32)
    g["k2d"] = k2
    x2c = arr((20, 30))
    g["conv2d_x"] = np.array(x2c)
    c2d = LinearFFTConvolver(k2, (20, 30))
    g["conv2d_fwd"] = np.array(c2d.forward(x2c))
    g["conv2d_adj"] = np.array(c2d.adjoint(x2c))

    # --- Hessian / gradient ----------------------------------------------
    xh = arr((8, 10, 12))
    g["hess_x"] = np.array(xh)
    h = Hessian3D(r=0.7)
    g["hess_fwd"] = np.array(h.forward(xh))
    yh = mx.array(rng.standard_normal((6, 8, 10, 12)).astype(np.float32))
    g["hess_y"] = np.array(yh)
    g["hess_adj"] = np.array(h.adjoint(yh))
    gr = Gradient3D(r=0.7)
    g["grad_fwd"] = np.array(gr.forward(xh))
    g["grad_adj"] = np.array(gr.adjoint(yh[:3]))

    # --- Proximal maps ----------------------------------------------------
    yp = mx.array(rng.standard_normal((7, 9)).astype(np.float32))
    dp = mx.array((rng.poisson(3.0, (7, 9)) * (rng.random((7, 9)) > 0.3)).astype(np.float32))
    g["prox_y"], g["prox_d"] = np.array(yp), np.array(dp)
    g["prox_poisson"] = np.array(prox_poisson_dual(yp, 0.3, dp, 2.0))
    g["prox_gauss"] = np.array(prox_gaussian_dual(yp, 0.3, dp, 2.0))
    g["prox_l1"] = np.array(prox_l1_dual(yp, 0.5))
    y3 = mx.array(rng.standard_normal((6, 4, 5)).astype(np.float32))
    g["prox_l12_y"] = np.array(y3)
    g["prox_l12"] = np.array(prox_l1_2_dual(y3, 0.5))

    # --- Richardson-Lucy ---------------------------------------------------
    truth = _beads((16, 32, 32), 40, seed=5)
    blur = np.array(LinearFFTConvolver(psf, (16, 32, 32)).forward(mx.array(truth)))
    blur = np.asarray(blur, np.float64)
    obs = np.random.default_rng(6).poisson(blur / blur.max() * 500.0 + 10.0).astype(np.float32)
    g["rl_obs"] = obs
    r = richardson_lucy_with_operator(obs, LinearFFTConvolver(psf, (16, 32, 32)),
                                      num_iter=12, background=10.0, eval_interval=5)
    g["rl_x"] = np.array(r.restored)
    g["rl_pred"] = np.array(r.pred)
    g["rl_loss"] = np.array(r.loss_history)
    g["rl_iters"] = np.array(r.iterations)
    # composed operator with a crop (the reference's padded-domain use)
    opc = compose(Crop((16, 32, 32), (12, 26, 28), start=(2, 3, 2)), LinearFFTConvolver(psf, (16, 32, 32)))
    obs_c = obs[2:14, 3:29, 2:30].copy()
    g["rlc_obs"] = obs_c
    rc = richardson_lucy_with_operator(obs_c, opc, num_iter=8, background=10.0, eval_interval=3)
    g["rlc_x"] = np.array(rc.restored)
    g["rlc_pred"] = np.array(rc.pred)
    g["rlc_loss"] = np.array(rc.loss_history)

    # --- PDHG: sampling_factors=2 (the super-resolved Hessian case) -----------
    psf_hr = _psf((16, 32, 32), 0.05, 0.0425, aberr=True)
    g["psf_hr"] = psf_hr
    truth_hr = _beads((16, 32, 32), 60, seed=7)
    fwd = compose(FractionalAreaDownsample(2.0, in_shape=(16, 32, 32)), LinearFFTConvolver(psf_hr, (16, 32, 32)))
    b = np.asarray(np.array(fwd.forward(mx.array(truth_hr))), np.float64)
    obs_p = np.random.default_rng(8).poisson(b / b.max() * 500.0 + 5.0).astype(np.float32)
    g["pd_obs"] = obs_p
    cases = {
        "pd_h_l1": dict(regularization="hessian", norm="L1"),
        "pd_h_l12": dict(regularization="hessian", norm="L1_2"),
        "pd_g_l1": dict(regularization="gradient", norm="L1"),
        "pd_i_l1": dict(regularization="identity", norm="L1"),
        "pd_h_gauss": dict(regularization="hessian", norm="L1", loss_type="gaussian"),
    }
    for name, kw in cases.items():
        res = solve_pdhg_mlx(mx.array(obs_p), psf_hr, alpha=1e-3, sampling_factors=2.0,
                             spacing=(0.05, 0.0425, 0.0425), background=5.0, num_iter=30,
                             eval_interval=10, **kw)
        g[name + "_x"] = np.array(res.restored)
        g[name + "_tau"] = np.array(res.tau_history)
        g[name + "_sigma"] = np.array(res.sigma_history)
        g[name + "_loss"] = np.array(res.loss_history)
        g[name + "_iters"] = np.array(res.iterations)
    # early stop by convergence (tight tol is met quickly with a large alpha)
    res = solve_pdhg_mlx(mx.array(obs_p), psf_hr, alpha=5.0, sampling_factors=2.0,
                         background=5.0, num_iter=60, tol=5e-2, min_iter=3, patience=2)
    g["pd_conv_x"] = np.array(res.restored)
    g["pd_conv_iters"] = np.array(res.iterations)
    g["pd_conv_converged"] = np.array(res.converged)
    g["pd_conv_tau"] = np.array(res.tau_history)
    # bin_factors and the plain PSF model
    res = solve_pdhg_mlx(mx.array(obs_p), psf_hr, alpha=1e-3, bin_factors=2, background=5.0,
                         num_iter=15)
    g["pd_bin_x"] = np.array(res.restored)
    g["pd_bin_tau"] = np.array(res.tau_history)
    res = solve_pdhg_mlx(mx.array(obs), psf, alpha=1e-3, background=10.0, num_iter=15,
                         spacing=(0.1, 0.085, 0.085))
    g["pd_plain_x"] = np.array(res.restored)
    g["pd_plain_tau"] = np.array(res.tau_history)
    g["pd_plain_loss"] = np.array(res.loss_history)
    # solve_pdhg_with_operator on a same-shape composed operator
    op = LinearFFTConvolver(psf, (16, 32, 32))
    losses = []
    res = solve_pdhg_with_operator(mx.array(obs), op, alpha=1e-3, regularization="hessian",
                                   background=10.0, num_iter=15,
                                   callback=lambda k, x, loss: losses.append(loss))
    g["pdo_x"] = np.array(res.restored)
    g["pdo_tau"] = np.array(res.tau_history)
    g["pdo_sigma"] = np.array(res.sigma_history)
    g["pdo_loss"] = np.array(res.loss_history)

    # --- tiling geometry, shapes, canonical forward model -----------------
    from deconlib.deconvolution.forward_model import make_forward_model
    from deconlib.deconvolution.shapes import compute_padded_shape, get_valid_slices
    from deconlib.deconvolution.tile_processing import optimal_tile_size, plan_tiles

    def enc(sl):
        return [[x.start, x.stop] for x in sl]

    tile_cases = [((64, 300, 300), 2.0, 16, 128, 48), ((40, 257, 190), 1.0, 8, 64, 48),
                  ((100, 512, 512), (1.0, 1.5, 1.5), 20, 200, 48), ((30, 90), 2.0, 4, 40, 48),
                  ((96, 700, 333), 1.0, 31, 256, 32)]
    for i, (shape, zoom, guard, ts, mz) in enumerate(tile_cases):
        plan = plan_tiles(shape, zoom, guard, ts, mz)
        g[f"tile{i}_tile_shape"] = np.array(plan.tile_shape)
        g[f"tile{i}_visible"] = np.array(plan.visible_shape)
        g[f"tile{i}_specs"] = np.array([[enc(t.read), enc(t.write), enc(t.crop)] for t in plan.tiles])
        g[f"tile{i}_index"] = np.array([t.index for t in plan.tiles])
    ots = []
    for N in (50, 64, 100, 257, 512, 1000, 1024, 2048):
        for guard in (0, 8, 31):
            for ts in (64, 128, 300, 512):
                try:
                    ots.append((N, guard, ts, optimal_tile_size(N, guard, ts)))
                except ValueError:
                    ots.append((N, guard, ts, -1))
    g["optimal_tile_size"] = np.array(ots)
    for i, (sig, ker) in enumerate([((100, 100), (31, 31)), ((64, 128, 128), (64, 128, 128)),
                                    ((17, 40, 33), (8, 9, 12))]):
        shp, pad = compute_padded_shape(sig, ker)
        g[f"pad{i}_shape"] = np.array(shp)
        g[f"pad{i}_pad"] = np.array(pad)
        g[f"pad{i}_valid"] = np.array(enc(get_valid_slices(shp, sig, pad)))
        g[f"pad{i}_valid_default"] = np.array(enc(get_valid_slices(shp, sig)))
    # forward model with zoom 2 on an even PSF (the registration fix)
    psf_fm = _psf((8, 16, 16), 0.2, 0.17)
    fm = make_forward_model(psf_fm, (6, 12, 10), 2.0)
    g["fm_psf"] = np.asarray(psf_fm, np.float32)
    g["fm_padded"] = np.array(fm.padded_shape)
    g["fm_valid"] = np.array(enc(fm.valid_slices))
    xin = rng.random(fm.padded_shape, dtype=np.float32)
    g["fm_x"] = xin
    g["fm_fwd"] = np.array(fm.op.forward(mx.array(xin)))
    yin = rng.random((6, 12, 10), dtype=np.float32)
    g["fm_y"] = yin
    g["fm_adj"] = np.array(fm.op.adjoint(mx.array(yin)))

    np.savez_compressed(out_path, **{k: np.asarray(v) for k, v in g.items()})
    print(f"wrote {out_path}: {len(g)} arrays")


def _run_psf(out_path):
    """pupil_to_psf cases: inputs (pupil, kz, z), the normalize flag and the
    reference's PSF.  pupil_to_psf is plain NumPy; the stand-in is on the path
    only because the package's imports name ``mlx.core``."""
    from deconlib.psf import Optics, make_geometry, make_pupil, pupil_to_psf
    from deconlib.psf.aberrations import (IndexMismatch, ZernikeAberration, ZernikeMode,
                                         apply_aberrations)
    from deconlib.utils import fft_coords

    cases = [  # (nz, ny, nx), dz, dxy, apodize, aberrated, normalize
        ((16, 64, 64), 0.1, 0.085, False, False, True),
        ((7, 36, 50), 0.2, 0.1, False, True, False),
        ((6, 120, 256), 0.15, 0.065, True, True, True),
        ((1, 48, 63), 0.1, 0.09, True, False, True),
    ]
    g = {}
    for i, (shape, dz, dxy, apod, aberr, norm) in enumerate(cases):
        optics = Optics(wavelength=0.525, na=1.4, ni=1.515, ns=1.334)
        geom = make_geometry(shape[1:], dxy, optics)
        pupil = make_pupil(geom, apodize=apod)
        if aberr:
            pupil = apply_aberrations(
                pupil, geom, optics,
                [IndexMismatch(depth=6.0),
                 ZernikeAberration({ZernikeMode.SPHERICAL: 0.4, ZernikeMode.COMA_X: 0.3})])
        z = fft_coords(shape[0], dz)
        psf = pupil_to_psf(pupil, geom, z, normalize=norm)
        g[f"psf{i}_pupil"] = np.asarray(pupil, np.complex128)
        g[f"psf{i}_kz"] = np.asarray(geom.kz, np.float64)
        g[f"psf{i}_z"] = np.asarray(z, np.float64)
        g[f"psf{i}_normalize"] = np.array(bool(norm))
        g[f"psf{i}_psf"] = np.asarray(psf, np.float32)
    g["psf_cases"] = np.array(len(cases))
    np.savez_compressed(out_path, **g)
    print(f"wrote {out_path}: {len(g)} arrays")


def _run_nlcg(out_path):
    """Nonlinear CG (nlcg_mlx.py): full solves on plain, regularised and
    composed operators, and the helper functions at a fixed point."""
    import mlx.core as mx
    from deconlib.deconvolution import (
        Crop, FractionalAreaDownsample, Gradient3D, Hessian3D, LinearFFTConvolver, compose,
    )
    from deconlib.deconvolution.nlcg_mlx import (
        i_divergence_between, nlcg_gradient, nlcg_hessian_quadform, nlcg_objective,
        nlcg_step_length, nlcg_with_operator,
    )

    g = {}
    shape = (16, 32, 32)
    psf = _psf(shape, 0.1, 0.085)
    g["psf"] = psf
    truth = _beads(shape, 40, seed=5)
    blur = np.asarray(np.array(LinearFFTConvolver(psf, shape).forward(mx.array(truth))), np.float64)
    obs = np.random.default_rng(6).poisson(blur / blur.max() * 500.0 + 10.0).astype(np.float32)
    g["obs"] = obs

    def rec(name, res):
        g[name + "_x"] = np.array(res.restored)
        g[name + "_pred"] = np.array(res.pred)
        g[name + "_loss"] = np.array(res.loss_history)
        g[name + "_iters"] = np.array(res.iterations)
        g[name + "_converged"] = np.array(res.converged)

    op = LinearFFTConvolver(psf, shape)
    rec("plain", nlcg_with_operator(obs, op, num_iter=15, background=10.0, eval_interval=4,
                                    min_iter=100))
    # discrepancy-principle stop (a loose slack makes it trigger early)
    rec("stop", nlcg_with_operator(obs, op, num_iter=40, background=10.0, slack=6.0, min_iter=3))
    rec("hess", nlcg_with_operator(obs, op, num_iter=12, background=10.0, regularizer=Hessian3D(),
                                   reg_weight=1e-3, tol=1e-4, min_iter=5, eval_interval=3))
    # Eq. 17 stop: relative change of successive iterates under a loose tol
    rec("tol", nlcg_with_operator(obs, op, num_iter=40, background=10.0, regularizer=Hessian3D(),
                                  reg_weight=1e-3, tol=3e-2, min_iter=5))
    rec("grad", nlcg_with_operator(obs, op, num_iter=10, background=10.0,
                                   regularizer=Gradient3D(r=0.85), reg_weight=2e-3,
                                   restart_interval=4, min_iter=100, eval_interval=2))
    init = np.full(shape, float(obs.mean()), np.float32)
    rec("init", nlcg_with_operator(obs, op, num_iter=6, background=10.0, init=init, min_iter=100,
                                   newton_iters=2))
    # composed operators: a crop (padded domain) and a 2x fractional-area downsample
    opc = compose(Crop(shape, (12, 26, 28), start=(2, 3, 2)), LinearFFTConvolver(psf, shape))
    obs_c = obs[2:14, 3:29, 2:30].copy()
    g["obs_c"] = obs_c
    rec("crop", nlcg_with_operator(obs_c, opc, num_iter=8, background=10.0, min_iter=100))
    fwd = compose(FractionalAreaDownsample(2.0, in_shape=shape), LinearFFTConvolver(psf, shape))
    b = np.asarray(np.array(fwd.forward(mx.array(_beads(shape, 60, seed=7)))), np.float64)
    obs_d = np.random.default_rng(8).poisson(b / b.max() * 500.0 + 5.0).astype(np.float32)
    g["obs_d"] = obs_d
    rec("down", nlcg_with_operator(obs_d, fwd, num_iter=8, background=5.0, min_iter=100,
                                   regularizer=Hessian3D(r=0.5), reg_weight=1e-3))

    # helpers at a fixed point s, direction d
    rng = np.random.default_rng(9)
    s = (rng.random(shape, dtype=np.float32) * 20 + 1).astype(np.float32)
    d = (rng.standard_normal(shape).astype(np.float32) * 0.5).astype(np.float32)
    g["h_s"], g["h_d"] = s, d
    for tag, reg, beta in (("n", None, 0.0), ("r", Hessian3D(), 1e-3)):
        g[f"h{tag}_obj"] = np.array(nlcg_objective(mx.array(s), op, mx.array(obs), 10.0, reg, beta))
        grad, aux = nlcg_gradient(mx.array(s), op, mx.array(obs), 10.0, reg, beta)
        g[f"h{tag}_grad"] = np.array(grad)
        g[f"h{tag}_quad"] = np.array(nlcg_hessian_quadform(mx.array(s), mx.array(d), op, mx.array(obs),
                                                           10.0, reg, beta, aux=aux))
        f = mx.array(s) * mx.array(s)
        lam, m_lam = nlcg_step_length(mx.array(s), mx.array(d), f, aux[0], op, mx.array(obs), 10.0,
                                      reg, beta)
        g[f"h{tag}_lam"] = np.array(lam)
        g[f"h{tag}_mlam"] = np.array(m_lam)
    f1 = rng.random(shape, dtype=np.float32) + 0.1
    f2 = f1 * (1 + 0.1 * rng.standard_normal(shape).astype(np.float32))
    g["h_f1"], g["h_f2"] = f1, f2
    g["h_idiv"] = np.array(i_divergence_between(mx.array(f1), mx.array(f2)))

    np.savez_compressed(out_path, **{k: np.asarray(v) for k, v in g.items()})
    print(f"wrote {out_path}: {len(g)} arrays")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="root of the deconlib 0.4.0 source tree (read-only)")
    ap.add_argument("--worker", choices=["fp32", "fp64", "psf", "nlcg32", "nlcg64"], default=None)
    a = ap.parse_args()
    if a.worker == "psf":
        sys.path[:0] = [STANDIN, a.reference]
        _run_psf(os.path.join(HERE, "golden_psf.npz"))
        return
    if a.worker in ("nlcg32", "nlcg64"):
        sys.path[:0] = [STANDIN, a.reference]
        _run_nlcg(os.path.join(HERE, f"golden_nlcg_fp{a.worker[4:]}.npz"))
        return
    if a.worker:
        sys.path[:0] = [STANDIN, a.reference]
        _run(os.path.join(HERE, f"golden_{a.worker}.npz"))
        return
    subprocess.run([sys.executable, os.path.abspath(__file__), "--reference", a.reference,
                    "--worker", "psf"], check=True)
    for mode in ("fp32", "fp64"):
        env = dict(os.environ)
        env["DECON_STANDIN_FP64"] = "1" if mode == "fp64" else "0"
        for w in (mode, "nlcg" + mode[2:]):
            subprocess.run([sys.executable, os.path.abspath(__file__), "--reference", a.reference,
                            "--worker", w], check=True, env=env)


if __name__ == "__main__":
    main()
