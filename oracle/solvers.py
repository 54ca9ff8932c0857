"""CPU oracle for the 3D deconvolution path: Richardson-Lucy and adaptive PDHG.

TEST INFRASTRUCTURE ONLY (the checker, never the product): only ``tests/``,
``__graft_entry__.smoke()`` and the CPU baseline leg of ``bench.py`` use it.

A NumPy restatement of deconlib 0.4.0's solvers:
  * ``richardson_lucy_with_operator``  -> deconvolution/rl_mlx.py:83-185
  * ``solve_pdhg_mlx``                 -> deconvolution/pdhg_mlx.py:507-920
  * ``solve_pdhg_with_operator``       -> deconvolution/pdhg_mlx.py:928-1242
  * proximal maps                      -> deconvolution/pdhg_mlx.py:115-233

``dtype=np.float32`` follows the reference's device precision, including the
float32 evaluation of the scalar step-size arithmetic (the reference does
``mx.sqrt(1.0 + theta) * tau`` on 0-d float32 device arrays and only then
converts to a Python float, pdhg_mlx.py:767-797, 851-853).  ``dtype=np.float64``
is the double-precision oracle.
"""

from __future__ import annotations

import math
from typing import Optional

import numpy as np

from . import ops


# ---------------------------------------------------------------------------
# Proximal maps (pdhg_mlx.py:115-233)
# ---------------------------------------------------------------------------


def prox_poisson_dual(y, sigma, data, background):
    """1 - z with z the positive root of z^2 - c z - sigma D = 0,
    c = 1 - y - sigma b; z = max(c, 1e-6) where D < 1e-6; z >= 1e-6
    (pdhg_mlx.py:115-166)."""
    t = y.dtype.type
    sigma = t(sigma)
    c = t(1.0) - y - sigma * t(background)
    d = np.maximum(data, t(0.0))
    disc = c * c + t(4.0) * sigma * d
    z = (t(2.0) * sigma * d) / (np.sqrt(disc) - c + t(1e-12))
    z = np.where(d < t(1e-6), np.maximum(c, t(1e-6)), z)
    z = np.maximum(z, t(1e-6))
    return t(1.0) - z


def prox_gaussian_dual(y, sigma, data, background):
    """(y - sigma (D - b)) / (1 + sigma) (pdhg_mlx.py:169-189)."""
    t = y.dtype.type
    return (y - t(sigma) * (data - t(background))) / (t(1.0) + t(sigma))


def prox_nonneg(x):
    """max(0, x) (pdhg_mlx.py:192-194)."""
    return np.maximum(x, x.dtype.type(0.0))


def prox_l1_dual(y, bound):
    """clip(y, -bound, bound) (pdhg_mlx.py:197-209)."""
    t = y.dtype.type
    return np.clip(y, t(-bound), t(bound))


def prox_l1_2_dual(y, bound):
    """y / max(sqrt(sum_c y^2 + 1e-12) / bound, 1) (pdhg_mlx.py:212-233)."""
    t = y.dtype.type
    n = np.sqrt(np.sum(y * y, axis=0, keepdims=True) + t(1e-12))
    return y / np.maximum(n / t(bound), t(1.0))


# ---------------------------------------------------------------------------
# Regularisers (pdhg_mlx.py:241-451)
# ---------------------------------------------------------------------------


class Regularizer:
    """identity / gradient / hessian operator L with its dual projection
    (pdhg_mlx.py:241-451, _create_regularizer :485-499)."""

    def __init__(self, kind, ndim, r, norm, dtype):
        self.kind, self.ndim, self.norm = kind, ndim, norm
        if kind == "identity":
            self.ncomp, self.operator_norm_sq = 1, 1.0
            self._f = lambda x: x[None]
            self._a = lambda y: y[0]
        elif kind in ("gradient", "hessian"):
            if ndim not in (1, 2, 3):
                raise ValueError(f"ndim must be 1, 2, or 3, got {ndim}")
            if kind == "gradient":
                op = {1: ops.Gradient1D(), 2: ops.Gradient2D(), 3: ops.Gradient3D(r, dtype)}[ndim]
                self.ncomp = ndim
            else:
                op = {1: ops.Hessian1D(), 2: ops.Hessian2D(dtype), 3: ops.Hessian3D(r, dtype)}[ndim]
                self.ncomp = {1: 1, 2: 3, 3: 6}[ndim]
            self.operator_norm_sq = op.operator_norm_sq
            if ndim == 1:
                self._f = lambda x: op.forward(x)[None]
                self._a = lambda y: op.adjoint(y[0])
            else:
                self._f, self._a = op.forward, op.adjoint
        else:
            raise ValueError(f"Unknown regularization: {kind}")

    def forward(self, x):
        return self._f(x)

    def adjoint(self, y):
        return self._a(y)

    def prox_dual(self, y, alpha):
        return prox_l1_dual(y, alpha) if self.norm == "L1" else prox_l1_2_dual(y, alpha)


def spacing_ratio(spacing, ndim):
    """r = mean(dy, dx) / dz for 3D, else 1 (pdhg_mlx.py:459-482)."""
    if spacing is None or ndim in (1, 2):
        return 1.0
    if len(spacing) != ndim:
        raise ValueError(f"spacing must have {ndim} elements, got {len(spacing)}")
    dz = spacing[0]
    lat = (spacing[1] + spacing[2]) / 2.0
    return lat / dz if dz > 0 else 1.0


# ---------------------------------------------------------------------------
# Richardson-Lucy (rl_mlx.py:58-185)
# ---------------------------------------------------------------------------


def poisson_i_divergence(observed, model, eps=1e-6):
    """mean(y log(max(y,eps)/max(m,eps)) - (y - max(m,eps))) (rl_mlx.py:58-80)."""
    t = observed.dtype.type
    ys = np.maximum(observed, t(eps))
    ms = np.maximum(model, t(eps))
    return float(np.mean(observed * np.log(ys / ms) - (observed - ms)))


def richardson_lucy_with_operator(observed, blur_op, num_iter=50, background=0.0,
                                  init=None, eval_interval=10, dtype=np.float32,
                                  callback=None):
    """Multiplicative RL with sensitivity A^T 1 and active-support mask
    (rl_mlx.py:83-185).  Returns a dict with the RLResult fields."""
    t = np.dtype(dtype).type
    y = np.asarray(observed).astype(dtype)
    eps = t(1e-10)
    bg = t(background)
    dmb = np.maximum(y - bg, t(1e-6))
    if init is None:
        x = np.maximum(blur_op.adjoint(dmb), t(1e-6))
    else:
        x = np.maximum(np.asarray(init).astype(dtype), t(1e-6))
    sens_raw = blur_op.adjoint(np.ones_like(y))
    floor = np.maximum(np.max(sens_raw) * t(1e-6), eps)
    active = sens_raw > floor
    sens = np.where(active, sens_raw, t(1.0))
    x = np.where(active, x, t(0.0))
    losses = []
    k = -1
    for k in range(num_iter):
        model = blur_op.forward(x) + bg
        ratio = y / np.maximum(model, eps)
        corr = np.where(active, blur_op.adjoint(ratio) / sens, t(0.0))
        x = np.maximum(x * corr, eps)
        if k % eval_interval == 0 or k == num_iter - 1:
            losses.append(poisson_i_divergence(y, blur_op.forward(x) + bg))
        if callback is not None and callback(k, x):
            break
    pred = blur_op.forward(x) + bg
    return dict(restored=x, pred=pred, iterations=k + 1, loss_history=losses,
                background=float(background), full_shape=tuple(x.shape),
                active=active, sensitivity=sens)


# ---------------------------------------------------------------------------
# Malitsky-Pock adaptive PDHG (pdhg_mlx.py:507-1242)
# ---------------------------------------------------------------------------


def _pdhg_loop(y, blur_op, reg, x, alpha, loss_type, num_iter, background, delta, eta,
               eval_interval, tol, min_iter, patience, dtype, generic, callback=None):
    """The shared iteration of both PDHG entry points (pdhg_mlx.py:717-900 and
    :1066-1221).  Scalars follow the reference: computed on 0-d device arrays
    (so in ``dtype``), then rounded to Python floats at the end of each
    iteration (:851-853)."""
    t = np.dtype(dtype).type
    bg = t(background)
    y1 = np.zeros(y.shape, dtype=dtype)
    y2 = np.zeros((reg.ncomp,) + tuple(x.shape), dtype=dtype)
    x_bar = x
    step_scale = 0.99 / (blur_op.operator_norm_sq + reg.operator_norm_sq) ** 0.5
    tau = sigma = step_scale
    theta = 1.0
    losses, taus, sigmas = [], [], []
    converged = False
    count = 0
    final_iter = num_iter
    prox = prox_poisson_dual if loss_type == "poisson" else prox_gaussian_dual
    for k in range(num_iter):
        s = t(sigma)
        y1n = prox(y1 + s * blur_op.forward(x_bar), sigma, y, bg)
        y2n = reg.prox_dual(y2 + s * reg.forward(x_bar), alpha)
        g = blur_op.adjoint(y1n) + reg.adjoint(y2n)
        xn = prox_nonneg(x - t(tau) * g)
        dx = xn - x
        dx2 = np.sum(dx * dx)
        dAx = blur_op.forward(xn) - blur_op.forward(x)
        dLx = reg.forward(xn) - reg.forward(x)
        dK2 = np.sum(dAx * dAx) + np.sum(dLx * dLx)
        dK2s = np.maximum(dK2, t(1e-12))
        ratio = dx2 / (t(2.0) * s * dK2s)
        tau_c = np.minimum(np.sqrt(t(1.0 + theta)) * t(tau), t(delta) * np.sqrt(ratio))
        cond = tau_c * s * dK2
        thr = t(delta) * dx2
        tau_n = np.where(cond > thr, t(eta) * tau_c, tau_c)
        tau_n = np.maximum(tau_n, t(step_scale * 1e-4))
        theta_n = tau_n / t(tau)
        sigma_n = s / np.maximum(theta_n, t(0.1))
        sigma_n = np.clip(sigma_n, t(step_scale * 1e-4), t(step_scale * 1e4))
        xx = np.sum(x * x)
        xnxn = np.sum(xn * xn)
        rel = float(np.sqrt(dx2 / (np.maximum(xx, xnxn) + t(1e-12))))
        if k >= min_iter:
            if rel < tol:
                count += 1
                if count >= patience:
                    converged = True
                    final_iter = k + 1
                    x, y1, y2 = xn, y1n, y2n
                    taus.append(float(tau_n))
                    sigmas.append(float(sigma_n))
                    break
            else:
                count = 0
        x_bar = xn + t(theta_n) * (xn - x)
        x, y1, y2 = xn, y1n, y2n
        tau, sigma, theta = float(tau_n), float(sigma_n), float(theta_n)
        taus.append(tau)
        sigmas.append(sigma)
        want_loss = (callback is not None) if generic else ((k + 1) % eval_interval == 0)
        if want_loss:
            fm = blur_op.forward(x) + bg
            fms = np.maximum(fm, t(1e-6))
            if loss_type == "poisson":
                dl = np.sum(y * np.log((y + t(1e-6)) / fms) - (y - fm))
            else:
                dl = t(0.5) * np.sum((y - fm) ** 2)
            lx = reg.forward(x)
            if reg.norm == "L1":
                rl = t(alpha) * np.sum(np.abs(lx))
            else:
                rl = t(alpha) * np.sum(np.sqrt(np.sum(lx * lx, axis=0) + t(1e-12)))
            losses.append(float(dl + rl))
            if generic and callback is not None:
                callback(k, x, losses[-1])
        if not generic and callback is not None and callback(k, x):
            final_iter = k + 1
            break
    return dict(restored=x, iterations=final_iter, loss_history=losses, converged=converged,
                tau_history=taus, sigma_history=sigmas, y1=y1, y2=y2)


def solve_pdhg_mlx(observed, psf, alpha=0.01, regularization="hessian", norm="L1",
                   loss_type="poisson", num_iter=200, background=0.0, spacing=None,
                   bin_factors=None, sampling_factors=None, init=None, delta=0.99, eta=0.5,
                   eval_interval=10, tol=1e-5, min_iter=20, patience=5, dtype=np.float32,
                   callback=None):
    """PSF entry point: builds A (plain / bin / sampling) and L
    (pdhg_mlx.py:507-700), then runs the shared loop."""
    y = np.asarray(observed).astype(dtype)
    psf = np.asarray(psf)
    nd = y.ndim
    if bin_factors is not None and sampling_factors is not None:
        raise ValueError("bin_factors and sampling_factors are mutually exclusive")
    if sampling_factors is not None:
        f = sampling_factors
        f = (float(f),) * nd if isinstance(f, (int, float)) else tuple(float(v) for v in f)
        if len(f) != nd:
            raise ValueError(f"sampling_factors has length {len(f)}, expected {nd}")
        if any(v <= 0 for v in f):
            raise ValueError("sampling_factors must all be positive")
        hr = tuple(max(1, int(round(n * v))) for n, v in zip(y.shape, f))
        if tuple(psf.shape) != hr:
            raise ValueError(
                "For sampling_factors, psf.shape must match the reconstructed "
                f"high-resolution shape {hr}; got {tuple(psf.shape)}"
            )
        conv = ops.LinearFFTConvolver(psf, hr, normalize=True, dtype=dtype)
        A = ops.compose(ops.FractionalAreaDownsample(f, dtype=dtype), conv)
    elif bin_factors is not None:
        b = bin_factors
        b = (int(b),) * nd if isinstance(b, int) else tuple(int(v) for v in b)
        if len(b) != nd:
            raise ValueError(f"bin_factors has length {len(b)}, expected {nd}")
        if any(v <= 0 for v in b):
            raise ValueError("bin_factors must all be positive")
        hr = tuple(psf.shape)
        for i, (n, v) in enumerate(zip(hr, b)):
            if n % v:
                raise ValueError(f"PSF dim {i} size {n} is not divisible by bin factor {v}")
        lr = tuple(n // v for n, v in zip(hr, b))
        if tuple(y.shape) != lr:
            raise ValueError(
                "For bin_factors, observed.shape must match psf.shape divided "
                f"by bin_factors; expected {lr}, got {tuple(y.shape)}"
            )
        conv = ops.LinearFFTConvolver(psf, hr, normalize=True, dtype=dtype)
        A = ops.compose(ops.FractionalAreaDownsample(b, dtype=dtype), conv)
    else:
        A = ops.LinearFFTConvolver(psf, tuple(y.shape), normalize=True, dtype=dtype)
        hr = tuple(y.shape)
    r = spacing_ratio(spacing, nd)
    reg = Regularizer(regularization, nd, r, norm, dtype)
    if init is not None:
        x = np.asarray(init).astype(dtype)
    else:
        x = A.adjoint(y) if (sampling_factors is not None or bin_factors is not None) else y.copy()
        x = np.maximum(x, np.dtype(dtype).type(0.0))
    out = _pdhg_loop(y, A, reg, x, alpha, loss_type, num_iter, background, delta, eta,
                     eval_interval, tol, min_iter, patience, dtype, generic=False,
                     callback=callback)
    out["blur_op"] = A
    return out


def solve_pdhg_with_operator(observed, blur_op, alpha=0.01, regularization="identity",
                             norm="L1", loss_type="poisson", num_iter=200, background=0.0,
                             init=None, delta=0.99, eta=0.5, eval_interval=10, tol=1e-5,
                             min_iter=20, patience=5, dtype=np.float32, callback=None,
                             solution_shape=None):
    """Operator entry point (pdhg_mlx.py:928-1242): x sized from ``observed``
    (the reference's rule, :1011-1018) unless ``solution_shape`` is given;
    r = 1; x0 = 0.01 unless ``init``."""
    y = np.asarray(observed).astype(dtype)
    shp = tuple(solution_shape) if solution_shape is not None else tuple(y.shape)
    reg = Regularizer(regularization, len(shp), 1.0, norm, dtype)
    t = np.dtype(dtype).type
    x = np.ones(shp, dtype=dtype) * t(0.01) if init is None else np.asarray(init).astype(dtype)
    x = np.maximum(x, t(0.0))
    return _pdhg_loop(y, blur_op, reg, x, alpha, loss_type, num_iter, background, delta, eta,
                      eval_interval, tol, min_iter, patience, dtype, generic=True,
                      callback=callback)
