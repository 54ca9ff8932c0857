"""Malitsky-Pock adaptive PDHG on the B200.

Mirrors deconlib's ``deconvolution/pdhg_mlx.py``: the proximal maps
(:115-233), Identity/Gradient/HessianRegularizer (:241-451),
_compute_spacing_ratio / _create_regularizer (:459-499), solve_pdhg_mlx
(:507-920) and solve_pdhg_with_operator (:928-1242), with the same
arguments, validation messages and result fields.

Device design.  tau, sigma, theta, the convergence counter and the
tau/sigma/objective histories live in device memory (``decon_pdhg``); one
FP64 step kernel per iteration performs the reference's scalar block
(:749-857) from deterministic FP64 reductions.  The host therefore queues
iterations without reading scalars back and only checks the stop flag every
``_CHUNK`` iterations (or every iteration when a callback needs x).  By
linearity A x_bar = (1 + theta) A x - theta A x_prev, so an iteration costs
one forward and one adjoint application of A (the reference spends three
forward and one adjoint), and ||L x_new - L x|| is computed as ||L (x_new - x)||.
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Callable, List, Literal, Optional, Tuple, Union

import numpy as np
import torch

from .. import _lib
from ._device import empty, fill, stream, to_device, zeros
from .base import MLXDeconvolutionResult
from .composition import LinearOperator, compose
from .core_operators import FractionalAreaDownsample
from .linops import (Gradient1D, Gradient2D, Gradient3D, Hessian1D, Hessian2D, Hessian3D,
                     LinearFFTConvolver)

__all__ = [
    "solve_pdhg_mlx", "solve_pdhg_with_operator", "IdentityRegularizer", "GradientRegularizer",
    "HessianRegularizer", "prox_poisson_dual", "prox_gaussian_dual", "prox_nonneg",
    "prox_l1_dual", "prox_l1_2_dual", "PDHGRunner", "pdhg_mlx_runner", "pdhg_result",
]

_CHUNK = 16


def _fused_stencil() -> bool:
    """DECON_FUSED_STENCIL=1: the Hessian dual and primal updates in one
    z-walk kernel instead of two kernels (identical values; on the B200 the
    two kernels measured faster, 260 vs 414 us at 128x256x256)."""
    return os.environ.get("DECON_FUSED_STENCIL") == "1"


def _overlap() -> bool:
    """The Hessian dual update and ||H dx||^2 on a second stream, beside the
    adjoint and the forward convolution (they read nothing those produce);
    DECON_PDHG_OVERLAP=0 queues everything on one stream.  Same kernels and
    values either way (on the B200: 1.056 vs 1.069 ms per iteration at
    128x256x256)."""
    return os.environ.get("DECON_PDHG_OVERLAP", "1") != "0"


# ---------------------------------------------------------------------------
# proximal maps (element-wise; exposed for API parity, pdhg_mlx.py:115-233)
# ---------------------------------------------------------------------------


class _Scalars:
    """A throw-away device state whose sigma/theta are fixed, used to run the
    PDHG dual kernels as stand-alone proximal maps."""

    def __init__(self, sigma: float):
        lib = _lib.load()
        h = C.c_void_p()
        _lib.check(lib.decon_pdhg_create(1, float(sigma), 0.99, 0.5, 0.0, 0, 1, C.byref(h)))
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib._lib is not None:
            torch.cuda.synchronize()
            _lib._lib.decon_pdhg_destroy(self.h)


def _prox_data(y, sigma, data, background, loss_type):
    y = to_device(y)
    d = to_device(data)
    out = y.clone()
    zero = torch.zeros_like(y)
    sc = _Scalars(sigma)
    # dual_data computes prox(y1 + sigma * A xbar); with A xbar = 0 it is prox(y)
    _lib.call("decon_pdhg_dual_data", sc.h, _lib.ptr(out), _lib.ptr(zero), _lib.ptr(zero),
              _lib.ptr(d), C.c_float(background), loss_type, out.numel(), stream())
    torch.cuda.current_stream().synchronize()
    return out


def prox_poisson_dual(y, sigma: float, data, background: float):
    """Poisson-dual prox: 1 - z, z the positive root (pdhg_mlx.py:115-166)."""
    return _prox_data(y, sigma, data, background, 0)


def prox_gaussian_dual(y, sigma: float, data, background: float):
    """(y - sigma (D - b)) / (1 + sigma) (pdhg_mlx.py:169-189)."""
    return _prox_data(y, sigma, data, background, 1)


def prox_nonneg(x):
    """max(0, x) (pdhg_mlx.py:192-194)."""
    x = to_device(x)
    out = empty(x.shape)
    _lib.call("decon_clamp_min", _lib.ptr(x), C.c_float(0.0), _lib.ptr(out), x.numel(), stream())
    return out


def _prox_reg(y, bound, norm):
    y = to_device(y)
    out = y.clone()
    zero = torch.zeros_like(y)
    sc = _Scalars(1.0)
    ncomp = y.shape[0] if (norm == 1 and y.dim() > 1) else 1
    n = y.numel() // ncomp
    _lib.call("decon_pdhg_dual_reg", sc.h, _lib.ptr(out), _lib.ptr(zero), C.c_float(bound), norm,
              ncomp, n, stream())
    torch.cuda.current_stream().synchronize()
    return out


def prox_l1_dual(y, bound: float):
    """clip(y, -bound, bound) (pdhg_mlx.py:197-209)."""
    return _prox_reg(y, bound, 0)


def prox_l1_2_dual(y, bound: float):
    """y / max(||y||_2 over axis 0 / bound, 1) (pdhg_mlx.py:212-233)."""
    return _prox_reg(y, bound, 1)


# ---------------------------------------------------------------------------
# regularisers (pdhg_mlx.py:241-451)
# ---------------------------------------------------------------------------


class IdentityRegularizer:
    """L = I with a leading component axis (pdhg_mlx.py:241-306)."""

    def __init__(self, norm: Literal["L1", "L1_2"] = "L1"):
        self.norm = norm
        self._operator_norm_sq = 1.0

    @property
    def output_components(self) -> int:
        return 1

    @property
    def operator_norm_sq(self) -> float:
        return self._operator_norm_sq

    def forward(self, x):
        return to_device(x).unsqueeze(0)

    def adjoint(self, y):
        return to_device(y)[0]

    def prox_dual(self, y, sigma: float, alpha: float):
        return prox_l1_dual(y, alpha) if self.norm == "L1" else prox_l1_2_dual(y, alpha)

    def __call__(self, x):
        return self.forward(x)


class GradientRegularizer:
    """TV operator (pdhg_mlx.py:309-377)."""

    def __init__(self, ndim: int, r: float = 1.0, norm: Literal["L1", "L1_2"] = "L1"):
        if ndim not in (1, 2, 3):
            raise ValueError(f"ndim must be 1, 2, or 3, got {ndim}")
        self.ndim, self.r, self.norm = ndim, r, norm
        self._op = Gradient1D() if ndim == 1 else (Gradient2D() if ndim == 2 else Gradient3D(r=r))

    @property
    def output_components(self) -> int:
        return self.ndim

    @property
    def operator_norm_sq(self) -> float:
        return self._op.operator_norm_sq

    def forward(self, x):
        g = self._op.forward(x)
        return g.unsqueeze(0) if self.ndim == 1 else g

    def adjoint(self, y):
        y = to_device(y)
        return self._op.adjoint(y[0] if self.ndim == 1 else y)

    def prox_dual(self, y, sigma: float, alpha: float):
        return prox_l1_dual(y, alpha) if self.norm == "L1" else prox_l1_2_dual(y, alpha)

    def __call__(self, x):
        return self.forward(x)


class HessianRegularizer:
    """Second-order operator (pdhg_mlx.py:380-451)."""

    def __init__(self, ndim: int, r: float = 1.0, norm: Literal["L1", "L1_2"] = "L1"):
        if ndim not in (1, 2, 3):
            raise ValueError(f"ndim must be 1, 2, or 3, got {ndim}")
        self.ndim, self.r, self.norm = ndim, r, norm
        self._op = Hessian1D() if ndim == 1 else (Hessian2D() if ndim == 2 else Hessian3D(r=r))

    @property
    def output_components(self) -> int:
        return 1 if self.ndim == 1 else (3 if self.ndim == 2 else 6)

    @property
    def operator_norm_sq(self) -> float:
        return self._op.operator_norm_sq

    def forward(self, x):
        h = self._op.forward(x)
        return h.unsqueeze(0) if self.ndim == 1 else h

    def adjoint(self, y):
        y = to_device(y)
        return self._op.adjoint(y[0] if self.ndim == 1 else y)

    def prox_dual(self, y, sigma: float, alpha: float):
        return prox_l1_dual(y, alpha) if self.norm == "L1" else prox_l1_2_dual(y, alpha)

    def __call__(self, x):
        return self.forward(x)


def _compute_spacing_ratio(spacing, ndim: int) -> float:
    """r = mean(dy, dx) / dz for 3-D, else 1 (pdhg_mlx.py:459-482)."""
    if spacing is None or ndim in (1, 2):
        return 1.0
    if len(spacing) != ndim:
        raise ValueError(f"spacing must have {ndim} elements, got {len(spacing)}")
    dz = spacing[0]
    lat = (spacing[1] + spacing[2]) / 2.0
    return lat / dz if dz > 0 else 1.0


def _create_regularizer(regularization, ndim, r, norm):
    if regularization == "identity":
        return IdentityRegularizer(norm=norm)
    if regularization == "gradient":
        return GradientRegularizer(ndim=ndim, r=r, norm=norm)
    if regularization == "hessian":
        return HessianRegularizer(ndim=ndim, r=r, norm=norm)
    raise ValueError(f"Unknown regularization: {regularization}")


def _normalize_sampling_factors(factors, ndim):
    if isinstance(factors, (int, float)):
        factors = (float(factors),) * ndim
    elif len(factors) != ndim:
        raise ValueError(f"sampling_factors has length {len(factors)}, expected {ndim}")
    else:
        factors = tuple(float(f) for f in factors)
    if any(f <= 0 for f in factors):
        raise ValueError("sampling_factors must all be positive")
    return factors


def _normalize_bin_factors(factors, ndim):
    if isinstance(factors, int):
        factors = (factors,) * ndim
    elif len(factors) != ndim:
        raise ValueError(f"bin_factors has length {len(factors)}, expected {ndim}")
    else:
        factors = tuple(int(f) for f in factors)
    if any(f <= 0 for f in factors):
        raise ValueError("bin_factors must all be positive")
    return factors


# ---------------------------------------------------------------------------
# the shared iteration
# ---------------------------------------------------------------------------


class _State:
    def __init__(self, num_iter, step_scale, delta, eta, tol, min_iter, patience):
        lib = _lib.load()
        h = C.c_void_p()
        _lib.check(lib.decon_pdhg_create(int(num_iter), float(step_scale), float(delta), float(eta),
                                         float(tol), int(min_iter), int(patience), C.byref(h)))
        self.h = h
        self.num_iter = num_iter
        self.capacity = max(int(num_iter), 1)

    def reset(self, num_iter, step_scale, delta, eta, tol, min_iter, patience):
        """Start a new solve in this state (num_iter <= capacity), queued on
        the current stream."""
        _lib.call("decon_pdhg_reset", self.h, int(num_iter), float(step_scale), float(delta),
                  float(eta), float(tol), int(min_iter), int(patience), stream())
        self.num_iter = num_iter
        return self

    def read(self, hist=False):
        k, fi, cv, st = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        sc = (C.c_double * 3)()
        n = max(self.num_iter, 1)
        arrs = [np.zeros(n) for _ in range(4)] if hist else [None] * 4
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None  # noqa: E731
        _lib.check(_lib.load().decon_pdhg_read(self.h, C.byref(k), C.byref(fi), C.byref(cv),
                                               C.byref(st), sc, *[dp(a) for a in arrs], stream()))
        return dict(k=k.value, final_iter=fi.value, converged=bool(cv.value), stop=bool(st.value),
                    tau=sc[0], sigma=sc[1], theta=sc[2], tau_hist=arrs[0], sigma_hist=arrs[1],
                    loss_hist=arrs[2], rel_hist=arrs[3])

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib._lib is not None:
            try:
                torch.cuda.synchronize()
                _lib._lib.decon_pdhg_destroy(self.h)
            except Exception:
                pass
            self.h = None


def _norm_code(norm):
    return 0 if norm == "L1" else 1


class PDHGRunner:
    """The shared iteration of both entry points (pdhg_mlx.py:717-900 and
    :1066-1221), split into set-up / ``iterate`` / ``result`` so a caller
    (the benchmark, the serving loop) can time or interleave iterations.

    Buffers: x is triple-buffered (slot k % 3 holds x_k, slot (k + 2) % 3
    x_{k-1}; iteration k writes x_{k+1} into slot (k + 1) % 3, so the fused
    Hessian kernel never writes a buffer it still reads with halos); A x is
    double-buffered (slot k % 2).  x_bar and A x_bar are never stored: they
    are formed from the slots inside the kernels."""

    def __init__(self, data, A, reg, x0, alpha, loss_type, num_iter, background, delta, eta,
                 eval_interval, tol, min_iter, patience, verbose=False, callback=None,
                 generic=False, fused=True, state=None, async_status=False):
        self.s = stream()
        # async_status: poll the device's stop flag through a page-locked copy
        # and an event instead of synchronising every _CHUNK iterations (a
        # host that feeds many solves from one thread must not block on one);
        # iterations queued after the stop are no-ops on the device
        self.async_status = bool(async_status) and callback is None and not verbose
        self._status = None
        self._status_ev = None
        self.data, self.A, self.reg = data, A, reg
        self.alpha = float(alpha)
        self.bg = float(background)
        self.lcode = 0 if loss_type == "poisson" else 1
        self.ncode = _norm_code(reg.norm)
        self.num_iter, self.eval_interval = int(num_iter), int(eval_interval)
        self.tol, self.patience = tol, patience
        self.verbose, self.callback, self.generic = verbose, callback, generic
        step_scale = 0.99 / (A.operator_norm_sq + reg.operator_norm_sq) ** 0.5
        if state is not None and state.capacity >= max(int(num_iter), 1):
            # pooled state (serving loop): no allocation
            self.state = state.reset(num_iter, step_scale, delta, eta, tol, min_iter, patience)
        else:
            self.state = _State(num_iter, step_scale, delta, eta, tol, min_iter, patience)
        self.h = self.state.h
        self.ncomp = reg.output_components
        self.X = [x0.contiguous(), x0.clone(), x0.clone()]
        ax0 = to_device(A.forward(self.X[0])).clone()
        if tuple(ax0.shape) != tuple(data.shape):
            raise ValueError(
                f"blur_op maps the solution to {tuple(ax0.shape)} but observed is "
                f"{tuple(data.shape)}"
            )
        self.AX = [ax0, ax0.clone()]
        self.m = data.numel()
        self.n = x0.numel()
        self.y1 = zeros(data.shape)
        self.y2 = zeros((self.ncomp,) + tuple(x0.shape))
        self.xbar = empty(x0.shape)
        self.dxb = empty(x0.shape)
        self.want_loss_each = generic and (verbose or callback is not None)
        self.stopped_at = None
        self.k = 0
        # fused Hessian3D kernels (fused=False keeps the operator-by-operator path)
        self.fused = (fused and isinstance(reg, HessianRegularizer) and reg.ndim == 3
                      and x0.dim() == 3)
        self.side = None
        if self.fused:
            self.shp = _lib.i64arr(tuple(x0.shape))
            self.r = float(reg.r)
            self.xbar = self.dxb = None
            # the fused dual + primal kernel reads y2 of iteration k from one
            # buffer and writes iteration k + 1's into the other
            self.fused_stencil = _fused_stencil()
            self.y2s = [self.y2, zeros((self.ncomp,) + tuple(x0.shape))] if self.fused_stencil else None
            if _overlap() and not self.fused_stencil:
                self.side = torch.cuda.Stream()
                self.evs = [torch.cuda.Event() for _ in range(4)]

    def iterate(self) -> bool:
        """Queue iteration k; returns False once the solve has stopped."""
        k, s, h, A, reg = self.k, self.s, self.h, self.A, self.reg
        if k >= self.num_iter or self.stopped_at is not None:
            return False
        m, n = self.m, self.n
        xc, xp, xo = self.X[k % 3], self.X[(k + 2) % 3], self.X[(k + 1) % 3]
        axc, axp = self.AX[k % 2], self.AX[(k + 1) % 2]
        side = self.side if self.fused else None
        if side is not None:
            # the Hessian dual update reads x_k, x_{k-1} and the step sizes
            # only: queue it on the side stream beside the adjoint
            cur = torch.cuda.current_stream()
            e0, e1, e2, e3 = self.evs
            e0.record(cur)
            side.wait_event(e0)
            _lib.call("decon_pdhg_hess_dual", h, _lib.ptr(self.y2), _lib.ptr(xc), _lib.ptr(xp),
                      self.shp, C.c_float(self.r), C.c_float(self.alpha), self.ncode,
                      C.c_void_p(side.cuda_stream))
            e1.record(side)
        _lib.call("decon_pdhg_dual_data", h, _lib.ptr(self.y1), _lib.ptr(axc), _lib.ptr(axp),
                  _lib.ptr(self.data), C.c_float(self.bg), self.lcode, m, s)
        aty = to_device(A.adjoint(self.y1))
        do_loss = self.want_loss_each or ((not self.generic) and (k + 1) % self.eval_interval == 0)
        if self.fused:
            # Hessian3D: L x_bar, L^T y2 and L (x_new - x) evaluated on the fly
            shp, r = self.shp, C.c_float(self.r)
            if side is not None:
                # primal update after the side stream's dual, then
                # ||H (x_new - x)||^2 on the side stream beside the forward
                # convolution, ||A x_new - A x||^2 here, the step after both
                cur.wait_event(e1)
                _lib.call("decon_pdhg_hess_primal", h, _lib.ptr(xc), _lib.ptr(aty),
                          _lib.ptr(self.y2), _lib.ptr(xo), shp, r, s)
                e2.record(cur)
                side.wait_event(e2)
                _lib.call("decon_pdhg_hess_dk", h, None, None, 0, _lib.ptr(xo), _lib.ptr(xc), shp, r,
                          C.c_void_p(side.cuda_stream))
                e3.record(side)
                xn = xo
                axn = to_device(A.forward(xn))
                _lib.call("decon_pdhg_dk", h, _lib.ptr(axn), _lib.ptr(axc), m, None, 0, s)
                cur.wait_event(e3)
            elif not self.fused_stencil:
                # the dual and the primal update as two kernels (same values)
                _lib.call("decon_pdhg_hess_dual", h, _lib.ptr(self.y2), _lib.ptr(xc), _lib.ptr(xp),
                          shp, r, C.c_float(self.alpha), self.ncode, s)
                _lib.call("decon_pdhg_hess_primal", h, _lib.ptr(xc), _lib.ptr(aty),
                          _lib.ptr(self.y2), _lib.ptr(xo), shp, r, s)
            else:
                y2i, y2o = self.y2s[k % 2], self.y2s[(k + 1) % 2]
                _lib.call("decon_pdhg_hess_dual_primal", h, _lib.ptr(y2i), _lib.ptr(y2o),
                          _lib.ptr(xc), _lib.ptr(xp), _lib.ptr(aty), _lib.ptr(xo), shp, r,
                          C.c_float(self.alpha), self.ncode, s)
                self.y2 = y2o
            if side is None:
                xn = xo
                axn = to_device(A.forward(xn))
                # ||A dx||^2 and ||H dx||^2 as the two sums of the two-stream
                # schedule (same bits on either schedule)
                _lib.call("decon_pdhg_dk", h, _lib.ptr(axn), _lib.ptr(axc), m, None, 0, s)
                _lib.call("decon_pdhg_hess_dk", h, None, None, 0, _lib.ptr(xn), _lib.ptr(xc), shp, r, s)
            _lib.call("decon_pdhg_step", h, s)
            if do_loss:
                _lib.call("decon_pdhg_hess_loss", h, _lib.ptr(axn), _lib.ptr(self.data),
                          C.c_float(self.bg), self.lcode, m, _lib.ptr(xn), shp, r, self.ncode,
                          C.c_double(self.alpha), k, s)
        else:
            _lib.call("decon_pdhg_xbar", h, _lib.ptr(xc), _lib.ptr(xp), _lib.ptr(self.xbar), n, s)
            lxb = to_device(reg.forward(self.xbar))
            _lib.call("decon_pdhg_dual_reg", h, _lib.ptr(self.y2), _lib.ptr(lxb),
                      C.c_float(self.alpha), self.ncode, self.ncomp, n, s)
            lty = to_device(reg.adjoint(self.y2))
            _lib.call("decon_pdhg_primal", h, _lib.ptr(xc), _lib.ptr(aty), _lib.ptr(lty),
                      _lib.ptr(xo), n, s)
            xn = xo
            axn = to_device(A.forward(xn))
            _lib.call("decon_pdhg_sub", h, _lib.ptr(xn), _lib.ptr(xc), _lib.ptr(self.dxb), n, s)
            ldx = to_device(reg.forward(self.dxb))
            _lib.call("decon_pdhg_dk", h, _lib.ptr(axn), _lib.ptr(axc), m, _lib.ptr(ldx), ldx.numel(),
                      s)
            _lib.call("decon_pdhg_step", h, s)
            if do_loss:
                lx = to_device(reg.forward(xn))
                _lib.call("decon_pdhg_loss", h, _lib.ptr(axn), _lib.ptr(self.data),
                          C.c_float(self.bg), self.lcode, m, _lib.ptr(lx), self.ncode, self.ncomp,
                          n, C.c_double(self.alpha), k, s)
        self.AX[(k + 1) % 2] = axn
        self.k = k + 1
        cb, verbose = self.callback, self.verbose
        if self.async_status:
            return self._poll_status()
        if cb is not None or (verbose and do_loss) or self.k % _CHUNK == 0:
            info = self.state.read(hist=bool(verbose and do_loss) or (self.generic and cb is not None))
            # Stop here if the solve ended before this iteration, or broke on
            # convergence at it (the reference breaks before the loss and the
            # callback, pdhg_mlx.py:812-833); reaching num_iter still runs them.
            ended_before = info["stop"] and info["final_iter"] < k + 1
            converged_here = info["converged"] and info["final_iter"] == k + 1
            if ended_before or converged_here:
                self.stopped_at = info["final_iter"]
                if verbose and info["converged"]:
                    rel = info["rel_hist"][self.stopped_at - 1] if info["rel_hist"] is not None else float("nan")
                    print(f"Converged at iteration {self.stopped_at}: rel_change={rel:.2e} "
                          f"< tol={self.tol:.2e} for {self.patience} consecutive iterations")
                return False
            if verbose and do_loss and (not self.generic or self.k % self.eval_interval == 0):
                print(f"Iter {k + 1:4d}: loss={info['loss_hist'][k]:.4e}, "
                      f"tau={info['tau']:.4e}, sigma={info['sigma']:.4e}")
            if cb is not None:
                if self.generic:
                    cb(k, xn, float(info["loss_hist"][k]))
                elif cb(k, xn):
                    _lib.call("decon_pdhg_set_stop", h, k + 1, s)
                    self.stopped_at = k + 1
                    return False
        return True

    def _poll_status(self) -> bool:
        """Non-blocking stop check: examine the last completed status copy,
        queue a new one every _CHUNK iterations."""
        ev = self._status_ev
        if ev is not None and ev.query():
            k, _, converged, final_iter, stop = (int(v) for v in self._status.tolist())
            self._status_ev = None
            if stop and final_iter <= k:
                self.stopped_at = final_iter
                return False
        if self._status_ev is None and self.k % _CHUNK == 0:
            if self._status is None:
                self._status = torch.zeros(5, dtype=torch.int32, pin_memory=True)
            _lib.call("decon_pdhg_status_async", self.h, C.c_void_p(self._status.data_ptr()), self.s)
            self._status_ev = torch.cuda.Event()
            self._status_ev.record(torch.cuda.current_stream())
        return True

    def run(self):
        while self.iterate():
            pass
        return self

    def result(self):
        info = self.state.read(hist=True)
        final_iter = info["final_iter"] if self.stopped_at is None else self.stopped_at
        final_iter = min(final_iter, self.k) if self.num_iter > 0 else 0
        converged = info["converged"]
        x = self.X[final_iter % 3]
        taus = [float(v) for v in info["tau_hist"][:final_iter]]
        sigmas = [float(v) for v in info["sigma_hist"][:final_iter]]
        lh = info["loss_hist"]
        if self.generic:
            loss_k = list(range(final_iter)) if self.want_loss_each else []
        else:
            loss_k = [k for k in range(final_iter) if (k + 1) % self.eval_interval == 0]
        if converged:
            loss_k = [k for k in loss_k if k != final_iter - 1]
        losses = [float(lh[k]) for k in loss_k]
        return x, final_iter, converged, taus, sigmas, losses


def _conv_for(conv, psf, signal_shape, precision="fp32", fft_shape=None):
    """A normalised LinearFFTConvolver of ``psf`` on ``signal_shape``: the
    given pooled one with its OTF rebuilt, or a new one (on ``fft_shape``,
    default the reference's 5-smooth canvas)."""
    if conv is None:
        return LinearFFTConvolver(psf, signal_shape=signal_shape, normalize=True, precision=precision,
                                  fft_shape=fft_shape)
    if tuple(conv.signal_shape) != tuple(signal_shape) or not conv.normalize:
        raise ValueError(f"pooled convolver is for {conv.signal_shape}, the solve needs {signal_shape}")
    if conv.precision != precision:
        conv.set_precision(precision)
    return conv.set_kernel(psf)


def solve_pdhg_mlx(observed, psf, alpha: float = 0.01,
                   regularization: Literal["identity", "gradient", "hessian"] = "hessian",
                   norm: Literal["L1", "L1_2"] = "L1",
                   loss_type: Literal["poisson", "gaussian"] = "poisson", num_iter: int = 200,
                   background: float = 0.0, spacing: Optional[Tuple[float, ...]] = None,
                   bin_factors=None, sampling_factors=None, icf_sigmas=None, icf_spacings=None,
                   init=None, verbose: bool = False, callback: Optional[Callable] = None,
                   delta: float = 0.99, eta: float = 0.5, eval_interval: int = 10,
                   tol: float = 1e-5, min_iter: int = 20, patience: int = 5,
                   precision: str = "fp32", fft_shape=None) -> MLXDeconvolutionResult:
    """PSF entry point of adaptive PDHG (pdhg_mlx.py:507-920).

    Not in the reference: ``precision="mixed"`` stores the OTF as FP16 with
    per-plane scales (``LinearFFTConvolver.set_precision``); ``fft_shape``
    chooses the convolution canvas (e.g. ``static_fft_shape``)."""
    runner, meta = pdhg_mlx_runner(
        observed, psf, alpha=alpha, regularization=regularization, norm=norm, loss_type=loss_type,
        num_iter=num_iter, background=background, spacing=spacing, bin_factors=bin_factors,
        sampling_factors=sampling_factors, icf_sigmas=icf_sigmas, icf_spacings=icf_spacings,
        init=init, verbose=verbose, callback=callback, delta=delta, eta=eta,
        eval_interval=eval_interval, tol=tol, min_iter=min_iter, patience=patience,
        precision=precision, fft_shape=fft_shape)
    return pdhg_result(runner.run(), meta)


def pdhg_result(runner: "PDHGRunner", metadata: dict) -> MLXDeconvolutionResult:
    """The result record of a finished runner (synchronises its stream)."""
    x, fi, cv, taus, sigmas, losses = runner.result()
    return MLXDeconvolutionResult(restored=x, iterations=fi, loss_history=losses, converged=cv,
                                  tau_history=taus, sigma_history=sigmas, metadata=metadata)


def pdhg_mlx_runner(observed, psf, alpha: float = 0.01,
                    regularization: Literal["identity", "gradient", "hessian"] = "hessian",
                    norm: Literal["L1", "L1_2"] = "L1",
                    loss_type: Literal["poisson", "gaussian"] = "poisson", num_iter: int = 200,
                    background: float = 0.0, spacing: Optional[Tuple[float, ...]] = None,
                    bin_factors=None, sampling_factors=None, icf_sigmas=None, icf_spacings=None,
                    init=None, verbose: bool = False, callback: Optional[Callable] = None,
                    delta: float = 0.99, eta: float = 0.5, eval_interval: int = 10,
                    tol: float = 1e-5, min_iter: int = 20, patience: int = 5,
                    conv: Optional[LinearFFTConvolver] = None, state=None,
                    precision: str = "fp32", async_status: bool = False, fft_shape=None):
    """Set-up of ``solve_pdhg_mlx`` without the iterations: returns the
    ``PDHGRunner`` (iterations queued on the current stream by ``iterate``)
    and the result metadata, for callers that interleave solves.

    ``conv`` / ``state`` (serving loop): a pooled LinearFFTConvolver of the
    right kernel and signal shapes, whose OTF is rebuilt for ``psf`` in place,
    and a pooled PDHG state; both avoid device allocation and cudaFree."""
    data = to_device(observed)
    psf_shape = tuple(int(s) for s in (psf.shape if hasattr(psf, "shape") else np.shape(psf)))
    ndim = data.dim()
    if bin_factors is not None and sampling_factors is not None:
        raise ValueError("bin_factors and sampling_factors are mutually exclusive")
    if icf_sigmas is not None:
        raise NotImplementedError(
            "ICF (icf_sigmas) is not yet supported with atomic operators. "
            "Use the composed operator API directly or remove icf_sigmas parameter."
        )
    if sampling_factors is not None:
        factors = _normalize_sampling_factors(sampling_factors, ndim)
        highres = tuple(max(1, int(round(n * f))) for n, f in zip(data.shape, factors))
        if psf_shape != highres:
            raise ValueError(
                "For sampling_factors, psf.shape must match the reconstructed "
                f"high-resolution shape {highres}; got {psf_shape}"
            )
        conv = _conv_for(conv, psf, highres, precision, fft_shape)
        blur_op = compose(FractionalAreaDownsample(scale=factors), conv)
    elif bin_factors is not None:
        factors = _normalize_bin_factors(bin_factors, ndim)
        highres = psf_shape
        for i, (nn, f) in enumerate(zip(highres, factors)):
            if nn % f != 0:
                raise ValueError(f"PSF dim {i} size {nn} is not divisible by bin factor {f}")
        lowres = tuple(nn // f for nn, f in zip(highres, factors))
        if tuple(data.shape) != lowres:
            raise ValueError(
                "For bin_factors, observed.shape must match psf.shape divided "
                f"by bin_factors; expected {lowres}, got {tuple(data.shape)}"
            )
        conv = _conv_for(conv, psf, highres, precision, fft_shape)
        blur_op = compose(FractionalAreaDownsample(scale=factors), conv)
    else:
        blur_op = _conv_for(conv, psf, tuple(data.shape), precision, fft_shape)
        highres = tuple(data.shape)
    r = _compute_spacing_ratio(spacing, ndim)
    reg = _create_regularizer(regularization, ndim, r, norm)
    if init is not None:
        x0 = to_device(init).clone()
    else:
        x0 = to_device(blur_op.adjoint(data)) if (sampling_factors is not None or bin_factors is not None) else data.clone()
        x0 = prox_nonneg(x0)
    runner = PDHGRunner(data, blur_op, reg, x0, alpha, loss_type, num_iter, background, delta, eta,
                        eval_interval, tol, min_iter, patience, verbose, callback, generic=False,
                        state=state, async_status=async_status)
    meta = {"algorithm": "malitsky_pock_pdhg", "regularization": regularization, "norm": norm,
            "loss_type": loss_type, "alpha": alpha, "background": background, "tol": tol,
            "min_iter": min_iter, "patience": patience}
    return runner, meta


def solve_pdhg_with_operator(observed, blur_op: LinearOperator, alpha: float = 0.01,
                             regularization: Literal["identity", "gradient", "hessian"] = "identity",
                             norm: Literal["L1", "L1_2"] = "L1",
                             loss_type: Literal["poisson", "gaussian"] = "poisson",
                             num_iter: int = 200, background: float = 0.0, init=None,
                             verbose: bool = False, callback: Optional[Callable] = None,
                             delta: float = 0.99, eta: float = 0.5, eval_interval: int = 10,
                             tol: float = 1e-5, min_iter: int = 20, patience: int = 5,
                             use_in_shape: bool = False) -> MLXDeconvolutionResult:
    """Operator entry point of adaptive PDHG (pdhg_mlx.py:928-1242).

    As in the reference, the solution takes ``observed.shape`` (or
    ``(blur_op.shape[1],)`` for a 2-D matrix operator) and r = 1.
    ``use_in_shape=True`` (opt-in, not in the reference) sizes x and y2 from
    ``blur_op.in_shape`` instead, which lets operators that change shape
    (e.g. ``compose(Crop, FractionalAreaDownsample, LinearFFTConvolver)``)
    run here; the reference fails on them at the first iteration."""
    data = to_device(observed)
    if hasattr(blur_op, "shape") and len(blur_op.shape) == 2:
        solution_shape = (int(blur_op.shape[1]),)
    elif use_in_shape and getattr(blur_op, "in_shape", None) is not None:
        solution_shape = tuple(int(s) for s in blur_op.in_shape)
    else:
        solution_shape = tuple(data.shape)
    reg = _create_regularizer(regularization, len(solution_shape), 1.0, norm)
    if init is not None:
        x0 = to_device(init)
    else:
        x0 = fill(empty(solution_shape), 0.01)
    x0 = prox_nonneg(x0)
    x, fi, cv, taus, sigmas, losses = PDHGRunner(
        data, blur_op, reg, x0, alpha, loss_type, num_iter, background, delta, eta, eval_interval,
        tol, min_iter, patience, verbose, callback, generic=True).run().result()
    return MLXDeconvolutionResult(
        restored=x, iterations=fi, loss_history=losses, converged=cv, tau_history=taus,
        sigma_history=sigmas,
        metadata={"algorithm": "malitsky_pock_pdhg", "regularization": regularization, "norm": norm,
                  "loss_type": loss_type, "alpha": alpha, "background": background, "tol": tol,
                  "min_iter": min_iter, "patience": patience, "operator_type": "generic"})
