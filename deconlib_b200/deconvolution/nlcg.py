"""Accelerated Poisson maximum likelihood by nonlinear conjugate gradients.

Mirrors deconlib's ``deconvolution/nlcg_mlx.py``: NLCGResult (:59-83),
nlcg_objective (:118-134), nlcg_gradient (:137-154), nlcg_hessian_quadform
(:157-194), nlcg_step_length (:197-300), i_divergence_between (:303-323),
nlcg_with_operator (:326-545) and nlcg_solver (:548-588).  Same objective
(Schaefer, Schuster & Herz 2001, f = s^2), Fletcher-Reeves directions and the
exact Newton-Raphson step length along the direction (Valdimarsson & Preza's
COSM), with the same stopping rules (discrepancy principle, Eq. 17).

Device path: the caller's ``blur_op`` and ``regularizer`` apply the
convolutions and the smoothness operator (three convolutions per iteration
at steady state; for ``Hessian3D`` the Gram matrix and energy of its images
are evaluated on the fly by ``decon_nlcg_hess_*`` and only C^T C f is formed);
every other pass is one fused kernel of libdecon_b200
(``decon_nlcg_*``) with FP64 sums.  The Newton refinements update the step
length on the device, so an iteration synchronises with the host once: each
step is carried through to the new gradient speculatively and kept only if
it lowers the objective, exactly the reference's acceptance test.  Sums are
FP64 where the reference sums in float32, so step lengths agree to float32
round-off rather than bit for bit.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Any, Callable, Optional, Tuple

import numpy as np
import torch

from .. import _lib
from ._device import empty, fill, stream, to_device
from .linops import Hessian3D

__all__ = ["NLCGResult", "nlcg_objective", "nlcg_gradient", "nlcg_hessian_quadform",
           "nlcg_step_length", "i_divergence_between", "nlcg_with_operator", "nlcg_solver"]

_EPS = 1e-10


@dataclass
class NLCGResult:
    """Result of nonlinear conjugate-gradient deconvolution (nlcg_mlx.py:59-83)."""

    restored: Any
    pred: Any
    iterations: int
    loss_history: list
    converged: bool = False
    background: float = 0.0
    full_shape: Optional[Tuple[int, ...]] = None
    valid_slices: Optional[Tuple[slice, ...]] = None


class _Scalars:
    """The device scalar block of one solve (``decon_nlcg`` handle)."""

    def __init__(self):
        h = C.c_void_p()
        _lib.call("decon_nlcg_create", C.byref(h))
        self.h = h
        self._out = (C.c_double * 18)()

    def read(self) -> dict:
        _lib.call("decon_nlcg_read", self.h, self._out, stream())
        o = list(self._out)
        return dict(lam=o[0], newton_stopped=bool(o[1]), newton_run=int(o[2]), sum_m=o[3],
                    sum_glogm=o[4], idiv_data=o[5], reg=o[6], rr=o[7], idiv=o[8], sum_f=o[9],
                    quad=(o[10], o[11]), gram=o[12:18])

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value and _lib._lib is not None:
            try:
                torch.cuda.synchronize()
                _lib._lib.decon_nlcg_destroy(h)
            except Exception:
                pass
            self.h = None


def _p(t):
    return None if t is None else _lib.ptr(t)


def _fwd(op, x):
    return to_device(op.forward(x))


def _adj(op, y):
    return to_device(op.adjoint(y))


def _model(blur_op, f, b: float):
    """m = K f + b (nlcg_mlx.py:86-90)."""
    kf = _fwd(blur_op, f)
    m = empty(kf.shape)
    _lib.call("decon_affine", _lib.ptr(kf), C.c_float(1.0), C.c_float(b), _lib.ptr(m), kf.numel(),
              stream())
    return m


def _square(s):
    f = empty(s.shape)
    _lib.call("decon_nlcg_init", _lib.ptr(s), None, _lib.ptr(f), s.numel(), 1, stream())
    return f


def _objective(sc, beta, use_reg):
    """phi = sum m - sum g ln max(m, eps) [+ beta ||C f||^2] (nlcg_mlx.py:93-102)."""
    val = sc["sum_m"] - sc["sum_glogm"]
    return val + beta * sc["reg"] if use_reg else val


def _use_reg(regularizer, reg_weight):
    return regularizer is not None and float(reg_weight) != 0.0


def _fused(reg, x) -> bool:
    """Hessian3D on a 3-D object: its Gram matrix and energy are evaluated on
    the fly (decon_nlcg_hess_*), the 6-component images are never stored."""
    return isinstance(reg, Hessian3D) and x.dim() == 3


def _energy(h, reg, x):
    """||C x||^2 into the handle's regulariser slot."""
    if _fused(reg, x):
        _lib.call("decon_nlcg_hess_energy", h.h, _lib.ptr(x), _lib.i64arr(tuple(x.shape)),
                  C.c_float(reg.r), stream())
    else:
        cx = _fwd(reg, x)
        _lib.call("decon_nlcg_energy", h.h, _lib.ptr(cx), cx.numel(), stream())


def nlcg_objective(s, blur_op, observed, background: float = 0.0, regularizer=None,
                   reg_weight: float = 0.0, eps: float = 1e-10) -> float:
    """phi(s) = sum(Kf) - sum(g ln(Kf + b)) + beta ||C f||^2, f = s^2 (nlcg_mlx.py:118-134)."""
    s = to_device(s)
    g = to_device(observed)
    use_reg = _use_reg(regularizer, reg_weight)
    h = _Scalars()
    f = _square(s)
    m = _model(blur_op, f, float(background))
    _lib.call("decon_nlcg_model", h.h, _lib.ptr(m), _lib.ptr(g), C.c_float(eps), None, g.numel(),
              stream())
    if use_reg:
        _energy(h, regularizer, f)
    return float(_objective(h.read(), float(reg_weight), use_reg))


def _gradient_parts(h, s, f, m, g, blur_op, regularizer, beta, use_reg, eps):
    w = empty(g.shape)
    _lib.call("decon_nlcg_model", h.h, _lib.ptr(m), _lib.ptr(g), C.c_float(eps), _lib.ptr(w),
              g.numel(), stream())
    ktw = _adj(blur_op, w)
    ctcf = None
    if use_reg:
        ctcf = _adj(regularizer, _fwd(regularizer, f))
    r = empty(s.shape)
    _lib.call("decon_nlcg_gradient", h.h, _lib.ptr(s), _lib.ptr(f), None, _lib.ptr(ktw), _p(ctcf),
              C.c_float(4.0 * beta), C.c_float(eps), _lib.ptr(r), s.numel(), stream())
    return r, ktw, ctcf


def nlcg_gradient(s, blur_op, observed, background: float = 0.0, regularizer=None,
                  reg_weight: float = 0.0, eps: float = 1e-10):
    """grad phi = 2 s K^T(1 - g/(Kf+b)) + 4 beta s C^T C f (nlcg_mlx.py:137-154).
    Returns ``(grad, (m, KTw, CtCf))``."""
    s = to_device(s)
    g = to_device(observed)
    beta = float(reg_weight)
    use_reg = _use_reg(regularizer, reg_weight)
    h = _Scalars()
    f = _square(s)
    m = _model(blur_op, f, float(background))
    r, ktw, ctcf = _gradient_parts(h, s, f, m, g, blur_op, regularizer, beta, use_reg, eps)
    grad = empty(r.shape)
    _lib.call("decon_affine", _lib.ptr(r), C.c_float(-1.0), C.c_float(0.0), _lib.ptr(grad), r.numel(),
              stream())
    return grad, (m, ktw, ctcf)


def nlcg_hessian_quadform(s, d, blur_op, observed, background: float = 0.0, regularizer=None,
                          reg_weight: float = 0.0, aux=None, eps: float = 1e-10) -> float:
    """<d, A(s) d> (Eq. 13) with one extra forward convolution (nlcg_mlx.py:157-194)."""
    s = to_device(s)
    d = to_device(d)
    g = to_device(observed)
    beta = float(reg_weight)
    use_reg = _use_reg(regularizer, reg_weight)
    if aux is None:
        _, aux = nlcg_gradient(s, blur_op, g, background, regularizer, reg_weight, eps)
    m, ktw, ctcf = aux
    h = _Scalars()
    sd = empty(s.shape)
    dd = empty(s.shape)
    _lib.call("decon_nlcg_products", h.h, 0, C.c_float(0.0), _lib.ptr(s), _lib.ptr(d), None, None,
              _lib.ptr(sd), _lib.ptr(dd), s.numel(), stream())
    ksd = _fwd(blur_op, sd)
    _lib.call("decon_nlcg_quad", h.h, _lib.ptr(g), _lib.ptr(m), _lib.ptr(ksd), g.numel(), _lib.ptr(ktw),
              _lib.ptr(d), d.numel(), C.c_float(eps), stream())
    q = h.read()["quad"]
    quad = 4.0 * q[0] + 2.0 * q[1]
    if use_reg:
        _energy(h, regularizer, sd)
        _lib.call("decon_nlcg_quad", h.h, _lib.ptr(g), _lib.ptr(m), _lib.ptr(ksd), g.numel(),
                  _lib.ptr(ctcf), _lib.ptr(d), d.numel(), C.c_float(eps), stream())
        sc = h.read()
        quad += 8.0 * beta * sc["reg"] + 4.0 * beta * sc["quad"][1]
    return float(quad)


def _products(h, mode, gamma, s, d, r):
    sd = empty(s.shape)
    dd = empty(s.shape)
    d_out = empty(s.shape) if mode == 1 else d
    _lib.call("decon_nlcg_products", h.h, mode, C.c_float(gamma), _lib.ptr(s), _lib.ptr(d), _p(r),
              _lib.ptr(d_out) if mode == 1 else None, _lib.ptr(sd), _lib.ptr(dd), s.numel(), stream())
    return d_out, sd, dd


def _line(h, s, d_sd_dd, f, cf, m, g, blur_op, regularizer, b, beta, use_reg, newton_iters, eps):
    """K(sd), K(dd) [, the regulariser's Gram matrix of C f, C(sd), C(dd); cf =
    C f when the images are materialised] and the Newton refinements."""
    _, sd, dd = d_sd_dd
    ksd = _fwd(blur_op, sd)
    kdd = _fwd(blur_op, dd)
    if use_reg:
        if _fused(regularizer, f):
            _lib.call("decon_nlcg_hess_gram", h.h, _lib.ptr(f), _lib.ptr(sd), _lib.ptr(dd),
                      _lib.i64arr(tuple(f.shape)), C.c_float(regularizer.r), stream())
        else:
            csd = _fwd(regularizer, sd)
            cdd = _fwd(regularizer, dd)
            _lib.call("decon_nlcg_gram", h.h, _lib.ptr(cf), _lib.ptr(csd), _lib.ptr(cdd), csd.numel(),
                      stream())
    _lib.call("decon_nlcg_newton", h.h, _lib.ptr(m), _lib.ptr(ksd), _lib.ptr(kdd), _lib.ptr(g),
              C.c_float(b), C.c_float(eps), C.c_double(beta), int(use_reg), int(newton_iters),
              g.numel(), stream())
    return ksd, kdd


def nlcg_step_length(s, d, f, m, blur_op, observed, background: float = 0.0, regularizer=None,
                     reg_weight: float = 0.0, newton_iters: int = 3, eps: float = 1e-10):
    """Exact step length along d by Newton-Raphson on the closed-form
    quadratic-in-lambda model K f(lambda) = Kss + 2 lambda K(sd) +
    lambda^2 K(dd) (nlcg_mlx.py:197-300).  Returns ``(lam, m_lam)``."""
    s, d, f, m = to_device(s), to_device(d), to_device(f), to_device(m)
    g = to_device(observed)
    b = float(background)
    beta = float(reg_weight)
    use_reg = _use_reg(regularizer, reg_weight)
    h = _Scalars()
    prods = _products(h, 0, 0.0, s, d, None)
    cf = _fwd(regularizer, f) if use_reg and not _fused(regularizer, f) else None
    ksd, kdd = _line(h, s, prods, f, cf, m, g, blur_op, regularizer, b, beta, use_reg, newton_iters, eps)
    m_lam = empty(g.shape)
    _lib.call("decon_nlcg_accept", h.h, _lib.ptr(m), _lib.ptr(ksd), _lib.ptr(kdd), _lib.ptr(g),
              C.c_float(b), C.c_float(eps), _lib.ptr(m_lam), None, g.numel(), None, None, None, None,
              0, stream())
    return float(h.read()["lam"]), m_lam


def i_divergence_between(f_prev, f_curr, eps: float = 1e-10) -> float:
    """sum f_k ln(f_k / f_{k+1}) - f_k + f_{k+1} (Eq. 17, nlcg_mlx.py:303-323)."""
    fp = to_device(f_prev)
    fc = to_device(f_curr)
    h = _Scalars()
    _lib.call("decon_nlcg_gradient", h.h, None, _lib.ptr(fc), _lib.ptr(fp), None, None, C.c_float(0.0),
              C.c_float(eps), None, fc.numel(), stream())
    return float(h.read()["idiv"])


def nlcg_with_operator(observed, blur_op, num_iter: int = 50, background: float = 0.0,
                       regularizer=None, reg_weight: float = 0.0, init=None,
                       callback: Optional[Callable] = None, eval_interval: int = 10,
                       slack: float = 1.0, tol: float = 1e-4, min_iter: int = 10,
                       restart_interval: Optional[int] = None, newton_iters: int = 3,
                       verbose: bool = False) -> NLCGResult:
    """Poisson-ML deconvolution by nonlinear CG with an exact Newton step
    length (nlcg_mlx.py:326-545).  ``restored`` is the full reconstruction
    domain; the stopping rules, loss logging and the steepest-descent fallback
    follow the reference."""
    g = to_device(observed)
    b = float(background)
    beta = float(reg_weight)
    use_reg = _use_reg(regularizer, reg_weight)
    reg = regularizer if use_reg else None
    eps = _EPS
    nd = g.numel()
    h = _Scalars()

    if init is None:
        dmb = empty(g.shape)
        _lib.call("decon_rl_data_floor", _lib.ptr(g), C.c_float(b), _lib.ptr(dmb), nd, stream())
        x0 = _adj(blur_op, dmb)
    else:
        x0 = to_device(init)
    s = empty(x0.shape)
    f = empty(x0.shape)
    _lib.call("decon_nlcg_init", _lib.ptr(x0), _lib.ptr(s), _lib.ptr(f), s.numel(), 0, stream())
    no = s.numel()
    m = _model(blur_op, f, b)
    if tuple(m.shape) != tuple(g.shape):
        raise ValueError(f"blur_op.forward produced {tuple(m.shape)}, observed is {tuple(g.shape)}")
    fused = use_reg and _fused(reg, f)
    cf = None
    if use_reg:
        if fused:
            _energy(h, reg, f)
        else:
            cf = _fwd(reg, f)
            _lib.call("decon_nlcg_energy", h.h, _lib.ptr(cf), cf.numel(), stream())
    r, _, _ = _gradient_parts(h, s, f, m, g, blur_op, reg, beta, use_reg, eps)
    sc = h.read()
    phi0 = _objective(sc, beta, use_reg)
    loss_cur = sc["idiv_data"] / nd
    rr = sc["rr"]

    def attempt(mode, gamma, d_in):
        """One trial step along d (mode 0) or r + gamma d (mode 1), carried
        through to the new gradient; None if rejected (nlcg_mlx.py:462-489)."""
        prods = _products(h, mode, gamma, s, d_in, r)
        ksd, kdd = _line(h, s, prods, f, cf, m, g, blur_op, reg, b, beta, use_reg, newton_iters, eps)
        d_used = prods[0]
        m_new = empty(g.shape)
        w_new = empty(g.shape)
        s_new = empty(s.shape)
        f_new = empty(s.shape)
        _lib.call("decon_nlcg_accept", h.h, _lib.ptr(m), _lib.ptr(ksd), _lib.ptr(kdd), _lib.ptr(g),
                  C.c_float(b), C.c_float(eps), _lib.ptr(m_new), _lib.ptr(w_new), nd, _lib.ptr(s),
                  _lib.ptr(d_used), _lib.ptr(s_new), _lib.ptr(f_new), no, stream())
        cf_new = ctcf_new = None
        if use_reg:
            if fused:
                _energy(h, reg, f_new)
                ctcf_new = _adj(reg, _fwd(reg, f_new))
            else:
                cf_new = _fwd(reg, f_new)
                _lib.call("decon_nlcg_energy", h.h, _lib.ptr(cf_new), cf_new.numel(), stream())
                ctcf_new = _adj(reg, cf_new)
        ktw = _adj(blur_op, w_new)
        r_new = empty(s.shape)
        _lib.call("decon_nlcg_gradient", h.h, _lib.ptr(s_new), _lib.ptr(f_new), _lib.ptr(f),
                  _lib.ptr(ktw), _p(ctcf_new), C.c_float(4.0 * beta), C.c_float(eps), _lib.ptr(r_new),
                  no, stream())
        st = h.read()
        lam = st["lam"]
        if not math.isfinite(lam):
            return None
        phi = _objective(st, beta, use_reg)
        if not phi < phi0:
            return None
        return dict(d=d_used, s=s_new, f=f_new, m=m_new, r=r_new, cf=cf_new, lam=lam, phi=phi,
                    loss=st["idiv_data"] / nd, rr=st["rr"], idiv=st["idiv"], sum_f=st["sum_f"])

    loss_history: list = []
    window: list = []
    converged = False
    d_prev = None
    gamma = 0.0
    k = 0
    for k in range(num_iter):
        if k == 0:
            step = attempt(0, 0.0, r)  # d is r: no steepest-descent retry
        else:
            step = attempt(1, gamma, d_prev)
            if step is None:
                step = attempt(0, 0.0, r)
        if step is None:
            converged = True
            loss_history.append(loss_cur)
            break
        s, f, m, r, cf = step["s"], step["f"], step["m"], step["r"], step["cf"]
        d_prev = step["d"]
        phi0 = step["phi"]
        rr_new = step["rr"]
        gamma = rr_new / rr if rr > eps else 0.0
        if restart_interval is not None and (k + 1) % restart_interval == 0:
            gamma = 0.0
        rr = rr_new
        loss = step["loss"]
        loss_cur = loss
        logged = k % eval_interval == 0 or k == num_iter - 1
        if logged:
            loss_history.append(loss)
            if verbose:
                print(f"  Iter {k:4d}: mean I-div = {loss:.6g}, lambda = {step['lam']:.4g}, "
                      f"gamma = {gamma:.4g}")
        rel = step["idiv"] / max(step["sum_f"], eps)
        window.append(rel)
        if len(window) > 5:
            window.pop(0)
        rel_avg = sum(window) / len(window)
        stop = False
        reason = None
        if callback is not None:
            stop = bool(callback(k, f))
        ready = not stop and k + 1 >= min_iter
        if ready and not use_reg and slack > 0.0 and loss <= 0.5 * slack:
            converged = stop = True
            reason = "discrepancy principle"
        elif ready and tol > 0.0 and len(window) == 5 and rel_avg < tol:
            converged = stop = True
            reason = "relative divergence change (Eq. 17)"
        if stop:
            if not logged:
                loss_history.append(loss)
            if verbose and reason is not None:
                print(f"  Stopped at iter {k}: {reason}")
            break

    x = _square(s)
    pred = _model(blur_op, x, b)
    return NLCGResult(restored=x, pred=pred, iterations=k + 1, loss_history=loss_history,
                      converged=converged, background=b, full_shape=tuple(x.shape), valid_slices=None)


def nlcg_solver(num_iter: int = 50, background: float = 0.0, regularizer=None,
                reg_weight: float = 0.0, init_value: Optional[float] = None, **nlcg_kwargs: Any):
    """``solve(data, model)`` adapter for tile processing (nlcg_mlx.py:548-588)."""

    def solve(data, model):
        init = None
        if init_value is not None:
            init = fill(empty(model.padded_shape), float(init_value))
        result = nlcg_with_operator(observed=data, blur_op=model.op, num_iter=num_iter,
                                    background=background, regularizer=regularizer,
                                    reg_weight=reg_weight, init=init, **nlcg_kwargs)
        return result.restored[model.valid_slices].detach().cpu().numpy()

    return solve
