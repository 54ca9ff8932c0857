"""CPU oracle for the nonlinear conjugate-gradient Poisson solver.

TEST INFRASTRUCTURE ONLY.  The checker that the CUDA NLCG path is compared
against; only ``tests/`` may import it.

A NumPy restatement of deconlib's ``nlcg_mlx.py`` (Schaefer, Schuster & Herz
2001 objective with f = s^2, Fletcher-Reeves directions, and the exact
Newton-Raphson step length of Valdimarsson & Preza's COSM).  Every routine
takes a ``dtype``: float32 follows the reference's device precision (its sums
are float32 reductions), float64 gives the double-precision oracle.  The
operators are the oracle's own (``oracle.ops``), called through
``forward`` / ``adjoint``.

Parity pin: ``tests/test_oracle_golden.py::test_nlcg`` checks it against
fixtures written by the reference's own source (``tests/golden/make_golden.py``).
"""

from __future__ import annotations

from typing import Optional

import numpy as np

from .solvers import poisson_i_divergence


def _sum(a):
    return a.sum(dtype=a.dtype)


def _objective_from_m(m, g, f, reg, beta, eps):
    """nlcg_mlx.py:96-102."""
    val = _sum(m) - _sum(g * np.log(np.maximum(m, eps)))
    if reg is not None and beta != 0.0:
        cf = reg.forward(f)
        val = val + m.dtype.type(beta) * _sum(cf * cf)
    return float(val)


def _gradient_from_m(s, f, m, g, blur_op, reg, beta, eps):
    """nlcg_mlx.py:105-115: grad = 2 s K^T(1 - g/m) + 4 beta s C^T C f."""
    t = s.dtype.type
    w = t(1.0) - g / np.maximum(m, eps)
    ktw = blur_op.adjoint(w)
    grad = t(2.0) * s * ktw
    ctcf = None
    if reg is not None and beta != 0.0:
        ctcf = reg.adjoint(reg.forward(f))
        grad = grad + t(4.0 * beta) * s * ctcf
    return grad, (m, ktw, ctcf)


def nlcg_objective(s, blur_op, observed, background=0.0, regularizer=None, reg_weight=0.0,
                   eps=1e-10, dtype=np.float32):
    """nlcg_mlx.py:118-134."""
    t = np.dtype(dtype).type
    s = np.asarray(s).astype(dtype)
    f = s * s
    m = blur_op.forward(f) + t(background)
    return _objective_from_m(m, np.asarray(observed).astype(dtype), f, regularizer, reg_weight, t(eps))


def nlcg_gradient(s, blur_op, observed, background=0.0, regularizer=None, reg_weight=0.0,
                  eps=1e-10, dtype=np.float32):
    """nlcg_mlx.py:137-154."""
    t = np.dtype(dtype).type
    s = np.asarray(s).astype(dtype)
    f = s * s
    m = blur_op.forward(f) + t(background)
    return _gradient_from_m(s, f, m, np.asarray(observed).astype(dtype), blur_op, regularizer,
                            reg_weight, t(eps))


def nlcg_hessian_quadform(s, d, blur_op, observed, background=0.0, regularizer=None, reg_weight=0.0,
                          aux=None, eps=1e-10, dtype=np.float32):
    """<d, A(s) d> with one extra forward convolution (nlcg_mlx.py:157-194)."""
    t = np.dtype(dtype).type
    s = np.asarray(s).astype(dtype)
    d = np.asarray(d).astype(dtype)
    g = np.asarray(observed).astype(dtype)
    if aux is None:
        _, aux = nlcg_gradient(s, blur_op, g, background, regularizer, reg_weight, eps, dtype)
    m, ktw, ctcf = aux
    sd = s * d
    ksd = blur_op.forward(sd)
    quad = t(4.0) * _sum((g / np.maximum(m * m, t(eps))) * (ksd * ksd)) + t(2.0) * _sum(ktw * (d * d))
    if regularizer is not None and reg_weight != 0.0:
        csd = regularizer.forward(sd)
        quad = quad + t(8.0 * reg_weight) * _sum(csd * csd) + t(4.0 * reg_weight) * _sum(ctcf * (d * d))
    return float(quad)


def nlcg_step_length(s, d, f, m, blur_op, observed, background=0.0, regularizer=None,
                     reg_weight=0.0, newton_iters=3, eps=1e-10, dtype=np.float32):
    """Exact step length by Newton-Raphson on phi(s + lam d), using that
    K f(lam) = Kss + 2 lam K(sd) + lam^2 K(dd) is exactly quadratic in lam
    (nlcg_mlx.py:197-300).  Returns (lam, m_lam)."""
    t = np.dtype(dtype).type
    g = np.asarray(observed).astype(dtype)
    b = t(background)
    beta = float(reg_weight)
    use_reg = regularizer is not None and beta != 0.0
    eps_t = t(eps)
    kss = m - b
    ksd = blur_op.forward(s * d)
    kdd = blur_op.forward(d * d)
    if use_reg:
        cf0 = regularizer.forward(f)
        csd = regularizer.forward(s * d)
        cdd = regularizer.forward(d * d)
    lam = 0.0
    for _ in range(newton_iters):
        m_lam = np.maximum(kss + t(2.0 * lam) * ksd + t(lam * lam) * kdd + b, eps_t)
        ksd_lam = ksd + t(lam) * kdd
        w_lam = t(1.0) - g / m_lam
        dphi1 = t(2.0) * _sum(ksd_lam * w_lam)
        dphi2 = t(2.0) * _sum(kdd * w_lam) + t(4.0) * _sum(g * (ksd_lam * ksd_lam) / (m_lam * m_lam))
        if use_reg:
            u = cf0 + t(2.0 * lam) * csd + t(lam * lam) * cdd
            csd_lam = csd + t(lam) * cdd
            dphi1 = dphi1 + t(4.0 * beta) * _sum(u * csd_lam)
            dphi2 = dphi2 + t(8.0 * beta) * _sum(csd_lam * csd_lam) + t(4.0 * beta) * _sum(u * cdd)
        dphi1 = float(dphi1)
        dphi2 = float(dphi2)
        if not np.isfinite(dphi2) or abs(dphi2) < eps:
            break
        lam = lam - dphi1 / dphi2
        if not np.isfinite(lam):
            break
    m_lam = kss + t(2.0 * lam) * ksd + t(lam * lam) * kdd + b
    return lam, m_lam


def i_divergence_between(f_prev, f_curr, eps=1e-10):
    """sum f_k ln(f_k / f_{k+1}) - f_k + f_{k+1} (nlcg_mlx.py:303-323)."""
    t = f_prev.dtype.type
    fp = np.maximum(f_prev, t(eps))
    fc = np.maximum(f_curr, t(eps))
    return float(_sum(f_prev * (np.log(fp) - np.log(fc)) - f_prev + f_curr))


def nlcg_with_operator(observed, blur_op, num_iter=50, background=0.0, regularizer=None,
                       reg_weight=0.0, init=None, callback=None, eval_interval=10, slack=1.0,
                       tol=1e-4, min_iter=10, restart_interval: Optional[int] = None,
                       newton_iters=3, dtype=np.float32):
    """The solver loop of nlcg_mlx.py:326-545.  Returns a dict with the
    NLCGResult fields."""
    t = np.dtype(dtype).type
    g = np.asarray(observed).astype(dtype)
    eps = 1e-10
    eps_t = t(eps)
    b = t(background)
    beta = float(reg_weight)
    use_reg = regularizer is not None and beta != 0.0
    dmb = np.maximum(g - b, t(1e-6))
    if init is None:
        f0 = np.maximum(blur_op.adjoint(dmb), t(1e-6))
    else:
        f0 = np.maximum(np.asarray(init).astype(dtype), t(1e-6))
    s = np.sqrt(f0)
    reg = regularizer if use_reg else None
    f = s * s
    m = blur_op.forward(f) + b
    grad, aux = _gradient_from_m(s, f, m, g, blur_op, reg, beta, eps_t)
    r = -grad
    d = r
    rr = float(_sum(r * r))
    loss_history = []
    window = []
    converged = False
    k = 0

    def step(direction, phi0):
        lam, m_lam = nlcg_step_length(s, direction, f, aux[0], blur_op, g, b, reg, beta,
                                      newton_iters=newton_iters, eps=eps, dtype=dtype)
        if not np.isfinite(lam):
            return None
        s_new = s + t(lam) * direction
        f_new = s_new * s_new
        if _objective_from_m(m_lam, g, f_new, reg, beta, eps_t) >= phi0:
            return None
        return s_new, f_new, m_lam, lam

    for k in range(num_iter):
        phi0 = _objective_from_m(aux[0], g, f, reg, beta, eps_t)
        st = step(d, phi0)
        if st is None and d is not r:
            d = r
            st = step(d, phi0)
        if st is None:
            converged = True
            loss_history.append(poisson_i_divergence(g, aux[0]))
            break
        f_prev = f
        s, f, m, lam = st
        grad, aux = _gradient_from_m(s, f, m, g, blur_op, reg, beta, eps_t)
        r_new = -grad
        rr_new = float(_sum(r_new * r_new))
        gamma = rr_new / rr if rr > eps else 0.0
        if restart_interval is not None and (k + 1) % restart_interval == 0:
            gamma = 0.0
        d = r_new + t(gamma) * d
        r = r_new
        rr = rr_new
        loss = poisson_i_divergence(g, m)
        logged = k % eval_interval == 0 or k == num_iter - 1
        if logged:
            loss_history.append(loss)
        rel = i_divergence_between(f_prev, f) / max(float(_sum(f)), eps)
        window.append(rel)
        if len(window) > 5:
            window.pop(0)
        rel_avg = sum(window) / len(window)
        stop = False
        if callback is not None:
            stop = bool(callback(k, f))
        ready = not stop and k + 1 >= min_iter
        if ready and not use_reg and slack > 0.0 and loss <= 0.5 * slack:
            converged = True
            stop = True
        elif ready and tol > 0.0 and len(window) == 5 and rel_avg < tol:
            converged = True
            stop = True
        if stop:
            if not logged:
                loss_history.append(loss)
            break
    x = s * s
    pred = blur_op.forward(x) + b
    return dict(restored=x, pred=pred, iterations=k + 1, loss_history=loss_history,
                converged=converged, background=float(background), full_shape=tuple(x.shape))
