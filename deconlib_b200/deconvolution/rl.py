"""Richardson-Lucy deconvolution on the B200.

Mirrors deconlib's ``deconvolution/rl_mlx.py``: RLResult (:35-55),
poisson_i_divergence (:58-80), richardson_lucy_with_operator (:83-185) and
richardson_lucy_solver (:188-226).

Two device paths, both through libdecon_b200:
  * ``blur_op`` is a LinearFFTConvolver: each iteration is two pruned
    convolutions whose last FFT pass carries the RL arithmetic: the forward
    pass writes ``y / max(Ax + b, 1e-10)``, the adjoint pass writes the
    updated ``x``; the I-divergence of iteration k is summed (FP64) inside the
    forward pass of iteration k + 1, so logging costs no extra convolution.
  * any other operator (compositions with Crop / Pad / resampling, ...):
    ``blur_op.forward`` / ``adjoint`` plus fused element-wise RL kernels.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Any, Callable, Optional, Tuple

import numpy as np
import torch

from .. import _lib
from ._device import empty, fill, stream, to_device, workspace
from .linops import LinearFFTConvolver

__all__ = ["RLResult", "RLRunner", "poisson_i_divergence", "richardson_lucy_with_operator",
           "richardson_lucy_solver"]


@dataclass
class RLResult:
    """Result of Richardson-Lucy deconvolution (rl_mlx.py:35-55)."""

    restored: Any
    pred: Any
    iterations: int
    loss_history: list
    background: float = 0.0
    full_shape: Optional[Tuple[int, ...]] = None
    valid_slices: Optional[Tuple[slice, ...]] = None


def poisson_i_divergence(observed, model, eps: float = 1e-6) -> float:
    """Mean Poisson I-divergence, FP64 accumulation on the device (rl_mlx.py:58-80)."""
    y = to_device(observed)
    m = to_device(model)
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    _lib.call("decon_rl_ratio", _lib.ptr(m), _lib.ptr(y), C.c_float(0.0), None, y.numel(),
              _lib.ptr(out), _lib.ptr(workspace()), stream())
    return float(out.item()) / y.numel()


def _want_loss(k, num_iter, eval_interval):
    return k % eval_interval == 0 or k == num_iter - 1


def richardson_lucy_with_operator(observed, blur_op, num_iter: int = 50, background: float = 0.0,
                                  init=None, callback: Optional[Callable] = None,
                                  eval_interval: int = 10, verbose: bool = False) -> RLResult:
    """Multiplicative RL with sensitivity ``A^T 1`` and active-support mask
    (rl_mlx.py:83-185).  Returns CUDA tensors in ``restored`` / ``pred``."""
    y = to_device(observed)
    bg = float(background)
    if isinstance(blur_op, LinearFFTConvolver) and tuple(y.shape) == blur_op.signal_shape:
        return _rl_fused(y, blur_op, num_iter, bg, init, callback, eval_interval, verbose)
    return _rl_generic(y, blur_op, num_iter, bg, init, callback, eval_interval, verbose)


class RLRunner:
    """Fused RL iterations of one job on a LinearFFTConvolver, split into
    set-up / ``iterate`` / ``finish`` so that a caller (the serving loop) can
    queue iterations of several jobs on their own streams and interleave them.

    Everything is queued on the stream that is current at construction; no
    call synchronises before ``finish``.  The I-divergence of iteration k is
    summed inside the forward pass of iteration k + 1 (and of the final
    prediction), so loss logging costs no extra convolution."""

    def __init__(self, observed, op: LinearFFTConvolver, num_iter: int = 50,
                 background: float = 0.0, init=None, eval_interval: int = 10):
        self.s = stream()
        self.y = to_device(observed)
        self.op, self.plan = op, op.plan
        self.bg = float(background)
        self.num_iter, self.eval_interval = int(num_iter), int(eval_interval)
        self.n = self.y.numel()
        self.x = empty(self.y.shape)
        self.sens = empty(self.y.shape)
        self.ratio = empty(self.y.shape)
        self.pred = empty(self.y.shape)
        x_init = to_device(init) if init is not None else None
        _lib.call("decon_rl_setup", self.plan, _lib.ptr(self.y), C.c_float(self.bg),
                  _lib.ptr(x_init), _lib.ptr(self.x), _lib.ptr(self.sens), self.s)
        self.losses_dev = torch.zeros(max(self.num_iter, 1), dtype=torch.float64, device="cuda")
        self.loss_idx = []
        self.k = 0

    def iterate(self) -> bool:
        """Queue iteration k; returns False once all iterations are queued."""
        if self.k >= self.num_iter:
            return False
        prev = self.k - 1
        lp = None
        if prev >= 0 and _want_loss(prev, self.num_iter, self.eval_interval):
            lp = _lib.ptr(self.losses_dev[prev:])
            self.loss_idx.append(prev)
        _lib.call("decon_rl_iteration", self.plan, _lib.ptr(self.y), C.c_float(self.bg),
                  _lib.ptr(self.sens), _lib.ptr(self.x), _lib.ptr(self.ratio), lp, self.s)
        self.k += 1
        return self.k < self.num_iter

    def finish(self) -> RLResult:
        """Queue the final prediction (with the last iteration's loss) and
        read the loss history (synchronises this runner's stream)."""
        last = self.k - 1
        lp = None
        if last >= 0:
            lp = _lib.ptr(self.losses_dev[last:])
            self.loss_idx.append(last)
        _lib.call("decon_rl_predict", self.plan, _lib.ptr(self.y), C.c_float(self.bg),
                  _lib.ptr(self.x), _lib.ptr(self.pred), lp, self.s)
        vals = self.losses_dev.cpu().numpy()
        losses = [float(vals[i]) / self.n for i in self.loss_idx]
        return RLResult(restored=self.x, pred=self.pred, iterations=self.k, loss_history=losses,
                        background=self.bg, full_shape=tuple(self.x.shape), valid_slices=None)


def _rl_fused(y, op, num_iter, bg, init, callback, eval_interval, verbose):
    if callback is None and not verbose:
        r = RLRunner(y, op, num_iter, bg, init, eval_interval)
        while r.iterate():
            pass
        return r.finish()
    plan = op.plan
    n = y.numel()
    x = empty(y.shape)
    sens = empty(y.shape)
    ratio = empty(y.shape)
    x_init = to_device(init) if init is not None else None
    _lib.call("decon_rl_setup", plan, _lib.ptr(y), C.c_float(bg), _lib.ptr(x_init), _lib.ptr(x),
              _lib.ptr(sens), stream())
    losses_dev = torch.zeros(max(num_iter, 1), dtype=torch.float64, device="cuda")
    pred = empty(y.shape)
    k = -1
    losses = []
    for k in range(num_iter):
        _lib.call("decon_rl_iteration", plan, _lib.ptr(y), C.c_float(bg), _lib.ptr(sens),
                  _lib.ptr(x), _lib.ptr(ratio), None, stream())
        if _want_loss(k, num_iter, eval_interval):
            _lib.call("decon_rl_predict", plan, _lib.ptr(y), C.c_float(bg), _lib.ptr(x),
                      _lib.ptr(ratio), _lib.ptr(losses_dev[k:]), stream())
            loss = float(losses_dev[k].item()) / n
            losses.append(loss)
            if verbose:
                print(f"  Iter {k:4d}: mean I-div = {loss:.6g}")
        if callback is not None and callback(k, x):
            break
    _lib.call("decon_rl_predict", plan, _lib.ptr(y), C.c_float(bg), _lib.ptr(x), _lib.ptr(pred),
              None, stream())
    return RLResult(restored=x, pred=pred, iterations=k + 1, loss_history=losses,
                    background=bg, full_shape=tuple(x.shape), valid_slices=None)


def _rl_generic(y, op, num_iter, bg, init, callback, eval_interval, verbose):
    n = y.numel()
    s = stream()
    ws = workspace()
    if init is None:
        dmb = empty(y.shape)
        _lib.call("decon_rl_data_floor", _lib.ptr(y), C.c_float(bg), _lib.ptr(dmb), n, s)
        x = to_device(op.adjoint(dmb)).clone()
    else:
        x = to_device(init).clone()
    ones = fill(empty(y.shape), 1.0)
    sens = to_device(op.adjoint(ones)).clone()
    if sens.shape != x.shape:
        raise ValueError(f"blur_op.adjoint produced {tuple(sens.shape)}, init is {tuple(x.shape)}")
    # x = where(active, max(x, 1e-6), 0); sens = where(active, sens, 0)
    _lib.call("decon_rl_mask", _lib.ptr(x), _lib.ptr(sens), x.numel(), _lib.ptr(ws), s)
    losses = []
    loss_t = torch.empty(1, dtype=torch.float64, device="cuda")
    ratio = empty(y.shape)
    k = -1
    for k in range(num_iter):
        model = to_device(op.forward(x))
        _lib.call("decon_rl_ratio", _lib.ptr(model), _lib.ptr(y), C.c_float(bg), _lib.ptr(ratio), n,
                  None, None, s)
        corr = to_device(op.adjoint(ratio))
        _lib.call("decon_rl_update", _lib.ptr(x), _lib.ptr(corr), _lib.ptr(sens), x.numel(), s)
        if _want_loss(k, num_iter, eval_interval):
            model = to_device(op.forward(x))
            _lib.call("decon_rl_ratio", _lib.ptr(model), _lib.ptr(y), C.c_float(bg), None, n,
                      _lib.ptr(loss_t), _lib.ptr(ws), s)
            loss = float(loss_t.item()) / n
            losses.append(loss)
            if verbose:
                print(f"  Iter {k:4d}: mean I-div = {loss:.6g}")
        if callback is not None and callback(k, x):
            break
    model = to_device(op.forward(x))
    pred = empty(model.shape)
    _lib.call("decon_affine", _lib.ptr(model), C.c_float(1.0), C.c_float(bg), _lib.ptr(pred),
              model.numel(), s)
    return RLResult(restored=x, pred=pred, iterations=k + 1, loss_history=losses, background=bg,
                    full_shape=tuple(x.shape), valid_slices=None)


def richardson_lucy_solver(num_iter: int = 50, background: float = 0.0,
                           init_value: Optional[float] = None, **rl_kwargs: Any):
    """``solve(data, model)`` adapter for tile processing (rl_mlx.py:188-226)."""

    def solve(data, model):
        init = None
        if init_value is not None:
            init = fill(empty(model.padded_shape), float(init_value))
        result = richardson_lucy_with_operator(observed=data, blur_op=model.op, num_iter=num_iter,
                                               background=background, init=init, **rl_kwargs)
        return result.restored[model.valid_slices].detach().cpu().numpy()

    return solve
