"""Operator protocol, composition and the NumPy adapter.

Mirrors deconlib's ``deconvolution/composition.py`` (LinearOperator :25-49,
Compose :52-106, compose :109-122, as_numpy_op :140-159): same names,
argument meaning and error text.  Arrays are CUDA ``torch.Tensor`` float32.
"""

from __future__ import annotations

import os
from typing import Any, Callable, Protocol, Tuple, runtime_checkable

import numpy as np
import torch

__all__ = ["LinearOperator", "Compose", "compose", "as_numpy_op"]


@runtime_checkable
class LinearOperator(Protocol):
    """forward / adjoint / __call__ plus an ``operator_norm_sq`` bound;
    optional ``in_shape`` / ``out_shape`` (composition.py:25-49)."""

    operator_norm_sq: float

    def forward(self, x: Any) -> Any: ...

    def adjoint(self, y: Any) -> Any: ...

    def __call__(self, x: Any) -> Any: ...


class Compose:
    """``Compose(A, B)(x) = A(B(x))``; adjoint reversed; norm bound = product.

    Shapes declared by both operators are checked at construction
    (composition.py:67-97)."""

    def __init__(self, outer: LinearOperator, inner: LinearOperator):
        outer_in = getattr(outer, "in_shape", None)
        inner_out = getattr(inner, "out_shape", None)
        if outer_in is not None and inner_out is not None and tuple(outer_in) != tuple(inner_out):
            hint = ""
            if "LinearFFTConvolver" in (type(outer).__name__, type(inner).__name__):
                hint = (
                    " Note: LinearFFTConvolver pads internally for wrap-free "
                    "convolution — its input and output are both signal_shape; "
                    "do not pad its input or output yourself."
                )
            raise ValueError(
                f"Cannot compose {type(outer).__name__} after "
                f"{type(inner).__name__}: {type(outer).__name__} expects "
                f"input of shape {tuple(outer_in)} but "
                f"{type(inner).__name__} produces {tuple(inner_out)}.{hint}"
            )
        self.outer = outer
        self.inner = inner
        self.in_shape = getattr(inner, "in_shape", None)
        self.out_shape = getattr(outer, "out_shape", None)
        self.operator_norm_sq = float(outer.operator_norm_sq * inner.operator_norm_sq)
        # DECON_NO_DOWN2=1 applies the two operators in turn (same values;
        # for measurement)
        self._down2 = None if os.environ.get("DECON_NO_DOWN2") == "1" else _down2_plan(outer, inner)

    def forward(self, x):
        if self._down2 is not None:
            y = self._fused("decon_conv_forward_down2", x, self._down2[1], self._down2[2])
            if y is not None:
                return y
        return self.outer.forward(self.inner.forward(x))

    def adjoint(self, y):
        if self._down2 is not None:
            x = self._fused("decon_conv_adjoint_up2", y, self._down2[2], self._down2[1])
            if x is not None:
                return x
        return self.inner.adjoint(self.outer.adjoint(y))

    def _fused(self, name, x, in_shape, out_shape):
        """The recognised composition FractionalAreaDownsample(2) o
        LinearFFTConvolver as one pass sequence (the area sum fused into the
        convolution's last FFT pass, its adjoint into the first); the same
        float32 values as applying the two operators in turn.  None if the
        plan cannot (the caller then applies them in turn)."""
        from .. import _lib
        from ._device import empty, stream, to_device

        x = to_device(x)
        if tuple(x.shape) != in_shape:
            return None
        out = empty(out_shape)
        st = getattr(_lib.load(), name)(self._down2[0].plan, _lib.ptr(x), _lib.ptr(out), stream())
        if st == _lib.ERR_UNSUPPORTED:
            self._down2 = None
            return None
        _lib.check(st)
        return out

    def __call__(self, x):
        return self.forward(x)


def _down2_plan(outer, inner):
    """(conv, N, N / 2) when ``outer`` is a FractionalAreaDownsample that
    halves every axis of a 3-D LinearFFTConvolver ``inner`` exactly
    (n_large = 2 n_small, so the band weights are 1 and 0), else None."""
    from .core_operators import FractionalAreaDownsample
    from .linops import LinearFFTConvolver

    if not (isinstance(outer, FractionalAreaDownsample) and isinstance(inner, LinearFFTConvolver)):
        return None
    n = tuple(inner.signal_shape)
    if len(n) != 3 or any(v % 2 for v in n) or inner.fft_shape[2] % 2:
        return None
    pairs = outer.axis_pairs(n)
    if sorted((a % 3, nl, ns) for a, nl, ns in pairs) != [(a, n[a], n[a] // 2) for a in range(3)]:
        return None
    return inner, n, tuple(v // 2 for v in n)


def compose(*ops: LinearOperator) -> LinearOperator:
    """``compose(A, B, C)(x) = A(B(C(x)))`` (composition.py:109-122)."""
    if not ops:
        raise ValueError("compose() requires at least one operator")
    if len(ops) == 1:
        return ops[0]
    result: LinearOperator = ops[-1]
    for op in reversed(ops[:-1]):
        result = Compose(op, result)
    return result


def flatten(op) -> list:
    """The chain of a composition in application order (innermost first)."""
    if isinstance(op, Compose):
        return flatten(op.inner) + flatten(op.outer)
    return [op]


def _call_numpy(fn: Callable, x: np.ndarray) -> np.ndarray:
    """Call an operator method with a NumPy array and return a NumPy array
    (composition.py:125-137): the array itself first, so pure NumPy operators
    take part too; this package's operators copy it to the device and return
    a CUDA tensor, which is read back.  A ``TypeError`` retries with the
    array on the device."""
    x_np = np.ascontiguousarray(x)
    try:
        out = fn(x_np)
    except TypeError:
        from ._device import to_device

        out = fn(to_device(x_np))
    if isinstance(out, torch.Tensor):
        return out.detach().cpu().numpy()
    return np.asarray(out)


def as_numpy_op(op: LinearOperator) -> Tuple[Callable[[np.ndarray], np.ndarray],
                                             Callable[[np.ndarray], np.ndarray]]:
    """``(R, Rt)`` NumPy callables for external solvers (composition.py:140-159)."""

    def R(x: np.ndarray) -> np.ndarray:
        return _call_numpy(op.forward, x)

    def Rt(y: np.ndarray) -> np.ndarray:
        return _call_numpy(op.adjoint, y)

    return R, Rt
