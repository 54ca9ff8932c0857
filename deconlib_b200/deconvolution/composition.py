"""Operator protocol, composition and the NumPy adapter.

Mirrors deconlib's ``deconvolution/composition.py`` (LinearOperator :25-49,
Compose :52-106, compose :109-122, as_numpy_op :140-159): same names,
argument meaning and error text.  Arrays are CUDA ``torch.Tensor`` float32.
"""

from __future__ import annotations

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

    def forward(self, x):
        return self.outer.forward(self.inner.forward(x))

    def adjoint(self, y):
        return self.inner.adjoint(self.outer.adjoint(y))

    def __call__(self, x):
        return self.forward(x)


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
