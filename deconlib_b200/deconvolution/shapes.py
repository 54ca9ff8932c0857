"""Shape and padding helpers across data / visible / padded grids.

Mirrors deconlib's ``deconvolution/shapes.py``: compute_visible_shape
(:31-98), compute_padded_shape (:101-164), get_valid_slices (:167-224).
Host-only integer arithmetic.
"""

from __future__ import annotations

from typing import Optional, Tuple, Union

__all__ = ["compute_visible_shape", "compute_padded_shape", "get_valid_slices"]


def _per_axis(value, ndim, name):
    if isinstance(value, (int, float)):
        return (float(value),) * ndim
    out = tuple(float(v) for v in value)
    if len(out) != ndim:
        raise ValueError(f"{name} has {len(out)} elements, expected {ndim} to match data_shape")
    return out


def compute_visible_shape(data_shape: Tuple[int, ...],
                          bin_factor: Union[float, Tuple[float, ...]] = 1.0) -> Tuple[int, ...]:
    """Visible grid of a data grid: round(data_dim / bin_factor) per axis (shapes.py:31-98)."""
    data_shape = tuple(int(s) for s in data_shape)
    f = _per_axis(bin_factor, len(data_shape), "bin_factor")
    return tuple(int(round(d / b)) for d, b in zip(data_shape, f))


def compute_padded_shape(signal_shape: Tuple[int, ...], kernel_shape: Tuple[int, ...], *,
                         min_pad: Optional[Union[int, Tuple[Optional[int], ...]]] = None):
    """Wrap-free padding M - 1 per axis (or the ``min_pad`` override), split
    floor(half) before / rest after (shapes.py:101-164).

    Returns (padded_shape, ((before, after), ...))."""
    s = tuple(int(v) for v in signal_shape)
    k = tuple(int(v) for v in kernel_shape)
    if len(k) != len(s):
        raise ValueError(f"kernel_shape has {len(k)} dimensions, expected {len(s)} to match "
                         "signal_shape")
    if min_pad is None:
        over = (None,) * len(s)
    elif isinstance(min_pad, int):
        over = (min_pad,) * len(s)
    else:
        over = tuple(min_pad)
    padded, pads = [], []
    for n, m, o in zip(s, k, over):
        total = (m - 1) if o is None else int(o)
        before = total // 2
        pads.append((before, total - before))
        padded.append(n + total)
    return tuple(padded), tuple(pads)


def get_valid_slices(padded_shape: Tuple[int, ...], signal_shape: Tuple[int, ...],
                     padding=None) -> Tuple[slice, ...]:
    """Slices of the signal region inside a padded array (shapes.py:167-224);
    without ``padding`` the padding is taken as floor-half before."""
    p = tuple(int(v) for v in padded_shape)
    s = tuple(int(v) for v in signal_shape)
    if len(s) != len(p):
        raise ValueError(f"padded_shape has {len(p)} dimensions, but signal_shape has {len(s)} "
                         "dimensions. Both must have the same ndim.")
    if padding is None:
        padding = tuple(((a - b) // 2, (a - b) - (a - b) // 2) for a, b in zip(p, s))
    return tuple(slice(before, n - after) for n, (before, after) in zip(p, padding))
