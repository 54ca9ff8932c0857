"""Pad, Crop and fractional-area resampling on the device.

Mirrors deconlib's ``deconvolution/core_operators.py``: Pad (:29-59), Crop
(:62-137), the banded overlap weights (:151-202) and their gather + weighted
sum (:205-219), FractionalAreaDownsample (:222-352) and FractionalAreaUpsample
(:355-450).  Same constructor arguments, attributes and ``ValueError`` text;
arrays are CUDA float32 tensors.  Pad/Crop run one window-copy kernel,
resampling one banded kernel per axis (``decon_window_copy``,
``decon_banded_axis``).
"""

from __future__ import annotations

import math
from typing import Tuple, Union

import numpy as np
import torch

from .. import _lib
from ._device import empty, stream, to_device

__all__ = ["Pad", "Crop", "FractionalAreaDownsample", "FractionalAreaUpsample"]


def _window(src: torch.Tensor, src_start, dst_shape, dst_start, ext) -> torch.Tensor:
    nd = src.dim()
    if nd > 4:
        raise ValueError("Pad/Crop support arrays of at most 4 dimensions")
    out = empty(dst_shape)
    if out.numel() == 0:
        return out
    _lib.call("decon_window_copy", _lib.ptr(src), _lib.i64arr(src.shape), _lib.i64arr(src_start),
              _lib.ptr(out), _lib.i64arr(dst_shape), _lib.i64arr(dst_start), _lib.i64arr(ext), nd,
              stream())
    return out


class Pad:
    """Zero padding by per-axis (before, after); adjoint crops (core_operators.py:29-59)."""

    def __init__(self, padding: Tuple[Tuple[int, int], ...]):
        self.padding = tuple((int(pb), int(pa)) for pb, pa in padding)
        self.operator_norm_sq = 1.0

    def forward(self, x):
        x = to_device(x)
        shape = [s + pb + pa for (pb, pa), s in zip(self.padding, x.shape)]
        return _window(x, [0] * x.dim(), shape, [pb for pb, _ in self.padding], list(x.shape))

    def adjoint(self, y):
        y = to_device(y)
        ext = [s - pb - pa for (pb, pa), s in zip(self.padding, y.shape)]
        return _window(y, [pb for pb, _ in self.padding], ext, [0] * y.dim(), ext)

    def __call__(self, x):
        return self.forward(x)


class Crop:
    """Centre (or explicit ``start``) crop; adjoint zero-pads (core_operators.py:62-137)."""

    def __init__(self, original_shape, target_shape, start=None):
        if len(original_shape) != len(target_shape):
            raise ValueError(
                f"original_shape {original_shape} and target_shape {target_shape} "
                "must have same number of dimensions"
            )
        self.original_shape = tuple(int(s) for s in original_shape)
        self.target_shape = tuple(int(s) for s in target_shape)
        self.in_shape = self.original_shape
        self.out_shape = self.target_shape
        self.operator_norm_sq = 1.0
        if start is not None and len(start) != len(self.original_shape):
            raise ValueError(
                f"start {start} must have same number of dimensions as "
                f"original_shape {self.original_shape}"
            )
        self._slices = ()
        self._padding = ()
        self.start = ()
        for i, (orig, tgt) in enumerate(zip(self.original_shape, self.target_shape)):
            if tgt > orig:
                raise ValueError(f"Target size {tgt} > original size {orig}. Use Pad for upsizing.")
            if start is None:
                s0 = (orig - tgt) // 2
            else:
                s0 = int(start[i])
                if s0 < 0 or s0 + tgt > orig:
                    raise ValueError(
                        f"start {s0} on axis {i} puts crop window "
                        f"[{s0}, {s0 + tgt}) outside original size {orig}"
                    )
            self.start += (s0,)
            self._slices += (slice(s0, s0 + tgt),)
            self._padding += ((s0, orig - s0 - tgt),)

    def forward(self, x):
        x = to_device(x)
        return _window(x, self.start, self.target_shape, [0] * x.dim(), self.target_shape)

    def adjoint(self, y):
        y = to_device(y)
        return _window(y, [0] * y.dim(), self.original_shape, self.start, self.target_shape)

    def __call__(self, x):
        return self.forward(x)


# ---------------------------------------------------------------------------
# banded weights (host tables from the library, cached on the device)
# ---------------------------------------------------------------------------

_BANDS = {}
_TABLE_STREAM = {}


def _upload_table(a: np.ndarray) -> torch.Tensor:
    """A device copy of a host table that every stream may read at once: the
    copy runs on a private stream that is synchronised before the table is
    cached.  (Uploaded on the caller's stream, a table first used by one job
    could be read by a concurrent job on another stream before its copy
    landed.)"""
    dev = torch.cuda.current_device()
    st = _TABLE_STREAM.get(dev)
    if st is None:
        st = _TABLE_STREAM[dev] = torch.cuda.Stream()
    with torch.cuda.stream(st):
        t = torch.from_numpy(np.ascontiguousarray(a)).to("cuda")
    st.synchronize()
    return t


def banded_overlap_weights(n_large: int, n_small: int):
    """Host (idx_fwd, w_fwd, idx_adj, w_adj) of core_operators.py:151-202."""
    return _lib.band_weights(int(n_large), int(n_small))


def _device_band(n_large: int, n_small: int, scale: float = 1.0):
    key = (torch.cuda.current_device(), n_large, n_small, scale)
    hit = _BANDS.get(key)
    if hit is None:
        i_f, w_f, i_a, w_a = banded_overlap_weights(n_large, n_small)
        if scale != 1.0:
            # FractionalAreaUpsample pre-scales by n_small / n_large in float32
            w_f = (w_f * np.float32(scale)).astype(np.float32)
            w_a = (w_a * np.float32(scale)).astype(np.float32)
        hit = tuple(_upload_table(a) for a in (i_f, w_f, i_a, w_a))
        _BANDS[key] = hit
    return hit


def _apply_banded(x: torch.Tensor, idx: torch.Tensor, w: torch.Tensor, axis: int) -> torch.Tensor:
    """out[..., i, ...] = sum_k w[i,k] x[..., idx[i,k], ...] (core_operators.py:205-219)."""
    axis = axis % x.dim()
    shape = list(x.shape)
    outer = int(np.prod(shape[:axis])) if axis > 0 else 1
    inner = int(np.prod(shape[axis + 1:])) if axis + 1 < len(shape) else 1
    n_out, width = idx.shape
    shape[axis] = n_out
    out = empty(shape)
    if out.numel() == 0:
        return out
    _lib.call("decon_banded_axis", _lib.ptr(x), _lib.ptr(out), outer, x.shape[axis], inner, n_out,
              _lib.ptr(idx), _lib.ptr(w), int(width), stream())
    return out


def _per_axis(scale, axes):
    return scale * len(axes) if (len(scale) == 1 and len(axes) > 1) else scale


class FractionalAreaDownsample:
    """Fine -> coarse intensity-preserving area sum; adjoint = exact transpose
    (core_operators.py:222-352)."""

    def __init__(self, scale: Union[float, Tuple[float, ...]], axes: Tuple[int, ...] = None,
                 in_shape: Tuple[int, ...] = None):
        if isinstance(scale, (int, float)):
            scale = (float(scale),)
        self.scale = tuple(float(s) for s in scale)
        if any(s < 1.0 for s in self.scale):
            raise ValueError(
                f"FractionalAreaDownsample requires scale >= 1 (fine -> coarse); "
                f"got {self.scale}. Use FractionalAreaUpsample to upsample."
            )
        self.axes = axes
        self._axis_map = {}
        self.in_shape = None
        self.out_shape = None
        if in_shape is not None:
            ax = axes if axes is not None else tuple(range(len(in_shape)))
            for a, s in zip(ax, _per_axis(self.scale, ax)):
                nl = in_shape[a]
                self._axis_map[a] = (nl, max(1, int(round(nl / s))))
            self.in_shape = tuple(int(s) for s in in_shape)
            out = list(self.in_shape)
            for a, (_, ns) in self._axis_map.items():
                out[a % len(out)] = ns
            self.out_shape = tuple(out)
        if self._axis_map:
            n2 = 1.0
            for nl, ns in self._axis_map.values():
                n2 *= nl / ns
        else:
            n2 = math.prod(self.scale)
        self.operator_norm_sq = float(n2)

    def axis_pairs(self, shape, adjoint=False):
        """[(axis, n_large, n_small)] in application order for an input of ``shape``."""
        axes = self.axes if self.axes is not None else tuple(range(len(shape)))
        cur = list(shape)
        out = []
        for a, s in zip(axes, _per_axis(self.scale, axes)):
            if a in self._axis_map:
                nl, ns = self._axis_map[a]
            elif adjoint:
                ns = cur[a]
                nl = max(1, int(round(ns * s)))
            else:
                nl = cur[a]
                ns = max(1, int(round(nl / s)))
            if nl == ns:
                continue
            out.append((a, nl, ns))
            cur[a] = nl if adjoint else ns
        return out

    def forward(self, x):
        r = to_device(x)
        for a, nl, ns in self.axis_pairs(r.shape):
            i_f, w_f, _, _ = _device_band(nl, ns)
            r = _apply_banded(r, i_f, w_f, a)
        return r

    def adjoint(self, y):
        r = to_device(y)
        for a, nl, ns in self.axis_pairs(r.shape, adjoint=True):
            _, _, i_a, w_a = _device_band(nl, ns)
            r = _apply_banded(r, i_a, w_a, a)
        return r

    def __call__(self, x):
        return self.forward(x)


class FractionalAreaUpsample:
    """Coarse -> fine spreading W_up = (n_small/n_large) W_dn^T; adjoint is the
    transpose (core_operators.py:355-450)."""

    def __init__(self, scale: Union[float, Tuple[float, ...]], axes: Tuple[int, ...] = None):
        if isinstance(scale, (int, float)):
            scale = (float(scale),)
        self.scale = tuple(float(s) for s in scale)
        if any(s < 1.0 for s in self.scale):
            raise ValueError(
                f"FractionalAreaUpsample requires scale >= 1 (coarse -> fine); "
                f"got {self.scale}. Use FractionalAreaDownsample to downsample."
            )
        self.axes = axes
        self.operator_norm_sq = 1.0

    def forward(self, x):
        r = to_device(x)
        axes = self.axes if self.axes is not None else tuple(range(r.dim()))
        for a, s in zip(axes, _per_axis(self.scale, axes)):
            ns = r.shape[a]
            nl = max(1, int(round(ns * s)))
            if nl == ns:
                continue
            _, _, i_a, w_a = _device_band(nl, ns, np.float32(ns / nl).item())
            r = _apply_banded(r, i_a, w_a, a)
        return r

    def adjoint(self, y):
        r = to_device(y)
        axes = self.axes if self.axes is not None else tuple(range(r.dim()))
        for a, s in zip(axes, _per_axis(self.scale, axes)):
            nl = r.shape[a]
            ns = max(1, int(round(nl / s)))
            if nl == ns:
                continue
            i_f, w_f, _, _ = _device_band(nl, ns, np.float32(ns / nl).item())
            r = _apply_banded(r, i_f, w_f, a)
        return r

    def __call__(self, x):
        return self.forward(x)
