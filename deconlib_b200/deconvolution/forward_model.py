"""Canonical forward model: padded visible grid -> convolve -> crop -> downsample -> data.

Mirrors deconlib's ``deconvolution/forward_model.py`` (ForwardModel :30-48,
make_forward_model :51-121).  The reconstruction lives on the padded visible
grid (visible grid extended by the PSF margins); the crop to the visible grid
uses the exact pad-before offset and happens on the fine grid, before the
fractional-area downsampling, so even-sized PSFs register correctly
(forward_model.py:99-107).
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Tuple, Union

import numpy as np

from .composition import LinearOperator, compose
from .core_operators import Crop, FractionalAreaDownsample
from .linops import LinearFFTConvolver
from .shapes import compute_padded_shape, get_valid_slices

__all__ = ["ForwardModel", "make_forward_model"]


@dataclass(frozen=True)
class ForwardModel:
    """op maps padded_shape -> data_shape; valid_slices crop padded -> visible."""

    op: LinearOperator
    data_shape: Tuple[int, ...]
    visible_shape: Tuple[int, ...]
    padded_shape: Tuple[int, ...]
    valid_slices: Tuple[slice, ...]


def make_forward_model(psf, data_shape: Tuple[int, ...],
                       zoom: Union[float, Tuple[float, ...]] = 1.0) -> ForwardModel:
    """Build convolve -> crop (-> downsample when zoom > 1) (forward_model.py:51-121)."""
    ndim = len(data_shape)
    if isinstance(zoom, (int, float)):
        zoom = (float(zoom),) * ndim
    else:
        zoom = tuple(float(z) for z in zoom)
    if len(zoom) != ndim:
        raise ValueError(f"zoom has {len(zoom)} entries, expected {ndim}")
    if any(z < 1.0 for z in zoom):
        raise ValueError(f"zoom must be >= 1 (visible grid at least as fine as data); got {zoom}")
    psf_shape = tuple(int(s) for s in (psf.shape if hasattr(psf, "shape") else np.shape(psf)))
    if len(psf_shape) != ndim:
        raise ValueError(f"psf is {len(psf_shape)}D but data_shape is {ndim}D")
    data_shape = tuple(int(d) for d in data_shape)
    visible = tuple(max(1, round(d * z)) for d, z in zip(data_shape, zoom))
    padded, padding = compute_padded_shape(visible, psf_shape)
    valid = get_valid_slices(padded, visible, padding)
    conv = LinearFFTConvolver(psf, signal_shape=padded, normalize=True)
    crop = Crop(padded, visible, start=tuple(b for b, _ in padding))
    if visible == data_shape:
        op = compose(crop, conv)
    else:
        scale = tuple(v / d for v, d in zip(visible, data_shape))
        op = compose(FractionalAreaDownsample(scale=scale, in_shape=visible), crop, conv)
    return ForwardModel(op=op, data_shape=data_shape, visible_shape=visible, padded_shape=padded,
                        valid_slices=valid)
