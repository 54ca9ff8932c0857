"""Tiled deconvolution of volumes too large for one solve.

Mirrors deconlib's ``deconvolution/tile_processing.py``: TileSpec (:60-75),
TilePlan (:78-94), the per-axis overlap-save windows (:97-125),
optimal_tile_size (:128-156), plan_tiles (:159-224) and process_tiles
(:227-288).  Geometry is host integer arithmetic; ``process_tiles`` runs any
``solve(data_tile, model)`` per tile with ONE forward model shared by all
tiles (every read window has the same shape).

Per axis of length N with read window T and guard g, the core C = T - 2g
steps the windows; window i owns output [i C, min((i + 1) C, N)) and reads
[clamp(i C - g, 0, N - T), + T); ownership boundaries are rounded from global
data positions (times zoom) so they never drift; owned intervals partition
the output, so every visible voxel is written exactly once.
"""

from __future__ import annotations

from dataclasses import dataclass
from itertools import product
from typing import Callable, List, Optional, Tuple, Union

import numpy as np

from .forward_model import ForwardModel, make_forward_model
from .linops import _next_smooth_number

__all__ = ["TileSpec", "TilePlan", "plan_tiles", "process_tiles", "optimal_tile_size"]

Solver = Callable[[np.ndarray, ForwardModel], np.ndarray]


@dataclass(frozen=True)
class TileSpec:
    """read: data-space window; write: owned core in the output; crop: that
    core inside the tile's visible-space result."""

    index: Tuple[int, ...]
    read: Tuple[slice, ...]
    write: Tuple[slice, ...]
    crop: Tuple[slice, ...]


@dataclass(frozen=True)
class TilePlan:
    data_shape: Tuple[int, ...]
    tile_shape: Tuple[int, ...]
    visible_shape: Tuple[int, ...]
    tiles: List[TileSpec]


def _axis_windows(N: int, V: int, T: int, guard: int, zoom: float):
    """(read, write, crop) slices along one axis (tile_processing.py:97-125)."""
    if T >= N:
        return [(slice(0, N), slice(0, V), slice(0, V))]
    core = T - 2 * guard
    if core <= 0:
        raise ValueError(f"tile size ({T}) must be > 2 * guard ({2 * guard})")
    out = []
    for i in range(-(-N // core)):
        lo, hi = i * core, min((i + 1) * core, N)
        r0 = min(max(lo - guard, 0), N - T)
        w0, w1, v0 = round(lo * zoom), round(hi * zoom), round(r0 * zoom)
        out.append((slice(r0, r0 + T), slice(w0, w1), slice(w0 - v0, w1 - v0)))
    return out


def optimal_tile_size(N: int, guard: int, tile_size: int) -> int:
    """Balanced, 5-smooth read window for one tiled axis (tile_processing.py:128-156):
    n = ceil(N / tile_size) tiles, core ceil(N / n), window core + 2 guard
    rounded up to 5-smooth and capped at N."""
    if N <= tile_size:
        return N
    n = -(-N // tile_size)
    core = -(-N // n)
    window = core + 2 * guard
    if window > N:
        raise ValueError(
            f"guard ({guard}) too large for tile_size ({tile_size}) on an axis of length {N}: "
            f"balanced core {core} + 2*guard = {window} would exceed the axis")
    return min(_next_smooth_number(window), N)


def plan_tiles(data_shape: Tuple[int, ...], zoom: Union[float, Tuple[float, ...]], guard: int,
               tile_size: int = 512, min_z_slices: int = 48) -> TilePlan:
    """Fixed-shape tiling of (..., Z, Y, X) data (tile_processing.py:159-224):
    Y and X always tiled, Z only when Nz > min_z_slices."""
    ndim = len(data_shape)
    if ndim < 2:
        raise ValueError("data_shape must be at least 2D")
    zoom = (float(zoom),) * ndim if isinstance(zoom, (int, float)) else tuple(float(z) for z in zoom)
    data_shape = tuple(int(n) for n in data_shape)
    visible = tuple(max(1, round(n * z)) for n, z in zip(data_shape, zoom))
    tiled = {ndim - 1, ndim - 2}
    if ndim >= 3 and data_shape[ndim - 3] > min_z_slices:
        tiled.add(ndim - 3)
    tile_shape, axes = [], []
    for i, (N, V, z) in enumerate(zip(data_shape, visible, zoom)):
        T = optimal_tile_size(N, guard, tile_size) if i in tiled else N
        tile_shape.append(T)
        axes.append(_axis_windows(N, V, T, guard, z))
    tiles = [TileSpec(index=tuple(i for i, _ in combo), read=tuple(w[0] for _, w in combo),
                      write=tuple(w[1] for _, w in combo), crop=tuple(w[2] for _, w in combo))
             for combo in product(*(list(enumerate(a)) for a in axes))]
    return TilePlan(data_shape=data_shape, tile_shape=tuple(tile_shape), visible_shape=visible,
                    tiles=tiles)


def process_tiles(data, psf, zoom, solve: Solver, *, guard: Optional[int] = None,
                  tile_size: int = 512, min_z_slices: int = 48,
                  on_tile_done: Optional[Callable] = None, verbose: bool = False) -> np.ndarray:
    """Tile-by-tile deconvolution with any solver (tile_processing.py:227-288).
    ``guard`` defaults to half the PSF's lateral width."""
    psf_shape = tuple(psf.shape)
    if guard is None:
        guard = max(psf_shape[-2:]) // 2
    plan = plan_tiles(tuple(data.shape), zoom, guard, tile_size, min_z_slices)
    model = make_forward_model(psf, plan.tile_shape, zoom)
    output = np.zeros(plan.visible_shape, dtype=np.float32)
    for i, spec in enumerate(plan.tiles):
        tile = np.asarray(data[spec.read], dtype=np.float32)
        restored = np.asarray(solve(tile, model))
        # rounding guard: clip the crop to the result, size the write to the core
        crop = tuple(slice(c.start, min(c.stop, restored.shape[j])) for j, c in enumerate(spec.crop))
        core = restored[crop]
        write = tuple(slice(w.start, w.start + core.shape[j]) for j, w in enumerate(spec.write))
        output[write] = core
        if verbose:
            print(f"  tile {i + 1}/{len(plan.tiles)} {spec.index} done")
        if on_tile_done is not None and on_tile_done(spec, output):
            break
    return output
