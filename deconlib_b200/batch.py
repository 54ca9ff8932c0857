"""Batched tiled Richardson-Lucy on one GPU.

A large volume is split into overlapping tiles of uneven shape (a seeded
core size per tile and axis plus a halo), and independent volumes with their
own PSFs join the same batch.  Every problem gets its own convolution plan,
with an FFT canvas and a pass schedule chosen by ``autotune_schedule`` (each
candidate canvas is a different radix factorisation of the axes, each
schedule a different family of equivalent FFT kernels: fused or separate
Y / axial passes, pipelined / one-tile / plain-load column kernels, one- or
two-CTA axial kernel, radix order, lines per CTA; the fastest measured
forward + adjoint convolution wins, cached per shape in memory and in a JSON
file), and K iterations of
all problems are recorded into one CUDA graph by the native batch runtime
(``decon_batch_rl_*``): the graph forks the problems over internal streams,
so one replay advances every tile and volume together.  The stitched result
takes each tile's core (its halo discarded).

The reference solves uniform tiles one at a time (tile_processing.py:226-288,
``richardson_lucy_with_operator`` per tile, rl_mlx.py:83-185); a tile here
computes exactly that solve on its own window, up to the rounding of a
different FFT canvas, which the tests bound.
"""

from __future__ import annotations

import ctypes as C
import json
import os
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .deconvolution._device import empty, stream, to_device
from .deconvolution.linops import LinearFFTConvolver, _next_smooth_number, static_fft_shape

__all__ = ["BatchTile", "plan_uneven_tiles", "fft_shape_candidates", "autotune_fft_shape",
           "autotune_schedule", "SCHEDULES", "tune_cache_path", "BatchedRL", "batched_tiled_rl"]


# ---------------------------------------------------------------------------
# uneven overlapping tiles
# ---------------------------------------------------------------------------


@dataclass(frozen=True)
class BatchTile:
    """read: the tile's window (core + halo, clipped to the volume); write:
    its core in the output; crop: the core inside the tile."""

    read: Tuple[slice, ...]
    write: Tuple[slice, ...]
    crop: Tuple[slice, ...]

    @property
    def shape(self) -> Tuple[int, ...]:
        return tuple(s.stop - s.start for s in self.read)


def _axis_cores(N: int, lo: int, hi: int, rng: np.random.Generator) -> List[Tuple[int, int]]:
    """Cores of seeded length in [lo, hi] covering [0, N).  With hi >= 2 lo
    every core, the last included, lies in [lo, hi] (N >= lo)."""
    if N <= hi:
        return [(0, N)]
    cores, pos = [], 0
    while N - pos > hi:
        s = int(rng.integers(lo, hi + 1))
        rest = N - pos - s
        if 0 < rest < lo:
            s = N - pos - lo
        cores.append((pos, pos + s))
        pos += s
    cores.append((pos, N))
    return cores


def plan_uneven_tiles(shape: Sequence[int], core_ranges: Sequence[Tuple[int, int]], halo: int,
                      rng: np.random.Generator) -> List[BatchTile]:
    """Tiles whose cores partition ``shape`` with seeded per-axis core lengths
    in ``core_ranges`` and a ``halo`` on every side (clipped at the border)."""
    per_axis = []
    for N, (lo, hi) in zip(shape, core_ranges):
        if hi < 2 * lo:
            raise ValueError(f"core range ({lo}, {hi}) needs hi >= 2 lo")
        per_axis.append(_axis_cores(int(N), int(lo), int(hi), rng))
    tiles = []
    for combo in np.ndindex(*[len(a) for a in per_axis]):
        read, write, crop = [], [], []
        for ax, i in enumerate(combo):
            c0, c1 = per_axis[ax][i]
            r0, r1 = max(0, c0 - halo), min(int(shape[ax]), c1 + halo)
            read.append(slice(r0, r1))
            write.append(slice(c0, c1))
            crop.append(slice(c0 - r0, c1 - r0))
        tiles.append(BatchTile(tuple(read), tuple(write), tuple(crop)))
    return tiles


# ---------------------------------------------------------------------------
# FFT canvas autotuner
# ---------------------------------------------------------------------------


def _next_pow2(n: int) -> int:
    return 1 << max(0, int(n - 1).bit_length())


def _next_23(n: int) -> int:
    best = _next_pow2(n)
    p3 = 1
    while p3 < best:
        m = p3
        while m < n:
            m *= 2
        best = min(best, m)
        p3 *= 3
    return best


def fft_shape_candidates(signal_shape, kernel_shape, max_growth: float = 1.35) -> List[tuple]:
    """Canvases to try: the reference's 5-smooth minimum on every axis, and
    variants with 2^a 3^b or power-of-two lengths (other radix sequences;
    power-of-two y / z lengths <= 512 also select the TMA-pipelined column
    kernels) where they grow an axis by <= max_growth, and the lengths of
    ``static_fft_shape`` (compile-time radix sequences).  Sorted by volume."""
    m = [int(n) + int(k) - 1 for n, k in zip(signal_shape, kernel_shape)]
    s5 = [_next_smooth_number(v) for v in m]
    st = static_fft_shape(signal_shape, kernel_shape)
    alt = []
    for v, base, sl in zip(m, s5, st):
        opts = {base, sl}
        for f in (_next_23, _next_pow2):
            c = f(v)
            if c <= max_growth * base:
                opts.add(c)
        alt.append(sorted(opts))
    cands = {tuple(s5)}
    for ax in range(len(m)):
        for c in alt[ax]:
            t = list(s5)
            t[ax] = c
            cands.add(tuple(t))
    if len(m) >= 2:
        for cy in alt[-2]:
            for cx in alt[-1]:
                t = list(s5)
                t[-2], t[-1] = cy, cx
                cands.add(tuple(t))
    cands.add(tuple(max(a) for a in alt))
    cands.add(tuple(st))
    return sorted(cands, key=lambda t: (int(np.prod(t)), t))


# Schedules the autotuner tries per canvas (decon_conv_set_schedule bits):
# each names an equivalent family of FFT passes, so the winner changes the
# speed, not the result (beyond FP32 rounding).
SCHED_FUSED, SCHED_NO_PIPE, SCHED_NO_TMA, SCHED_LEAN_OFF, SCHED_ODD_RADIX, SCHED_HALF_LINES = (
    1, 2, 4, 8, 16, 32)
SCHEDULES = {
    "default": 0,
    "fused-y-axial": SCHED_FUSED,
    "one-tile": SCHED_NO_PIPE,
    "plain-loads": SCHED_NO_TMA,
    "one-cta-axial": SCHED_LEAN_OFF,
    "odd-radix-first": SCHED_ODD_RADIX,
    "half-lines": SCHED_HALF_LINES,
}

_TUNED: Dict[str, tuple] = {}
_CACHE_LOADED = False


def tune_cache_path() -> str:
    """JSON file the autotuner persists its choices to: $DECON_AUTOTUNE_CACHE,
    else ~/.cache/deconlib_b200/autotune.json."""
    return os.environ.get("DECON_AUTOTUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "deconlib_b200", "autotune.json")


def _device_tag() -> str:
    p = torch.cuda.get_device_properties(torch.cuda.current_device())
    return f"{p.name}|sm{p.major}{p.minor}|{p.multi_processor_count}"


def _load_cache() -> None:
    global _CACHE_LOADED
    if _CACHE_LOADED:
        return
    _CACHE_LOADED = True
    try:
        with open(tune_cache_path()) as f:
            for k, v in json.load(f).items():
                _TUNED[k] = (tuple(v["fft_shape"]), int(v["schedule"]), float(v.get("ms", -1.0)))
    except (OSError, ValueError, KeyError):
        pass


def _save_cache() -> None:
    path = tune_cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        out = {k: {"fft_shape": list(v[0]), "schedule": v[1], "ms": v[2]} for k, v in _TUNED.items()}
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def _time_pair(conv, x, reps) -> float:
    conv.adjoint(conv.forward(x))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        conv.adjoint(conv.forward(x))
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def autotune_schedule(signal_shape, psf, candidates: Optional[List[tuple]] = None,
                      max_candidates: int = 6, reps: int = 3, schedules=None) -> Tuple[tuple, int]:
    """Fastest (canvas, schedule) for a LinearFFTConvolver of ``psf`` on
    ``signal_shape``: every candidate canvas (a different radix factorisation)
    is timed under every applicable schedule (fused or separate Y / axial
    passes, pipelined / one-tile / plain-load column kernels, one- or two-CTA
    axial kernel, radix order, lines per CTA), forward + adjoint with CUDA
    events after a warm-up.  The winner is cached per (device, signal shape,
    kernel shape) in memory and in the JSON file of ``tune_cache_path()``;
    shapes with the same candidate canvases share one timing."""
    _load_cache()
    kshape = tuple(int(s) for s in psf.shape)
    sig = tuple(int(s) for s in signal_shape)
    dev = _device_tag()
    key = f"{dev}|{sig}|{kshape}"
    if key in _TUNED:
        return _TUNED[key][0], _TUNED[key][1]
    cands = list((candidates or fft_shape_candidates(sig, kshape))[:max_candidates])
    if candidates is None:
        # always time the canvas of compile-time FFT lengths
        st = tuple(static_fft_shape(sig, kshape))
        if st not in cands:
            cands[-1:] = [st]
    ckey = f"{dev}|canvases|{tuple(cands)}"
    if ckey in _TUNED:
        _TUNED[key] = _TUNED[ckey]
        _save_cache()
        return _TUNED[key][0], _TUNED[key][1]
    scheds = list(SCHEDULES.values()) if schedules is None else list(schedules)
    x = empty(sig)
    x.fill_(1.0)
    best, best_ms = (tuple(cands[0]), 0), float("inf")
    for fs in cands:
        conv = LinearFFTConvolver(psf, sig, fft_shape=fs)
        seen = set()
        for sc in scheds:
            conv.set_schedule(sc)
            # the fused pass ignores the column-kernel bits; a canvas it does
            # not serve ignores the fused bit: time each distinct family once
            fused = conv.fused_yz
            eff = sc & (SCHED_FUSED | SCHED_ODD_RADIX | SCHED_HALF_LINES) if fused else sc & ~SCHED_FUSED
            if eff in seen:
                continue
            seen.add(eff)
            conv.set_schedule(eff)
            ms = _time_pair(conv, x, reps)
            if ms < best_ms:
                best, best_ms = (tuple(fs), eff), ms
        del conv
    _TUNED[key] = _TUNED[ckey] = (best[0], best[1], best_ms)
    _save_cache()
    return best


def autotune_fft_shape(signal_shape, psf, candidates: Optional[List[tuple]] = None,
                       max_candidates: int = 6, reps: int = 3) -> tuple:
    """The canvas of ``autotune_schedule`` (kept for callers that choose the
    canvas only)."""
    return autotune_schedule(signal_shape, psf, candidates, max_candidates, reps)[0]


# ---------------------------------------------------------------------------
# the batch
# ---------------------------------------------------------------------------


def _ptrs(ts):
    return (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


class BatchedRL:
    """Independent RL problems (observation, PSF) solved together through
    one CUDA graph per K iterations (``decon_batch_rl_*``).

    ``fft_shapes``: None (5-smooth default per problem), "auto" (autotuned)
    or a list of canvases.  ``restored`` / ``predict()`` give CUDA tensors on
    each problem's own grid."""

    def __init__(self, problems: Sequence[Tuple[object, object]], background=0.0, fft_shapes=None,
                 nstreams: int = 8, iters_per_graph: int = 10):
        n = len(problems)
        if n == 0:
            raise ValueError("BatchedRL needs at least one problem")
        bgs = list(background) if isinstance(background, (list, tuple)) else [float(background)] * n
        self.obs = [to_device(o) for o, _ in problems]
        psfs = [p for _, p in problems]
        scheds = [0] * n
        if isinstance(fft_shapes, str) and fft_shapes == "auto":
            tuned = [autotune_schedule(tuple(o.shape), p) for o, p in zip(self.obs, psfs)]
            fft_shapes = [t[0] for t in tuned]
            scheds = [t[1] for t in tuned]
        elif fft_shapes is None:
            fft_shapes = [None] * n
        self.convs = [LinearFFTConvolver(p, tuple(o.shape), fft_shape=fs, schedule=sc)
                      for o, p, fs, sc in zip(self.obs, psfs, fft_shapes, scheds)]
        self.fft_shapes = [c.fft_shape for c in self.convs]
        self.schedules = [c.schedule for c in self.convs]
        self.x = [empty(o.shape) for o in self.obs]
        self.sens = [empty(o.shape) for o in self.obs]
        self.ratio = [empty(o.shape) for o in self.obs]
        self.background = [float(b) for b in bgs]
        self.iters_per_graph = int(iters_per_graph)
        h = C.c_void_p()
        plans = (C.c_void_p * n)(*[c.plan.value for c in self.convs])
        _lib.check(_lib.load().decon_batch_rl_create(
            n, plans, _ptrs(self.obs), (C.c_float * n)(*self.background), _ptrs(self.x),
            _ptrs(self.sens), _ptrs(self.ratio), int(nstreams), C.byref(h)))
        self.h = h
        _lib.call("decon_batch_rl_setup", h, None, stream())
        self.iterations = 0

    def run(self, num_iter: int) -> "BatchedRL":
        _lib.call("decon_batch_rl_run", self.h, int(num_iter), self.iters_per_graph, stream())
        self.iterations += int(num_iter)
        if num_iter > 0:
            self.last_graph_iters = min(self.iters_per_graph, int(num_iter))
        return self

    def graph_kernels(self) -> int:
        """Kernel nodes of the graph the last run replayed (K = min(iters_per_graph, n))."""
        k = C.c_int64()
        _lib.call("decon_batch_graph_nodes", self.h, getattr(self, "last_graph_iters", 0), C.byref(k))
        return int(k.value)

    @property
    def restored(self) -> List[torch.Tensor]:
        return self.x

    def predict(self) -> List[torch.Tensor]:
        pred = [empty(o.shape) for o in self.obs]
        _lib.call("decon_batch_rl_predict", self.h, _ptrs(pred), stream())
        return pred

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value and _lib._lib is not None:
            try:
                torch.cuda.synchronize()
                _lib._lib.decon_batch_destroy(h)
            except Exception:
                pass
            self.h = None


def batched_tiled_rl(data, psf, tiles: Sequence[BatchTile], num_iter: int, background: float = 0.0,
                     extra: Sequence[Tuple[object, object, float]] = (), fft_shapes="auto",
                     nstreams: int = 8, iters_per_graph: int = 10):
    """RL of every tile of ``data`` (one PSF) and of the ``extra`` volumes
    (observation, PSF, background) in one batch; returns (stitched volume as
    a CUDA tensor, [restored extra volumes], the BatchedRL)."""
    vol = to_device(data)
    probs = [(vol[t.read].contiguous(), psf) for t in tiles]
    probs += [(o, p) for o, p, _ in extra]
    bgs = [float(background)] * len(tiles) + [float(b) for _, _, b in extra]
    batch = BatchedRL(probs, bgs, fft_shapes=fft_shapes, nstreams=nstreams,
                      iters_per_graph=iters_per_graph).run(num_iter)
    out = empty(vol.shape)
    for t, x in zip(tiles, batch.restored[:len(tiles)]):
        out[t.write] = x[t.crop]
    return out, batch.restored[len(tiles):], batch
