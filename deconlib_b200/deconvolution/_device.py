"""Device-array helpers: conversion to CUDA float32 tensors, workspaces, reductions."""

from __future__ import annotations

import ctypes as C
from typing import Tuple

import numpy as np
import torch

from .. import _lib


def to_device(x, dtype=torch.float32) -> torch.Tensor:
    """A C-contiguous CUDA float32 tensor holding ``x`` (NumPy, torch or scalar).

    NumPy input is copied to the device, as the reference copies NumPy input
    into an ``mx.array`` (rl_mlx.py:117-120)."""
    _lib.require_cuda()
    if isinstance(x, torch.Tensor):
        t = x
        if not t.is_cuda:
            t = t.to("cuda")
    else:
        a = np.asarray(x)
        if a.dtype != np.float32:
            a = a.astype(np.float32)
        t = torch.from_numpy(np.ascontiguousarray(a)).to("cuda")
    if t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()


def empty(shape, dtype=torch.float32) -> torch.Tensor:
    return torch.empty(tuple(int(s) for s in shape), dtype=dtype, device="cuda")


def zeros(shape, dtype=torch.float32) -> torch.Tensor:
    return torch.zeros(tuple(int(s) for s in shape), dtype=dtype, device="cuda")


def shape3(shape) -> Tuple[int, int, int]:
    """(z, y, x) view of a 1-3 dimensional shape (leading extents of 1)."""
    s = tuple(int(v) for v in shape)
    if not 1 <= len(s) <= 3:
        raise ValueError(f"only 1-, 2- and 3-dimensional arrays are supported, got shape {s}")
    return (1,) * (3 - len(s)) + s


def stream():
    return _lib.stream_ptr()


_WS = {}


def workspace() -> torch.Tensor:
    """Reduction workspace of the current stream: reductions queued on one
    stream run in order, so one workspace per (device, stream) is race-free
    even when several solves run on different streams."""
    key = (torch.cuda.current_device(), torch.cuda.current_stream().cuda_stream)
    ws = _WS.get(key)
    if ws is None:
        n = int(_lib.load().decon_reduce_workspace_bytes()) // 8
        ws = torch.empty(n + 8, dtype=torch.float64, device="cuda")
        _WS[key] = ws
    return ws


def reduce(a: torch.Tensor, op: int, b: torch.Tensor = None, out: torch.Tensor = None) -> torch.Tensor:
    """FP64 deterministic reduction on the device; returns a 1-element float64 tensor."""
    if out is None:
        out = torch.empty(1, dtype=torch.float64, device="cuda")
    _lib.call("decon_reduce", _lib.ptr(a), _lib.ptr(b), a.numel(), op, _lib.ptr(out),
              _lib.ptr(workspace()), stream())
    return out


def fill(t: torch.Tensor, v: float) -> torch.Tensor:
    _lib.call("decon_fill", _lib.ptr(t), C.c_float(v), t.numel(), stream())
    return t
