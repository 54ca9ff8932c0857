"""FFT convolution and finite-difference operators on the B200.

Mirrors deconlib's ``deconvolution/linops_mlx.py``: Gradient1D/2D/3D
(:46-122), Hessian1D/2D/3D (:130-262), FFTConvolver (:384-432),
LinearFFTConvolver (:435-533), _next_smooth_number / fast_padded_shape
(:956-1032).  Same constructors, attributes and errors.  The convolutions
run the pruned R2C/C2R FFT kernels of ``libdecon_b200`` (one plan per
operator: OTF, spectra and twiddles resident on the device); the stencils
run the library's Hessian / gradient kernels.
"""

from __future__ import annotations

import ctypes as C
import math
from typing import Optional, Tuple, Union

import numpy as np
import torch

from .. import _lib
from ._device import empty, shape3, stream, to_device

__all__ = [
    "Gradient1D", "Gradient2D", "Gradient3D", "Hessian1D", "Hessian2D", "Hessian3D",
    "FFTConvolver", "LinearFFTConvolver", "fast_padded_shape", "pad_corner_origin_kernel",
    "STATIC_FFT_LENGTHS", "static_fft_shape",
]

SQRT2 = float(np.sqrt(np.float32(2.0)))


def _next_smooth_number(n: int) -> int:
    """Smallest integer >= n with prime factors 2, 3, 5 only (linops_mlx.py:956-972)."""
    m = n
    while True:
        r = m
        for p in (2, 3, 5):
            while r % p == 0:
                r //= p
        if r == 1:
            return m
        m += 1


def fast_padded_shape(signal_shape, kernel_shape, min_pad=None) -> Tuple[int, ...]:
    """5-smooth canvas for wrap-free convolution (linops_mlx.py:975-1032)."""
    ndim = len(signal_shape)
    if min_pad is None:
        pads = (None,) * ndim
    elif isinstance(min_pad, int):
        pads = (min_pad,) * ndim
    else:
        pads = tuple(min_pad)
    out = []
    for n, m, p in zip(signal_shape, kernel_shape, pads):
        need = (m - 1) if p is None else int(p)
        out.append(_next_smooth_number(max(n + need, m)))
    return tuple(out)


# FFT lengths with a compile-time radix sequence in the library (2^a x {1, 3,
# 5, 15}, 64 to 1024): the strided passes of these lengths run straight-line
# stages; other 7-smooth lengths take the runtime-radix path, which measured
# ~4x slower per canvas voxel on the B200.
STATIC_FFT_LENGTHS = (64, 80, 96, 128, 160, 192, 240, 256, 320, 384, 480, 512, 640, 768, 960, 1024)


def static_fft_shape(signal_shape, kernel_shape) -> Tuple[int, ...]:
    """Wrap-free canvas on the compile-time FFT lengths (not in the reference).

    Per axis the smallest length >= N + M - 1 in ``STATIC_FFT_LENGTHS`` (the
    last axis, transformed as packed complex pairs, twice such a length), when
    that grows the axis by at most 1/3 over ``fast_padded_shape``'s 5-smooth
    length; otherwise the 5-smooth length.  The axial (first) axis of a 3-D
    canvas takes 64, 128 or 256 instead when that is at most twice the
    length chosen so: those lengths run the TMA-pipelined axial kernels,
    which measured faster per iteration on the B200 even on the larger canvas
    (RL at 76x362x244: 1.43 ms on 256x768x512 vs 2.29 ms on 160x768x512).
    A convolution's result does not depend on the canvas beyond FP32
    rounding."""
    ref = fast_padded_shape(signal_shape, kernel_shape)
    nd = len(ref)
    out = []
    for ax, (n, m, r) in enumerate(zip(signal_shape, kernel_shape, ref)):
        need = max(int(n) + int(m) - 1, int(m))
        scale = 2 if ax == nd - 1 else 1
        c = next((scale * L for L in STATIC_FFT_LENGTHS if scale * L >= need), None)
        out.append(c if c is not None and 3 * c <= 4 * r else r)
    if nd == 3:
        need = max(int(signal_shape[0]) + int(kernel_shape[0]) - 1, int(kernel_shape[0]))
        p = 1 << max(0, (need - 1).bit_length())
        if p in (64, 128, 256) and p <= 2 * out[0]:
            out[0] = p
    return tuple(out)


def pad_corner_origin_kernel(kernel: np.ndarray, output_shape) -> np.ndarray:
    """Host form of the corner-origin embedding (utils/padding.py:142-190).

    The convolution plans do this embedding on the device inside the OTF
    build; this host version is kept for API completeness."""
    kernel = np.asarray(kernel)
    out_shape = tuple(int(s) for s in output_shape)
    if len(out_shape) != kernel.ndim:
        raise ValueError(f"output_shape has {len(out_shape)} dims, expected {kernel.ndim}")
    for ax, (m, f) in enumerate(zip(kernel.shape, out_shape)):
        if f < m:
            raise ValueError(
                f"output size {f} cannot be smaller than kernel size {m} in dimension {ax}"
            )
    idx = []
    for m, f in zip(kernel.shape, out_shape):
        i = np.arange(m)
        npos = (m + 1) // 2
        idx.append(np.where(i < npos, i, f - (m - i)))
    out = np.zeros(out_shape, dtype=kernel.dtype)
    out[np.ix_(*idx)] = kernel
    return out


# ---------------------------------------------------------------------------
# FFT convolution
# ---------------------------------------------------------------------------


class _ConvPlan:
    """Owns one ``decon_conv`` plan (OTF + spectra) on the current device."""

    def __init__(self, kernel: torch.Tensor, kshape3, sshape3, fshape3, normalize, circular):
        lib = _lib.load()
        h = C.c_void_p()
        if circular:
            st = lib.decon_conv_create_circular(_lib.ptr(kernel), _lib.i64arr(kshape3),
                                                int(bool(normalize)), stream(), C.byref(h))
        else:
            st = lib.decon_conv_create(_lib.ptr(kernel), _lib.i64arr(kshape3), _lib.i64arr(sshape3),
                                       _lib.i64arr(fshape3), int(bool(normalize)), stream(),
                                       C.byref(h))
        _lib.check(st)
        self.handle = h
        self.device = torch.cuda.current_device()
        nrm = C.c_double()
        _lib.check(lib.decon_conv_norm_sq(h, C.byref(nrm)))
        self.norm_sq = float(nrm.value)
        self.fshape3 = tuple(fshape3)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value and _lib._lib is not None:
            try:
                with torch.cuda.device(self.device):
                    torch.cuda.synchronize()
                    _lib._lib.decon_conv_destroy(h)
            except Exception:
                pass
            self.handle = None

    def otf(self) -> torch.Tensor:
        fz, fy, fx = self.fshape3
        out = torch.empty((fz, fy, fx // 2 + 1), dtype=torch.complex64, device="cuda")
        _lib.call("decon_conv_get_otf", self.handle, _lib.ptr(out), stream())
        return out


class FFTConvolver:
    """Circular convolution by a resident OTF (linops_mlx.py:384-432)."""

    def __init__(self, kernel, normalize: bool = True):
        k = to_device(kernel)
        self.shape = tuple(int(s) for s in k.shape)
        self.in_shape = self.shape
        self.out_shape = self.shape
        self.axes = tuple(range(-len(self.shape), 0))
        s3 = shape3(self.shape)
        self._plan = _ConvPlan(k, s3, s3, s3, normalize, circular=True)
        self.operator_norm_sq = self._plan.norm_sq

    @property
    def otf(self) -> torch.Tensor:
        return self._plan.otf().reshape(self.shape[:-1] + (self.shape[-1] // 2 + 1,))

    @property
    def otf_conj(self) -> torch.Tensor:
        return torch.conj(self.otf)

    def _run(self, name, x):
        x = to_device(x)
        if tuple(x.shape) != self.shape:
            raise ValueError(f"expected input of shape {self.shape}, got {tuple(x.shape)}")
        out = empty(self.shape)
        _lib.call(name, self._plan.handle, _lib.ptr(x), _lib.ptr(out), stream())
        return out

    def forward(self, x):
        return self._run("decon_conv_forward", x)

    def adjoint(self, y):
        return self._run("decon_conv_adjoint", y)

    def __call__(self, x):
        return self.forward(x)


class LinearFFTConvolver:
    """Wrap-free convolution on ``signal_shape`` (linops_mlx.py:435-533).

    The canvas ``fft_shape`` (default: 5-smooth >= N + M - 1) is never
    materialised: the zero padding is implicit in the first FFT pass and the
    crop in the last (pruned transforms)."""

    def __init__(self, kernel, signal_shape: Tuple[int, ...], normalize: bool = True,
                 fft_shape: Optional[Tuple[int, ...]] = None, precision: str = "fp32",
                 schedule: int = 0):
        if isinstance(kernel, torch.Tensor):
            kshape = tuple(int(s) for s in kernel.shape)
        else:
            kshape = tuple(int(s) for s in np.shape(kernel))
        self.signal_shape = tuple(int(s) for s in signal_shape)
        self.in_shape = self.signal_shape
        self.out_shape = self.signal_shape
        self.kernel_shape = kshape
        if len(self.signal_shape) != len(self.kernel_shape):
            raise ValueError("signal_shape and kernel must have the same number of dimensions")
        minimum = tuple(n + m - 1 for n, m in zip(self.signal_shape, self.kernel_shape))
        if fft_shape is None:
            fft_shape = fast_padded_shape(self.signal_shape, self.kernel_shape)
        self.fft_shape = tuple(int(s) for s in fft_shape)
        if len(self.fft_shape) != len(self.signal_shape):
            raise ValueError("fft_shape must match signal_shape ndim")
        if any(p < q for p, q in zip(self.fft_shape, minimum)):
            raise ValueError(
                f"fft_shape {self.fft_shape} is too small for linear "
                f"convolution; minimum is {minimum}"
            )
        self.normalize = bool(normalize)
        k = to_device(kernel)
        self._n3 = shape3(self.signal_shape)
        self._f3 = shape3(self.fft_shape)
        self._plan = _ConvPlan(k, shape3(self.kernel_shape), self._n3, self._f3, normalize,
                               circular=False)
        self.operator_norm_sq = self._plan.norm_sq
        self.precision = "fp32"
        if precision != "fp32":
            self.set_precision(precision)
        self.schedule = 0
        if schedule:
            self.set_schedule(schedule)

    def set_schedule(self, schedule: int) -> "LinearFFTConvolver":
        """Choose among equivalent FFT pass families for this plan (not in the
        reference; ``decon_conv_set_schedule`` bits, see ``SCHEDULES``):
        results agree with the default to FP32 rounding.  Used by the
        batched-workload autotuner."""
        _lib.call("decon_conv_set_schedule", self._plan.handle, int(schedule))
        self.schedule = int(schedule)
        return self

    @property
    def fused_yz(self) -> bool:
        """True when this plan runs the fused Y / axial cluster pass."""
        f = C.c_int()
        _lib.check(_lib.load().decon_conv_fused_yz(self._plan.handle, C.byref(f)))
        return bool(f.value)

    def set_precision(self, precision: str) -> "LinearFFTConvolver":
        """"fp32" or "mixed" (not in the reference): "mixed" stores the OTF as
        FP16 complex with a power-of-two scale per kz plane for the axial FFT
        pass; transforms and products stay FP32, reductions FP64.  Raises
        RuntimeError when this canvas has no pipelined axial pass."""
        codes = {"fp32": 0, "mixed": 1}
        if precision not in codes:
            raise ValueError(f"precision must be 'fp32' or 'mixed', got {precision!r}")
        _lib.call("decon_conv_set_precision", self._plan.handle, codes[precision], stream())
        self.precision = precision
        return self

    def set_kernel(self, kernel) -> "LinearFFTConvolver":
        """Replace the kernel by another of the same shape, rebuilding the OTF
        in this plan's device buffers (no allocation, no cudaFree).  Not in
        the reference; a serving loop uses it to hand a pooled plan to the next
        job of the same shape.  Synchronises the current stream."""
        k = to_device(kernel)
        if tuple(k.shape) != self.kernel_shape:
            raise ValueError(f"set_kernel expects a kernel of shape {self.kernel_shape}, "
                             f"got {tuple(k.shape)}")
        _lib.call("decon_conv_set_kernel", self._plan.handle, _lib.ptr(k), int(self.normalize),
                  stream())
        nrm = C.c_double()
        _lib.check(_lib.load().decon_conv_norm_sq(self._plan.handle, C.byref(nrm)))
        self._plan.norm_sq = float(nrm.value)
        self.operator_norm_sq = self._plan.norm_sq
        return self

    @property
    def otf(self) -> torch.Tensor:
        """rfftn of the (normalised) kernel canvas, complex64 on the device."""
        f = self.fft_shape
        return self._plan.otf().reshape(f[:-1] + (f[-1] // 2 + 1,))

    @property
    def plan(self):
        return self._plan.handle

    def _run(self, name, x):
        x = to_device(x)
        if tuple(x.shape) != self.signal_shape:
            raise ValueError(
                f"LinearFFTConvolver expects input of shape {self.signal_shape}, "
                f"got {tuple(x.shape)}"
            )
        out = empty(self.signal_shape)
        _lib.call(name, self._plan.handle, _lib.ptr(x), _lib.ptr(out), stream())
        return out

    def forward(self, x):
        """Zero-boundary linear convolution (linops_mlx.py:520-524)."""
        return self._run("decon_conv_forward", x)

    def adjoint(self, y):
        """Adjoint correlation (linops_mlx.py:526-530)."""
        return self._run("decon_conv_adjoint", y)

    def __call__(self, x):
        return self.forward(x)


# ---------------------------------------------------------------------------
# Finite-difference operators (Neumann boundaries)
# ---------------------------------------------------------------------------


def _stencil(name, src, out_shape, shp3, r):
    out = empty(out_shape)
    _lib.call(name, _lib.ptr(src), _lib.ptr(out), _lib.i64arr(shp3), C.c_float(r), stream())
    return out


class Hessian3D:
    """[r^2 zz, yy, xx, sqrt2 r yz, sqrt2 r xz, sqrt2 xy]; norm^2 = 16 r^4 + 4 r^2 + 34
    (linops_mlx.py:182-262)."""

    def __init__(self, r: float = 1.0):
        self.r = r
        self.operator_norm_sq = 16.0 * (r ** 4) + 4.0 * (r ** 2) + 34.0

    @classmethod
    def from_spacing(cls, spacing: Tuple[float, float, float]) -> "Hessian3D":
        dz, dy, dx = spacing
        if abs(dy - dx) > 1e-2 * max(dy, dx):
            raise ValueError(
                f"Hessian3D.from_spacing assumes isotropic lateral sampling "
                f"(dy == dx); got dy={dy}, dx={dx}. Construct Hessian3D(r=...) "
                f"directly for anisotropic lateral spacing."
            )
        return cls(r=dy / dz)

    def forward(self, f):
        f = to_device(f)
        if f.dim() != 3:
            raise ValueError("Hessian3D expects a 3-D array")
        return _stencil("decon_hessian3d_forward", f, (6,) + tuple(f.shape), f.shape, self.r)

    def adjoint(self, H):
        H = to_device(H)
        if H.dim() != 4 or H.shape[0] != 6:
            raise ValueError("Hessian3D.adjoint expects an array of shape (6, Z, Y, X)")
        return _stencil("decon_hessian3d_adjoint", H, tuple(H.shape[1:]), H.shape[1:], self.r)

    def __call__(self, f):
        return self.forward(f)


class Hessian2D:
    """[yy, xx, sqrt2 xy]; norm^2 = 48 (linops_mlx.py:153-179).  Runs the 3-D
    stencil on a (1, H, W) view, whose zz / yz / xz components vanish."""

    operator_norm_sq = 48.0
    _COMP = (1, 2, 5)

    def forward(self, f):
        f = to_device(f)
        h = _stencil("decon_hessian3d_forward", f, (6, 1) + tuple(f.shape), (1,) + tuple(f.shape), 1.0)
        return h[list(self._COMP), 0].contiguous()

    def adjoint(self, H):
        H = to_device(H)
        full = torch.zeros((6, 1) + tuple(H.shape[1:]), dtype=torch.float32, device="cuda")
        full[list(self._COMP), 0] = H
        return _stencil("decon_hessian3d_adjoint", full, tuple(H.shape[1:]), (1,) + tuple(H.shape[1:]), 1.0)

    def __call__(self, f):
        return self.forward(f)


class Hessian1D:
    """d2 along the only axis; norm^2 = 16 (linops_mlx.py:130-150)."""

    operator_norm_sq = 16.0

    def forward(self, f):
        f = to_device(f)
        h = _stencil("decon_hessian3d_forward", f, (6, 1, 1) + tuple(f.shape), (1, 1) + tuple(f.shape), 1.0)
        return h[2, 0, 0].contiguous()

    def adjoint(self, g):
        g = to_device(g)
        full = torch.zeros((6, 1, 1) + tuple(g.shape), dtype=torch.float32, device="cuda")
        full[2, 0, 0] = g
        return _stencil("decon_hessian3d_adjoint", full, tuple(g.shape), (1, 1) + tuple(g.shape), 1.0)

    def __call__(self, f):
        return self.forward(f)


class Gradient3D:
    """(r dz, dy, dx) forward differences; norm^2 = 4 (r^2 + 2) (linops_mlx.py:92-122)."""

    def __init__(self, r: float = 1.0):
        self.r = r
        self.operator_norm_sq = 4.0 * (r * r + 2.0)

    def forward(self, f):
        f = to_device(f)
        return _stencil("decon_gradient3d_forward", f, (3,) + tuple(f.shape), f.shape, self.r)

    def adjoint(self, g):
        g = to_device(g)
        return _stencil("decon_gradient3d_adjoint", g, tuple(g.shape[1:]), g.shape[1:], self.r)

    def __call__(self, f):
        return self.forward(f)


class Gradient2D:
    """(dy, dx); norm^2 = 8 (linops_mlx.py:69-89)."""

    operator_norm_sq = 8.0

    def forward(self, f):
        f = to_device(f)
        g = _stencil("decon_gradient3d_forward", f, (3, 1) + tuple(f.shape), (1,) + tuple(f.shape), 1.0)
        return g[1:, 0].contiguous()

    def adjoint(self, g):
        g = to_device(g)
        full = torch.zeros((3, 1) + tuple(g.shape[1:]), dtype=torch.float32, device="cuda")
        full[1:, 0] = g
        return _stencil("decon_gradient3d_adjoint", full, tuple(g.shape[1:]), (1,) + tuple(g.shape[1:]), 1.0)

    def __call__(self, f):
        return self.forward(f)


class Gradient1D:
    """Forward difference along the only axis; norm^2 = 4 (linops_mlx.py:46-66)."""

    operator_norm_sq = 4.0

    def forward(self, f):
        f = to_device(f)
        g = _stencil("decon_gradient3d_forward", f, (3, 1, 1) + tuple(f.shape), (1, 1) + tuple(f.shape), 1.0)
        return g[2, 0, 0].contiguous()

    def adjoint(self, g):
        g = to_device(g)
        full = torch.zeros((3, 1, 1) + tuple(g.shape), dtype=torch.float32, device="cuda")
        full[2, 0, 0] = g
        return _stencil("decon_gradient3d_adjoint", full, tuple(g.shape), (1, 1) + tuple(g.shape), 1.0)

    def __call__(self, f):
        return self.forward(f)
