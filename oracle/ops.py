"""CPU oracle for the 3D deconvolution path: operators.

TEST INFRASTRUCTURE ONLY.  This module is the checker that the CUDA path is
compared against.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` may import it; the product package
(``deconlib_b200``) never does.

It is a plain NumPy restatement of deconlib 0.4.0's operator algebra.  Each
function cites the reference file and line it follows.  Every routine takes a
``dtype`` (``np.float32`` or ``np.float64``): float32 reproduces the
reference's device precision, float64 gives the double-precision oracle.

Parity pin: ``tests/test_oracle_golden.py`` checks this module against golden
vectors produced by the reference's own source (``tests/golden/make_golden.py``).
"""

from __future__ import annotations

import math
from typing import Optional, Sequence, Tuple

import numpy as np

SQRT2 = math.sqrt(2.0)

# FFT backend: NumPy's pocketfft (single thread) by default; set_fft_workers(n)
# switches to scipy.fft (the same pocketfft algorithm) with n host threads,
# which the timed CPU baseline uses to give the reference every core.
_WORKERS = 1


def set_fft_workers(n: int) -> None:
    global _WORKERS
    _WORKERS = max(1, int(n))


def _rfftn(x):
    if _WORKERS > 1:
        import scipy.fft as sf

        return sf.rfftn(x, workers=_WORKERS)
    return np.fft.rfftn(x)


def _irfftn(x, s):
    if _WORKERS > 1:
        import scipy.fft as sf

        return sf.irfftn(x, s=s, workers=_WORKERS)
    return np.fft.irfftn(x, s=s)


def _c(dtype):
    return np.complex64 if np.dtype(dtype) == np.float32 else np.complex128


# ---------------------------------------------------------------------------
# FFT sizing (deconvolution/linops_mlx.py:956-1032)
# ---------------------------------------------------------------------------


def next_smooth_number(n: int) -> int:
    """Smallest m >= n whose only prime factors are 2, 3 and 5
    (linops_mlx.py:956-972)."""
    m = max(int(n), 1)
    while True:
        r = m
        for p in (2, 3, 5):
            while r % p == 0:
                r //= p
        if r == 1:
            return m
        m += 1


def fast_padded_shape(signal_shape, kernel_shape, min_pad=None):
    """Per-axis 5-smooth size >= max(N + pad, M), pad = M - 1 by default
    (linops_mlx.py:975-1032)."""
    nd = len(signal_shape)
    if min_pad is None:
        pads = (None,) * nd
    elif isinstance(min_pad, int):
        pads = (min_pad,) * nd
    else:
        pads = tuple(min_pad)
    out = []
    for n, m, p in zip(signal_shape, kernel_shape, pads):
        need = (m - 1) if p is None else int(p)
        out.append(next_smooth_number(max(n + need, m)))
    return tuple(out)


def pad_corner_origin_kernel(kernel: np.ndarray, out_shape) -> np.ndarray:
    """Embed a corner-origin kernel in a larger canvas: the first ceil(m/2)
    samples of each axis stay at the low end, the remaining ones move to the
    high end (utils/padding.py:142-190)."""
    kernel = np.asarray(kernel)
    out_shape = tuple(int(s) for s in out_shape)
    if len(out_shape) != kernel.ndim:
        raise ValueError(f"output_shape has {len(out_shape)} dims, expected {kernel.ndim}")
    for ax, (m, f) in enumerate(zip(kernel.shape, out_shape)):
        if f < m:
            raise ValueError(
                f"output size {f} cannot be smaller than kernel size {m} in dimension {ax}"
            )
    # Destination index of every source index, per axis.
    dest = []
    for m, f in zip(kernel.shape, out_shape):
        i = np.arange(m)
        npos = (m + 1) // 2
        dest.append(np.where(i < npos, i, f - (m - i)))
    out = np.zeros(out_shape, dtype=kernel.dtype)
    out[np.ix_(*dest)] = kernel
    return out


# ---------------------------------------------------------------------------
# Pad / Crop (deconvolution/core_operators.py:29-137)
# ---------------------------------------------------------------------------


class Pad:
    """Zero padding; adjoint crops (core_operators.py:29-59)."""

    def __init__(self, padding):
        self.padding = tuple((int(a), int(b)) for a, b in padding)
        self.operator_norm_sq = 1.0

    def forward(self, x):
        return np.pad(x, self.padding, mode="constant")

    def adjoint(self, y):
        sl = tuple(slice(a, s - b) for (a, b), s in zip(self.padding, y.shape))
        return y[sl]


class Crop:
    """Centre (or explicit-start) crop; adjoint zero-pads
    (core_operators.py:62-137)."""

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
        self.start = []
        for i, (o, t) in enumerate(zip(self.original_shape, self.target_shape)):
            if t > o:
                raise ValueError(f"Target size {t} > original size {o}. Use Pad for upsizing.")
            s0 = (o - t) // 2 if start is None else int(start[i])
            if start is not None and (s0 < 0 or s0 + t > o):
                raise ValueError(
                    f"start {s0} on axis {i} puts crop window [{s0}, {s0 + t}) "
                    f"outside original size {o}"
                )
            self.start.append(s0)
        self.start = tuple(self.start)

    def forward(self, x):
        return x[tuple(slice(s, s + t) for s, t in zip(self.start, self.target_shape))]

    def adjoint(self, y):
        pw = tuple((s, o - s - t) for s, t, o in zip(self.start, self.target_shape, self.original_shape))
        return np.pad(y, pw, mode="constant")


# ---------------------------------------------------------------------------
# Fractional-area resampling (core_operators.py:151-450)
# ---------------------------------------------------------------------------


def banded_overlap_weights(n_large: int, n_small: int):
    """Interval-overlap weights |[i*s,(i+1)s) ∩ [j,j+1)| as fixed-width
    windows, s = n_large / n_small, computed in float64
    (core_operators.py:151-202).

    Returns (idx_fwd int32 (n_small, wf), w_fwd f32, idx_adj int32
    (n_large, wa), w_adj f32).
    """
    s = n_large / n_small
    wf = min(n_large, int(math.ceil(s)) + 2)
    i = np.arange(n_small)
    first = np.clip(np.floor(i * s).astype(np.int64), 0, n_large - wf)
    idx_f = first[:, None] + np.arange(wf)[None, :]
    lo = (i * s)[:, None]
    hi = ((i + 1) * s)[:, None]
    jf = idx_f.astype(np.float64)
    w_f = np.maximum(0.0, np.minimum(hi, jf + 1) - np.maximum(lo, jf))

    wa = min(n_small, int(math.ceil(1.0 / s)) + 3)
    j = np.arange(n_large)
    first_a = np.clip(np.floor(j / s).astype(np.int64) - 1, 0, n_small - wa)
    idx_a = first_a[:, None] + np.arange(wa)[None, :]
    a_lo = idx_a.astype(np.float64) * s
    a_hi = (idx_a.astype(np.float64) + 1) * s
    jj = j[:, None].astype(np.float64)
    w_a = np.maximum(0.0, np.minimum(a_hi, jj + 1) - np.maximum(a_lo, jj))
    return (idx_f.astype(np.int32), w_f.astype(np.float32),
            idx_a.astype(np.int32), w_a.astype(np.float32))


def apply_banded(x, idx, w, axis, dtype):
    """out[..., i, ...] = sum_k w[i, k] * x[..., idx[i, k], ...]
    (core_operators.py:205-219)."""
    xm = np.moveaxis(x, axis, -1)
    g = xm[..., idx]  # (..., out, width)
    out = np.sum(g * w.astype(dtype), axis=-1)
    return np.moveaxis(out, -1, axis)


def _expand_scale(scale, axes):
    return scale * len(axes) if (len(scale) == 1 and len(axes) > 1) else scale


class FractionalAreaDownsample:
    """Fine -> coarse banded area sum; adjoint is the exact transpose
    (core_operators.py:222-352)."""

    def __init__(self, scale, axes=None, in_shape=None, dtype=np.float32):
        if isinstance(scale, (int, float)):
            scale = (float(scale),)
        self.scale = tuple(float(s) for s in scale)
        if any(s < 1.0 for s in self.scale):
            raise ValueError(
                f"FractionalAreaDownsample requires scale >= 1 (fine -> coarse); "
                f"got {self.scale}. Use FractionalAreaUpsample to upsample."
            )
        self.axes = axes
        self.dtype = dtype
        self.axis_map = {}
        self.in_shape = None
        self.out_shape = None
        if in_shape is not None:
            ax = axes if axes is not None else tuple(range(len(in_shape)))
            for a, s in zip(ax, _expand_scale(self.scale, ax)):
                nl = in_shape[a]
                self.axis_map[a] = (nl, max(1, int(round(nl / s))))
            self.in_shape = tuple(int(s) for s in in_shape)
            out = list(self.in_shape)
            for a, (_, ns) in self.axis_map.items():
                out[a % len(out)] = ns
            self.out_shape = tuple(out)
        if self.axis_map:
            n2 = 1.0
            for nl, ns in self.axis_map.values():
                n2 *= nl / ns
        else:
            n2 = math.prod(self.scale)
        self.operator_norm_sq = float(n2)

    def forward(self, x):
        axes = self.axes if self.axes is not None else tuple(range(x.ndim))
        out = x
        for a, s in zip(axes, _expand_scale(self.scale, axes)):
            if a in self.axis_map:
                nl, ns = self.axis_map[a]
            else:
                nl = out.shape[a]
                ns = max(1, int(round(nl / s)))
            if nl == ns:
                continue
            i_f, w_f, _, _ = banded_overlap_weights(nl, ns)
            out = apply_banded(out, i_f, w_f, a, self.dtype)
        return out

    def adjoint(self, y):
        axes = self.axes if self.axes is not None else tuple(range(y.ndim))
        out = y
        for a, s in zip(axes, _expand_scale(self.scale, axes)):
            if a in self.axis_map:
                nl, ns = self.axis_map[a]
            else:
                ns = out.shape[a]
                nl = max(1, int(round(ns * s)))
            if nl == ns:
                continue
            _, _, i_a, w_a = banded_overlap_weights(nl, ns)
            out = apply_banded(out, i_a, w_a, a, self.dtype)
        return out


class FractionalAreaUpsample:
    """Coarse -> fine spreading W_up = (n_small/n_large) W_dn^T; adjoint is
    ratio * W_dn (core_operators.py:355-450)."""

    def __init__(self, scale, axes=None, dtype=np.float32):
        if isinstance(scale, (int, float)):
            scale = (float(scale),)
        self.scale = tuple(float(s) for s in scale)
        if any(s < 1.0 for s in self.scale):
            raise ValueError(
                f"FractionalAreaUpsample requires scale >= 1 (coarse -> fine); "
                f"got {self.scale}. Use FractionalAreaDownsample to downsample."
            )
        self.axes = axes
        self.dtype = dtype
        self.operator_norm_sq = 1.0

    def _band(self, nl, ns):
        i_f, w_f, i_a, w_a = banded_overlap_weights(nl, ns)
        r = ns / nl
        return i_a, w_a * r, i_f, w_f * r

    def forward(self, x):
        axes = self.axes if self.axes is not None else tuple(range(x.ndim))
        out = x
        for a, s in zip(axes, _expand_scale(self.scale, axes)):
            ns = out.shape[a]
            nl = max(1, int(round(ns * s)))
            if nl == ns:
                continue
            iu, wu, _, _ = self._band(nl, ns)
            out = apply_banded(out, iu, wu, a, self.dtype)
        return out

    def adjoint(self, y):
        axes = self.axes if self.axes is not None else tuple(range(y.ndim))
        out = y
        for a, s in zip(axes, _expand_scale(self.scale, axes)):
            nl = out.shape[a]
            ns = max(1, int(round(nl / s)))
            if nl == ns:
                continue
            _, _, idn, wdn = self._band(nl, ns)
            out = apply_banded(out, idn, wdn, a, self.dtype)
        return out


# ---------------------------------------------------------------------------
# FFT convolution (deconvolution/linops_mlx.py:384-533)
# ---------------------------------------------------------------------------


class FFTConvolver:
    """Circular convolution by a stored OTF = rfftn(kernel / sum(kernel))
    (linops_mlx.py:384-432)."""

    def __init__(self, kernel, normalize=True, dtype=np.float32):
        k = np.asarray(kernel).astype(dtype)
        self.shape = k.shape
        self.in_shape = self.out_shape = tuple(int(s) for s in k.shape)
        self.dtype = dtype
        if normalize:
            k = k / np.sum(k)
        self.otf = _rfftn(k).astype(_c(dtype))
        self.operator_norm_sq = float(np.max(np.abs(self.otf) ** 2))

    def forward(self, x):
        return _irfftn(_rfftn(x) * self.otf, self.shape).astype(self.dtype)

    def adjoint(self, y):
        return _irfftn(_rfftn(y) * np.conj(self.otf), self.shape).astype(self.dtype)


class LinearFFTConvolver:
    """Wrap-free convolution on ``signal_shape``: zero-pad to ``fft_shape``,
    circular convolution with the corner-embedded kernel, crop
    (linops_mlx.py:435-533)."""

    def __init__(self, kernel, signal_shape, normalize=True, fft_shape=None, dtype=np.float32):
        k = np.asarray(kernel)
        self.signal_shape = tuple(int(s) for s in signal_shape)
        self.in_shape = self.out_shape = self.signal_shape
        self.kernel_shape = tuple(int(s) for s in k.shape)
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
                f"fft_shape {self.fft_shape} is too small for linear convolution; "
                f"minimum is {minimum}"
            )
        # The reference embeds the float32-cast kernel (linops_mlx.py:508-511).
        padded = pad_corner_origin_kernel(k.astype(np.float32), self.fft_shape)
        self._pad = Pad(tuple((0, f - n) for n, f in zip(self.signal_shape, self.fft_shape)))
        self._conv = FFTConvolver(padded, normalize=normalize, dtype=dtype)
        self.otf = self._conv.otf
        self.operator_norm_sq = self._conv.operator_norm_sq

    def forward(self, x):
        return self._pad.adjoint(self._conv.forward(self._pad.forward(x)))

    def adjoint(self, y):
        return self._pad.adjoint(self._conv.adjoint(self._pad.forward(y)))


# ---------------------------------------------------------------------------
# Composition (deconvolution/composition.py:52-122)
# ---------------------------------------------------------------------------


class Compose:
    """outer(inner(x)); adjoint reversed; norm = product
    (composition.py:52-106)."""

    def __init__(self, outer, inner):
        oi = getattr(outer, "in_shape", None)
        io = getattr(inner, "out_shape", None)
        if oi is not None and io is not None and tuple(oi) != tuple(io):
            raise ValueError(
                f"Cannot compose {type(outer).__name__} after {type(inner).__name__}"
            )
        self.outer, self.inner = outer, inner
        self.in_shape = getattr(inner, "in_shape", None)
        self.out_shape = getattr(outer, "out_shape", None)
        self.operator_norm_sq = float(outer.operator_norm_sq * inner.operator_norm_sq)

    def forward(self, x):
        return self.outer.forward(self.inner.forward(x))

    def adjoint(self, y):
        return self.inner.adjoint(self.outer.adjoint(y))


def compose(*ops):
    """compose(A, B, C)(x) = A(B(C(x))) (composition.py:109-122)."""
    if not ops:
        raise ValueError("compose() requires at least one operator")
    out = ops[-1]
    for op in reversed(ops[:-1]):
        out = Compose(op, out)
    return out


# ---------------------------------------------------------------------------
# Finite differences, Neumann boundary (deconvolution/linops_core_mlx.py:25-80)
# ---------------------------------------------------------------------------


def _edge_pad(f, axis):
    f = np.moveaxis(f, axis, 0)
    return np.concatenate([f[:1], f, f[-1:]], axis=0)


def d1_fwd(f, axis):
    """(Df)[i] = f[i+1] - f[i], f[n] = f[n-1] (linops_core_mlx.py:25-32)."""
    g = np.moveaxis(f, axis, 0)
    r = np.concatenate([g[1:], g[-1:]], axis=0) - g
    return np.moveaxis(r, 0, axis)


def d1_fwd_adj(g, axis):
    """Adjoint of d1_fwd (linops_core_mlx.py:35-39)."""
    h = np.moveaxis(g, axis, 0)
    r = np.concatenate([-h[:1], h[:-2] - h[1:-1], h[-2:-1]], axis=0)
    return np.moveaxis(r, 0, axis)


def d1_cen(f, axis):
    """(f[i+1] - f[i-1]) / 2 with edge replication (linops_core_mlx.py:42-50)."""
    p = _edge_pad(f, axis)
    return np.moveaxis((p[2:] - p[:-2]) / 2.0, 0, axis)


def d1_cen_adj(g, axis):
    """Adjoint of d1_cen (linops_core_mlx.py:53-58)."""
    h = np.moveaxis(g, axis, 0)
    p = np.concatenate([-h[:1], h, -h[-1:]], axis=0)
    return np.moveaxis((p[:-2] - p[2:]) / 2.0, 0, axis)


def d2(f, axis):
    """f[i-1] - 2 f[i] + f[i+1] with edge replication; self-adjoint
    (linops_core_mlx.py:66-80)."""
    p = _edge_pad(f, axis)
    return np.moveaxis(p[:-2] - 2 * p[1:-1] + p[2:], 0, axis)


class Hessian3D:
    """Six weighted second differences [zz, yy, xx, yz, xz, xy] x
    [r^2, 1, 1, sqrt2 r, sqrt2 r, sqrt2]; norm^2 = 16 r^4 + 4 r^2 + 34
    (linops_mlx.py:182-262)."""

    def __init__(self, r=1.0, dtype=np.float32):
        self.r = r
        self.dtype = dtype
        self.operator_norm_sq = 16.0 * r ** 4 + 4.0 * r ** 2 + 34.0
        self.weights = np.array([r ** 2, 1.0, 1.0, r * SQRT2, r * SQRT2, SQRT2]).astype(dtype)

    def forward(self, f):
        dz = d1_cen(f, 0)
        dy = d1_cen(f, 1)
        h = np.stack([d2(f, 0), d2(f, 1), d2(f, 2), d1_cen(dz, 1), d1_cen(dz, 2), d1_cen(dy, 2)])
        return h * self.weights.reshape(6, 1, 1, 1)

    def adjoint(self, h):
        hw = h * self.weights.reshape(6, 1, 1, 1)
        return (d2(hw[0], 0) + d2(hw[1], 1) + d2(hw[2], 2)
                + d1_cen_adj(d1_cen_adj(hw[3], 1), 0)
                + d1_cen_adj(d1_cen_adj(hw[4], 2), 0)
                + d1_cen_adj(d1_cen_adj(hw[5], 2), 1))


class Hessian2D:
    """[yy, xx, sqrt2 xy]; norm^2 = 48 (linops_mlx.py:153-179)."""

    operator_norm_sq = 48.0

    def __init__(self, dtype=np.float32):
        self.dtype = dtype

    def forward(self, f):
        s2 = self.dtype(SQRT2)
        return np.stack([d2(f, 0), d2(f, 1), s2 * d1_cen(d1_cen(f, 0), 1)])

    def adjoint(self, h):
        s2 = self.dtype(SQRT2)
        return d2(h[0], 0) + d2(h[1], 1) + s2 * d1_cen_adj(d1_cen_adj(h[2], 0), 1)


class Hessian1D:
    """d2 along axis 0; norm^2 = 16 (linops_mlx.py:130-150)."""

    operator_norm_sq = 16.0

    def forward(self, f):
        return d2(f, 0)

    def adjoint(self, h):
        return d2(h, 0)


class Gradient3D:
    """(r dz, dy, dx) forward differences; norm^2 = 4 (r^2 + 2)
    (linops_mlx.py:92-122)."""

    def __init__(self, r=1.0, dtype=np.float32):
        self.r = r
        self.operator_norm_sq = 4.0 * (r * r + 2.0)

    def forward(self, f):
        return np.stack([self.r * d1_fwd(f, 0), d1_fwd(f, 1), d1_fwd(f, 2)])

    def adjoint(self, g):
        return d1_fwd_adj(self.r * g[0], 0) + d1_fwd_adj(g[1], 1) + d1_fwd_adj(g[2], 2)


class Gradient2D:
    """(dy, dx); norm^2 = 8 (linops_mlx.py:69-89)."""

    operator_norm_sq = 8.0

    def forward(self, f):
        return np.stack([d1_fwd(f, 0), d1_fwd(f, 1)])

    def adjoint(self, g):
        return d1_fwd_adj(g[0], 0) + d1_fwd_adj(g[1], 1)


class Gradient1D:
    """d1_fwd along axis 0; norm^2 = 4 (linops_mlx.py:46-66)."""

    operator_norm_sq = 4.0

    def forward(self, f):
        return d1_fwd(f, 0)

    def adjoint(self, g):
        return d1_fwd_adj(g, 0)
