"""NumPy stand-in for the subset of ``mlx.core`` that deconlib's deconvolution
path calls.  Test infrastructure only: it lets ``make_golden.py`` run the
reference's own solver source (which imports ``mlx.core``) on the CPU so that
its outputs can be frozen as golden fixtures.

Semantics kept from MLX:
  * ``mx.array(...)`` produces float32 / complex64 arrays (float64 input is
    narrowed), and ``isinstance(np_array, mx.array)`` is true.
  * A bare Python float handed to an ``mx`` function becomes a float32
    0-d array, so scalar arithmetic such as ``mx.sqrt(1.0 + theta) * tau``
    runs in float32 as it does on the device.

Setting ``DECON_STANDIN_FP64=1`` before import widens every float to float64
and every complex to complex128, which turns the same reference source into
a double-precision run.
"""

import os

import numpy as np

_FP64 = os.environ.get("DECON_STANDIN_FP64", "0") == "1"

float32 = np.float64 if _FP64 else np.float32
complex64 = np.complex128 if _FP64 else np.complex64
float64 = np.float64
float16 = np.float16
int32 = np.int32
int64 = np.int64
bool_ = np.bool_
uint32 = np.uint32

_FT = np.dtype(float32)
_CT = np.dtype(complex64)


def _narrow(a):
    a = np.asarray(a)
    if a.dtype.kind == "f" and a.dtype != _FT:
        return a.astype(_FT)
    if a.dtype.kind == "c" and a.dtype != _CT:
        return a.astype(_CT)
    return a


def _arg(x):
    """Python scalars become device-precision 0-d arrays (MLX behaviour)."""
    if isinstance(x, bool):
        return np.bool_(x)
    if isinstance(x, float):
        return _FT.type(x)
    if isinstance(x, complex):
        return _CT.type(x)
    return x


class _ArrayMeta(type):
    def __instancecheck__(cls, obj):
        return isinstance(obj, (np.ndarray, np.generic))

    def __call__(cls, x, dtype=None):
        a = np.asarray(x)
        if dtype is not None:
            return a.astype(dtype)
        if a.dtype.kind in "fc":
            return _narrow(a)
        if a.dtype == np.int64:
            return a.astype(np.int32)
        return a


class array(metaclass=_ArrayMeta):
    pass


def eval(*args):  # noqa: A001 - mirrors mlx.core.eval
    return None


def compile(fn, *args, **kwargs):  # noqa: A001 - mirrors mlx.core.compile
    return fn


def _unary(fn):
    def wrapped(x, *a, **k):
        return fn(_arg(x), *a, **k)

    return wrapped


def _binary(fn):
    def wrapped(x, y, *a, **k):
        return fn(_arg(x), _arg(y), *a, **k)

    return wrapped


maximum = _binary(np.maximum)
minimum = _binary(np.minimum)
sqrt = _unary(np.sqrt)
log = _unary(np.log)
exp = _unary(np.exp)
abs = _unary(np.abs)  # noqa: A001
conj = _unary(np.conj)
isfinite = _unary(np.isfinite)
square = _unary(np.square)
sign = _unary(np.sign)


def where(c, a, b):
    return np.where(c, _arg(a), _arg(b))


def clip(x, a_min, a_max):
    return np.clip(_arg(x), _arg(a_min), _arg(a_max))


def sum(x, axis=None, keepdims=False):  # noqa: A001
    return np.sum(_arg(x), axis=axis, keepdims=keepdims)


def mean(x, axis=None, keepdims=False):
    return np.mean(_arg(x), axis=axis, keepdims=keepdims)


def max(x, axis=None, keepdims=False):  # noqa: A001
    return np.max(_arg(x), axis=axis, keepdims=keepdims)


def min(x, axis=None, keepdims=False):  # noqa: A001
    return np.min(_arg(x), axis=axis, keepdims=keepdims)


def all(x, axis=None, keepdims=False):  # noqa: A001
    return np.all(x, axis=axis, keepdims=keepdims)


def allclose(a, b, rtol=1e-5, atol=1e-8, equal_nan=False):
    return np.bool_(np.allclose(a, b, rtol=rtol, atol=atol, equal_nan=equal_nan))


def zeros(shape, dtype=None):
    return np.zeros(shape, dtype=dtype or float32)


def ones(shape, dtype=None):
    return np.ones(shape, dtype=dtype or float32)


def full(shape, vals, dtype=None):
    return np.full(shape, vals, dtype=dtype or float32)


def zeros_like(x):
    return np.zeros_like(x)


def ones_like(x):
    return np.ones_like(x)


def pad(x, pad_width, mode="constant", constant_values=0):
    return np.pad(x, pad_width, mode=mode, constant_values=constant_values)


def take(x, idx, axis=None):
    return np.take(x, idx, axis=axis)


def moveaxis(x, a, b):
    return np.moveaxis(x, a, b)


def swapaxes(x, a, b):
    return np.swapaxes(x, a, b)


def concatenate(xs, axis=0):
    return np.concatenate(xs, axis=axis)


def stack(xs, axis=0):
    return np.stack(xs, axis=axis)


def expand_dims(x, axis):
    return np.expand_dims(x, axis)


def reshape(x, shape):
    return np.reshape(x, shape)


def arange(*args, dtype=None):
    return np.arange(*args, dtype=dtype)


class fft:  # noqa: N801 - mirrors the mlx.core.fft namespace
    @staticmethod
    def rfftn(x, s=None, axes=None):
        return np.fft.rfftn(x, s=s, axes=axes)

    @staticmethod
    def irfftn(x, s=None, axes=None):
        return np.fft.irfftn(x, s=s, axes=axes)

    @staticmethod
    def fftn(x, s=None, axes=None):
        return np.fft.fftn(x, s=s, axes=axes)

    @staticmethod
    def ifftn(x, s=None, axes=None):
        return np.fft.ifftn(x, s=s, axes=axes)

    @staticmethod
    def rfft(x, n=None, axis=-1):
        return np.fft.rfft(x, n=n, axis=axis)

    @staticmethod
    def irfft(x, n=None, axis=-1):
        return np.fft.irfft(x, n=n, axis=axis)

    @staticmethod
    def fft2(x, s=None, axes=(-2, -1)):
        return np.fft.fft2(x, s=s, axes=axes)

    @staticmethod
    def ifft2(x, s=None, axes=(-2, -1)):
        return np.fft.ifft2(x, s=s, axes=axes)


class random:  # noqa: N801 - mirrors the mlx.core.random namespace
    _rng = np.random.default_rng(0)

    @classmethod
    def seed(cls, s):
        cls._rng = np.random.default_rng(s)

    @classmethod
    def normal(cls, shape=(), dtype=None, loc=0.0, scale=1.0, key=None):
        return cls._rng.normal(loc, scale, size=shape).astype(dtype or float32)

    @classmethod
    def uniform(cls, low=0.0, high=1.0, shape=(), dtype=None, key=None):
        return cls._rng.uniform(low, high, size=shape).astype(dtype or float32)
