"""CPU-only checks: the C ABI library loads and exports every declared
symbol; host-side logic (FFT sizing, band tables, shape validation, operator
composition) matches the reference's rules.  No device compute is called."""

import ctypes
import os
import re

import numpy as np
import pytest

from oracle import ops

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "decon_b200.h")
LIB = os.path.join(ROOT, "deconlib_b200", "libdecon_b200.so")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(decon_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.skip("libdecon_b200.so not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(LIB)
    names = declared_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from deconlib_b200 import _lib

    missing = set(declared_symbols()) - set(_lib.exported_names())
    assert not missing, missing


def test_sizing_matches_reference_rules():
    from deconlib_b200 import _lib
    from deconlib_b200.deconvolution import fast_padded_shape

    for n in [1, 2, 7, 11, 13, 17, 31, 97, 127, 255, 257, 511, 847, 1000, 1021, 4097]:
        assert _lib.next_smooth(n) == ops.next_smooth_number(n)
    # linops_mlx.py:1008-1017 docstring examples
    assert fast_padded_shape((101, 589, 549), (101, 256, 256)) == (216, 864, 810)
    assert fast_padded_shape((101, 589, 549), (101, 256, 256), min_pad=(0, None, None)) == (108, 864, 810)
    assert fast_padded_shape((34, 311, 311), (101, 160, 160), min_pad=(0, None, None)) == (108, 480, 480)


@pytest.mark.parametrize("nl,ns", [(12, 6), (20, 16), (18, 7), (256, 128), (5, 4), (9, 1), (7, 7)])
def test_band_tables_bitwise_vs_oracle(nl, ns):
    from deconlib_b200 import _lib

    got = _lib.band_weights(nl, ns)
    ref = ops.banded_overlap_weights(nl, ns)
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)


def test_shape_validation_errors():
    from deconlib_b200.deconvolution import (Crop, FractionalAreaDownsample,
                                             FractionalAreaUpsample, compose)

    with pytest.raises(ValueError, match="Use Pad for upsizing"):
        Crop((10, 10), (12, 10))
    with pytest.raises(ValueError, match="must have same number of dimensions"):
        Crop((10, 10), (5,))
    with pytest.raises(ValueError, match="outside original size"):
        Crop((10, 10), (5, 5), start=(6, 0))
    with pytest.raises(ValueError, match="requires scale >= 1"):
        FractionalAreaDownsample(0.5)
    with pytest.raises(ValueError, match="requires scale >= 1"):
        FractionalAreaUpsample(0.9)
    with pytest.raises(ValueError, match="compose\\(\\) requires at least one operator"):
        compose()
    d = FractionalAreaDownsample(2.0, in_shape=(16, 32, 32))
    assert d.out_shape == (8, 16, 16) and d.operator_norm_sq == 8.0
    c = Crop((16, 32, 32), (8, 16, 16))
    with pytest.raises(ValueError, match="Cannot compose Crop after FractionalAreaDownsample"):
        compose(Crop((10, 16, 16), (8, 16, 16)), d)
    op = compose(c, Crop((20, 40, 40), (16, 32, 32)))
    assert op.in_shape == (20, 40, 40) and op.out_shape == (8, 16, 16)


def test_regulariser_norms_and_spacing():
    from deconlib_b200.deconvolution import Gradient3D, Hessian3D
    from deconlib_b200.deconvolution.pdhg import _compute_spacing_ratio, _create_regularizer

    assert Hessian3D(0.5).operator_norm_sq == 16 * 0.5 ** 4 + 4 * 0.25 + 34
    assert Gradient3D(2.0).operator_norm_sq == 4 * (4 + 2)
    r = _compute_spacing_ratio((0.05, 0.0425, 0.0425), 3)
    assert abs(r - 0.85) < 1e-12
    assert _compute_spacing_ratio(None, 3) == 1.0
    assert _create_regularizer("hessian", 2, 1.0, "L1").output_components == 3
    with pytest.raises(ValueError, match="Unknown regularization"):
        _create_regularizer("tv", 3, 1.0, "L1")
    with pytest.raises(ValueError, match="ndim must be 1, 2, or 3"):
        _create_regularizer("hessian", 4, 1.0, "L1")
    with pytest.raises(ValueError, match="spacing must have 3 elements"):
        _compute_spacing_ratio((1.0, 1.0), 3)


def test_no_cpu_fallback_without_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from deconlib_b200.deconvolution import LinearFFTConvolver

    with pytest.raises(RuntimeError, match="no CPU fallback"):
        LinearFFTConvolver(np.ones((3, 3, 3), np.float32), (8, 8, 8))


def test_product_package_never_imports_oracle():
    pkg = os.path.join(ROOT, "deconlib_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith(".py"):
                src = open(os.path.join(dirpath, f)).read()
                assert "import oracle" not in src and "from oracle" not in src, f
