"""The bounded mbarrier wait of the TMA kernels, driven to its limit.

``decon_test_wait_timeout`` makes one CTA wait, through the same bounded wait
the column passes use, on an mbarrier that nothing completes.  The wait gives
up after the given number of polls and the kernel returns: no fault, no hang,
the context stays usable.  ``decon_device_status`` must then report
DECON_ERR_TIMEOUT, ``decon_device_status_clear`` must reset it, and a
convolution afterwards must run and report a clean status.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_is_reported():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from deconlib_b200 import _lib
    import deconlib_b200.deconvolution as D

    lib = _lib.load()
    st = _lib.stream_ptr()
    assert lib.decon_device_status_clear(st) == _lib.OK
    assert lib.decon_device_status(st) == _lib.OK
    assert lib.decon_test_wait_timeout(1024, st) == _lib.OK
    assert lib.decon_device_status(st) == _lib.ERR_TIMEOUT
    assert b"bounded" in lib.decon_last_error()
    # sticky until cleared
    assert lib.decon_device_status(st) == _lib.ERR_TIMEOUT
    assert lib.decon_device_status_clear(st) == _lib.OK
    assert lib.decon_device_status(st) == _lib.OK
    # argument check on the host
    assert lib.decon_test_wait_timeout(0, st) == _lib.ERR_VALUE
    # the context is still usable: a convolution runs and reports clean
    rng = np.random.default_rng(0)
    k = rng.random((5, 7, 9)).astype(np.float32)
    x = rng.random((16, 32, 32)).astype(np.float32)
    c = D.LinearFFTConvolver(k, x.shape)
    y = c.forward(x)
    torch.cuda.synchronize()
    assert torch.isfinite(y).all()
    assert lib.decon_device_status(st) == _lib.OK
