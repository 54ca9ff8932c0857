"""deconlib_b200: B200-native (sm_100a) 3D deconvolution behind deconlib's API.

The device work runs in ``libdecon_b200.so`` (hand-written CUDA, C ABI in
``include/decon_b200.h``); this package is the Python host side that mirrors
``deconlib.deconvolution``.  There is no CPU fallback.
"""

from . import deconvolution  # noqa: F401

__version__ = "0.1.0"
