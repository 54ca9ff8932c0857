"""ctypes binding of ``libdecon_b200.so`` (the C ABI in ``include/decon_b200.h``).

The product path has no CPU fallback: every array operation of the package
goes through this library on a CUDA device.  Importing works without a GPU
(so shape logic and the exported symbols can be checked on any host); the
first call that needs the device raises ``RuntimeError`` if there is none.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdecon_b200.so")

OK, ERR_VALUE, ERR_UNSUPPORTED, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_NULL = range(7)
RED_SUM, RED_SUMSQ, RED_DIFFSQ, RED_MAX, RED_DOT = range(5)

_i64 = C.c_int64
_p = C.c_void_p
_i64p = C.POINTER(C.c_int64)
_dp = C.POINTER(C.c_double)

# name -> (restype, argtypes)
_SIGS = {
    "decon_last_error": (C.c_char_p, []),
    "decon_version": (C.c_int, []),
    "decon_launch_count": (_i64, []),
    "decon_device_status": (C.c_int, [_p]),
    "decon_device_status_clear": (C.c_int, [_p]),
    "decon_pdhg_solver_create": (C.c_int, [_p, _p, _i64p, _dp, C.c_float, C.c_int, _p, C.c_double,
                                           C.c_double, C.c_int, C.c_int, C.c_double, C.c_double,
                                           C.c_double, C.c_int, C.c_int, C.c_int, _p, C.POINTER(_p)]),
    "decon_pdhg_run": (C.c_int, [_p, C.c_int, _p]),
    "decon_pdhg_solver_x": (C.c_int, [_p, _p, _p]),
    "decon_pdhg_solver_state": (C.c_int, [_p, C.POINTER(_p), C.POINTER(C.c_int)]),
    "decon_pdhg_solver_destroy": (C.c_int, [_p]),
    "decon_test_wait_timeout": (C.c_int, [C.c_uint, _p]),
    "decon_next_smooth": (_i64, [_i64]),
    "decon_fast_padded_shape": (C.c_int, [C.c_int, _i64p, _i64p, _i64p, _i64p]),
    "decon_conv_create": (C.c_int, [_p, _i64p, _i64p, _i64p, C.c_int, _p, C.POINTER(_p)]),
    "decon_conv_destroy": (C.c_int, [_p]),
    "decon_conv_set_kernel": (C.c_int, [_p, _p, C.c_int, _p]),
    "decon_conv_set_precision": (C.c_int, [_p, C.c_int, _p]),
    "decon_conv_norm_sq": (C.c_int, [_p, _dp]),
    "decon_conv_fused_yz": (C.c_int, [_p, C.POINTER(C.c_int)]),
    "decon_conv_set_schedule": (C.c_int, [_p, C.c_int]),
    "decon_conv_get_schedule": (C.c_int, [_p, C.POINTER(C.c_int)]),
    "decon_conv_shape": (C.c_int, [_p, _i64p, _i64p]),
    "decon_conv_get_otf": (C.c_int, [_p, _p, _p]),
    "decon_conv_forward": (C.c_int, [_p, _p, _p, _p]),
    "decon_conv_adjoint": (C.c_int, [_p, _p, _p, _p]),
    "decon_conv_forward_down2": (C.c_int, [_p, _p, _p, _p]),
    "decon_conv_adjoint_up2": (C.c_int, [_p, _p, _p, _p]),
    "decon_rl_setup": (C.c_int, [_p, _p, C.c_float, _p, _p, _p, _p]),
    "decon_rl_iteration": (C.c_int, [_p, _p, C.c_float, _p, _p, _p, _p, _p]),
    "decon_rl_predict": (C.c_int, [_p, _p, C.c_float, _p, _p, _p, _p]),
    "decon_rl_run": (C.c_int, [_p, _p, C.c_float, _p, _p, _p, C.c_int, _p]),
    "decon_pupil_to_psf": (C.c_int, [_p, _p, _p, _i64, _i64, _i64, C.c_int, _p, _p]),
    "decon_psf_geometry": (C.c_int, [_i64, _i64, C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_int, C.c_double, _p, _p, _p, _p, _p, _p, _p,
                                     _p, _p, _p, _p]),
    "decon_psf_pupil": (C.c_int, [_p, _p, _p, _i64, C.c_int, _p, _p]),
    "decon_psf_defocus": (C.c_int, [_p, _i64, C.c_double, _p, _p]),
    "decon_psf_index_mismatch": (C.c_int, [_p, _p, _i64, C.c_double, C.c_double, C.c_double,
                                           C.c_double, _p, _p]),
    "decon_psf_zernike": (C.c_int, [_p, _p, _p, _i64, C.c_int, C.POINTER(C.c_int),
                                    C.POINTER(C.c_double), _p, _p]),
    "decon_nlcg_create": (C.c_int, [_p]),
    "decon_nlcg_destroy": (C.c_int, [_p]),
    "decon_nlcg_init": (C.c_int, [_p, _p, _p, _i64, C.c_int, _p]),
    "decon_nlcg_model": (C.c_int, [_p, _p, _p, C.c_float, _p, _i64, _p]),
    "decon_nlcg_products": (C.c_int, [_p, C.c_int, C.c_float, _p, _p, _p, _p, _p, _p, _i64, _p]),
    "decon_nlcg_gram": (C.c_int, [_p, _p, _p, _p, _i64, _p]),
    "decon_nlcg_newton": (C.c_int, [_p, _p, _p, _p, _p, C.c_float, C.c_float, C.c_double, C.c_int,
                                    C.c_int, _i64, _p]),
    "decon_nlcg_accept": (C.c_int, [_p, _p, _p, _p, _p, C.c_float, C.c_float, _p, _p, _i64, _p, _p, _p,
                                    _p, _i64, _p]),
    "decon_nlcg_energy": (C.c_int, [_p, _p, _i64, _p]),
    "decon_nlcg_gradient": (C.c_int, [_p, _p, _p, _p, _p, _p, C.c_float, C.c_float, _p, _i64, _p]),
    "decon_nlcg_quad": (C.c_int, [_p, _p, _p, _p, _i64, _p, _p, _i64, C.c_float, _p]),
    "decon_nlcg_hess_gram": (C.c_int, [_p, _p, _p, _p, _p, C.c_float, _p]),
    "decon_nlcg_hess_energy": (C.c_int, [_p, _p, _p, C.c_float, _p]),
    "decon_nlcg_read": (C.c_int, [_p, _p, _p]),
    "decon_batch_rl_create": (C.c_int, [C.c_int, _p, _p, _p, _p, _p, _p, C.c_int, C.POINTER(_p)]),
    "decon_batch_rl_setup": (C.c_int, [_p, _p, _p]),
    "decon_batch_rl_run": (C.c_int, [_p, C.c_int, C.c_int, _p]),
    "decon_batch_rl_predict": (C.c_int, [_p, _p, _p]),
    "decon_batch_graph_nodes": (C.c_int, [_p, C.c_int, _i64p]),
    "decon_batch_destroy": (C.c_int, [_p]),
    "decon_rl_ratio": (C.c_int, [_p, _p, C.c_float, _p, _i64, _p, _p, _p]),
    "decon_rl_update": (C.c_int, [_p, _p, _p, _i64, _p]),
    "decon_rl_data_floor": (C.c_int, [_p, C.c_float, _p, _i64, _p]),
    "decon_rl_mask": (C.c_int, [_p, _p, _i64, _p, _p]),
    "decon_fill": (C.c_int, [_p, C.c_float, _i64, _p]),
    "decon_clamp_min": (C.c_int, [_p, C.c_float, _p, _i64, _p]),
    "decon_affine": (C.c_int, [_p, C.c_float, C.c_float, _p, _i64, _p]),
    "decon_conv_create_circular": (C.c_int, [_p, _i64p, C.c_int, _p, C.POINTER(_p)]),
    "decon_window_copy": (C.c_int, [_p, _i64p, _i64p, _p, _i64p, _i64p, _i64p, C.c_int, _p]),
    "decon_band_widths": (C.c_int, [_i64, _i64, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "decon_band_weights": (C.c_int, [_i64, _i64, _p, _p, _p, _p]),
    "decon_banded_axis": (C.c_int, [_p, _p, _i64, _i64, _i64, _i64, _p, _p, C.c_int, _p]),
    "decon_hessian3d_forward": (C.c_int, [_p, _p, _i64p, C.c_float, _p]),
    "decon_hessian3d_adjoint": (C.c_int, [_p, _p, _i64p, C.c_float, _p]),
    "decon_gradient3d_forward": (C.c_int, [_p, _p, _i64p, C.c_float, _p]),
    "decon_gradient3d_adjoint": (C.c_int, [_p, _p, _i64p, C.c_float, _p]),
    "decon_reduce_workspace_bytes": (_i64, []),
    "decon_reduce": (C.c_int, [_p, _p, _i64, C.c_int, _p, _p, _p]),
    "decon_reduce_noalloc": (C.c_int, [_p, _p, _i64, C.c_int, _p, _p]),
    "decon_pdhg_create": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_int, C.c_int, C.POINTER(_p)]),
    "decon_pdhg_destroy": (C.c_int, [_p]),
    "decon_pdhg_reset": (C.c_int, [_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_int, C.c_int, _p]),
    "decon_pdhg_dual_data": (C.c_int, [_p, _p, _p, _p, _p, C.c_float, C.c_int, _i64, _p]),
    "decon_pdhg_dual_reg": (C.c_int, [_p, _p, _p, C.c_float, C.c_int, C.c_int, _i64, _p]),
    "decon_pdhg_xbar": (C.c_int, [_p, _p, _p, _p, _i64, _p]),
    "decon_pdhg_primal": (C.c_int, [_p, _p, _p, _p, _p, _i64, _p]),
    "decon_pdhg_sub": (C.c_int, [_p, _p, _p, _p, _i64, _p]),
    "decon_pdhg_dk": (C.c_int, [_p, _p, _p, _i64, _p, _i64, _p]),
    "decon_pdhg_step": (C.c_int, [_p, _p]),
    "decon_pdhg_loss": (C.c_int, [_p, _p, _p, C.c_float, C.c_int, _i64, _p, C.c_int, C.c_int,
                                  _i64, C.c_double, C.c_int, _p]),
    "decon_pdhg_status_async": (C.c_int, [_p, _p, _p]),
    "decon_pdhg_read": (C.c_int, [_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), C.POINTER(C.c_int), _dp, _dp, _dp, _dp,
                                  _dp, _p]),
    "decon_pdhg_set_stop": (C.c_int, [_p, C.c_int, _p]),
    "decon_pdhg_hess_dual": (C.c_int, [_p, _p, _p, _p, _i64p, C.c_float, C.c_float, C.c_int, _p]),
    "decon_pdhg_hess_primal": (C.c_int, [_p, _p, _p, _p, _p, _i64p, C.c_float, _p]),
    "decon_pdhg_hess_dual_primal": (C.c_int, [_p, _p, _p, _p, _p, _p, _p, _i64p, C.c_float,
                                              C.c_float, C.c_int, _p]),
    "decon_pdhg_hess_dk": (C.c_int, [_p, _p, _p, _i64, _p, _p, _i64p, C.c_float, _p]),
    "decon_pdhg_hess_loss": (C.c_int, [_p, _p, _p, C.c_float, C.c_int, _i64, _p, _i64p, C.c_float,
                                       C.c_int, C.c_double, C.c_int, _p]),
    "decon_profile_start": (C.c_int, [C.c_int]),
    "decon_profile_stop": (C.c_int, [_dp, _i64p]),
}

PROF_XR2C, PROF_COL, PROF_ZOTF, PROF_XC2R = 1, 2, 4, 8

_lib = None
_lock = threading.Lock()


class DeconError(RuntimeError):
    """A CUDA-side failure reported by libdecon_b200 (status code + message)."""

    def __init__(self, code, msg):
        super().__init__(f"[decon_b200 status {code}] {msg}")
        self.code = code


def load():
    """Load the shared library (once) and declare every signature."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python deconlib_b200/csrc/build.py` "
                "(deconlib_b200 has no CPU fallback)"
            )
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def exported_names():
    return list(_SIGS)


def check(status):
    """Map a status code to the reference's exception types."""
    if status == OK:
        return
    msg = load().decon_last_error().decode(errors="replace")
    if status == ERR_VALUE:
        raise ValueError(msg)
    if status == ERR_OOM:
        raise MemoryError(msg)
    raise DeconError(status, msg)


def call(name, *args):
    check(getattr(load(), name)(*args))


def i64arr(vals):
    a = (C.c_int64 * len(vals))(*[int(v) for v in vals])
    return a


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    if t is None:
        return None
    return C.c_void_p(t.data_ptr())


def stream_ptr(torch_mod=None):
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def require_cuda():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError(
            "deconlib_b200 needs a CUDA device (sm_100a); it has no CPU fallback"
        )
    load()


def next_smooth(n: int) -> int:
    return int(load().decon_next_smooth(int(n)))


def band_weights(n_large: int, n_small: int):
    """Host band tables from the library (FP64 math, float32 weights)."""
    lib = load()
    wf, wa = C.c_int(), C.c_int()
    check(lib.decon_band_widths(n_large, n_small, C.byref(wf), C.byref(wa)))
    idx_f = np.zeros((n_small, wf.value), np.int32)
    w_f = np.zeros((n_small, wf.value), np.float32)
    idx_a = np.zeros((n_large, wa.value), np.int32)
    w_a = np.zeros((n_large, wa.value), np.float32)
    check(lib.decon_band_weights(n_large, n_small, idx_f.ctypes.data_as(C.c_void_p),
                                 w_f.ctypes.data_as(C.c_void_p), idx_a.ctypes.data_as(C.c_void_p),
                                 w_a.ctypes.data_as(C.c_void_p)))
    return idx_f, w_f, idx_a, w_a
