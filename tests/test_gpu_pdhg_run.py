"""decon_pdhg_run: the resident Hessian-PDHG solve behind the C ABI.

A C caller creates a solver from a convolution plan, the observation and the
sampling factors, queues iterations with decon_pdhg_run and reads x and the
histories back.  It runs the same kernels in the same order as
solve_pdhg_mlx's fused Hessian path, so its iterates and tau / sigma / loss
histories must equal the Python driver's exactly, and lie within the PDHG
tolerance of the reference's FP64 golden trajectory
(deconlib/deconvolution/pdhg_mlx.py:717-900).
"""

import ctypes as C
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def env():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import deconlib_b200.deconvolution as D
    from deconlib_b200 import _lib

    g32 = np.load(os.path.join(HERE, "golden", "golden_fp32.npz"))
    g64 = np.load(os.path.join(HERE, "golden", "golden_fp64.npz"))
    return D, _lib, g32, g64


def _solve_c(D, _lib, conv, obs, scale, iters, chunks, norm=0, loss=0, r=1.0, alpha=1e-3, bg=5.0,
             tol=1e-5, eval_interval=10):
    lib = _lib.load()
    st = _lib.stream_ptr()
    data = torch.from_numpy(np.ascontiguousarray(obs, np.float32)).cuda()
    h = C.c_void_p()
    sc = (C.c_double * 3)(*scale)
    _lib.check(lib.decon_pdhg_solver_create(conv.plan, _lib.ptr(data), _lib.i64arr(obs.shape), sc,
                                            C.c_float(bg), loss, None, C.c_double(r),
                                            C.c_double(alpha), norm, iters, 0.99, 0.5, tol, 20, 5,
                                            eval_interval, st, C.byref(h)))
    try:
        done = 0
        for c in chunks:
            _lib.check(lib.decon_pdhg_run(h, c, st))
            done += c
        x = torch.empty(conv.signal_shape, device="cuda")
        _lib.check(lib.decon_pdhg_solver_x(h, _lib.ptr(x), st))
        state, queued = C.c_void_p(), C.c_int()
        _lib.check(lib.decon_pdhg_solver_state(h, C.byref(state), C.byref(queued)))
        assert queued.value == min(done, iters)
        k, fi, cv, stop = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        sc3 = (C.c_double * 3)()
        hist = [np.zeros(max(iters, 1)) for _ in range(4)]
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        _lib.check(lib.decon_pdhg_read(state, C.byref(k), C.byref(fi), C.byref(cv), C.byref(stop),
                                       sc3, *[dp(a) for a in hist], st))
        torch.cuda.synchronize()
        return x.cpu().numpy(), fi.value, bool(cv.value), hist
    finally:
        lib.decon_pdhg_solver_destroy(h)


@pytest.mark.parametrize("norm", [0, 1])
def test_pdhg_run_equals_python_driver_and_golden(env, norm):
    D, _lib, g32, g64 = env
    from deconlib_b200.deconvolution.pdhg import _compute_spacing_ratio

    obs, psf = g32["pd_obs"], g32["psf_hr"]
    spacing = (0.05, 0.0425, 0.0425)
    r = _compute_spacing_ratio(spacing, 3)
    nm = "L1" if norm == 0 else "L1_2"
    ref = D.solve_pdhg_mlx(obs, psf, alpha=1e-3, sampling_factors=2.0, spacing=spacing,
                           background=5.0, num_iter=30, eval_interval=10, norm=nm)
    conv = D.LinearFFTConvolver(psf, psf.shape)
    x, fi, cv, (tau, sigma, loss, _) = _solve_c(D, _lib, conv, obs, (2.0, 2.0, 2.0), 30,
                                                 [7, 16, 7, 5], norm=norm, r=r)
    assert fi == ref.iterations == 30 and cv == ref.converged
    np.testing.assert_array_equal(x, ref.restored.cpu().numpy())
    np.testing.assert_array_equal(tau[:30], ref.tau_history)
    np.testing.assert_array_equal(sigma[:30], ref.sigma_history)
    np.testing.assert_array_equal(loss[[9, 19, 29]], ref.loss_history)
    name = "pd_h_l1" if norm == 0 else "pd_h_l12"
    spread = np.linalg.norm(g32[name + "_x"] - g64[name + "_x"]) / np.linalg.norm(g64[name + "_x"])
    tol = max(1e-4, 2 * spread)
    err = np.linalg.norm(x - g64[name + "_x"]) / np.linalg.norm(g64[name + "_x"])
    assert err < tol


def test_pdhg_run_plain_operator_and_convergence(env):
    D, _lib, g32, g64 = env
    obs, psf = g32["rl_obs"], g32["psf16"]
    conv = D.LinearFFTConvolver(psf, obs.shape)
    ref = D.solve_pdhg_mlx(obs, psf, alpha=1e-3, background=10.0, num_iter=15,
                           spacing=(0.1, 0.085, 0.085))
    from deconlib_b200.deconvolution.pdhg import _compute_spacing_ratio

    r = _compute_spacing_ratio((0.1, 0.085, 0.085), 3)
    x, fi, cv, (tau, _, loss, _) = _solve_c(D, _lib, conv, obs, (1.0, 1.0, 1.0), 15, [15],
                                             r=r, bg=10.0)
    np.testing.assert_array_equal(x, ref.restored.cpu().numpy())
    np.testing.assert_array_equal(tau[:15], ref.tau_history)
    assert np.linalg.norm(x - g64["pd_plain_x"]) / np.linalg.norm(g64["pd_plain_x"]) < 1e-4
    # early stop: the reference's convergence rule, queued far past the stop
    ref = D.solve_pdhg_mlx(g32["pd_obs"], g32["psf_hr"], alpha=5.0, sampling_factors=2.0,
                           background=5.0, num_iter=60, tol=5e-2, min_iter=3, patience=2)
    lib = _lib.load()
    conv2 = D.LinearFFTConvolver(g32["psf_hr"], g32["psf_hr"].shape)
    data = torch.from_numpy(np.ascontiguousarray(g32["pd_obs"])).cuda()
    h = C.c_void_p()
    st = _lib.stream_ptr()
    _lib.check(lib.decon_pdhg_solver_create(conv2.plan, _lib.ptr(data),
                                            _lib.i64arr(g32["pd_obs"].shape),
                                            (C.c_double * 3)(2.0, 2.0, 2.0), C.c_float(5.0), 0,
                                            None, C.c_double(1.0), C.c_double(5.0), 0, 60, 0.99, 0.5,
                                            5e-2, 3, 2, 10, st, C.byref(h)))
    try:
        _lib.check(lib.decon_pdhg_run(h, 60, st))
        x = torch.empty(g32["psf_hr"].shape, device="cuda")
        _lib.check(lib.decon_pdhg_solver_x(h, _lib.ptr(x), st))
        state = C.c_void_p()
        _lib.check(lib.decon_pdhg_solver_state(h, C.byref(state), None))
        fi, cv = C.c_int(), C.c_int()
        _lib.check(lib.decon_pdhg_read(state, None, C.byref(fi), C.byref(cv), None, None, None,
                                       None, None, None, st))
        assert fi.value == ref.iterations == int(g64["pd_conv_iters"])
        assert bool(cv.value) == ref.converged == bool(g64["pd_conv_converged"])
        np.testing.assert_array_equal(x.cpu().numpy(), ref.restored.cpu().numpy())
    finally:
        lib.decon_pdhg_solver_destroy(h)


def test_pdhg_solver_rejects_bad_arguments(env):
    D, _lib, g32, _ = env
    lib = _lib.load()
    conv = D.LinearFFTConvolver(g32["psf16"], (16, 32, 32))
    data = torch.zeros((8, 16, 40), device="cuda")
    h = C.c_void_p()
    st = lib.decon_pdhg_solver_create(conv.plan, _lib.ptr(data), _lib.i64arr((8, 16, 40)),
                                      (C.c_double * 3)(2.0, 2.0, 2.0), C.c_float(0.0), 0, None,
                                      C.c_double(1.0), C.c_double(1e-3), 0, 10, 0.99, 0.5, 1e-5, 20,
                                      5, 10, _lib.stream_ptr(), C.byref(h))
    assert st == _lib.ERR_VALUE and not h.value
    st = lib.decon_pdhg_solver_create(conv.plan, _lib.ptr(data), _lib.i64arr((8, 16, 16)),
                                      (C.c_double * 3)(2.0, 2.0, 2.0), C.c_float(0.0), 3, None,
                                      C.c_double(1.0), C.c_double(1e-3), 0, 10, 0.99, 0.5, 1e-5, 20,
                                      5, 10, _lib.stream_ptr(), C.byref(h))
    assert st == _lib.ERR_VALUE


def test_async_status_polling_gives_the_same_solve(env):
    # the serving loop's PDHG runners poll the stop flag through a pinned copy
    # instead of synchronising; iterations queued after the device stopped are
    # no-ops, so the result equals the synchronous driver's (early stop case)
    D, _lib, g32, g64 = env
    from deconlib_b200.deconvolution.pdhg import pdhg_mlx_runner, pdhg_result

    kw = dict(alpha=5.0, sampling_factors=2.0, background=5.0, num_iter=60, tol=5e-2, min_iter=3,
              patience=2)
    ref = D.solve_pdhg_mlx(g32["pd_obs"], g32["psf_hr"], **kw)
    runner, meta = pdhg_mlx_runner(g32["pd_obs"], g32["psf_hr"], async_status=True, **kw)
    assert runner.async_status
    res = pdhg_result(runner.run(), meta)
    assert res.iterations == ref.iterations == int(g64["pd_conv_iters"])
    assert res.converged == ref.converged
    np.testing.assert_array_equal(res.restored.cpu().numpy(), ref.restored.cpu().numpy())
    np.testing.assert_array_equal(res.tau_history, ref.tau_history)
