"""decon_pdhg_hess_dual_primal (the dual and primal Hessian updates in one
z-walk) against decon_pdhg_hess_dual followed by decon_pdhg_hess_primal.

Both evaluate the same float32 operations, so y2 and x_new must agree
bit for bit.  The FP64 sums (||dx||^2, ||x||^2, ||x_new||^2) are folded in a
different block order; a 40-iteration PDHG trajectory with the fused kernel
must stay within 1e-6 of the operator-by-operator path.  Shapes cover one and
two planes,
z-chunks that end inside the volume, partial x / y tiles and 1-voxel-wide
volumes; both norms (L1 clip, L1,2 ball).
"""

import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

SHAPES = [(1, 9, 40), (2, 9, 33), (17, 10, 35), (33, 16, 64), (40, 70, 90), (5, 1, 1), (3, 20, 1),
          # partial x / y tiles whose x extent is a multiple of 4, one row,
          # four columns
          (17, 10, 36), (40, 70, 92), (5, 1, 4), (3, 20, 4)]


@pytest.fixture(scope="module")
def env():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from deconlib_b200 import _lib

    return _lib


def _state(_lib, step):
    # a fresh state has tau = sigma = step and theta = 1
    lib = _lib.load()
    h = C.c_void_p()
    _lib.check(lib.decon_pdhg_create(4, step, 0.99, 0.5, 0.0, 0, 1, C.byref(h)))
    return h


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("norm", [0, 1])
def test_fused_dual_primal_equals_separate_kernels(env, shape, norm):
    _lib = env
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(sum(shape) + norm)
    xc = torch.rand(shape, device="cuda", generator=g)
    xp = torch.rand(shape, device="cuda", generator=g)
    aty = torch.rand(shape, device="cuda", generator=g) - 0.5
    y2 = 0.01 * torch.randn((6,) + shape, device="cuda", generator=g)
    shp = _lib.i64arr(shape)
    r, alpha = 0.7, 0.02
    st = _lib.stream_ptr()
    outs = []
    for fused in (True, False):
        h = _state(_lib, 0.3)
        xn = torch.full(shape, float("nan"), device="cuda")
        if fused:
            y2o = torch.full_like(y2, float("nan"))
            _lib.check(lib.decon_pdhg_hess_dual_primal(h, _lib.ptr(y2), _lib.ptr(y2o), _lib.ptr(xc),
                                                       _lib.ptr(xp), _lib.ptr(aty), _lib.ptr(xn), shp,
                                                       C.c_float(r), C.c_float(alpha), norm, st))
        else:
            y2o = y2.clone()
            _lib.check(lib.decon_pdhg_hess_dual(h, _lib.ptr(y2o), _lib.ptr(xc), _lib.ptr(xp), shp,
                                                C.c_float(r), C.c_float(alpha), norm, st))
            _lib.check(lib.decon_pdhg_hess_primal(h, _lib.ptr(xc), _lib.ptr(aty), _lib.ptr(y2o),
                                                  _lib.ptr(xn), shp, C.c_float(r), st))
        torch.cuda.synchronize()
        outs.append((y2o.clone(), xn.clone()))
        lib.decon_pdhg_destroy(h)
    assert torch.equal(outs[0][0], outs[1][0])
    assert torch.equal(outs[0][1], outs[1][1])
    assert not torch.isnan(outs[0][1]).any()


@pytest.mark.parametrize("switch", ["DECON_FUSED_STENCIL", "DECON_PDHG_OVERLAP"])
def test_pdhg_fused_stencil_trajectory_matches_operator_path(monkeypatch, switch):
    """The opt-in schedules of the Hessian path (one fused dual + primal
    kernel; dual and ||H dx||^2 on a second stream) follow the
    operator-by-operator trajectory."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    monkeypatch.setenv(switch, "1")
    import os

    import deconlib_b200.deconvolution as D
    from deconlib_b200.deconvolution._device import to_device
    from deconlib_b200.deconvolution.pdhg import (HessianRegularizer, PDHGRunner,
                                                   _compute_spacing_ratio)

    g32 = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_fp32.npz"))
    data = to_device(g32["pd_obs"])
    conv = D.LinearFFTConvolver(g32["psf_hr"], (16, 32, 32))
    A = D.compose(D.FractionalAreaDownsample(2.0), conv)
    reg = HessianRegularizer(3, _compute_spacing_ratio((0.05, 0.0425, 0.0425), 3), "L1")
    out = []
    for fused in (True, False):
        x0 = D.prox_nonneg(A.adjoint(data))
        run = PDHGRunner(data, A, reg, x0, 1e-3, "poisson", 40, 5.0, 0.99, 0.5, 10, 1e-5, 20, 5,
                         fused=fused)
        assert run.fused == fused
        if fused:
            assert (run.fused_stencil if switch == "DECON_FUSED_STENCIL" else run.side is not None)
        out.append(run.run().result())
    x = out[0][0].cpu().numpy()
    ref = out[1][0].cpu().numpy()
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-6
    np.testing.assert_allclose(out[0][3], out[1][3], rtol=1e-6)


def test_pdhg_two_stream_schedule_bit_identical(monkeypatch):
    """The default two-stream schedule (Hessian dual update and ||H dx||^2 on
    a second stream) and DECON_PDHG_OVERLAP=0 (one stream) run the same
    kernels on the same data: identical iterates and step histories."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import os

    import deconlib_b200.deconvolution as D

    g32 = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_fp32.npz"))
    out = []
    for v in ("1", "0"):
        monkeypatch.setenv("DECON_PDHG_OVERLAP", v)
        r = D.solve_pdhg_mlx(g32["pd_obs"], g32["psf_hr"], alpha=1e-3, regularization="hessian",
                             sampling_factors=2.0, spacing=(0.05, 0.0425, 0.0425), background=5.0,
                             num_iter=30, tol=0.0)
        out.append(r)
    np.testing.assert_array_equal(out[0].restored.cpu().numpy(), out[1].restored.cpu().numpy())
    assert out[0].tau_history == out[1].tau_history
    assert out[0].sigma_history == out[1].sigma_history

