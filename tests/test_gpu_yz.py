"""The fused Y / axial pass (one thread-block cluster per kx column, the
spectrum kx-major between the X passes; an opt-in schedule,
DECON_SCHED_FUSED) against the FP64 oracle and against the default separate
passes, on the canvases it serves: Fy in {256,
512}, Fz in {128, 256}, the signal in the first half of both, Ny even; odd
and non-power-of-two Fx; planes that leave CTAs of a cluster without z rows.
Tolerance: 1e-6 relative L2 against FP64 (2e-6 for the 64x128x128 canvas of
the 5-smooth sizes, as the other convolution parity tests); fused vs unfused
1e-6.  Also: the RL fused iteration through the new layout, and a shape the
pass does not serve (odd Ny) falling back to the unfused passes.
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

CASES = [((128, 256, 256), (256, 512, 512)),
         ((64, 128, 128), (128, 256, 256)),
         ((60, 200, 90), (128, 512, 200)),
         ((100, 128, 77), (256, 256, 160)),
         ((5, 30, 33), (128, 256, 75)),
         ((20, 31, 40), (128, 256, 64))]


def rel(a, b):
    a = np.asarray(a.detach().cpu().numpy() if hasattr(a, "detach") else a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def D():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import deconlib_b200.deconvolution as d

    return d


@pytest.mark.parametrize("shape,fft", CASES)
def test_fused_yz_pass_vs_fp64_and_unfused(D, shape, fft):
    from oracle import ops

    rng = np.random.default_rng(sum(shape) + sum(fft))
    kshape = tuple(f - n + 1 for n, f in zip(shape, fft))
    k = (rng.random(kshape, dtype=np.float32) ** 4).astype(np.float32)
    x = rng.random(shape, dtype=np.float32)
    o = ops.LinearFFTConvolver(k, shape, fft_shape=fft, dtype=np.float64)
    c = D.LinearFFTConvolver(k, shape, fft_shape=fft, schedule=1)
    assert c.fused_yz == (shape[1] % 2 == 0)  # every case but the odd-Ny one is served
    f1, a1 = c.forward(x), c.adjoint(x)
    tol = 2e-6 if fft == (128, 256, 256) else 1e-6
    ef, ea = rel(f1, o.forward(x.astype(np.float64))), rel(a1, o.adjoint(x.astype(np.float64)))
    print(f"\nfused Y/axial {shape} canvas {fft}: forward {ef:.2e}, adjoint {ea:.2e}")
    assert ef < tol and ea < tol
    c0 = D.LinearFFTConvolver(k, shape, fft_shape=fft)
    assert not c0.fused_yz
    assert rel(f1, c0.forward(x).cpu().numpy()) < 1e-6
    assert rel(a1, c0.adjoint(x).cpu().numpy()) < 1e-6
    # switching the schedule back on the same plan gives the separate passes
    c.set_schedule(0)
    assert not c.fused_yz
    assert rel(c.forward(x), c0.forward(x).cpu().numpy()) < 1e-6
    from deconlib_b200 import _lib

    _lib.call("decon_device_status", _lib.stream_ptr())


def test_rl_through_fused_pass_matches_unfused(D):
    rng = np.random.default_rng(3)
    shape = (64, 128, 128)
    psf = (rng.random(shape, dtype=np.float32) ** 6).astype(np.float32)
    obs = rng.poisson(200 * rng.random(shape) + 10).astype(np.float32)
    out = []
    for sched in (1, 0):
        c = D.LinearFFTConvolver(psf, shape, schedule=sched)
        assert c.fused_yz == bool(sched)
        r = D.richardson_lucy_with_operator(obs, c, num_iter=10, background=10.0)
        out.append((r.restored.cpu().numpy(), r.loss_history))
    assert rel(out[0][0], out[1][0]) < 1e-5
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-6)


@pytest.mark.parametrize("shape,fft", [((128, 256, 256), None), ((16, 32, 32), None),
                                       ((20, 64, 48), (64, 128, 96)), ((40, 32, 64), None)])
@pytest.mark.parametrize("sched", [0, 1])
def test_fused_area_sum_composition_equals_operators(D, shape, fft, sched):
    # compose(FractionalAreaDownsample(2), LinearFFTConvolver): the 2x area sum
    # fused into the last FFT pass and its adjoint into the first give the
    # float32 values of the two operators applied in turn (unit weights, the
    # passes' summation order), on fused and unfused column passes alike.
    rng = np.random.default_rng(sum(shape))
    k = (rng.random(shape if fft is None else tuple(f - n + 1 for n, f in zip(shape, fft)),
                    dtype=np.float32) ** 4).astype(np.float32)
    conv = D.LinearFFTConvolver(k, shape, fft_shape=fft, schedule=sched)
    down = D.FractionalAreaDownsample(2.0)
    A = D.compose(down, conv)
    assert A._down2 is not None
    x = torch.from_numpy(rng.random(shape, dtype=np.float32)).cuda()
    y = torch.from_numpy(rng.random(tuple(s // 2 for s in shape), dtype=np.float32)).cuda()
    f1, a1 = A.forward(x), A.adjoint(y)
    assert A._down2 is not None  # the fused path ran
    f0 = down.forward(conv.forward(x))
    a0 = conv.adjoint(down.adjoint(y))
    assert torch.equal(f1, f0)
    assert torch.equal(a1, a0)


def test_area_sum_composition_falls_back_for_odd_extents(D):
    rng = np.random.default_rng(1)
    shape = (10, 33, 40)
    k = rng.random((5, 7, 9)).astype(np.float32)
    conv = D.LinearFFTConvolver(k, shape)
    A = D.compose(D.FractionalAreaDownsample(2.0), conv)
    assert A._down2 is None
    x = rng.random(shape, dtype=np.float32)
    ref = D.FractionalAreaDownsample(2.0).forward(conv.forward(x))
    assert torch.equal(A.forward(x), ref)
