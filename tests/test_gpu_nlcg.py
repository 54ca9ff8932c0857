"""NLCG on the device against the reference's nlcg_with_operator.

Fixtures: ``tests/golden/golden_nlcg_fp{32,64}.npz`` (the reference's own
source, float32 and float64).  The device sums in FP64 where the reference
sums in float32, so its trajectory sits between the two fixtures: iterates
must match the float64 fixture within max(1e-4, 2 x the float32-float64
spread of the reference itself), with the same iteration count, stop
decision and loss history (rtol 1e-4).  Larger problems are checked against
the float64 oracle (oracle/nlcg.py) with the same rule, the loss history to
max(1e-4, 2 x the float32 oracle's own deviation): the regularised
trajectory at 64x128x128 amplifies float32 round-off to ~1e-2."""

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    b = b.detach().cpu().numpy() if hasattr(b, "detach") else np.asarray(b)
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def g32():
    return np.load(os.path.join(HERE, "golden", "golden_nlcg_fp32.npz"))


@pytest.fixture(scope="module")
def g64():
    return np.load(os.path.join(HERE, "golden", "golden_nlcg_fp64.npz"))


@pytest.fixture(scope="module")
def D():
    import deconlib_b200.deconvolution as D

    return D


SHAPE = (16, 32, 32)

CASES = {  # name: (observation key, operator, keyword arguments)
    "plain": ("obs", "conv", dict(num_iter=15, background=10.0, eval_interval=4, min_iter=100)),
    "stop": ("obs", "conv", dict(num_iter=40, background=10.0, slack=6.0, min_iter=3)),
    "hess": ("obs", "conv", dict(num_iter=12, background=10.0, reg="hess", reg_weight=1e-3, tol=1e-4,
                                 min_iter=5, eval_interval=3)),
    "tol": ("obs", "conv", dict(num_iter=40, background=10.0, reg="hess", reg_weight=1e-3, tol=3e-2,
                                min_iter=5)),
    "grad": ("obs", "conv", dict(num_iter=10, background=10.0, reg="grad", reg_weight=2e-3,
                                 restart_interval=4, min_iter=100, eval_interval=2)),
    "init": ("obs", "conv", dict(num_iter=6, background=10.0, init="mean", min_iter=100,
                                 newton_iters=2)),
    "crop": ("obs_c", "crop", dict(num_iter=8, background=10.0, min_iter=100)),
    "down": ("obs_d", "down", dict(num_iter=8, background=5.0, min_iter=100, reg="hess05",
                                   reg_weight=1e-3)),
}


def _op(D, psf, key):
    conv = D.LinearFFTConvolver(psf, SHAPE)
    if key == "conv":
        return conv
    if key == "crop":
        return D.compose(D.Crop(SHAPE, (12, 26, 28), start=(2, 3, 2)), conv)
    return D.compose(D.FractionalAreaDownsample(2.0, in_shape=SHAPE), conv)


def _kw(D, g, kw):
    kw = dict(kw)
    reg = kw.pop("reg", None)
    if reg is not None:
        kw["regularizer"] = {"hess": D.Hessian3D(), "hess05": D.Hessian3D(r=0.5),
                             "grad": D.Gradient3D(r=0.85)}[reg]
    if kw.get("init") == "mean":
        kw["init"] = np.full(SHAPE, float(g["obs"].mean()), np.float32)
    return kw


@pytest.mark.parametrize("name", list(CASES))
def test_nlcg_golden(D, g32, g64, name):
    obs_key, op_key, kw = CASES[name]
    r = D.nlcg_with_operator(g32[obs_key], _op(D, g32["psf"], op_key), **_kw(D, g32, kw))
    spread = rel(g32[name + "_x"], g64[name + "_x"])
    e64 = rel(r.restored, g64[name + "_x"])
    print(f"nlcg {name}: iterations {r.iterations}, rel-L2 vs fp64 reference {e64:.2e} "
          f"(reference fp32-fp64 spread {spread:.2e})")
    assert r.iterations == int(g64[name + "_iters"])
    assert r.converged == bool(g64[name + "_converged"])
    assert e64 < max(1e-4, 2 * spread)
    assert rel(r.pred, g64[name + "_pred"]) < max(1e-5, 2 * rel(g32[name + "_pred"], g64[name + "_pred"]))
    np.testing.assert_allclose(r.loss_history, g64[name + "_loss"], rtol=1e-4)


def test_nlcg_helpers(D, g32, g64):
    conv = D.LinearFFTConvolver(g32["psf"], SHAPE)
    s, d, y = g32["h_s"], g32["h_d"], g32["obs"]
    for tag, reg, beta in (("n", None, 0.0), ("r", D.Hessian3D(), 1e-3)):
        obj = D.nlcg_objective(s, conv, y, 10.0, reg, beta)
        assert obj == pytest.approx(float(g64[f"h{tag}_obj"]), rel=1e-6)
        grad, aux = D.nlcg_gradient(s, conv, y, 10.0, reg, beta)
        assert rel(grad, g64[f"h{tag}_grad"]) < 1e-5
        q = D.nlcg_hessian_quadform(s, d, conv, y, 10.0, reg, beta, aux=aux)
        assert q == pytest.approx(float(g64[f"h{tag}_quad"]), rel=1e-5)
        f = torch.from_numpy(s * s).cuda()
        lam, m_lam = D.nlcg_step_length(s, d, f, aux[0], conv, y, 10.0, reg, beta)
        print(f"step length {tag}: {lam:.9g} (fp64 reference {float(g64[f'h{tag}_lam']):.9g}, "
              f"fp32 {float(g32[f'h{tag}_lam']):.9g})")
        assert lam == pytest.approx(float(g64[f"h{tag}_lam"]), rel=1e-5)
        assert rel(m_lam, g64[f"h{tag}_mlam"]) < 1e-6
    v = D.i_divergence_between(g32["h_f1"], g32["h_f2"])
    assert v == pytest.approx(float(g64["h_idiv"]), rel=1e-5)


def test_nlcg_rejected_first_step(D, g32):
    """newton_iters=0 leaves lambda = 0: the first step cannot lower phi, so
    the solve stops at once as converged with the initial loss (the
    reference's step-failure branch, nlcg_mlx.py:476-479)."""
    from oracle import nlcg as O
    from oracle import ops

    conv = D.LinearFFTConvolver(g32["psf"], SHAPE)
    r = D.nlcg_with_operator(g32["obs"], conv, num_iter=5, background=10.0, newton_iters=0)
    ref = O.nlcg_with_operator(g32["obs"], ops.LinearFFTConvolver(g32["psf"], SHAPE, dtype=np.float64),
                               num_iter=5, background=10.0, newton_iters=0, dtype=np.float64)
    assert r.iterations == ref["iterations"] == 1 and r.converged and ref["converged"]
    np.testing.assert_allclose(r.loss_history, ref["loss_history"], rtol=1e-5)


def test_nlcg_callback_and_solver(D, g32):
    conv = D.LinearFFTConvolver(g32["psf"], SHAPE)
    seen = []
    r = D.nlcg_with_operator(g32["obs"], conv, num_iter=10, background=10.0, min_iter=100,
                             callback=lambda k, f: seen.append(k) or k == 3)
    assert r.iterations == 4 and seen == [0, 1, 2, 3] and not r.converged

    from deconlib_b200.deconvolution import make_forward_model

    fm = make_forward_model(g32["psf"], (12, 28, 30), 1.0)
    obs = g32["obs"][:12, :28, :30]
    out = D.nlcg_solver(num_iter=4, background=10.0, min_iter=100)(obs, fm)
    assert out.shape == (12, 28, 30) and np.isfinite(out).all()


@pytest.mark.parametrize("reg", [None, "hess"])
def test_nlcg_against_fp64_oracle_64x128x128(D, reg):
    from deconlib_b200 import synth
    from oracle import nlcg as O
    from oracle import ops

    shape = (64, 128, 128)
    rng = np.random.default_rng(11)
    psf = synth.widefield_psf(shape, 0.1, 0.085)
    truth = synth.beads(shape, 300, rng) + 0.05
    blur = D.LinearFFTConvolver(psf, shape).forward(truth).cpu().numpy()
    obs = synth.poisson_observation(blur, 800.0, 10.0, rng)
    kw = dict(num_iter=10, background=10.0, min_iter=100)
    if reg:
        kw.update(reg_weight=1e-4)
    r = D.nlcg_with_operator(obs, D.LinearFFTConvolver(psf, shape),
                             regularizer=D.Hessian3D() if reg else None, **kw)
    ops.set_fft_workers(8)
    ref64 = O.nlcg_with_operator(obs, ops.LinearFFTConvolver(psf, shape, dtype=np.float64),
                                 regularizer=ops.Hessian3D(1.0, np.float64) if reg else None,
                                 dtype=np.float64, **kw)
    ref32 = O.nlcg_with_operator(obs, ops.LinearFFTConvolver(psf, shape, dtype=np.float32),
                                 regularizer=ops.Hessian3D(1.0, np.float32) if reg else None,
                                 dtype=np.float32, **kw)
    spread = rel(ref32["restored"], ref64["restored"])
    e = rel(r.restored, ref64["restored"])
    print(f"nlcg {shape} reg={reg}: rel-L2 vs fp64 oracle {e:.2e} (fp32 oracle spread {spread:.2e})")
    assert r.iterations == ref64["iterations"]
    assert e < max(1e-4, 2 * spread)
    l32, l64 = np.asarray(ref32["loss_history"]), np.asarray(ref64["loss_history"])
    loss_spread = float(np.max(np.abs(l32 - l64) / np.abs(l64)))
    np.testing.assert_allclose(r.loss_history, l64, rtol=max(1e-4, 2 * loss_spread))


def test_nlcg_fused_hessian_matches_materialised_images(D, g32):
    """Hessian3D's Gram matrix and energy evaluated on the fly equal the sums
    over the materialised images (same float32 components, FP64 sums in
    another order): the trajectories agree to 1e-6."""
    H = D.Hessian3D(r=0.7)

    class Wrapped:  # not a Hessian3D: takes the generic, materialised path
        def forward(self, x):
            return H.forward(x)

        def adjoint(self, y):
            return H.adjoint(y)

    conv = D.LinearFFTConvolver(g32["psf"], SHAPE)
    kw = dict(num_iter=8, background=10.0, reg_weight=1e-3, min_iter=100)
    a = D.nlcg_with_operator(g32["obs"], conv, regularizer=H, **kw)
    b = D.nlcg_with_operator(g32["obs"], conv, regularizer=Wrapped(), **kw)
    assert a.iterations == b.iterations
    assert rel(a.restored, b.restored.cpu().numpy()) < 1e-6
    np.testing.assert_allclose(a.loss_history, b.loss_history, rtol=1e-6)
    s = np.random.default_rng(3).random(SHAPE).astype(np.float32) + 0.5
    assert D.nlcg_objective(s, conv, g32["obs"], 10.0, H, 1e-3) == pytest.approx(
        D.nlcg_objective(s, conv, g32["obs"], 10.0, Wrapped(), 1e-3), rel=1e-12)
