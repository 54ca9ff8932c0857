"""Canonical forward model, tile processing and the batched tiled RL on the GPU.

* make_forward_model: forward / adjoint of the composed operator against the
  reference's outputs on the same input (golden, FP32 rel-L2 1e-5).
* process_tiles with a pass-through solver reproduces the input exactly
  (reference tests/test_tile_processing.py:169-185), and with
  richardson_lucy_solver matches a full-image solve in the interior
  (:235-255).
* BatchedRL (one CUDA graph over all problems) against each problem solved
  alone with richardson_lucy_with_operator: identical canvases give identical
  results (rel-L2 <= 1e-6); autotuned canvases differ only by FFT rounding
  (rel-L2 <= 1e-4 after 20 iterations).  Stitching takes each tile's core.
"""

import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.fixture(scope="module")
def D():
    import deconlib_b200.deconvolution as D

    return D


@pytest.fixture(scope="module")
def g32():
    return np.load(os.path.join(HERE, "golden", "golden_fp32.npz"))


def test_forward_model_matches_reference(D, g32):
    fm = D.make_forward_model(g32["fm_psf"], (6, 12, 10), 2.0)
    assert list(fm.padded_shape) == g32["fm_padded"].tolist()
    assert [[s.start, s.stop] for s in fm.valid_slices] == g32["fm_valid"].tolist()
    assert rel(fm.op.forward(g32["fm_x"]), g32["fm_fwd"]) < 1e-5
    assert rel(fm.op.adjoint(g32["fm_y"]), g32["fm_adj"]) < 1e-5


def test_process_tiles_passthrough_is_exact(D):
    rng = np.random.default_rng(3)
    data = rng.random((20, 90, 70)).astype(np.float32)
    psf = np.ones((5, 9, 9), np.float32)

    def passthrough(tile, model):
        out = np.zeros(model.padded_shape, np.float32)
        out[model.valid_slices] = tile
        return out[model.valid_slices]

    out = D.process_tiles(data, psf, 1.0, passthrough, guard=4, tile_size=32)
    np.testing.assert_array_equal(out, data)


def test_tiled_rl_matches_full_image_in_interior(D):
    from deconlib_b200 import synth

    rng = np.random.default_rng(5)
    shape = (12, 96, 96)
    psf = synth.widefield_psf((8, 16, 16), 0.2, 0.1)
    truth = synth.beads(shape, 60, rng) + 0.1
    data = D.LinearFFTConvolver(psf, shape).forward(truth).cpu().numpy() * 200 + 5
    solve = D.richardson_lucy_solver(num_iter=10, background=5.0)
    tiled = D.process_tiles(data, psf, 1.0, solve, guard=12, tile_size=48)
    full = solve(data, D.make_forward_model(psf, shape, 1.0))
    sl = (slice(None), slice(24, 72), slice(24, 72))
    assert rel(tiled[sl], full[sl]) < 0.02


def _problems():
    from deconlib_b200 import synth

    rng = np.random.default_rng(9)
    probs = []
    for shp in [(16, 40, 36), (12, 32, 32), (20, 48, 44)]:
        psf = synth.widefield_psf((8, 16, 16), 0.2, 0.1, na=float(rng.uniform(1.0, 1.4)))
        truth = synth.beads(shp, 30, rng) + 0.05
        obs = synth.poisson_observation(truth, 300.0, 5.0, rng)
        probs.append((obs, psf))
    return probs


def _alone(D, obs, psf, n, fft_shape=None):
    op = D.LinearFFTConvolver(psf, obs.shape, fft_shape=fft_shape)
    return D.richardson_lucy_with_operator(obs, op, num_iter=n, background=5.0).restored.cpu().numpy()


@pytest.mark.parametrize("iters,per_graph", [(12, 5), (7, 10)])
def test_batched_rl_equals_each_problem_alone(D, iters, per_graph):
    from deconlib_b200 import _lib
    from deconlib_b200.batch import BatchedRL

    probs = _problems()
    n0 = _lib.load().decon_launch_count()
    b = BatchedRL(probs, 5.0, nstreams=2, iters_per_graph=per_graph).run(iters)
    torch.cuda.synchronize()
    assert b.graph_kernels() > 0
    assert _lib.load().decon_launch_count() > n0
    for (obs, psf), x in zip(probs, b.restored):
        assert rel(x, _alone(D, obs, psf, iters)) <= 1e-6
    pred = b.predict()
    assert all(p.shape == x.shape for p, x in zip(pred, b.restored))
    _lib.call("decon_device_status", _lib.stream_ptr())


def test_batched_tiles_with_autotuned_canvases(D):
    from deconlib_b200 import synth
    from deconlib_b200.batch import batched_tiled_rl, plan_uneven_tiles

    rng = np.random.default_rng(11)
    shape = (40, 120, 110)
    psf = synth.widefield_psf((8, 16, 16), 0.2, 0.1)
    truth = synth.beads(shape, 80, rng) + 0.05
    data = synth.poisson_observation(
        D.LinearFFTConvolver(psf, shape).forward(truth).cpu().numpy(), 300.0, 5.0, rng)
    tiles = plan_uneven_tiles(shape, [(12, 24), (30, 60), (30, 60)], 6, rng)
    extra = [(p[0], p[1], 5.0) for p in _problems()[:2]]
    out, vols, batch = batched_tiled_rl(data, psf, tiles, 20, 5.0, extra=extra, fft_shapes="auto",
                                        nstreams=4, iters_per_graph=10)
    torch.cuda.synchronize()
    assert len(vols) == 2
    o = out.cpu().numpy()
    for t, fs in zip(tiles, batch.fft_shapes):
        ref = _alone(D, data[t.read], psf, 20)
        assert rel(o[t.write], ref[t.crop]) <= 1e-4
    for (obs, psf_e, _), x in zip(extra, vols):
        assert rel(x, _alone(D, obs, psf_e, 20)) <= 1e-4


@pytest.mark.parametrize("shape,fft", [((20, 60, 45), (32, 120, 90)), ((64, 128, 128), None),
                                       ((30, 100, 90), (64, 256, 256))])
def test_every_schedule_gives_the_same_convolution(shape, fft):
    # the autotuner's schedules choose among equivalent pass families (fused
    # or separate Y / axial passes, pipelined / one-tile / plain-load column
    # kernels, one- or two-CTA axial kernel, radix order, lines per CTA):
    # every one must give the default's result to FP32 rounding
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import deconlib_b200.deconvolution as D
    from deconlib_b200.batch import SCHEDULES

    rng = np.random.default_rng(sum(shape))
    kshape = shape if fft is None else tuple(f - n + 1 for n, f in zip(shape, fft))
    k = (rng.random(kshape, dtype=np.float32) ** 4).astype(np.float32)
    x = rng.random(shape, dtype=np.float32)
    c = D.LinearFFTConvolver(k, shape, fft_shape=fft)
    f0, a0 = c.forward(x).cpu().numpy(), c.adjoint(x).cpu().numpy()
    for name, sc in SCHEDULES.items():
        c.set_schedule(sc)
        f, a = c.forward(x).cpu().numpy(), c.adjoint(x).cpu().numpy()
        assert np.linalg.norm(f - f0) / np.linalg.norm(f0) < 1e-6, name
        assert np.linalg.norm(a - a0) / np.linalg.norm(a0) < 1e-6, name


def test_autotuner_persists_its_choice(tmp_path, monkeypatch):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import json

    from deconlib_b200 import batch

    monkeypatch.setenv("DECON_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(batch, "_TUNED", {})
    monkeypatch.setattr(batch, "_CACHE_LOADED", False)
    rng = np.random.default_rng(0)
    psf = rng.random((9, 21, 17)).astype(np.float32)
    fs, sc = batch.autotune_schedule((24, 60, 50), psf, reps=1)
    saved = json.load(open(tmp_path / "tune.json"))
    assert any(v["fft_shape"] == list(fs) and v["schedule"] == sc for v in saved.values())
    # a fresh process state reads the file instead of timing again
    monkeypatch.setattr(batch, "_TUNED", {})
    monkeypatch.setattr(batch, "_CACHE_LOADED", False)
    assert batch.autotune_schedule((24, 60, 50), psf, reps=1) == (fs, sc)
