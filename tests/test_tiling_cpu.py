"""Tiling geometry and shape helpers (host integer arithmetic) against the
reference's own outputs (tests/golden, made by running deconlib's
tile_processing.py / shapes.py through the NumPy stand-in), plus the
properties the reference tests check (tests/test_tile_processing.py:70-165):
uniform read shape, write slices partitioning the output, reads in bounds."""

import os

import numpy as np
import pytest

from deconlib_b200.batch import _axis_cores, fft_shape_candidates, plan_uneven_tiles
from deconlib_b200.deconvolution.shapes import (compute_padded_shape, compute_visible_shape,
                                                get_valid_slices)
from deconlib_b200.deconvolution.tile_processing import optimal_tile_size, plan_tiles

HERE = os.path.dirname(os.path.abspath(__file__))
TILE_CASES = [((64, 300, 300), 2.0, 16, 128, 48), ((40, 257, 190), 1.0, 8, 64, 48),
              ((100, 512, 512), (1.0, 1.5, 1.5), 20, 200, 48), ((30, 90), 2.0, 4, 40, 48),
              ((96, 700, 333), 1.0, 31, 256, 32)]


@pytest.fixture(scope="module")
def g():
    return np.load(os.path.join(HERE, "golden", "golden_fp32.npz"))


def _enc(sl):
    return [[s.start, s.stop] for s in sl]


@pytest.mark.parametrize("i", range(len(TILE_CASES)))
def test_plan_tiles_matches_reference(g, i):
    shape, zoom, guard, ts, mz = TILE_CASES[i]
    plan = plan_tiles(shape, zoom, guard, ts, mz)
    assert list(plan.tile_shape) == g[f"tile{i}_tile_shape"].tolist()
    assert list(plan.visible_shape) == g[f"tile{i}_visible"].tolist()
    got = np.array([[_enc(t.read), _enc(t.write), _enc(t.crop)] for t in plan.tiles])
    np.testing.assert_array_equal(got, g[f"tile{i}_specs"])
    np.testing.assert_array_equal(np.array([t.index for t in plan.tiles]), g[f"tile{i}_index"])
    # reference properties: uniform reads in bounds, writes partition the output
    cover = np.zeros(plan.visible_shape, np.int32)
    for t in plan.tiles:
        assert tuple(s.stop - s.start for s in t.read) == plan.tile_shape
        assert all(0 <= s.start and s.stop <= n for s, n in zip(t.read, plan.data_shape))
        assert all(w.stop - w.start == c.stop - c.start for w, c in zip(t.write, t.crop))
        cover[t.write] += 1
    assert np.all(cover == 1)


def test_optimal_tile_size_matches_reference(g):
    for N, guard, ts, ref in g["optimal_tile_size"].tolist():
        if ref < 0:
            with pytest.raises(ValueError):
                optimal_tile_size(N, guard, ts)
        else:
            assert optimal_tile_size(N, guard, ts) == ref


def test_padded_shape_and_valid_slices_match_reference(g):
    cases = [((100, 100), (31, 31)), ((64, 128, 128), (64, 128, 128)), ((17, 40, 33), (8, 9, 12))]
    for i, (sig, ker) in enumerate(cases):
        shp, pad = compute_padded_shape(sig, ker)
        assert list(shp) == g[f"pad{i}_shape"].tolist()
        assert [list(p) for p in pad] == g[f"pad{i}_pad"].tolist()
        assert _enc(get_valid_slices(shp, sig, pad)) == g[f"pad{i}_valid"].tolist()
        assert _enc(get_valid_slices(shp, sig)) == g[f"pad{i}_valid_default"].tolist()
    assert compute_padded_shape((10, 10), (5, 5), min_pad=(None, 0)) == ((14, 10), ((2, 2), (0, 0)))
    assert compute_visible_shape((100, 100), 0.85) == (118, 118)
    assert compute_visible_shape((100, 100, 50), (1.0, 1.0, 2.0)) == (100, 100, 25)
    with pytest.raises(ValueError):
        compute_padded_shape((10, 10), (3,))


def test_plan_tiles_errors_like_the_reference():
    # tests/test_tile_processing.py:97-99 and :159-161
    with pytest.raises(ValueError):
        plan_tiles((100,), 1.0, 4)
    with pytest.raises(ValueError):
        optimal_tile_size(64, guard=20, tile_size=32)
    with pytest.raises(ValueError):
        plan_tiles((4, 64, 64), 1.0, guard=20, tile_size=32)
    for N in range(50, 80):
        assert optimal_tile_size(N, guard=4, tile_size=32) <= N


def test_uneven_tiles_partition_the_volume_with_seeded_cores():
    shape = (256, 1024, 1024)
    ranges = [(48, 96), (160, 320), (160, 320)]
    t1 = plan_uneven_tiles(shape, ranges, 32, np.random.default_rng(7))
    t2 = plan_uneven_tiles(shape, ranges, 32, np.random.default_rng(7))
    assert t1 == t2 and len(t1) > 1
    for ax, N in enumerate(shape):
        cores = sorted({(t.write[ax].start, t.write[ax].stop) for t in t1})
        assert cores[0][0] == 0 and cores[-1][1] == N
        assert all(a[1] == b[0] for a, b in zip(cores, cores[1:]))
        lo, hi = ranges[ax]
        assert all(lo <= c1 - c0 <= hi for c0, c1 in cores)
    for t in t1:
        for ax, N in enumerate(shape):
            r, w, c = t.read[ax], t.write[ax], t.crop[ax]
            assert r.start == max(0, w.start - 32) and r.stop == min(N, w.stop + 32)
            assert c.start == w.start - r.start and c.stop - c.start == w.stop - w.start


def test_axis_cores_edge_cases():
    rng = np.random.default_rng(0)
    assert _axis_cores(50, 48, 96, rng) == [(0, 50)]
    assert _axis_cores(97, 48, 96, rng)[-1][1] == 97
    for N in range(97, 400):
        cores = _axis_cores(N, 48, 96, np.random.default_rng(N))
        assert all(48 <= b - a <= 96 for a, b in cores)
    with pytest.raises(ValueError):
        plan_uneven_tiles((100,), [(40, 60)], 4, rng)


def test_fft_candidates_include_the_reference_canvas_and_are_linear_safe():
    c = fft_shape_candidates((136, 304, 304), (64, 128, 128))
    assert c[0] == (200, 432, 432)  # fast_padded_shape, the reference's choice
    assert (256, 480, 480) in c  # static_fft_shape: compile-time FFT lengths
    for t in c:
        assert all(f >= n + k - 1 for f, n, k in zip(t, (136, 304, 304), (64, 128, 128)))
        for f in t:
            m = f
            for p in (2, 3, 5):
                while m % p == 0:
                    m //= p
            assert m == 1
