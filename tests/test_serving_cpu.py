"""Host-side logic of the serving loop: FIFO admission by slots and HBM
budget, the device-footprint model and the seeded arrival process (no GPU)."""

import numpy as np
import pytest

from deconlib_b200.serving import (Job, Scheduler, job_device_bytes, job_signal_shape,
                                   poisson_arrivals)


def _job(i, shape=(8, 16, 16), kind="rl", psf_shape=None, **opts):
    obs = np.zeros(shape, np.float32)
    psf = np.zeros(psf_shape or shape, np.float32)
    return Job(job_id=i, kind=kind, observed=obs, psf=psf, num_iter=5, options=opts)


def test_admission_is_fifo_and_bounded_by_slots():
    s = Scheduler(budget_bytes=10**12, max_active=2, footprint=lambda j: 1)
    for i in range(4):
        s.arrive(_job(i))
    got = [j.job_id for j, _ in s.admit()]
    assert got == [0, 1]
    assert s.admit() == []
    s.release(0)
    assert [j.job_id for j, _ in s.admit()] == [2]
    s.release(1)
    s.release(2)
    assert [j.job_id for j, _ in s.admit()] == [3]
    s.release(3)
    assert s.idle


def test_admission_respects_budget_and_reserved_bytes():
    sizes = {0: 60, 1: 50, 2: 10}
    s = Scheduler(budget_bytes=100, max_active=8, footprint=lambda j: sizes[j.job_id])
    for i in range(3):
        s.arrive(_job(i))
    # job 1 does not fit beside job 0; strict FIFO keeps job 2 behind it
    assert [j.job_id for j, _ in s.admit()] == [0]
    assert s.head_blocked_by(0) == 10
    assert s.head_blocked_by(20) == 30
    s.release(0)
    assert [j.job_id for j, _ in s.admit(reserved=30)] == [1, 2]
    assert s.used == 60 and s.peak == 90


def test_oversized_job_is_rejected_on_arrival():
    s = Scheduler(budget_bytes=100, max_active=2, footprint=lambda j: 101)
    with pytest.raises(ValueError, match="more than the whole budget"):
        s.arrive(_job(0))


def test_footprint_model_counts_plan_and_arrays():
    # RL at 128x256x256 with a same-size PSF: canvas 256x512x512, pitch 272
    j = _job(0, shape=(128, 256, 256))
    pitch = 272
    plan = 8 * pitch * (256 * 512 + 128 * 256 + 128 * 512)
    n = 128 * 256 * 256
    assert job_device_bytes(j) == plan + 4 * (5 * n + n)
    # PDHG with sampling factors: the object grid is the PSF grid
    p = _job(1, shape=(64, 128, 128), kind="pdhg", psf_shape=(128, 256, 256), sampling_factors=2.0)
    assert job_signal_shape(p) == (128, 256, 256)
    m = 64 * 128 * 128
    assert job_device_bytes(p) == plan + 4 * (6 * m + 11 * n + n)


def test_static_canvas_policy_sizes_the_footprint():
    from deconlib_b200.serving import job_fft_shape

    j = _job(0, shape=(76, 362, 244))
    assert job_fft_shape(j, "reference") == (160, 729, 500)
    assert job_fft_shape(j, "static") == (256, 768, 512)
    pitch = 272  # 512 / 2 + 1 rounded up to 16
    plan = 8 * pitch * (256 * 768 + 76 * 362 + 76 * 768)
    n = 76 * 362 * 244
    assert job_device_bytes(j, "static") == plan + 4 * (5 * n + n)
    with pytest.raises(ValueError):
        job_fft_shape(j, "largest")


def test_poisson_arrivals_are_seeded_with_the_requested_rate():
    a = poisson_arrivals(4000, 20.0, np.random.default_rng(5))
    b = poisson_arrivals(4000, 20.0, np.random.default_rng(5))
    assert np.array_equal(a, b)
    assert np.all(np.diff(a) > 0)
    assert abs(4000 / a[-1] - 20.0) < 1.5
