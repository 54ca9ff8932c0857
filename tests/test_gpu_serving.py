"""The serving loop on the GPU: every job's result is the same alone (the
public API, one solve at a time) and inside the mix (continuous batching on
several streams, pooled plans whose OTF is rebuilt for the next job's PSF,
pooled PDHG states).  Tolerance: relative L2 <= 1e-6; the kernels, launch
shapes and FP64 reductions are identical, so the results are expected to be
bit-identical and the maximum absolute difference is reported."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _mix():
    from deconlib_b200 import synth
    from deconlib_b200.serving import Job

    rng = np.random.default_rng(42)
    jobs = []
    shapes = [(16, 32, 32), (16, 32, 32), (12, 40, 36), (16, 32, 32)]
    for i, shp in enumerate(shapes):
        psf = synth.widefield_psf(shp, 0.1, 0.085, na=float(rng.uniform(1.0, 1.4)),
                                  wavelength=float(rng.uniform(0.45, 0.65)),
                                  depth=float(rng.uniform(0, 20)))
        truth = synth.beads(shp, 20, rng)
        obs = synth.poisson_observation(truth + 0.05, 300.0, 5.0, rng)
        jobs.append(Job(job_id=i, kind="rl", observed=obs, psf=psf, num_iter=12, arrival=0.001 * i,
                        background=5.0))
    # PDHG with 2x sampling: object 16x32x32, data 8x16x16
    psf = synth.widefield_psf((16, 32, 32), 0.1, 0.085, depth=5.0)
    truth = synth.beads((16, 32, 32), 20, rng)
    obs = synth.poisson_observation(truth[::2, ::2, ::2] + 0.05, 300.0, 5.0, rng)
    opts = dict(alpha=1e-3, regularization="hessian", sampling_factors=2.0,
                spacing=(0.1, 0.085, 0.085), tol=0.0)
    jobs.append(Job(job_id=4, kind="pdhg", observed=obs, psf=psf, num_iter=15, arrival=0.002,
                    background=5.0, options=opts))
    jobs.append(Job(job_id=5, kind="pdhg", observed=obs * 1.5, psf=psf, num_iter=10, arrival=0.003,
                    background=5.0, options=opts))
    return jobs


def _alone(job, canvas="static"):
    """The job through the public API on the canvas the server gives it."""
    import deconlib_b200.deconvolution as D
    from deconlib_b200.serving import job_fft_shape

    fft = job_fft_shape(job, canvas)
    if job.kind == "rl":
        op = D.LinearFFTConvolver(job.psf, job.observed.shape, fft_shape=fft)
        r = D.richardson_lucy_with_operator(job.observed, op, num_iter=job.num_iter,
                                            background=job.background)
    else:
        r = D.solve_pdhg_mlx(job.observed, job.psf, num_iter=job.num_iter,
                             background=job.background, fft_shape=fft, **job.options)
    return r.restored.cpu().numpy(), r.iterations


@pytest.mark.parametrize("max_active,budget,canvas", [(3, 150 * 10**9, "static"),
                                                      (8, 150 * 10**9, "static"),
                                                      (8, 3 * 10**6, "static"),
                                                      (8, 150 * 10**9, "reference")])
def test_each_result_is_the_same_alone_and_in_the_mix(max_active, budget, canvas):
    from deconlib_b200.serving import DeconServer

    jobs = _mix()
    rep = DeconServer(budget_bytes=budget, max_active=max_active, chunk=4, canvas=canvas).run(
        jobs, realtime=False)
    assert [r.job_id for r in rep.results] == [j.job_id for j in jobs]
    if budget < 10**7:
        assert rep.peak_device_bytes <= budget
    for job, res in zip(jobs, rep.results):
        ref, iters = _alone(job, canvas)
        assert res.iterations == iters
        d = np.linalg.norm(res.restored - ref) / np.linalg.norm(ref)
        assert d <= 1e-6, (job.job_id, d, float(np.abs(res.restored - ref).max()))
        assert res.latency >= 0
    assert rep.p99_latency >= rep.p50_latency > 0
    assert rep.voxel_iters_per_s > 0


def test_realtime_arrivals_overlap_on_the_device():
    from deconlib_b200.serving import DeconServer

    jobs = _mix()
    rep = DeconServer(max_active=4, chunk=2).run(jobs, realtime=True)
    assert len(rep.results) == len(jobs)
    assert rep.max_concurrent >= 2
    for r in rep.results:
        assert r.finished >= r.admitted >= r.arrival - 1e-3


def test_mix_with_the_two_cta_axial_pass_is_bit_identical():
    """PDHG jobs whose axial canvas is 256 (object depth 128) run the two-CTA
    pipelined axial kernel; served beside RL jobs on other streams (other
    kernels sharing the SMs) every result must equal the job alone bit for
    bit."""
    from deconlib_b200 import synth
    from deconlib_b200.serving import DeconServer, Job

    rng = np.random.default_rng(7)
    jobs = []
    for i in range(4):
        shp = (128, 64 + 16 * i, 96)
        psf = synth.widefield_psf(shp, 0.05, 0.0425, depth=float(rng.uniform(0, 10)))
        truth = synth.beads(shp, 60, rng)
        obs = synth.poisson_observation(truth[::2, ::2, ::2] + 0.05, 400.0, 5.0, rng)
        opts = dict(alpha=1e-3, regularization="hessian", sampling_factors=2.0,
                    spacing=(0.05, 0.0425, 0.0425), tol=0.0)
        jobs.append(Job(job_id=i, kind="pdhg", observed=obs, psf=psf, num_iter=40, arrival=0.0,
                        background=5.0, options=opts))
    for i in range(4, 8):
        shp = (60 + 4 * i, 120, 100)
        psf = synth.widefield_psf(shp, 0.1, 0.085)
        truth = synth.beads(shp, 60, rng)
        obs = synth.poisson_observation(truth + 0.05, 300.0, 5.0, rng)
        jobs.append(Job(job_id=i, kind="rl", observed=obs, psf=psf, num_iter=40, arrival=0.0,
                        background=5.0))
    alone = [_alone(j) for j in jobs]
    for _ in range(3):
        rep = DeconServer(budget_bytes=150 * 10**9, max_active=8, chunk=4).run(jobs, realtime=False)
        for job, res, (ref, iters) in zip(jobs, rep.results, alone):
            assert res.iterations == iters
            assert np.array_equal(res.restored, ref), (job.job_id, float(np.abs(res.restored - ref).max()))
