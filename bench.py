"""Benchmark: voxel-iterations/s of Hessian-PDHG and Richardson-Lucy at 128x256x256.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (seeded synthetic inputs, no dataset exists for it): the
super-resolved Hessian-PDHG solve of a 128x256x256 object through
compose(FractionalAreaDownsample(2), LinearFFTConvolver) against a
64x128x128 Poisson observation (500 peak photons, background 5, PSF with a
10 um index mismatch, 0.5 rad spherical and -0.2 rad coma, filament + bead
phantom), alpha = 1e-3, L1 Hessian with r = dy/dz.  A step is one PDHG
iteration over the whole volume.  The same line carries Richardson-Lucy at
128x256x256 (beads + shells, 1000 photons, background 10) under "rl".

``value``: object voxels x timed iterations / device time (CUDA events, max
over ranks), inputs resident in HBM.  ``e2e``: the same metric through the
public API (``solve_pdhg_mlx`` with NumPy host arrays: host->device copies,
OTF set-up, iterations and the device->host copy of the result all inside the
timed region).  ``roofline``: the axial FFT x OTF pass (the largest FFT pass),
algorithmic bytes per launch / its average CUDA-event launch time.
``cpu_baseline``: the NumPy oracle port of the reference on this host.

Multi-GPU: the path does not shard; ``--gpus N`` runs N independent replicas
(one process per GPU, torchrun), value = all replicas' voxel-iterations /
max device time.  Timed iterations use tol = 0 so every one does full work.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

OBJ = (128, 256, 256)
DATA = (64, 128, 128)
SPACING_PD = (0.05, 0.0425, 0.0425)
SPACING_RL = (0.1, 0.085, 0.085)
METRIC = "voxel-iter/s RL & PDHG at 128x256^2 vs plain GPU; %HBM roofline; serve p50/p99"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 20 ms."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region starts only once samples flow
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 3.0:
                time.sleep(0.01)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], [], set()
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
                for nm, v in zip(names, r[4:8]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "samples": len(sm),
                "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# inputs
# ---------------------------------------------------------------------------


def pdhg_inputs(D):
    from deconlib_b200 import synth

    psf, truth = synth.pdhg_workload(OBJ, SPACING_PD, seed=2)
    fwd = D.compose(D.FractionalAreaDownsample(2.0, in_shape=OBJ), D.LinearFFTConvolver(psf, OBJ))
    blur = fwd.forward(truth).cpu().numpy()
    obs = synth.poisson_observation(blur, 500.0, 5.0, np.random.default_rng(3))
    return psf, obs


def rl_inputs(D):
    from deconlib_b200 import synth

    psf, truth = synth.rl_workload(OBJ, SPACING_RL, seed=0)
    blur = D.LinearFFTConvolver(psf, OBJ).forward(truth).cpu().numpy()
    obs = synth.poisson_observation(blur, 1000.0, 10.0, np.random.default_rng(1))
    return psf, obs


def serve_jobs(D, n_jobs, seed=4):
    """Seeded request stream of the served workload: Poisson arrivals at a
    rate drawn from [5, 50] jobs/s; each job is RL (50 iterations, beads +
    shells, 1000 photons, background 10) or Hessian-PDHG (100 iterations,
    2x sampling, 500 photons, background 5, default tol / min_iter /
    patience) on an object of even shape drawn from 32-128 x 128-512 x
    128-512, with its own widefield PSF (NA 1.0-1.45 capped below ni,
    wavelength 0.45-0.65 um, ni 1.33-1.52, ns = min(ni, 1.334), index-mismatch
    depth 0-20 um)."""
    from deconlib_b200 import synth
    from deconlib_b200.serving import Job, poisson_arrivals

    rng = np.random.default_rng(seed)
    rate = float(rng.uniform(5.0, 50.0))
    arrivals = poisson_arrivals(n_jobs, rate, rng)
    jobs = []
    for i in range(n_jobs):
        kind = "rl" if rng.random() < 0.5 else "pdhg"
        shp = (2 * int(rng.integers(16, 65)), 2 * int(rng.integers(64, 257)),
               2 * int(rng.integers(64, 257)))
        ni = float(rng.uniform(1.33, 1.52))
        na = min(float(rng.uniform(1.0, 1.45)), 0.98 * ni)
        wl = float(rng.uniform(0.45, 0.65))
        depth = float(rng.uniform(0.0, 20.0))
        sp = SPACING_RL if kind == "rl" else SPACING_PD
        psf = synth.widefield_psf(shp, sp[0], sp[1], wavelength=wl, na=na, ni=ni,
                                  ns=min(ni, 1.334), depth=depth)
        truth = synth.beads(shp, 200, rng)
        synth.shells(shp, sp, 5, rng, out=truth)
        if kind == "rl":
            blur = D.LinearFFTConvolver(psf, shp).forward(truth).cpu().numpy()
            obs = synth.poisson_observation(blur, 1000.0, 10.0, rng)
            jobs.append(Job(i, "rl", obs, psf, 50, float(arrivals[i]), 10.0))
        else:
            fwd = D.compose(D.FractionalAreaDownsample(2.0, in_shape=shp), D.LinearFFTConvolver(psf, shp))
            obs = synth.poisson_observation(fwd.forward(truth).cpu().numpy(), 500.0, 5.0, rng)
            opts = dict(alpha=1e-3, regularization="hessian", sampling_factors=2.0, spacing=SPACING_PD)
            jobs.append(Job(i, "pdhg", obs, psf, 100, float(arrivals[i]), 5.0, opts))
    return jobs, rate


def solve_alone(D, job, fft=None):
    """One job through the public API (the plain FP32 GPU form; ``fft``: the
    canvas, default the reference's)."""
    if job.kind == "rl":
        conv = D.LinearFFTConvolver(job.psf, job.observed.shape, fft_shape=fft)
        r = D.richardson_lucy_with_operator(job.observed, conv, num_iter=job.num_iter,
                                            background=job.background)
    else:
        r = D.solve_pdhg_mlx(job.observed, job.psf, num_iter=job.num_iter, background=job.background,
                             fft_shape=fft, **job.options)
    return r.restored.cpu().numpy(), r.iterations


def run_serving(D, n_jobs):
    """Served stream vs the same jobs solved one at a time through the API."""
    import torch

    from deconlib_b200.serving import DeconServer, job_fft_shape, job_signal_shape

    jobs, rate = serve_jobs(D, n_jobs)
    server = DeconServer(budget_bytes=150 * 10**9, max_active=8, chunk=8)
    server.run(jobs[:2], realtime=False)  # warm-up (first-use set-up of every kernel family)
    live = server.run(jobs, realtime=True)
    burst = server.run(jobs, realtime=False)
    flat = DeconServer(budget_bytes=150 * 10**9, max_active=8, chunk=8, prioritise=False).run(
        jobs, realtime=True)
    ref_canvas = DeconServer(budget_bytes=150 * 10**9, max_active=8, chunk=8,
                             canvas="reference").run(jobs, realtime=True)

    def sequential(fft_of):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = [solve_alone(D, j, fft_of(j)) for j in jobs]
        torch.cuda.synchronize()
        return res, time.perf_counter() - t0

    alone, t_seq = sequential(lambda j: None)
    alone_static, t_seq_static = sequential(lambda j: job_fft_shape(j, "static"))
    vi = sum(int(np.prod(job_signal_shape(j))) * it for j, (_, it) in zip(jobs, alone))

    def worst(results, refs):
        w = 0.0
        for res, (ref, _) in zip(results, refs):
            w = max(w, float(np.linalg.norm(res.restored - ref) / max(np.linalg.norm(ref), 1e-30)))
        return w

    out = {"workload": "poisson_stream_rl50_pdhg100_mixed_shapes", "jobs": len(jobs),
           "rate_jobs_per_s": rate, "budget_bytes": server.budget, "max_active": server.max_active,
           "canvas": server.canvas,
           "vs_fp64_oracle": _served_vs_oracle(D),
           "realtime": live.summary(), "all_at_once": burst.summary(),
           "realtime_equal_priority": flat.summary(),
           "realtime_reference_canvas": ref_canvas.summary(),
           "plain_sequential_voxel_iter_per_s": vi / t_seq, "plain_sequential_s": t_seq,
           "plain_sequential_static_canvas_voxel_iter_per_s": vi / t_seq_static,
           "served_vs_plain_sequential": live.voxel_iters_per_s / (vi / t_seq),
           "max_rel_l2_served_vs_alone_same_canvas": worst(live.results, alone_static),
           "max_rel_l2_served_static_vs_reference_canvas": worst(live.results, alone),
           "note": "latency = arrival to restored volume on the host; plain = the same jobs "
                   "one at a time through richardson_lucy_with_operator / solve_pdhg_mlx on the "
                   "reference's canvases (fast_padded_shape); the server puts each job on "
                   "static_fft_shape (compile-time FFT lengths)"}
    return out


def _served_vs_oracle(D):
    """Accuracy of the served form against the FP64 NumPy oracle (the
    reference's solvers restated in float64 on the reference's canvas,
    scipy.fft on every host core): one RL job (50 iterations) and one
    Hessian-PDHG job (100 iterations, sampling 2) of the stream's smallest
    object shape, 32x128x128, served together; relative L2 and max-abs error
    of each restored volume.  (The full-size jobs of the stream would keep
    the oracle busy for many minutes.)"""
    from deconlib_b200 import synth
    from deconlib_b200.serving import DeconServer, Job
    from oracle import ops, solvers

    ops.set_fft_workers(len(os.sched_getaffinity(0)))
    rng = np.random.default_rng(11)
    shp = (32, 128, 128)
    jobs = []
    for i, (kind, sp) in enumerate((("rl", SPACING_RL), ("pdhg", SPACING_PD))):
        psf = synth.widefield_psf(shp, sp[0], sp[1], wavelength=0.52, na=1.2, ni=1.45, ns=1.334,
                                  depth=8.0)
        truth = synth.beads(shp, 100, rng)
        synth.shells(shp, sp, 3, rng, out=truth)
        if kind == "rl":
            blur = ops.LinearFFTConvolver(psf, shp, dtype=np.float64).forward(truth.astype(np.float64))
            obs = synth.poisson_observation(blur, 1000.0, 10.0, rng)
            jobs.append(Job(i, "rl", obs, psf, 50, 0.0, 10.0))
        else:
            fwd = ops.compose(ops.FractionalAreaDownsample(2.0, in_shape=shp, dtype=np.float64),
                              ops.LinearFFTConvolver(psf, shp, dtype=np.float64))
            obs = synth.poisson_observation(fwd.forward(truth.astype(np.float64)), 500.0, 5.0, rng)
            opts = dict(alpha=1e-3, regularization="hessian", sampling_factors=2.0, spacing=SPACING_PD)
            jobs.append(Job(i, "pdhg", obs, psf, 100, 0.0, 5.0, opts))
    rep = DeconServer(budget_bytes=150 * 10**9, max_active=8, chunk=8).run(jobs, realtime=False)
    out = {"oracle": "oracle/ NumPy restatement of rl_mlx.py / pdhg_mlx.py in float64"}
    for job, res in zip(jobs, rep.results):
        if job.kind == "rl":
            o64 = ops.LinearFFTConvolver(job.psf, shp, dtype=np.float64)
            ref = solvers.richardson_lucy_with_operator(job.observed, o64, num_iter=job.num_iter,
                                                        background=job.background,
                                                        dtype=np.float64)["restored"]
        else:
            ref = solvers.solve_pdhg_mlx(job.observed, job.psf, num_iter=job.num_iter,
                                         background=job.background, dtype=np.float64,
                                         **job.options)["restored"]
        x = res.restored.astype(np.float64)
        out[f"{job.kind}_{'x'.join(map(str, shp))}_{job.num_iter}it"] = {
            "rel_l2": float(np.linalg.norm(x - ref) / np.linalg.norm(ref)),
            "max_abs": float(np.abs(x - ref).max()), "ref_max": float(np.abs(ref).max())}
    ops.set_fft_workers(1)
    return out


BATCH_VOLUME = (256, 1024, 1024)


def batch_inputs(D, seed=20):
    """Batched tiled workload: a 256x1024x1024 volume of the plain-RL object
    type scaled up (51,200 beads, 320 hollow shells; spacing 0.1 / 0.085 um;
    the 64x128x128 widefield PSF of the plain-RL case; 1000 peak photons,
    background 10, Poisson), split into overlapping tiles with seeded cores
    z 48-96, y / x 160-320 and a 32-voxel halo, plus 16 independent volumes
    of shape U(32-128 x 128-384 x 128-384), each with its own PSF (NA
    1.0-1.45 capped below ni, wavelength 0.45-0.65 um, ni 1.33-1.52)."""
    import torch

    from deconlib_b200 import synth
    from deconlib_b200.batch import plan_uneven_tiles

    rng = np.random.default_rng(seed)
    psf = synth.widefield_psf((64, 128, 128), SPACING_RL[0], SPACING_RL[1])
    truth = synth.beads(BATCH_VOLUME, 51200, rng)
    synth.shells(BATCH_VOLUME, SPACING_RL, 320, rng, out=truth)
    blur = D.LinearFFTConvolver(psf, BATCH_VOLUME).forward(truth)
    del truth
    blur = blur.cpu().numpy()
    data = synth.poisson_observation(blur, 1000.0, 10.0, rng)
    del blur
    torch.cuda.empty_cache()
    tiles = plan_uneven_tiles(BATCH_VOLUME, [(48, 96), (160, 320), (160, 320)], 32, rng)
    vols = []
    for _ in range(16):
        shp = (int(rng.integers(32, 129)), int(rng.integers(128, 385)), int(rng.integers(128, 385)))
        ni = float(rng.uniform(1.33, 1.52))
        p = synth.widefield_psf(shp, SPACING_RL[0], SPACING_RL[1], wavelength=float(rng.uniform(0.45, 0.65)),
                                na=min(float(rng.uniform(1.0, 1.45)), 0.98 * ni), ni=ni,
                                ns=min(ni, 1.334))
        t = synth.beads(shp, max(20, int(np.prod(shp)) // 5000), rng)
        synth.shells(shp, SPACING_RL, 5, rng, out=t)
        b = D.LinearFFTConvolver(p, shp).forward(t).cpu().numpy()
        vols.append((synth.poisson_observation(b, 1000.0, 10.0, rng), p, 10.0))
    return data, psf, tiles, vols


def _schedule_table(b):
    """The autotuner's choice per distinct problem shape: canvas and schedule."""
    from deconlib_b200.batch import SCHEDULES

    names = {v: k for k, v in SCHEDULES.items()}
    seen = {}
    for o, c in zip(b.obs, b.convs):
        key = "x".join(str(s) for s in o.shape)
        if key not in seen:
            seen[key] = {"fft_shape": list(c.fft_shape), "schedule": c.schedule,
                         "schedule_name": names.get(c.schedule, str(c.schedule)),
                         "fused_yz": c.fused_yz}
    return seen


def run_batched(D, iters=100):
    """All tiles + volumes in one batch (autotuned canvases, one CUDA graph of
    all iterations) vs the same problems solved one at a time through
    richardson_lucy_with_operator with the default canvas."""
    import torch

    from deconlib_b200 import _lib
    from deconlib_b200.batch import BatchedRL
    from deconlib_b200.deconvolution._device import to_device

    t0 = time.perf_counter()
    data, psf, tiles, vols = batch_inputs(D)
    vol = to_device(data)
    probs = [(vol[t.read].contiguous(), psf) for t in tiles] + [(o, p) for o, p, _ in vols]
    del vol
    t_inputs = time.perf_counter() - t0
    lib = _lib.load()
    # set-up: autotuning, plans and OTFs, RL initialisation
    t0 = time.perf_counter()
    b = BatchedRL(probs, 10.0, fft_shapes="auto", nstreams=8, iters_per_graph=iters)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t0
    # first run records the graph (all problems x all iterations) and replays it
    t0 = time.perf_counter()
    b.run(iters)
    torch.cuda.synchronize()
    t_first = time.perf_counter() - t0
    # timed: the same solve from a fresh start, one replay of the cached graph
    _lib.call("decon_batch_rl_setup", b.h, None, _lib.stream_ptr())
    torch.cuda.synchronize()
    n0 = lib.decon_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    b.run(iters)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = lib.decon_launch_count() - n0
    voxels_processed = sum(int(o.numel()) for o in b.obs)
    voxels_useful = int(np.prod(BATCH_VOLUME)) + sum(int(np.prod(v[0].shape)) for v in vols)
    stitched = torch.empty(BATCH_VOLUME, dtype=torch.float32, device="cuda")
    for t, x in zip(tiles, b.restored[:len(tiles)]):
        stitched[t.write] = x[t.crop]
    # per-problem plain solves (default canvas) and the stitched / batched results against them
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    worst = 0.0
    for i, (obs, p) in enumerate(probs):
        ref = D.richardson_lucy_with_operator(obs, D.LinearFFTConvolver(p, tuple(obs.shape)),
                                              num_iter=iters, background=10.0).restored
        if i < len(tiles):
            got, ref = stitched[tiles[i].write], ref[tiles[i].crop]
        else:
            got = b.restored[i]
        worst = max(worst, float(torch.linalg.vector_norm(got - ref) / torch.linalg.vector_norm(ref)))
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    out = {"workload": "batched_tiled_rl_256x1024x1024_uneven_tiles_plus_16_volumes",
           "tiles": len(tiles), "volumes": len(vols), "iterations": iters,
           "graph_replays": 1, "graph_kernels": b.graph_kernels(), "gpu_launches_counted": int(launches),
           "ms": ms, "useful_voxel_iter_per_s": voxels_useful * iters / (ms / 1e3),
           "processed_voxel_iter_per_s": voxels_processed * iters / (ms / 1e3),
           "plain_per_problem_s": t_plain,
           "plain_useful_voxel_iter_per_s": voxels_useful * iters / t_plain,
           "max_rel_l2_vs_plain_per_problem": worst,
           "setup_s": {"inputs": t_inputs, "autotune_plans_otf_init": t_setup,
                       "first_run_with_capture": t_first},
           "fft_shapes_distinct": len(set(b.fft_shapes)),
           "schedule_per_shape": _schedule_table(b),
           "note": "ms = device time of one replay of the captured graph (every problem, every "
                   "iteration); useful voxels = the stitched volume + the 16 volumes; plain = each "
                   "problem through richardson_lucy_with_operator one after another (wall clock, "
                   "includes its loss logging)"}
    del b, probs, stitched
    torch.cuda.empty_cache()
    return out


def _rl_fp64_reference(psf, obs, bg, checkpoints):
    """FP64 accuracy reference at full size: Richardson-Lucy with the same
    steps as rl_mlx.py:117-175 (A^T max(y - b, 1e-6) start, sensitivity
    A^T 1 with the active-support mask, multiplicative update floored at
    1e-10), the wrap-free convolution done with torch.fft in float64 on the
    GPU.  A measurement reference only: it is not timed and not the product."""
    import torch

    from deconlib_b200.deconvolution.linops import fast_padded_shape, pad_corner_origin_kernel

    N = tuple(obs.shape)
    F = fast_padded_shape(N, psf.shape)
    k = pad_corner_origin_kernel(psf.astype(np.float64) / psf.astype(np.float64).sum(), F)
    otf = torch.fft.rfftn(torch.from_numpy(k).cuda())
    crop = tuple(slice(0, n) for n in N)

    def conv(x, adj=False):
        X = torch.fft.rfftn(x, s=F)
        return torch.fft.irfftn(X * (otf.conj() if adj else otf), s=F)[crop]

    y = torch.from_numpy(obs.astype(np.float64)).cuda()
    x = torch.clamp(conv(torch.clamp(y - bg, min=1e-6), True), min=1e-6)
    sens_raw = conv(torch.ones_like(y), True)
    floor = max(float(sens_raw.max()) * 1e-6, 1e-10)
    active = sens_raw > floor
    sens = torch.where(active, sens_raw, torch.ones_like(sens_raw))
    x = torch.where(active, x, torch.zeros_like(x))
    snaps = {}
    for it in range(1, max(checkpoints) + 1):
        ratio = y / torch.clamp(conv(x) + bg, min=1e-10)
        x = torch.clamp(x * torch.where(active, conv(ratio, True) / sens, torch.zeros_like(x)), min=1e-10)
        if it in checkpoints:
            snaps[it] = x.float().clone()
    return snaps


def _errs(a, ref):
    import torch

    d = (a - ref).double()
    return {"rel_l2": float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(ref.double())),
            "max_abs": float(d.abs().max()), "ref_max": float(ref.abs().max())}


def run_mixed(D, iters=200):
    """Plain FP32 vs mixed precision (FP16 OTF with per-kz-plane power-of-two
    scales) for RL and Hessian-PDHG at 128x256x256: device time per
    iteration and the error at iterations 10 / 50 / 200 (PDHG: 10 / 50 /
    100) against an FP64 reference (RL) or the FP32 GPU path (PDHG)."""
    import torch

    from deconlib_b200.deconvolution.pdhg import pdhg_mlx_runner
    from deconlib_b200.deconvolution.rl import RLRunner

    checks = tuple(c for c in (10, 50, 200) if c <= iters)
    psf, obs = rl_inputs(D)
    ref = _rl_fp64_reference(psf, obs, 10.0, checks)
    n = int(np.prod(OBJ))
    out = {"workload": "rl_object128x256x256 + hessian_pdhg_sampling2_object128x256x256",
           "fp64_reference": "torch.fft float64 RL on the GPU (same steps as rl_mlx.py:117-175)",
           "rl": {}, "pdhg": {}}
    for prec in ("fp32", "mixed"):
        op = D.LinearFFTConvolver(psf, OBJ, precision=prec)
        r = RLRunner(obs, op, iters, 10.0, eval_interval=10**9)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        snaps, ms = {}, 0.0
        done = 0
        for c in checks:
            e0.record()
            while r.k < c:
                r.iterate()
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            snaps[c] = r.x.clone()
            done = c
        out["rl"][prec] = {"voxel_iter_per_s": n * done / (ms / 1e3), "ms_per_iter": ms / done,
                           "vs_fp64": {str(c): _errs(snaps[c], ref[c]) for c in checks}}
        del r, op
    pchecks = tuple(c for c in (10, 50, 100) if c <= iters)
    ppsf, pobs = pdhg_inputs(D)
    pres = {}
    for prec in ("fp32", "mixed"):
        runner, _ = pdhg_mlx_runner(pobs, ppsf, alpha=1e-3, regularization="hessian",
                                    sampling_factors=2.0, spacing=SPACING_PD, background=5.0,
                                    num_iter=max(pchecks), tol=0.0, precision=prec)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        snaps, ms = {}, 0.0
        for c in pchecks:
            e0.record()
            while runner.k < c:
                runner.iterate()
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            snaps[c] = runner.X[runner.k % 3].clone()
        pres[prec] = snaps
        out["pdhg"][prec] = {"voxel_iter_per_s": n * max(pchecks) / (ms / 1e3),
                             "ms_per_iter": ms / max(pchecks)}
        del runner
    out["pdhg"]["mixed"]["vs_fp32"] = {str(c): _errs(pres["mixed"][c], pres["fp32"][c]) for c in pchecks}
    torch.cuda.empty_cache()
    out["vs_fp64_oracle"] = _mixed_vs_oracle(D, checks=(10, 50, 200))
    return out


def _mixed_vs_oracle(D, checks=(10, 50, 200)):
    """FP32 and mixed precision against the FP64 NumPy oracle (the reference's
    RL and PDHG restated in float64, scipy.fft on every host core) at the
    given iterations: RL on the 64x128x128 bead / shell workload (canvas
    128x256x256) and Hessian-PDHG on a 64x128x128 object of the filament
    workload type (data 32x64x64, sampling 2), so the oracle finishes in
    about two minutes.  Relative L2 and max-abs error of x."""
    import torch

    from deconlib_b200 import synth
    from deconlib_b200.deconvolution.pdhg import pdhg_mlx_runner
    from deconlib_b200.deconvolution.rl import RLRunner
    from oracle import ops, solvers

    ops.set_fft_workers(len(os.sched_getaffinity(0)))
    out = {"oracle": "oracle/ NumPy restatement of rl_mlx.py / pdhg_mlx.py in float64",
           "checkpoints": list(checks)}
    # RL
    shape = (64, 128, 128)
    psf, truth = synth.rl_workload(shape, SPACING_RL, seed=0)
    o64 = ops.LinearFFTConvolver(psf, shape, dtype=np.float64)
    obs = synth.poisson_observation(o64.forward(truth.astype(np.float64)), 1000.0, 10.0,
                                    np.random.default_rng(1))
    ref = {}
    solvers.richardson_lucy_with_operator(
        obs, o64, num_iter=max(checks), background=10.0, dtype=np.float64, eval_interval=10**9,
        callback=lambda k, x: ref.__setitem__(k + 1, x.copy()) if k + 1 in checks else None)
    rl = {}
    for prec in ("fp32", "mixed"):
        r = RLRunner(obs, D.LinearFFTConvolver(psf, shape, precision=prec), max(checks), 10.0,
                     eval_interval=10**9)
        res = {}
        while r.k < max(checks):
            r.iterate()
            if r.k in checks:
                res[str(r.k)] = _errs(r.x, torch.from_numpy(ref[r.k]).cuda())
        rl[prec] = res
        del r
    out["rl_64x128x128"] = rl
    # Hessian-PDHG
    obj, data_shape = (64, 128, 128), (32, 64, 64)
    ppsf, ptruth = synth.pdhg_workload(obj, SPACING_PD, seed=2)
    fwd = ops.compose(ops.FractionalAreaDownsample(2.0, in_shape=obj, dtype=np.float64),
                      ops.LinearFFTConvolver(ppsf, obj, dtype=np.float64))
    pobs = synth.poisson_observation(fwd.forward(ptruth.astype(np.float64)), 500.0, 5.0,
                                     np.random.default_rng(3))
    kw = dict(alpha=1e-3, regularization="hessian", sampling_factors=2.0, spacing=SPACING_PD,
              background=5.0, num_iter=max(checks), tol=0.0)
    pref = {}
    solvers.solve_pdhg_mlx(pobs, ppsf, dtype=np.float64, eval_interval=10**9,
                           callback=lambda k, x: pref.__setitem__(k + 1, x.copy()) if k + 1 in checks else None,
                           **kw)
    pd = {}
    for prec in ("fp32", "mixed"):
        runner, _ = pdhg_mlx_runner(pobs, ppsf, precision=prec, eval_interval=10**9, **kw)
        res = {}
        while runner.k < max(checks):
            runner.iterate()
            if runner.k in checks:
                res[str(runner.k)] = _errs(runner.X[runner.k % 3], torch.from_numpy(pref[runner.k]).cuda())
        pd[prec] = res
        del runner
    out["pdhg_object64x128x128"] = pd
    ops.set_fft_workers(1)
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# algorithmic bytes of the axial pass (per launch)
# ---------------------------------------------------------------------------


def run_psf(reps=20, shape=(128, 256, 256), dxy=0.0425, dz=0.05):
    """Widefield PSF synthesis (pupil_to_psf) on the device for the PDHG
    workload's grid: an anti-aliased NA-1.4 pupil with a seeded smooth phase,
    FFT-order z.  Device time by CUDA events over ``reps`` calls (inputs
    resident); the NumPy loop of the same formula (psf/widefield.py:53-73)
    timed on two planes and scaled to nz, and the device PSF's relative error
    on those planes."""
    import numpy as np
    import torch

    from deconlib_b200 import _lib
    from deconlib_b200.deconvolution._device import stream

    nz, ny, nx = shape
    ky = np.fft.fftfreq(ny, dxy)[:, None]
    kx = np.fft.fftfreq(nx, dxy)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    kmax = 1.4 / 0.525
    w = np.clip((kmax - k) * max(ny, nx) * dxy + 0.5, 0.0, 1.0)
    kz = np.sqrt(np.maximum((1.515 / 0.525) ** 2 - k * k, 0.0))
    rho = np.clip(k / kmax, 0, 1)
    pupil = (w * np.exp(0.7j * (6 * rho ** 4 - 6 * rho ** 2 + 1))).astype(np.complex64)
    z = np.fft.fftfreq(nz) * nz * dz
    pd = torch.from_numpy(pupil).cuda()
    kzd = torch.from_numpy(kz).cuda()
    zd = torch.from_numpy(z).cuda()
    out = torch.empty(shape, device="cuda")
    lib = _lib.load()

    def call():
        _lib.call("decon_pupil_to_psf", pd.data_ptr(), kzd.data_ptr(), zd.data_ptr(), nz, ny, nx, 1,
                  out.data_ptr(), stream())

    for _ in range(3):
        call()
    torch.cuda.synchronize()
    n0 = lib.decon_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        call()
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    launches = (lib.decon_launch_count() - n0) / reps
    t = time.perf_counter()
    ref = np.empty((2, ny, nx))
    for i in range(2):
        a = np.fft.ifft2(pupil.astype(np.complex128) * np.exp(2j * np.pi * kz * z[i]))
        ref[i] = a.real ** 2 + a.imag ** 2
    np_ms = (time.perf_counter() - t) / 2 * nz * 1e3
    tot = nz * ny * nx * np.sum(np.abs(pupil.astype(np.complex128)) ** 2) / (ny * nx) ** 2
    got = out[:2].double().cpu().numpy()
    err = float(np.linalg.norm(got - ref / tot) / np.linalg.norm(ref / tot))
    vox = nz * ny * nx
    return {"shape": list(shape), "ms": ms, "gvox_per_s": vox / ms / 1e6,
            "algorithmic_bytes_per_voxel": 20, "achieved_gbs": 20 * vox / ms / 1e6,
            "launches_per_call": launches, "numpy_ms_estimate": np_ms,
            "rel_l2_vs_fp64_planes01": err}


def run_nlcg(D, iters=50):
    """Nonlinear CG (nlcg_with_operator) on the RL workload (128x256x256,
    LinearFFTConvolver, background 10), unregularised and with a Hessian
    smoothness prior (beta 1e-4), stopping rules off so every solve runs its
    iterations.  The steady-state time per iteration is the difference of a
    10-iteration and an ``iters``-iteration solve (CUDA events around each
    whole solve, its one host read per iteration included; the fastest of
    three solves of each length)."""
    import torch

    psf, obs = rl_inputs(D)
    lib = __import__("deconlib_b200._lib", fromlist=["load"]).load()
    n = int(np.prod(OBJ))
    out = {"workload": "rl_object128x256x256_beads_shells", "convolutions_per_iter": 3}
    op = D.LinearFFTConvolver(psf, OBJ)
    for tag, reg, beta in (("plain", None, 0.0), ("hessian", D.Hessian3D(), 1e-4)):
        def solve(k):
            return D.nlcg_with_operator(obs, op, num_iter=k, background=10.0, regularizer=reg,
                                        reg_weight=beta, slack=0.0, tol=0.0, min_iter=10 ** 9)

        solve(3)
        times, launches = {}, {}
        for k in (10, iters):
            best = float("inf")
            for _ in range(3):  # the fastest of three solves (host hiccups only add time)
                torch.cuda.synchronize()
                n0 = lib.decon_launch_count()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                res = solve(k)
                e1.record()
                e1.synchronize()
                best = min(best, e0.elapsed_time(e1))
                launches[k] = lib.decon_launch_count() - n0
            times[k] = best
        ms = (times[iters] - times[10]) / (iters - 10)
        out[tag] = {"ms_per_iter": ms, "voxel_iter_per_s": n / (ms / 1e3),
                    "launches_per_iter": (launches[iters] - launches[10]) / (iters - 10),
                    "iterations": res.iterations, "final_loss": res.loss_history[-1]}
    return out


def zpass_bytes(n_shape, f_shape, fused):
    """Algorithmic bytes of one launch of the axial pass: the fused Y / axial
    pass reads and writes the kx-major spectrum S1 (Nz x Ny x Hx) and reads the
    OTF; the unfused axial pass reads and writes S2 (Nz x Fy x Hx) and reads
    the OTF.  Complex values are 8 bytes."""
    nz, ny = n_shape[0], n_shape[1]
    fz, fy, fx = f_shape
    hx = fx // 2 + 1
    hf = fz * fy * hx
    if fused:
        return 8 * (2 * nz * ny * hx + hf)
    return 8 * (2 * nz * fy * hx + hf)


def conv_fused(lib, conv):
    import ctypes as C

    f = C.c_int()
    lib.decon_conv_fused_yz(conv.plan, C.byref(f))
    return bool(f.value)


def pdhg_model_bytes(n_shape, m_shape, f_shape, c=8):
    """Minimal bytes of one Hessian-PDHG iteration (linearity-cached, one
    forward and one adjoint convolution, fused stencil): 32 M + 72 N +
    8 c Hs + 2 c Hf, Hs = Nz Fy Hx, Hf = Fz Fy Hx."""
    n = int(np.prod(n_shape))
    m = int(np.prod(m_shape))
    fz, fy, fx = f_shape
    hx = fx // 2 + 1
    return 32 * m + 72 * n + 8 * c * n_shape[0] * fy * hx + 2 * c * fz * fy * hx


def profile_traffic(name):
    """DRAM bytes per launch from a committed ncu summary (profiles/<name>.json)."""
    p = os.path.join(ROOT, "profiles", name + ".json")
    try:
        with open(p) as f:
            return float(json.load(f)["dram_bytes_per_launch"])
    except Exception:
        return None


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------


def run_ours(args, ws, rank, local):
    import torch
    import ctypes as C

    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import deconlib_b200.deconvolution as D
    from deconlib_b200 import _lib
    from deconlib_b200.deconvolution.pdhg import HessianRegularizer, PDHGRunner, _compute_spacing_ratio

    lib = _lib.load()
    K, W = args.steps, args.warmup
    psf, obs = pdhg_inputs(D)
    n_obj = int(np.prod(OBJ))

    # --- PDHG, resident inputs ---------------------------------------------
    from deconlib_b200.deconvolution._device import to_device

    data = to_device(obs)
    conv = D.LinearFFTConvolver(psf, OBJ)
    A = D.compose(D.FractionalAreaDownsample((2.0, 2.0, 2.0)), conv)
    reg = HessianRegularizer(3, _compute_spacing_ratio(SPACING_PD, 3), "L1")
    x0 = D.prox_nonneg(A.adjoint(data))
    runner = PDHGRunner(data, A, reg, x0, 1e-3, "poisson", W + K, 5.0, 0.99, 0.5, 10, 0.0, 20, 5)
    for _ in range(W):
        runner.iterate()
    torch.cuda.synchronize()
    # --- RL at the same size (fused path), set up before the timed regions ---
    psf_rl, obs_rl = rl_inputs(D)
    y = to_device(obs_rl)
    c_rl = D.LinearFFTConvolver(psf_rl, OBJ)
    x = torch.empty_like(y)
    sens = torch.empty_like(y)
    ratio = torch.empty_like(y)
    s = _lib.stream_ptr()
    _lib.call("decon_rl_setup", c_rl.plan, _lib.ptr(y), C.c_float(10.0), None, _lib.ptr(x),
              _lib.ptr(sens), s)
    for _ in range(W):
        _lib.call("decon_rl_iteration", c_rl.plan, _lib.ptr(y), C.c_float(10.0), _lib.ptr(sens),
                  _lib.ptr(x), _lib.ptr(ratio), None, s)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = lib.decon_launch_count()
    lib.decon_profile_start(_lib.PROF_ZOTF)
    e0.record(st)
    for _ in range(K):
        runner.iterate()
    e1.record(st)
    torch.cuda.synchronize()
    ms_z, nz_launch = C.c_double(), C.c_int64()
    lib.decon_profile_stop(C.byref(ms_z), C.byref(nz_launch))
    launches = lib.decon_launch_count() - n0
    ms = e0.elapsed_time(e1)
    from deconlib_b200.replicas import aggregate

    ms, units = aggregate(ms, n_obj * K)  # max device time, total voxel-iterations
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
    info = runner.result()
    value = units / (ms / 1e3)

    # roofline of the axial pass (fused Y / axial pass where the canvas allows)
    fused = conv_fused(lib, conv)
    z_bytes = zpass_bytes(OBJ, conv.fft_shape, fused)
    z_ms = ms_z.value / max(nz_launch.value, 1)
    hbm, src = peaks()
    achieved = z_bytes / (z_ms / 1e3) / 1e9
    traffic = profile_traffic("yz_pdhg_128x256x256" if fused else "zotf_pdhg_128x256x256")

    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lib.decon_profile_start(_lib.PROF_ZOTF)
    r0.record(st)
    for _ in range(K):
        _lib.call("decon_rl_iteration", c_rl.plan, _lib.ptr(y), C.c_float(10.0), _lib.ptr(sens),
                  _lib.ptr(x), _lib.ptr(ratio), None, s)
    r1.record(st)
    torch.cuda.synchronize()
    ms_rz, n_rz = C.c_double(), C.c_int64()
    lib.decon_profile_stop(C.byref(ms_rz), C.byref(n_rz))
    clk = clocks.stop()  # sampled across the PDHG and RL timed regions
    ms_rl, rl_units = aggregate(r0.elapsed_time(r1), n_obj * K)
    rl_value = rl_units / (ms_rl / 1e3)
    fz, fy, fx = c_rl.fft_shape
    hx = fx // 2 + 1
    rl_model_bytes = 28 * n_obj + 8 * 8 * OBJ[0] * fy * hx + 2 * 8 * fz * fy * hx

    # --- e2e through the public API with host buffers ------------------------
    # inputs in pinned host memory (copied to the device inside the call), the
    # restored volume read back into a pinned host buffer
    obs_h = torch.from_numpy(np.ascontiguousarray(obs, dtype=np.float32)).pin_memory()
    psf_h = torch.from_numpy(np.ascontiguousarray(psf, dtype=np.float32)).pin_memory()
    out = torch.empty(OBJ, dtype=torch.float32, pin_memory=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = D.solve_pdhg_mlx(obs_h, psf_h, alpha=1e-3, regularization="hessian", sampling_factors=2.0,
                           spacing=SPACING_PD, background=5.0, num_iter=K, tol=0.0)
    out.copy_(res.restored)
    torch.cuda.synchronize()
    e2e_s, e2e_units = aggregate(time.perf_counter() - t0, n_obj * res.iterations)
    e2e_value = e2e_units / e2e_s

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "voxel-iter/s",
        "n_gpus": ws,
        "steps": K,
        "warmup": W,
        "ms_per_step": ms / K,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded filament+bead phantom, widefield PSF with aberrations, Poisson)",
        "config": {
            "workload": "hessian_pdhg_sampling2_object128x256x256_data64x128x128",
            "object_shape": list(OBJ), "data_shape": list(DATA),
            "fft_shape": list(conv.fft_shape), "alpha": 1e-3, "norm": "L1",
            "step": "one PDHG iteration (1 forward + 1 adjoint A, Hessian dual/primal, FP64 step)",
            "l2": "inputs larger than L2 (OTF 285 MB, Hessian dual 201 MB per iteration)",
            "parallelism": f"replicas x{ws}",
        },
        "iteration_model": {
            "bytes": pdhg_model_bytes(OBJ, DATA, conv.fft_shape),
            "hbm_frac": pdhg_model_bytes(OBJ, DATA, conv.fft_shape) / (ms / K / 1e3) / 1e9 / hbm,
            "note": "minimal-byte model of one PDHG iteration (X and Y transforms fused, FP32 spectra) / ms_per_step"},
        "roofline": {
            "bound": "hbm",
            "kernel": ("k_yz<512,256> fused Y FFT / axial FFT x OTF x IFFT / Y IFFT, one 8-CTA "
                       "cluster per kx column" if fused else
                       "k_col_pipe<16,1,OTF> axial FFT x OTF x IFFT (lean, 2 CTAs/SM)"),
            "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "peak_source": src, "traffic": traffic, "algorithmic_bytes_per_launch": z_bytes,
            "launch_ms": z_ms, "launches": nz_launch.value,
        },
        "e2e": {"value": e2e_value, "unit": "voxel-iter/s",
                "h2d_bytes_per_step": int((obs_h.nbytes + psf_h.nbytes) / max(res.iterations, 1)),
                "d2h_bytes_per_step": int(out.nbytes / max(res.iterations, 1)),
                "seconds": e2e_s, "iterations": res.iterations,
                "note": "solve_pdhg_mlx(pinned host observation + PSF in, restored volume read back "
                        "into pinned host memory) incl. OTF set-up; bytes amortised per iteration"},
        "gpu_launches": int(launches),
        "clocks": clk,
        "rl": {"value": rl_value, "unit": "voxel-iter/s", "ms_per_iter": ms_rl / K,
               "fused_yz": conv_fused(lib, c_rl),
               "model_bytes_per_iter": rl_model_bytes,
               "hbm_frac_model": rl_model_bytes / (ms_rl / K / 1e3) / 1e9 / hbm,
               "zpass_ms": ms_rz.value / max(n_rz.value, 1),
               "workload": "rl_object128x256x256_beads_shells"},
        "pdhg_iterations_run": info[1],
    }
    if args.serve_jobs > 0:
        line["serve"] = run_serving(D, args.serve_jobs)
    if args.batch_iters > 0:
        line["batched"] = run_batched(D, args.batch_iters)
    if args.mixed_iters > 0:
        line["mixed"] = run_mixed(D, args.mixed_iters)
    if args.psf_reps > 0:
        line["psf_synthesis"] = run_psf(args.psf_reps)
    if args.nlcg_iters > 0:
        line["nlcg"] = run_nlcg(D, args.nlcg_iters)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_pdhg(psf, obs, iters=1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# CPU oracle (reference restatement) timing
# ---------------------------------------------------------------------------


def _oracle_pdhg_setup(psf, obs, workers):
    from oracle import ops, solvers

    ops.set_fft_workers(workers)
    y = obs.astype(np.float32)
    conv = ops.LinearFFTConvolver(psf, OBJ, dtype=np.float32)
    A = ops.compose(ops.FractionalAreaDownsample(2.0, dtype=np.float32), conv)
    reg = solvers.Regularizer("hessian", 3, solvers.spacing_ratio(SPACING_PD, 3), "L1", np.float32)
    x0 = np.maximum(A.adjoint(y), np.float32(0))
    return solvers, y, A, reg, x0


def _oracle_iter(solvers, y, A, reg, x0):
    return solvers._pdhg_loop(y, A, reg, x0, 1e-3, "poisson", 1, 5.0, 0.99, 0.5, 10, 0.0, 20, 5,
                              np.float32, generic=False)


def cpu_baseline_pdhg(psf, obs, iters=1):
    workers = len(os.sched_getaffinity(0))
    solvers, y, A, reg, x0 = _oracle_pdhg_setup(psf, obs, workers)
    t0 = time.perf_counter()
    for _ in range(iters):
        _oracle_iter(solvers, y, A, reg, x0)
    dt = (time.perf_counter() - t0) / iters
    return {"value": int(np.prod(OBJ)) / dt, "unit": "voxel-iter/s", "cores": workers,
            "kind": "port",
            "sample": f"{iters} full PDHG iteration(s) of the NumPy oracle at 128x256x256 "
                      f"(3 forward + 1 adjoint convolution, as the reference), scipy.fft with "
                      f"{workers} threads; set-up excluded", "seconds_per_iter": dt}


def _synth_standalone():
    """deconlib_b200/synth.py loaded as a plain module (NumPy only), without
    importing the package, so the reference arm's process maps none of this
    repository's native libraries."""
    import importlib.util

    spec = importlib.util.spec_from_file_location(
        "_bench_synth", os.path.join(ROOT, "deconlib_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def run_reference(args, ws, rank, local):
    """The reference's CPU path on this host: the NumPy restatement of
    deconlib's PDHG loop (oracle/), inputs made by the same oracle.  No torch,
    no CUDA, nothing of deconlib_b200 but its NumPy input generators."""
    if rank != 0:
        return
    from oracle import ops

    synth = _synth_standalone()
    psf, truth = synth.pdhg_workload(OBJ, SPACING_PD, seed=2)
    fwd = ops.compose(ops.FractionalAreaDownsample(2.0, in_shape=OBJ, dtype=np.float64),
                      ops.LinearFFTConvolver(psf, OBJ, dtype=np.float64))
    workers = len(os.sched_getaffinity(0))
    ops.set_fft_workers(workers)
    obs = synth.poisson_observation(fwd.forward(truth.astype(np.float64)), 500.0, 5.0,
                                    np.random.default_rng(3))
    solvers, y, A, reg, x0 = _oracle_pdhg_setup(psf, obs, workers)
    W = min(args.warmup, 1)
    K = max(1, min(args.steps, 3))
    for _ in range(W):
        _oracle_iter(solvers, y, A, reg, x0)
    t0 = time.perf_counter()
    for _ in range(K):
        _oracle_iter(solvers, y, A, reg, x0)
    dt = time.perf_counter() - t0
    value = int(np.prod(OBJ)) * K / dt
    sample = (f"{K} timed PDHG iteration(s) (+{W} warm-up) of the NumPy restatement of the "
              f"reference at 128x256x256, scipy.fft with {workers} threads; the CPU arm times "
              f"min(steps, 3) iterations and min(warmup, 1) warm-up (asked: {args.steps} / "
              f"{args.warmup}), so that it ends within minutes")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "voxel-iter/s",
            "n_gpus": ws, "steps": K, "warmup": W, "steps_requested": args.steps,
            "warmup_requested": args.warmup, "ms_per_step": dt / K * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": "hessian_pdhg_sampling2_object128x256x256_data64x128x128"},
            "cpu_baseline": {"value": value, "unit": "voxel-iter/s", "cores": workers,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "voxel-iter/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_conv_only(args):
    """Forward + adjoint LinearFFTConvolver at 128x256x256 (canvas 256x512x512), seeded
    random PSF-like kernel; prints the device time per convolution pair."""
    import torch

    import deconlib_b200.deconvolution as D

    rng = np.random.default_rng(0)
    k = (rng.random(OBJ, dtype=np.float32) ** 8).astype(np.float32)
    from deconlib_b200.deconvolution._device import to_device

    x = to_device(rng.random(OBJ, dtype=np.float32))
    c = D.LinearFFTConvolver(k, OBJ)
    for _ in range(args.warmup):
        c.adjoint(c.forward(x))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        c.adjoint(c.forward(x))
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"mode": "conv", "fft_shape": list(c.fft_shape),
                      "ms_per_fwd_adj_pair": e0.elapsed_time(e1) / args.steps}), flush=True)


def run_pdhg_only(args):
    """The PDHG iterations of the headline workload only; prints ms per iteration."""
    import torch

    import deconlib_b200.deconvolution as D
    from deconlib_b200.deconvolution._device import to_device
    from deconlib_b200.deconvolution.pdhg import HessianRegularizer, PDHGRunner, _compute_spacing_ratio

    psf, obs = pdhg_inputs(D)
    data = to_device(obs)
    A = D.compose(D.FractionalAreaDownsample((2.0, 2.0, 2.0)), D.LinearFFTConvolver(psf, OBJ))
    reg = HessianRegularizer(3, _compute_spacing_ratio(SPACING_PD, 3), "L1")
    x0 = D.prox_nonneg(A.adjoint(data))
    run = PDHGRunner(data, A, reg, x0, 1e-3, "poisson", args.warmup + args.steps, 5.0, 0.99, 0.5,
                     10, 0.0, 20, 5)
    for _ in range(args.warmup):
        run.iterate()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        run.iterate()
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"mode": "pdhg", "ms_per_iter": e0.elapsed_time(e1) / args.steps}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mixed-iters", type=int, default=200,
                    help="RL iterations of the FP32 vs mixed-precision comparison (0: skip it)")
    ap.add_argument("--batch-iters", type=int, default=100,
                    help="RL iterations of the batched tiled workload (0: skip it)")
    ap.add_argument("--serve-jobs", type=int, default=16,
                    help="jobs in the served request stream (0: skip the serving measurement)")
    ap.add_argument("--psf-reps", type=int, default=20,
                    help="timed pupil_to_psf calls at 128x256x256 (0: skip the PSF synthesis line)")
    ap.add_argument("--nlcg-iters", type=int, default=50,
                    help="NLCG iterations per timed solve at 128x256x256 (0: skip the NLCG line)")
    ap.add_argument("--mode", choices=["full", "conv", "pdhg", "serve", "batch", "mixed", "psf",
                                       "nlcg"],
                    default="full",
                    help="conv: only warm-up + steps forward/adjoint convolutions of the PDHG "
                         "operator; pdhg: only the timed PDHG iterations (small, fixed launch "
                         "sequences for ncu captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_setup()
    if args.mode == "conv":
        run_conv_only(args)
        return
    if args.mode == "pdhg":
        run_pdhg_only(args)
        return
    if args.mode == "serve":
        import torch

        import deconlib_b200.deconvolution as D

        torch.cuda.set_device(local)
        print(json.dumps({"mode": "serve", **run_serving(D, max(args.serve_jobs, 1))}), flush=True)
        return
    if args.mode == "mixed":
        import torch

        import deconlib_b200.deconvolution as D

        torch.cuda.set_device(local)
        print(json.dumps({"mode": "mixed", **run_mixed(D, max(args.mixed_iters, 10))}), flush=True)
        return
    if args.mode == "nlcg":
        import torch

        import deconlib_b200.deconvolution as D

        torch.cuda.set_device(local)
        print(json.dumps({"mode": "nlcg", **run_nlcg(D, max(args.nlcg_iters, 11))}), flush=True)
        return
    if args.mode == "psf":
        import torch

        torch.cuda.set_device(local)
        print(json.dumps({"mode": "psf", **run_psf(max(args.psf_reps, 1))}), flush=True)
        return
    if args.mode == "batch":
        import torch

        import deconlib_b200.deconvolution as D

        torch.cuda.set_device(local)
        print(json.dumps({"mode": "batch", **run_batched(D, max(args.batch_iters, 1))}), flush=True)
        return
    if args.impl == "reference":
        run_reference(args, ws, rank, local)
    else:
        run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
