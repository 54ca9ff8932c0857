"""Served deconvolution on one GPU: continuous batching of RL and Hessian-PDHG jobs.

Jobs (an observation, its PSF, the solver and its parameters) arrive over
time.  The server

  * admits a job once it has arrived, a slot is free and its estimated device
    footprint fits the HBM budget beside the jobs already on the device
    (``Scheduler``: strict FIFO, so a large job is never starved);
  * keeps every admitted job's OTF, spectra and iterates resident in HBM and
    runs it on its own CUDA stream; each scheduling round queues ``chunk``
    iterations of every job whose previous chunk has finished, so kernels of
    different jobs overlap on the device (continuous batching: new jobs join
    while others are mid-solve, finished jobs leave at once);
  * pools device resources by shape bucket: a finished job hands its
    convolution plan (OTF + spectra buffers) to the next job with the same
    kernel and signal shapes, which rebuilds the OTF in place
    (``LinearFFTConvolver.set_kernel``), and its PDHG state to the next PDHG
    job (``decon_pdhg_reset``).  Nothing is freed while jobs run, because
    ``cudaFree`` synchronises the whole device and would drain every stream;
  * puts every job's convolution on a canvas of compile-time FFT lengths
    (``canvas="static"``: ``static_fft_shape``, each axis at most 1/3 longer
    than the reference's 5-smooth canvas), because the runtime-radix FFT path
    that most 5-smooth lengths take measured ~4x slower per canvas voxel;
    ``canvas="reference"`` keeps ``fast_padded_shape``.  The canvas changes a
    result by FP32 rounding only.

Latency is arrival -> restored volume on the host.  The reference has no
serving layer; each job computes exactly what ``richardson_lucy_with_operator``
/ ``solve_pdhg_mlx`` compute for it alone (same kernels, same launch shapes,
deterministic reductions), which the tests check.
"""

from __future__ import annotations

import collections
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

__all__ = ["Job", "JobResult", "ServeReport", "Scheduler", "DeconServer", "job_signal_shape",
           "job_fft_shape", "job_device_bytes", "poisson_arrivals"]


@dataclass
class Job:
    """One deconvolution request.

    ``kind``: "rl" (``richardson_lucy_with_operator`` on a LinearFFTConvolver
    of ``psf`` over ``observed.shape``) or "pdhg" (``solve_pdhg_mlx`` with
    ``options`` as keyword arguments, e.g. alpha, sampling_factors, spacing).
    ``arrival``: seconds after the start of the stream."""

    job_id: int
    kind: str
    observed: np.ndarray
    psf: np.ndarray
    num_iter: int
    arrival: float = 0.0
    background: float = 0.0
    options: dict = field(default_factory=dict)


@dataclass
class JobResult:
    job_id: int
    kind: str
    restored: np.ndarray
    iterations: int
    arrival: float
    admitted: float
    finished: float
    object_voxels: int
    device_bytes: int

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


@dataclass
class ServeReport:
    results: List[JobResult]
    makespan: float
    voxel_iters_per_s: float
    p50_latency: float
    p99_latency: float
    peak_device_bytes: int
    max_concurrent: int

    def summary(self) -> dict:
        return {"jobs": len(self.results), "makespan_s": self.makespan,
                "voxel_iter_per_s": self.voxel_iters_per_s, "p50_latency_s": self.p50_latency,
                "p99_latency_s": self.p99_latency, "peak_budgeted_bytes": self.peak_device_bytes,
                "max_concurrent_jobs": self.max_concurrent}


# ---------------------------------------------------------------------------
# footprint model
# ---------------------------------------------------------------------------


def _fast_padded(signal, kernel):
    from .deconvolution.linops import fast_padded_shape

    return tuple(int(v) for v in fast_padded_shape(tuple(signal), tuple(kernel)))


def job_signal_shape(job: Job) -> Tuple[int, ...]:
    """Object (reconstruction) grid of the job's convolution."""
    if job.kind == "pdhg" and (job.options.get("sampling_factors") is not None
                               or job.options.get("bin_factors") is not None):
        return tuple(int(s) for s in job.psf.shape)
    return tuple(int(s) for s in job.observed.shape)


def job_fft_shape(job: Job, canvas: str = "reference") -> Tuple[int, ...]:
    """The job's convolution canvas under a canvas policy ("reference":
    ``fast_padded_shape``; "static": ``static_fft_shape``)."""
    sig = job_signal_shape(job)
    if canvas == "reference":
        return _fast_padded(sig, job.psf.shape)
    if canvas == "static":
        from .deconvolution.linops import static_fft_shape

        return tuple(int(v) for v in static_fft_shape(sig, tuple(job.psf.shape)))
    raise ValueError(f"canvas must be 'reference' or 'static', got {canvas!r}")


def _plan_bytes(signal, kernel, fft=None) -> int:
    f = tuple(fft) if fft is not None else _fast_padded(signal, kernel)
    while len(f) < 3:
        f = (1,) + f
    s = (1,) * (3 - len(signal)) + tuple(signal)
    pitch = -(-(f[2] // 2 + 1) // 16) * 16
    return 8 * pitch * (f[0] * f[1] + s[0] * s[1] + s[0] * f[1])


def job_device_bytes(job: Job, canvas: str = "reference") -> int:
    """Device bytes the job holds while admitted: its convolution plan (OTF
    and the two scratch spectra) on the policy's canvas, its iterates and
    temporaries."""
    sig = job_signal_shape(job)
    n = int(np.prod(sig))
    m = int(np.prod(job.observed.shape))
    k = int(np.prod(job.psf.shape))
    plan = _plan_bytes(sig, job.psf.shape, job_fft_shape(job, canvas))
    if job.kind == "rl":
        arrays = 4 * (5 * n + k)
    else:
        # data, A x (x2), y1, resampling temporaries; x (x2), y2 (6), A^T y1, temporaries
        arrays = 4 * (6 * m + 11 * n + k)
    return plan + arrays


def poisson_arrivals(n: int, rate: float, rng: np.random.Generator) -> np.ndarray:
    """Arrival times (s) of a Poisson process of ``rate`` jobs/s."""
    return np.cumsum(rng.exponential(1.0 / rate, n))


# ---------------------------------------------------------------------------
# admission (host logic only)
# ---------------------------------------------------------------------------


class Scheduler:
    """FIFO admission by slots and an HBM byte budget.

    ``arrive`` queues a job; ``admit`` pops jobs from the head of the queue
    while a slot is free and the head's footprint fits beside the admitted
    jobs (and ``reserved`` bytes, e.g. idle pooled plans); ``release`` returns
    a finished job's bytes.  A job whose footprint exceeds the whole budget
    can never run and is rejected with ValueError on arrival."""

    def __init__(self, budget_bytes: int, max_active: int,
                 footprint: Callable[[Job], int] = job_device_bytes):
        if max_active < 1:
            raise ValueError("max_active must be >= 1")
        self.budget = int(budget_bytes)
        self.max_active = int(max_active)
        self.footprint = footprint
        self.pending: collections.deque = collections.deque()
        self.active: Dict[int, int] = {}
        self.used = 0
        self.peak = 0

    def arrive(self, job: Job) -> None:
        b = self.footprint(job)
        if b > self.budget:
            raise ValueError(f"job {job.job_id} needs {b} device bytes, more than the whole "
                             f"budget of {self.budget}")
        self.pending.append((job, b))

    def admit(self, reserved: int = 0) -> List[Tuple[Job, int]]:
        out = []
        while self.pending and len(self.active) < self.max_active:
            job, b = self.pending[0]
            if self.used + b + reserved > self.budget:
                break
            self.pending.popleft()
            self.active[job.job_id] = b
            self.used += b
            self.peak = max(self.peak, self.used + reserved)
            out.append((job, b))
        return out

    def head_blocked_by(self, reserved: int) -> int:
        """Bytes the head of the queue lacks (0 if it fits or nothing waits)."""
        if not self.pending or len(self.active) >= self.max_active:
            return 0
        _, b = self.pending[0]
        return max(0, self.used + b + reserved - self.budget)

    def release(self, job_id: int) -> None:
        self.used -= self.active.pop(job_id)

    @property
    def idle(self) -> bool:
        return not self.pending and not self.active


# ---------------------------------------------------------------------------
# device side
# ---------------------------------------------------------------------------


class _Pools:
    """Streams, convolution plans and PDHG states reused across jobs."""

    def __init__(self, n_streams: int, prioritise: bool = True):
        import torch

        # Stream priorities spread over the device's range: the scheduler
        # hands the highest-priority free stream to each admitted job, so the
        # jobs that arrived first keep the SMs when several compete and finish
        # first (lower latency at the same throughput).
        least, greatest = torch.cuda.Stream.priority_range() if prioritise else (0, 0)
        levels = list(range(greatest, least + 1)) or [0]
        prios = [levels[min(len(levels) - 1, i * len(levels) // max(n_streams, 1))]
                 for i in range(n_streams)]
        self.streams = [torch.cuda.Stream(priority=p) for p in prios]
        self.free_streams = list(reversed(self.streams))  # pop() takes the highest priority
        self.plans: Dict[tuple, list] = collections.defaultdict(list)
        self.plan_bytes: Dict[int, int] = {}
        self.states: list = []

    def idle_plan_bytes(self) -> int:
        return sum(self.plan_bytes[id(p)] for v in self.plans.values() for p in v)

    def take_plan(self, key):
        lst = self.plans.get(key)
        return lst.pop() if lst else None

    def give_plan(self, key, conv, nbytes):
        self.plan_bytes[id(conv)] = nbytes
        self.plans[key].append(conv)

    def evict_plans(self, nbytes: int) -> int:
        """Destroy idle plans (largest first) until ``nbytes`` are freed."""
        import torch

        freed = 0
        items = sorted(((self.plan_bytes[id(p)], k, p) for k, v in self.plans.items() for p in v),
                       key=lambda t: -t[0])
        victims = []
        for b, k, p in items:
            if freed >= nbytes:
                break
            self.plans[k].remove(p)
            self.plan_bytes.pop(id(p), None)
            victims.append(p)
            freed += b
        items = None
        victims.clear()  # last references: each plan synchronises the device and frees
        torch.cuda.synchronize()
        return freed

    def take_state(self, num_iter):
        for i, s in enumerate(self.states):
            if s.capacity >= max(int(num_iter), 1):
                return self.states.pop(i)
        return None


class _Slot:
    """One admitted job on its own stream."""

    def __init__(self, job: Job, nbytes: int, pools: _Pools, now: float, canvas: str = "reference"):
        import torch

        from .deconvolution.linops import LinearFFTConvolver
        from .deconvolution.pdhg import pdhg_mlx_runner
        from .deconvolution.rl import RLRunner

        self.job, self.nbytes, self.pools = job, nbytes, pools
        self.admitted = now
        self.stream = pools.free_streams.pop()
        self.event = None
        self.finished = False
        self.sig = job_signal_shape(job)
        self.fft = job_fft_shape(job, canvas)
        self.key = (tuple(job.psf.shape), self.sig, self.fft)
        with torch.cuda.stream(self.stream):
            conv = pools.take_plan(self.key)
            if job.kind == "rl":
                if conv is None:
                    conv = LinearFFTConvolver(job.psf, self.sig, fft_shape=self.fft)
                else:
                    conv.set_kernel(job.psf)
                self.conv = conv
                self.runner = RLRunner(job.observed, conv, job.num_iter, job.background)
                self.state = None
            elif job.kind == "pdhg":
                opts = dict(job.options)
                self.state = pools.take_state(job.num_iter)
                self.runner, self.meta = pdhg_mlx_runner(
                    job.observed, job.psf, num_iter=job.num_iter, background=job.background,
                    conv=conv, state=self.state, async_status=True, fft_shape=self.fft, **opts)
                self.conv = _find_conv(self.runner.A)
                self.state = self.runner.state
            else:
                raise ValueError(f"unknown job kind {job.kind!r}")

    def ready(self) -> bool:
        return self.event is None or self.event.query()

    def step(self, n: int) -> None:
        import torch

        with torch.cuda.stream(self.stream):
            for _ in range(n):
                if not self.runner.iterate():
                    self.finished = True
                    break
            self.event = torch.cuda.Event()
            self.event.record(self.stream)

    def collect(self) -> Tuple[np.ndarray, int]:
        import torch

        from .deconvolution.pdhg import pdhg_result

        with torch.cuda.stream(self.stream):
            if self.job.kind == "rl":
                res = self.runner.finish()
            else:
                res = pdhg_result(self.runner, self.meta)
            out = res.restored.cpu().numpy()
        return out, int(res.iterations)

    def release(self) -> None:
        pools = self.pools
        if self.conv is not None:
            pools.give_plan(self.key, self.conv, _plan_bytes(self.sig, self.job.psf.shape, self.fft))
        if self.state is not None:
            pools.states.append(self.state)
        self.runner = None
        self.conv = None
        self.state = None
        pools.free_streams.append(self.stream)
        pools.free_streams.sort(key=lambda st: -st.priority)


def _find_conv(op):
    from .deconvolution.composition import Compose
    from .deconvolution.linops import LinearFFTConvolver

    if isinstance(op, LinearFFTConvolver):
        return op
    if isinstance(op, Compose):
        return _find_conv(op.outer) or _find_conv(op.inner)
    return None


class DeconServer:
    """Continuous-batching request loop (see the module docstring).

    ``budget_bytes``: device bytes admitted jobs (plus idle pooled plans) may
    hold; ``max_active``: concurrent jobs (one stream each); ``chunk``:
    iterations queued per job per scheduling round; ``canvas``: "static"
    (compile-time FFT lengths) or "reference" (the reference's canvases)."""

    def __init__(self, budget_bytes: int = 150 * 10**9, max_active: int = 8, chunk: int = 8,
                 prioritise: bool = True, canvas: str = "static"):
        if canvas not in ("static", "reference"):
            raise ValueError(f"canvas must be 'static' or 'reference', got {canvas!r}")
        self.budget = int(budget_bytes)
        self.max_active = int(max_active)
        self.chunk = int(chunk)
        self.prioritise = bool(prioritise)
        self.canvas = canvas

    def run(self, jobs: Sequence[Job], clock: Callable[[], float] = time.perf_counter,
            realtime: bool = True) -> ServeReport:
        """Serve ``jobs`` (arrival times relative to the start of the call).
        ``realtime=False`` releases every job at once (arrival times are still
        used for the latency figures)."""
        import torch

        order = sorted(jobs, key=lambda j: j.arrival)
        sched = Scheduler(self.budget, self.max_active,
                          footprint=lambda j: job_device_bytes(j, self.canvas))
        pools = _Pools(self.max_active, self.prioritise)
        active: List[_Slot] = []
        results: List[JobResult] = []
        nxt = 0
        max_conc = 0
        torch.cuda.synchronize()
        t0 = clock()
        while True:
            now = clock() - t0
            while nxt < len(order) and (not realtime or order[nxt].arrival <= now):
                sched.arrive(order[nxt])
                nxt += 1
            lack = sched.head_blocked_by(pools.idle_plan_bytes())
            if lack > 0 and pools.idle_plan_bytes() > 0:
                pools.evict_plans(lack)
            for job, b in sched.admit(pools.idle_plan_bytes()):
                active.append(_Slot(job, b, pools, clock() - t0, self.canvas))
            max_conc = max(max_conc, len(active))
            progressed = False
            for slot in list(active):
                if not slot.ready():
                    continue
                progressed = True
                if slot.finished:
                    out, iters = slot.collect()
                    t_done = clock() - t0
                    j = slot.job
                    results.append(JobResult(j.job_id, j.kind, out, iters, j.arrival, slot.admitted,
                                             t_done, int(np.prod(slot.sig)), slot.nbytes))
                    slot.release()
                    sched.release(j.job_id)
                    active.remove(slot)
                else:
                    slot.step(self.chunk)
            if nxt >= len(order) and sched.idle and not active:
                break
            if not progressed:
                if not active and nxt < len(order) and realtime:
                    time.sleep(max(0.0, min(order[nxt].arrival - (clock() - t0), 0.01)))
                else:
                    time.sleep(20e-6)
        makespan = max((r.finished for r in results), default=0.0) - min(
            (r.arrival for r in results), default=0.0)
        vi = sum(r.object_voxels * r.iterations for r in results)
        lat = np.array([r.latency for r in results]) if results else np.zeros(1)
        results.sort(key=lambda r: r.job_id)
        return ServeReport(results=results, makespan=makespan,
                           voxel_iters_per_s=vi / makespan if makespan > 0 else 0.0,
                           p50_latency=float(np.percentile(lat, 50)),
                           p99_latency=float(np.percentile(lat, 99)),
                           peak_device_bytes=sched.peak, max_concurrent=max_conc)
