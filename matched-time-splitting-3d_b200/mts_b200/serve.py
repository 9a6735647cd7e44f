"""Serving: continuous batching of independent solves on one GPU.

Requests (grid, surface, beta, method, dt, number of steps) arrive over time.
Each goes through
  1. host setup (tags, crossings, MIB weights) on a pool of host threads,
  2. admission: it waits until its device memory (an upper bound computed
     from its grid and crossing count) fits in the HBM budget, then a pool
     thread uploads it (mts_create_from_crossings) and initializes it,
  3. the running batch: at every chunk boundary the server advances all
     admitted problems together by one mts_batch_advance_steps call (each by
     up to chunk_steps steps; one launch per kernel of a step for all of
     them), so problems that arrive while others run join the batch as soon
     as they are uploaded, and their work overlaps on the device,
  4. retirement: after its last step a pool thread reads the problem's
     error norms and frees its device memory; its budget is returned when
     that is done.  The loop goes on batching meanwhile.
Batching does not change any result: each problem's solution is the one it
gets alone, bit for bit (mts_batch_advance_steps' contract).
"""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from . import Solver, batch_advance_steps, setup_device, setup_host
from .workloads import Request, device_bytes_bound


@dataclass
class Result:
    id: int
    arrival: float
    admitted: float = 0.0
    done: float = 0.0
    steps: int = 0
    lmax: float = 0.0
    l2: float = 0.0
    t: float = 0.0
    device_bytes: int = 0
    solution: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class _Job:
    req: Request
    result: Result
    bound: int = 0
    tags: np.ndarray | None = None
    crossings: np.ndarray | None = None
    solver: Solver | None = None
    left: int = 0
    error: str | None = None


class Server:
    """Continuous-batching server over the C ABI.

    hbm_budget: bytes of device memory the admitted problems may hold.
    max_active: problems on the device at once (admitted and not retired); a
      batch call's cost grows faster than its problem count, so past a few
      hundred problems more of them in flight lower the throughput.
    chunk_steps: steps per batch call; new arrivals join at chunk boundaries.
    host_threads: pool for host setup and uploads.
    keep_solutions: keep each result's final field (for tests).
    setup: "host" (tags, crossings and MIB weights on the pool's host
      threads) or "device" (the same on the GPU, mts_setup_device)."""

    def __init__(self, hbm_budget: float = 120e9, chunk_steps: int = 32, host_threads: int = 16,
                 keep_solutions: bool = False, precision: str = "plain", max_active: int = 384,
                 setup: str = "host"):
        self.budget = int(hbm_budget)
        self.max_active = max(1, int(max_active))
        self.chunk = max(1, int(chunk_steps))
        self.threads = max(1, int(host_threads))
        self.keep = keep_solutions
        self.precision = precision
        if setup not in ("host", "device"):
            raise ValueError("setup must be host or device")
        self.setup = setup_device if setup == "device" else setup_host
        self.peak_bytes = 0
        self.peak_active = 0
        self.batches = 0
        # seconds of the loop in batch calls and in retirements (norms, field
        # read, free), for the breakdown of a run
        self.batch_s = 0.0
        self.retire_s = 0.0

    # -- pool tasks ----------------------------------------------------------
    def _setup(self, job: _Job) -> _Job:
        tags, cr, _ = self.setup(job.req.spec)
        job.tags, job.crossings = tags, cr
        job.bound = device_bytes_bound(job.req.spec, len(cr), precision=self.precision)
        return job

    def _retire(self, job: _Job, clock) -> _Job:
        res = job.result
        lmax, l2, _ = job.solver.norms()
        res.lmax, res.l2, res.t, res.steps = lmax, l2, job.solver.time, job.req.steps
        if self.keep:
            res.solution = job.solver.solution()
        job.solver.close()
        job.solver = None
        res.done = clock()
        return job

    def _upload(self, job: _Job) -> _Job:
        s = Solver(job.req.spec, tags=job.tags, crossings=job.crossings)
        if self.precision == "mixed" and job.req.spec.method == "adi":
            s.set_precision("mixed")
        s.initialize()
        s.synchronize()
        job.solver = s
        job.tags = job.crossings = None
        job.result.device_bytes = s.device_bytes()
        return job

    # -- the loop --------------------------------------------------------------
    def run(self, requests: list[Request]) -> list[Result]:
        reqs = sorted(requests, key=lambda r: r.arrival)
        results = {r.id: Result(r.id, r.arrival) for r in reqs}
        pool = ThreadPoolExecutor(max_workers=self.threads)
        setups, uploads, retires = [], [], []  # futures in flight
        ready: list[_Job] = []            # set up, waiting for budget
        active: list[_Job] = []           # on the device
        used = 0
        nxt = 0
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0  # noqa: E731
        try:
            while nxt < len(reqs) or setups or ready or uploads or active or retires:
                now = clock()
                # 1. arrivals -> host setup
                while nxt < len(reqs) and reqs[nxt].arrival <= now:
                    r = reqs[nxt]
                    setups.append(pool.submit(self._setup, _Job(r, results[r.id], left=r.steps)))
                    nxt += 1
                # 2. finished setups, in arrival order, wait for budget
                done_s = [f for f in setups if f.done()]
                for f in done_s:
                    setups.remove(f)
                    ready.append(f.result())
                ready.sort(key=lambda j: j.req.arrival)
                # 3. admission against the budget and the active cap (first
                # come, first served)
                while (ready and used + ready[0].bound <= self.budget
                       and len(active) + len(uploads) < self.max_active):
                    job = ready.pop(0)
                    used += job.bound
                    uploads.append(pool.submit(self._upload, job))
                # finished retirements return their budget
                for f in [f for f in retires if f.done()]:
                    retires.remove(f)
                    used -= f.result().bound
                if ready and not active and not uploads and not retires and ready[0].bound > self.budget:
                    raise RuntimeError(f"request {ready[0].req.id} needs {ready[0].bound} bytes, over the budget")
                done_u = [f for f in uploads if f.done()]
                for f in done_u:
                    uploads.remove(f)
                    job = f.result()
                    job.result.admitted = clock()
                    active.append(job)
                self.peak_bytes = max(self.peak_bytes, used)
                self.peak_active = max(self.peak_active, len(active))
                # 4. one chunk of the running batch
                if active:
                    ks = [min(self.chunk, j.left) for j in active]
                    tb = time.perf_counter()
                    batch_advance_steps([j.solver for j in active], ks)
                    self.batch_s += time.perf_counter() - tb
                    self.batches += 1
                    for j, k in zip(active, ks):
                        j.left -= k
                    tr = time.perf_counter()
                    for j in [j for j in active if j.left == 0]:
                        active.remove(j)
                        retires.append(pool.submit(self._retire, j, clock))
                    self.retire_s += time.perf_counter() - tr
                else:
                    time.sleep(0.0005)
        finally:
            pool.shutdown(wait=True)
            for j in active:
                j.solver.close()
        return [results[r.id] for r in reqs]


def solve_alone(req: Request, keep_solution: bool = False, precision: str = "plain") -> Result:
    """One request on its own: setup, upload, steps, norms (the sequential
    baseline's unit of work)."""
    res = Result(req.id, req.arrival)
    with Solver(req.spec) as s:
        if precision == "mixed" and req.spec.method == "adi":
            s.set_precision("mixed")
        s.initialize()
        s.advance(req.steps)
        lmax, l2, _ = s.norms()
        res.lmax, res.l2, res.t, res.steps = lmax, l2, s.time, req.steps
        if keep_solution:
            res.solution = s.solution()
    return res


def fifo_latencies(arrivals: np.ndarray, service: np.ndarray) -> np.ndarray:
    """Latencies of a single FIFO server with the given arrival and service
    times (the sequential baseline under the same arrival stream)."""
    free = 0.0
    out = np.empty(len(arrivals))
    for i, (a, s) in enumerate(zip(arrivals, service)):
        start = max(a, free)
        free = start + s
        out[i] = free - a
    return out
