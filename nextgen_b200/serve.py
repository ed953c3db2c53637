"""Served stream: continuous batching of periodic-box cases on one GPU.

Requests (a mesh, parameters, an initial state, a step count and a
precision) arrive over time; the server admits each one into the resident
batch of its precision as soon as it has arrived and its HBM footprint fits
the budget, keeps every admitted case's state on the device, advances all
resident cases together one graph replay per step (cgx_batch_step) and
retires each case at its own step count.  Requests that arrive while others
run join between steps.

`serve()` returns per-request records (arrival, admission, completion,
latency) and aggregate throughput; `run_sequential()` runs the same cases
one at a time on the plain FP64 path for comparison.
"""
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import cgx


@dataclass
class Request:
    rid: int
    mesh: object          # cgx.Mesh (device mesh, may be shared between requests)
    params: object        # cgx.Params
    rho: np.ndarray
    u: np.ndarray
    p: np.ndarray
    nsteps: int
    precision: int = cgx.CGX_FP64
    arrival: float = 0.0  # seconds after the start of the stream
    # filled by the server
    admitted: float = None
    finished: float = None
    case_id: int = None
    state: tuple = field(default=None, repr=False)

    @property
    def cell_steps(self):
        return self.mesh.ncv * self.nsteps


def poisson_arrivals(n, rate, seed=2024):
    """Arrival times of a seeded Poisson process of the given rate (1/s)."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def serve(requests, hbm_budget=96 << 30, chunk=8, max_cases=256, device=0, keep_state=True,
          concurrent=True):
    """Continuous batching over `requests` (sorted by arrival).  Each loop
    iteration admits every arrived request that fits, advances the resident
    cases `chunk` steps (a case stops at its own step count) and retires the
    finished ones.  With `concurrent`, the FP64 and the mixed-precision
    batches (each on its own CUDA stream) are stepped from two host threads
    at once, so their kernels overlap on the GPU.  Returns a summary dict;
    requests are updated in place."""
    pending = sorted(requests, key=lambda r: r.arrival)
    batches = {}
    resident = {}
    pool = ThreadPoolExecutor(max_workers=2) if concurrent else None
    busy = 0.0  # wall time with at least one batch stepping
    t0 = time.perf_counter()

    def now():
        return time.perf_counter() - t0

    def batch_of(prec):
        if prec not in batches:
            batches[prec] = cgx.Batch(device, prec, max_cases=max_cases, hbm_budget=hbm_budget)
        return batches[prec]

    waiting = []
    while pending or waiting or resident:
        t = now()
        while pending and pending[0].arrival <= t:
            waiting.append(pending.pop(0))
        # admit in arrival order while the budget allows (per precision)
        still = []
        for r in waiting:
            b = batch_of(r.precision)
            cid = b.add(r.mesh, r.params, r.rho, r.u, r.p, r.nsteps)
            if cid is None:
                still.append(r)
                continue
            r.case_id = cid
            r.admitted = now()
            resident[(r.precision, cid)] = r
        waiting = still
        if not resident:
            if pending:
                time.sleep(max(0.0, min(pending[0].arrival - now(), 0.01)))
            continue
        active = [b for prec, b in batches.items() if any(k[0] == prec for k in resident)]
        tb = time.perf_counter()
        if pool is not None and len(active) > 1:
            for f in [pool.submit(b.step, chunk) for b in active]:
                f.result()
        else:
            for b in active:
                b.step(chunk)
        busy += time.perf_counter() - tb
        for prec, b in batches.items():
            for cid in b.done():
                r = resident.pop((prec, cid))
                if keep_state:
                    r.state = b.get_state(cid)
                r.finished = now()
                b.remove(cid)
    makespan = now()
    if pool is not None:
        pool.shutdown()
    for b in batches.values():
        b.close()
    lat = np.array([r.finished - r.arrival for r in requests])
    cs = float(sum(r.cell_steps for r in requests))
    return {"requests": len(requests), "makespan_s": makespan, "solves_per_s": len(requests) / makespan,
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "cell_steps_per_s": cs / makespan, "cell_steps": cs, "stepping_s": busy,
            "concurrent_precisions": pool is not None}


def run_sequential(requests, precision=cgx.CGX_FP64, keep_state=False):
    """The same cases one at a time on the plain single-case path: set the
    state, initComplete, step to the case's count, read the state back."""
    t0 = time.perf_counter()
    states = []
    for r in requests:
        s = cgx.Solver(r.mesh, r.params, precision)
        s.set_state_primitive(r.rho, r.u, r.p)
        s.initComplete()
        s.step(r.nsteps)
        st = s.get_state()
        if keep_state:
            states.append(st)
        s.close()
    el = time.perf_counter() - t0
    cs = float(sum(r.cell_steps for r in requests))
    return {"seconds": el, "cell_steps_per_s": cs / el, "solves_per_s": len(requests) / el}, states
