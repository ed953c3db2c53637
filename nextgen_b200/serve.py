"""Served stream: continuous batching of periodic-box cases on one GPU.

Requests (a mesh, parameters, an initial state, a step count and a
precision) arrive over time.  A preparer thread builds each arrived
request's case (and its device mesh, when the request brings the mesher's
compact mesh) while the GPU steps the resident ones; the stepping loop admits
prepared cases into the batch of their precision between steps as their HBM
footprint fits the budget, keeps every admitted case's state on the device,
advances all resident cases together one graph replay per step
(cgx_batch_step) and retires each case at its own step count.

`serve()` returns per-request records (arrival, admission, completion,
latency) and aggregate throughput; `run_sequential()` runs the same cases
one at a time on the plain FP64 path for comparison.
"""
import os
import queue
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import cgx


@dataclass
class Request:
    rid: int
    mesh: object          # cgx.Mesh (device mesh, may be shared), or None with `compact`
    params: object        # cgx.Params
    rho: np.ndarray
    u: np.ndarray
    p: np.ndarray
    nsteps: int
    precision: int = cgx.CGX_FP64
    arrival: float = 0.0  # seconds after the start of the stream
    # a request may instead carry the mesher's compact mesh (meshgen's
    # compact_only output); admission then builds its operators on the GPU
    # (cgx_operators_build) and its device mesh, and retirement frees them
    compact: object = None
    ncv: int = 0
    # filled by the server
    admitted: float = None
    finished: float = None
    case_id: int = None
    state: tuple = field(default=None, repr=False)

    @property
    def cells(self):
        return self.mesh.ncv if self.mesh is not None else (self.compact.ncv if self.compact is not None else self.ncv)

    @property
    def cell_steps(self):
        return self.cells * self.nsteps


def poisson_arrivals(n, rate, seed=2024):
    """Arrival times of a seeded Poisson process of the given rate (1/s)."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


def device_mesh(r, device=0):
    """The request's device mesh: its own, or built from its compact mesh
    (GPU operator build, then cgx_mesh_create).  Returns (mesh, owned)."""
    if r.mesh is not None:
        return r.mesh, False
    from .meshgen import DeviceOperatorMesh
    ops = DeviceOperatorMesh(r.compact, device=device)
    try:
        return cgx.Mesh(ops, device=device), True
    finally:
        ops.close()


def serve(requests, hbm_budget=96 << 30, chunk=8, max_cases=256, device=0, keep_state=True,
          concurrent=True, prepare_ahead=4):
    """Continuous batching over `requests`.

    A preparer thread takes the requests in arrival order: once one has
    arrived it builds the request's device mesh if needed and its case
    (cgx_batch_prepare: solver, state, initComplete on the case's own
    stream), at most `prepare_ahead` cases ahead of admission, while the
    batches step.  The stepping loop joins prepared cases between steps
    (cgx_batch_admit, in arrival order, while the HBM budget allows),
    advances the resident cases `chunk` steps (a case stops at its own step
    count) and retires the finished ones.  With `concurrent`, the FP64 and
    the mixed-precision batches (each on its own CUDA stream) are stepped
    from two host threads at once.  Returns a summary dict; requests are
    updated in place."""
    order = sorted(requests, key=lambda r: r.arrival)
    batches = {prec: cgx.Batch(device, prec, max_cases=max_cases, hbm_budget=hbm_budget)
               for prec in sorted(set(r.precision for r in order))}
    ready = queue.Queue()
    slots = threading.Semaphore(prepare_ahead)
    stop = threading.Event()
    failure = []
    t0 = time.perf_counter()

    def now():
        return time.perf_counter() - t0

    def prepare_all():
        try:
            # leave host cores to the stepping threads while meshes are set up
            cgx.set_host_threads(max(1, (os.cpu_count() or 1) - 4))
            for r in order:
                while not stop.is_set() and now() < r.arrival:
                    time.sleep(min(0.005, max(0.0, r.arrival - now())))
                while not stop.is_set() and not slots.acquire(timeout=0.05):
                    pass
                if stop.is_set():
                    return
                r._dev_mesh, r._own_mesh = device_mesh(r, device)
                r._prepared = batches[r.precision].prepare(r._dev_mesh, r.params, r.rho, r.u, r.p, r.nsteps)
                ready.put(r)
        except Exception as e:  # reported by the stepping loop
            failure.append(e)

    prep = threading.Thread(target=prepare_all, daemon=True)
    prep.start()
    pool = ThreadPoolExecutor(max_workers=2) if concurrent and len(batches) > 1 else None
    busy = 0.0  # wall time with at least one batch stepping
    waiting, resident, n_done = [], {}, 0
    try:
        while n_done < len(order):
            if failure:
                raise failure[0]
            while True:
                try:
                    waiting.append(ready.get_nowait())
                except queue.Empty:
                    break
            still = []
            for r in sorted(waiting, key=lambda q: q.arrival):
                cid = batches[r.precision].admit(r._prepared)
                if cid is None:
                    still.append(r)
                    continue
                slots.release()
                r.case_id = cid
                r.admitted = now()
                resident[(r.precision, cid)] = r
            waiting = still
            if not resident:
                time.sleep(0.002)
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
                    if r._own_mesh:
                        r._dev_mesh.close()
                    r._dev_mesh = r._prepared = None
                    n_done += 1
        makespan = now()
    finally:
        stop.set()
        prep.join()
        if pool is not None:
            pool.shutdown()
        for r in waiting:
            r._prepared.release()
        for b in batches.values():
            b.close()
    lat = np.array([r.finished - r.arrival for r in requests])
    cs = float(sum(r.cell_steps for r in requests))
    return {"requests": len(requests), "makespan_s": makespan, "solves_per_s": len(requests) / makespan,
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "cell_steps_per_s": cs / makespan, "cell_steps": cs, "stepping_s": busy,
            "concurrent_precisions": pool is not None, "admission": "preparer thread, overlapped with stepping"}


def run_sequential(requests, precision=cgx.CGX_FP64, keep_state=False, device=0):
    """The same cases one at a time on the plain single-case path: the
    request's device mesh (built as admission builds it), set the state,
    initComplete, step to the case's count, read the state back.
    precision=None runs each request at its own precision."""
    t0 = time.perf_counter()
    states = []
    for r in requests:
        gm, owned = device_mesh(r, device)
        s = cgx.Solver(gm, r.params, r.precision if precision is None else precision)
        s.set_state_primitive(r.rho, r.u, r.p)
        s.initComplete()
        s.step(r.nsteps)
        st = s.get_state()
        if keep_state:
            states.append(st)
        s.close()
        if owned:
            gm.close()
    el = time.perf_counter() - t0
    cs = float(sum(r.cell_steps for r in requests))
    return {"seconds": el, "cell_steps_per_s": cs / el, "solves_per_s": len(requests) / el}, states
