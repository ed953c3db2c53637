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
import queue
import threading
import time
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
    batches step.  Each precision's batch (on its own CUDA stream) has its
    own stepping thread: it joins its prepared cases between steps
    (cgx_batch_admit, in arrival order, while the HBM budget allows),
    advances its resident cases `chunk` steps (a case stops at its own step
    count) and retires the finished ones, without waiting for the other
    batch.  Without `concurrent` one thread steps the batches in turn.
    Returns a summary dict; requests are updated in place."""
    order = sorted(requests, key=lambda r: r.arrival)
    precs = sorted(set(r.precision for r in order))
    batches = {prec: cgx.Batch(device, prec, max_cases=max_cases, hbm_budget=hbm_budget) for prec in precs}
    ready = {prec: queue.Queue() for prec in precs}
    total = {prec: sum(1 for r in order if r.precision == prec) for prec in precs}
    slots = threading.Semaphore(prepare_ahead)
    stop = threading.Event()
    failure = []
    lock = threading.Lock()
    busy = [0.0, 0, 0.0]  # wall time with a batch stepping; steppers active; since
    t0 = time.perf_counter()

    def now():
        return time.perf_counter() - t0

    def mark(delta):
        with lock:
            t = time.perf_counter()
            if busy[1] > 0:
                busy[0] += t - busy[2]
            busy[1] += delta
            busy[2] = t

    def prepare_all():
        try:
            for r in order:
                while not stop.is_set() and now() < r.arrival:
                    time.sleep(min(0.005, max(0.0, r.arrival - now())))
                while not stop.is_set() and not slots.acquire(timeout=0.05):
                    pass
                if stop.is_set():
                    return
                r._dev_mesh, r._own_mesh = device_mesh(r, device)
                r._prepared = batches[r.precision].prepare(r._dev_mesh, r.params, r.rho, r.u, r.p, r.nsteps)
                ready[r.precision].put(r)
        except Exception as e:  # reported by the stepping threads
            failure.append(e)

    class Lane:
        """One precision's stepping state."""

        def __init__(self, prec):
            self.prec, self.b = prec, batches[prec]
            self.waiting, self.resident, self.n_done = [], {}, 0

        def turn(self):
            """Admit, step `chunk` steps, retire; False if nothing is resident."""
            while True:
                try:
                    self.waiting.append(ready[self.prec].get_nowait())
                except queue.Empty:
                    break
            still = []
            for r in sorted(self.waiting, key=lambda q: q.arrival):
                cid = self.b.admit(r._prepared)
                if cid is None:
                    still.append(r)
                    continue
                slots.release()
                r.case_id = cid
                r.admitted = now()
                self.resident[cid] = r
            self.waiting = still
            if not self.resident:
                return False
            mark(1)
            try:
                self.b.step(chunk)
            finally:
                mark(-1)
            for cid in self.b.done():
                r = self.resident.pop(cid)
                if keep_state:
                    r.state = self.b.get_state(cid)
                r.finished = now()
                self.b.remove(cid)
                if r._own_mesh:
                    r._dev_mesh.close()
                r._dev_mesh = r._prepared = None
                self.n_done += 1
            return True

    lanes = [Lane(prec) for prec in precs]

    def run(ls):
        try:
            while not stop.is_set() and any(l.n_done < total[l.prec] for l in ls):
                if failure:
                    return
                stepped = False
                for l in ls:
                    if l.n_done < total[l.prec]:
                        stepped |= l.turn()
                if not stepped:
                    time.sleep(0.002)
        except Exception as e:
            failure.append(e)

    prep = threading.Thread(target=prepare_all, daemon=True)
    prep.start()
    groups = [[l] for l in lanes] if concurrent else [lanes]
    steppers = [threading.Thread(target=run, args=(g,)) for g in groups]
    try:
        for t in steppers:
            t.start()
        for t in steppers:
            t.join()
        if failure:
            raise failure[0]
        makespan = now()
    finally:
        stop.set()
        for t in steppers:
            t.join()
        prep.join()
        for l in lanes:
            for r in l.waiting:
                r._prepared.release()
        for b in batches.values():
            b.close()
    lat = np.array([r.finished - r.arrival for r in requests])
    cs = float(sum(r.cell_steps for r in requests))
    return {"requests": len(requests), "makespan_s": makespan, "solves_per_s": len(requests) / makespan,
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "cell_steps_per_s": cs / makespan, "cell_steps": cs, "stepping_s": busy[0],
            "concurrent_precisions": bool(concurrent and len(lanes) > 1),
            "admission": "preparer thread, overlapped with stepping"}


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
