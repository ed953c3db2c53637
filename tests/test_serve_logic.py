"""The served loop's host logic (nextgen_b200/serve.py) on CPU, against a
fake batch that counts steps instead of launching kernels: every request is
prepared after its arrival, admitted while the HBM budget allows, stepped to
exactly its own step count by its own precision's stepping thread, retired
once, and its latency is measured from its arrival; a failure in the
preparer or in a step reaches the caller.
"""
import threading
import time
from types import SimpleNamespace

import numpy as np
import pytest

from nextgen_b200 import cgx, serve


class FakePrepared:
    def __init__(self, r, nsteps, cells):
        self.r, self.nsteps, self.cells, self.released = r, nsteps, cells, False

    def release(self):
        self.released = True


class FakeBatch:
    """One precision's batch: cases advance `nsteps` per step() call up to
    their own count; the budget counts cells."""
    fail_step = False

    def __init__(self, device, prec, max_cases=256, hbm_budget=0):
        self.prec, self.budget = prec, hbm_budget
        self.cases, self.next_id, self.used = {}, 0, 0
        self.lock = threading.Lock()
        self.max_resident = 0
        self.max_used = 0
        self.closed = False

    def prepare(self, mesh, params, rho, u, p, nsteps):
        return FakePrepared(mesh, nsteps, len(rho))

    def admit(self, case):
        with self.lock:
            if self.used + case.cells > self.budget:
                return None
            cid = self.next_id
            self.next_id += 1
            self.cases[cid] = [case, 0]
            self.used += case.cells
            self.max_resident = max(self.max_resident, len(self.cases))
            self.max_used = max(self.max_used, self.used)
            return cid

    def step(self, nsteps):
        if FakeBatch.fail_step:
            raise cgx.CgxError(-3, "fake step failure")
        time.sleep(0.001)
        with self.lock:
            for c in self.cases.values():
                c[1] = min(c[0].nsteps, c[1] + nsteps)

    def done(self):
        with self.lock:
            return [cid for cid, (c, k) in self.cases.items() if k >= c.nsteps]

    def get_state(self, cid):
        c, k = self.cases[cid]
        return (np.full(c.cells, float(k)),)

    def remove(self, cid):
        with self.lock:
            c, _ = self.cases.pop(cid)
            self.used -= c.cells

    def close(self):
        self.closed = True


@pytest.fixture
def fake(monkeypatch):
    made = []

    def batch(*a, **k):
        b = FakeBatch(*a, **k)
        made.append(b)
        return b
    monkeypatch.setattr(cgx, "Batch", batch)
    monkeypatch.setattr(serve, "device_mesh", lambda r, device=0: (r.mesh, False))
    FakeBatch.fail_step = False
    return made


def _requests(n, seed=3):
    rng = np.random.default_rng(seed)
    arrivals = serve.poisson_arrivals(n, rate=400.0, seed=seed)
    reqs = []
    for k in range(n):
        cells = int(rng.integers(10, 60))
        prec = cgx.CGX_FP64 if k % 3 else cgx.CGX_MIXED
        reqs.append(serve.Request(k, SimpleNamespace(ncv=cells), None, np.zeros(cells), None, None,
                                  int(rng.integers(3, 40)), prec, float(arrivals[k])))
    return reqs


@pytest.mark.parametrize("concurrent", [True, False])
def test_every_request_served_once_at_its_own_count(fake, concurrent):
    reqs = _requests(24)
    out = serve.serve(reqs, hbm_budget=120, chunk=4, prepare_ahead=3, concurrent=concurrent)
    assert out["requests"] == 24 and out["cell_steps_per_s"] > 0
    assert out["p99_latency_s"] >= out["p50_latency_s"] > 0
    assert out["concurrent_precisions"] == concurrent
    for r in reqs:
        assert r.finished >= r.admitted >= r.arrival
        assert np.all(r.state[0] == r.nsteps)  # stepped to its own count, no further
    # the budget held: never more cells resident than allowed
    for b in fake:
        assert b.closed and b.used == 0
        assert 1 <= b.max_resident and b.max_used <= 120


def test_failure_in_a_step_reaches_the_caller(fake):
    FakeBatch.fail_step = True
    with pytest.raises(cgx.CgxError, match="fake step failure"):
        serve.serve(_requests(6), hbm_budget=1000, chunk=2)
    assert all(b.closed for b in fake)


def test_failure_in_the_preparer_reaches_the_caller(fake, monkeypatch):
    def bad_mesh(r, device=0):
        raise RuntimeError("no mesh")
    monkeypatch.setattr(serve, "device_mesh", bad_mesh)
    with pytest.raises(RuntimeError, match="no mesh"):
        serve.serve(_requests(4), hbm_budget=1000, chunk=2)
