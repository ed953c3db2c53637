"""Batched and served form: many resident cases advanced by one graph replay
per step over a packed work list; cases join and leave between steps.

Each result must match the same case run alone (single-case path) within
the stated tolerance: FP64 1e-12 relative (the per-cell sums may be grouped
differently when the batch and the lone case are tuned differently), mixed
1e-6 relative (FP32 arithmetic).
"""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx, serve
from nextgen_b200.meshgen import PeriodicBoxMesh

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def make_case(n, jit, kind, seed, Ma=0.1, Re=1600.0):
    m = PeriodicBoxMesh(n, jitter=jit, seed=seed)
    if kind == "tgv":
        prm = cases.tgv_params(Ma=Ma, Re=Re)
        rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    else:
        prm = cases.hit_params()
        rho, u, p = cases.hit_state(n, prm, k0=min(4.0, n / 4))
    prm.check_interval = 5
    return m, cgx.Mesh(m), prm, rho, u, p


def alone(gm, prm, rho, u, p, nsteps, prec):
    s = cgx.Solver(gm, prm, prec)
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    assert s.step(nsteps) == 0
    return s.get_state(), s.time()


@pytest.fixture(scope="module")
def three(built):
    return [make_case(8, 0.0, "tgv", 1, Ma=0.2), make_case(12, 0.25, "tgv", 2, Ma=0.4, Re=800.0),
            make_case(10, 0.25, "hit", 3)]


@pytest.mark.parametrize("prec,tol", [(cgx.CGX_FP64, 1e-12), (cgx.CGX_MIXED, 1e-6)])
def test_batch_matches_alone(three, prec, tol):
    steps = [5, 8, 3]
    b = cgx.Batch(0, prec, max_cases=8, hbm_budget=8 << 30)
    ids = [b.add(gm, prm, rho, u, p, n) for (m, gm, prm, rho, u, p), n in zip(three, steps)]
    assert None not in ids
    b.step(1)  # first step tunes the lane counts for this batch size
    n0 = b.launch_count()
    b.step(100)
    assert sorted(b.done()) == sorted(ids)
    # one graph replay (13 kernels) per step of the longest case, plus at most
    # one tuning (17 candidates x 4 timed launches) and the gradient's
    # re-derivation when the batch shrinks into a size bucket not tuned yet
    assert 7 * 13 <= b.launch_count() - n0 <= 7 * 13 + 17 * 4 + 1
    for cid, (m, gm, prm, rho, u, p), n in zip(ids, three, steps):
        got = b.get_state(cid)
        ref, (t_ref, dt_ref, st_ref) = alone(gm, prm, rho, u, p, n, prec)
        t, dt, st = b.time(cid)
        assert st == st_ref == n
        assert abs(t / t_ref - 1) <= tol
        for a, r in zip(got, ref):
            assert rel(a, r) <= tol
    for cid in ids:
        b.remove(cid)
    assert b.bytes()[0] == 0
    b.close()


def test_continuous_join_and_leave(three):
    """A case admitted while another is running, and one retired early."""
    (m0, g0, p0, r0, u0, q0), (m1, g1, p1, r1, u1, q1), _ = three
    b = cgx.Batch(0, cgx.CGX_FP64, max_cases=4, hbm_budget=8 << 30)
    a = b.add(g0, p0, r0, u0, q0, 10)
    b.step(4)
    c = b.add(g1, p1, r1, u1, q1, 6)  # joins mid-run
    b.step(100)
    assert sorted(b.done()) == sorted([a, c])
    ra, _ = alone(g0, p0, r0, u0, q0, 10, cgx.CGX_FP64)
    rc_, _ = alone(g1, p1, r1, u1, q1, 6, cgx.CGX_FP64)
    for x, y in zip(b.get_state(a), ra):
        assert rel(x, y) <= 1e-12
    for x, y in zip(b.get_state(c), rc_):
        assert rel(x, y) <= 1e-12
    b.close()


def test_admission_by_budget(three):
    m, gm, prm, rho, u, p = three[1]
    b = cgx.Batch(0, cgx.CGX_FP64, max_cases=4, hbm_budget=1 << 20)  # 1 MiB: too small
    assert b.add(gm, prm, rho, u, p, 5) is None
    assert b.bytes()[0] == 0
    b.close()
    b = cgx.Batch(0, cgx.CGX_FP64, max_cases=4, hbm_budget=64 << 20)
    first = b.add(gm, prm, rho, u, p, 5)
    assert first is not None
    used1 = b.bytes()[0]
    second = b.add(gm, prm, rho, u, p, 5)  # same mesh: counted once
    assert second is not None and b.bytes()[0] - used1 < used1
    b.step(10)
    b.remove(first)
    b.remove(second)
    assert b.bytes()[0] == 0
    b.close()


def test_served_stream_matches_sequential(built):
    """Poisson arrivals, uneven sizes and step counts, FP64 and mixed: every
    request completes and its result equals the same case run alone."""
    rng = np.random.default_rng(7)
    reqs = []
    arrivals = serve.poisson_arrivals(6, rate=200.0, seed=11)
    meshes = {}
    for k in range(6):
        n = int(rng.choice([8, 10, 12]))
        if n not in meshes:
            mm = PeriodicBoxMesh(n, jitter=0.25, seed=100 + n)
            meshes[n] = (mm, cgx.Mesh(mm))
        mm, gm = meshes[n]
        prm = cases.tgv_params(Ma=float(rng.uniform(0.1, 0.5)), Re=float(rng.uniform(400, 3200)))
        prm.check_interval = 5
        rho, u, p = cases.tgv_state(mm.x_cv[: mm.ncv], prm)
        prec = cgx.CGX_FP64 if k % 2 == 0 else cgx.CGX_MIXED
        reqs.append(serve.Request(k, gm, prm, rho, u, p, int(rng.integers(5, 25)), prec, float(arrivals[k])))
    out = serve.serve(reqs, hbm_budget=4 << 30, chunk=4)
    assert out["requests"] == 6 and out["p99_latency_s"] >= out["p50_latency_s"] > 0
    for r in reqs:
        assert r.finished >= r.admitted >= r.arrival
        ref, _ = alone(r.mesh, r.params, r.rho, r.u, r.p, r.nsteps, r.precision)
        tol = 1e-12 if r.precision == cgx.CGX_FP64 else 1e-6
        for a, b in zip(r.state, ref):
            assert rel(a, b) <= tol
