"""Source terms on the GPU, the counterpart of the subclass hook
addSourceHook(rhs, time, rk_stage) that calcRhs calls after the face sums
(IdealGasSolver.hpp:697-705, 713).

* cgx_set_source: a constant body force, and a relaxation force with a
  per-cell field, against the oracle's source (the force form of the
  reference's example hook, quiver/charles/charles.sphere.cpp:166-173):
  calcRhs per cell within 1e-12 of the face-sum scale, and the state after
  RK3 steps within 1e-10.
* cgx_set_source_hook: a host hook adding the same body force gives the
  device form's state within 1e-12, and sees the stage times t, t + dt,
  t + dt/2 and stages 1, 2, 3.
* cgx_set_frame_rotation: the rotating frame's centrifugal and Coriolis
  terms against the oracle (addRotationSourceTerms).
"""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import PeriodicBoxMesh
from oracle import Oracle

pytestmark = pytest.mark.gpu

G = (0.7, -0.4, 0.25)


@pytest.fixture(scope="module")
def setup(built):
    m = PeriodicBoxMesh(12, jitter=0.25, seed=77)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    return m, prm, (rho, u, p), cgx.Mesh(m, device=0)


def _pair(setup, **src):
    m, prm, (rho, u, p), gm = setup
    s = cgx.Solver(gm, prm)
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    if src:
        s.set_source(**src)
        o.set_source(**src)
    return s, o


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("kind", ["body_force", "relaxation_field"])
def test_source_matches_oracle(setup, kind):
    m = setup[0]
    if kind == "body_force":
        src = dict(g=G)
    else:
        rng = np.random.default_rng(5)
        src = dict(A=-2.0, g=(0.5, 0.0, -0.3), field=rng.normal(size=(m.ncv, 5)) * 1e-3 * np.array(m.vol_cv)[:, None])
    s, o = _pair(setup, **src)
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    err = (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max()
    assert err <= 1e-12, err
    # the source is really there: rhs without it differs by about the force
    s0, o0 = _pair(setup)
    ref0, _ = o0.calc_rhs(1)
    assert np.abs(ref - ref0).max() > 1e-3 * np.abs(ref).max()
    assert s.step(5) == 0 and o.step(5) == 0
    g, w = s.get_state(), o.get_state()
    for a, b in zip(g, w):
        assert _rel(a, b) <= 1e-10
    # momentum of a periodic box changes by the body force alone (face sums
    # cancel): d(sum rho u V)/dt = g sum rho V for the constant force
    if kind == "body_force":
        t0 = o0.totals()
        assert o0.step(5) == 0
        tg = s.totals()
        mass = t0[0]
        elapsed = s.time()[0]
        dmom = tg[1:4] - t0[1:4]
        expect = np.array(G) * mass * elapsed
        assert np.abs(dmom - expect).max() <= 1e-9 * np.abs(expect).max()
    for x in (s, s0):
        x.close()


def test_source_removed(setup):
    s, _ = _pair(setup, g=G)
    s.set_source()
    s0, o0 = _pair(setup)
    assert np.array_equal(s.calcRhs(1), s0.calcRhs(1))
    s.close()
    s0.close()


def test_host_hook_equals_device_form(setup):
    m, prm, (rho, u, p), gm = setup
    vol = np.array(m.vol_cv)
    calls = []

    def hook(r, uu, e, rhs, time, stage):
        f = (vol * r)[:, None] * np.array(G)[None, :]
        rhs[:, 1:4] += f
        rhs[:, 4] += (f * uu).sum(1)
        calls.append((time, stage))

    sh = cgx.Solver(gm, prm)
    sh.set_state_primitive(rho, u, p)
    sh.initComplete()
    sh.set_source_hook(hook)
    sd, o = _pair(setup, g=G)
    # calcRhs with the caller's time
    rh = sh.calcRhs(2, time=1.25)
    assert calls[-1] == (1.25, 2)
    rd = sd.calcRhs(2)
    ref, scale = o.calc_rhs(2)
    assert (np.abs(rh - rd) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    calls.clear()
    assert sh.step(2) == 0 and sd.step(2) == 0
    a, b = sh.get_state(), sd.get_state()
    for x, y in zip(a, b):
        assert _rel(x, y) <= 1e-12
    # stage times: t, t + dt, t + dt/2 per step
    assert [c[1] for c in calls] == [1, 2, 3, 1, 2, 3]
    t_end, dt_last, _ = sh.time()
    t1 = calls[3][0]
    assert calls[0][0] == 0.0 and abs(calls[2][0] - 0.5 * calls[1][0]) <= 1e-15
    assert abs(calls[4][0] - (t1 + dt_last)) <= 1e-14 and abs(t_end - (t1 + dt_last)) <= 1e-14
    sh.set_source_hook(None)
    assert sh.step(1) == 0 and len(calls) == 6
    sh.close()
    sd.close()


def test_rotating_frame_matches_oracle(setup):
    """ROTATING_REFERENCE_FRAME (addRotationSourceTerms, IdealGasSolver.cpp:
    695-733) with a body force beside it: calcRhs within 1e-12 of the
    face-sum scale, 10 RK3 steps within 1e-10 of the oracle; the mixed form
    within its tolerance of FP64; a zero rate removes the terms."""
    m, prm, (rho, u, p), gm = setup
    rev = (0.05, -0.02, 0.11)
    x = m.x_cv[: m.ncv]
    s, o = _pair(setup, g=G)
    s.set_frame_rotation(rev, x)
    o.set_frame_rotation(rev)
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert _rel(a, b) <= 1e-10
    s.close()
    o.close()
    res = {}
    for prec in (cgx.CGX_FP64, cgx.CGX_MIXED):
        s = cgx.Solver(gm, prm, prec)
        s.set_state_primitive(rho, u, p)
        s.initComplete()
        s.set_frame_rotation(rev, x)
        assert s.step(10) == 0
        res[prec] = s.get_state()
        s.close()
    for a64, a32 in zip(res[cgx.CGX_FP64], res[cgx.CGX_MIXED]):
        assert np.sqrt(((a32 - a64) ** 2).mean() / (a64 ** 2).mean()) <= 1e-5
    s = cgx.Solver(gm, prm)
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    r0 = s.calcRhs(1)
    s.set_frame_rotation(rev, x)
    s.set_frame_rotation((0.0, 0.0, 0.0), x)
    assert np.array_equal(s.calcRhs(1), r0)
    s.close()
