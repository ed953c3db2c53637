"""Restart through the C ABI: a solver set to a saved state, time and step
(cgx_set_state + cgx_init_complete + cgx_set_time, as a host solver does
after reading a restart file) continues the uninterrupted run.

The NaN checks and the restore point follow the global step count
(IdealGasSolver.hpp:807-811), so with check_interval 7 a run restarted at
step 30 checks at 35, 42, ... exactly as the uninterrupted one.
"""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import PeriodicBoxMesh

pytestmark = pytest.mark.gpu


def test_restart_continues_the_run(built):
    m = PeriodicBoxMesh(16, jitter=0.25, seed=8)
    prm = cases.tgv_params(Ma=0.2)
    prm.check_interval = 7
    rho, u, p = cases.tgv_state(np.array(m.x_cv[: m.ncv]), prm)
    gm = cgx.Mesh(m, device=0)
    a = cgx.Solver(gm, prm)
    a.set_state_primitive(rho, u, p)
    a.initComplete()
    assert a.step(30) == 0
    saved = a.get_state()
    t30, dt30, st30 = a.time()
    assert st30 == 30 and t30 > 0.0
    assert a.step(25) == 0
    ra, ua, ea = a.get_state()
    ta, _, sta = a.time()

    b = cgx.Solver(gm, prm)
    b.set_state(*saved)
    b.initComplete()
    b.set_time(t30, 30)
    assert b.time()[0] == t30 and b.time()[2] == 30
    assert b.step(25) == 0
    rb, ub, eb = b.get_state()
    tb, _, stb = b.time()
    assert stb == sta == 55
    assert abs(tb - ta) <= 1e-13 * ta
    for x, y in ((ra, rb), (ua, ub), (ea, eb)):
        assert np.abs(x - y).max() <= 1e-12 * np.abs(x).max()
    a.close()
    b.close()


def test_set_time_checks_arguments(built):
    m = PeriodicBoxMesh(8, jitter=0.2)
    s = cgx.Solver(cgx.Mesh(m, device=0), cases.tgv_params())
    with pytest.raises(cgx.CgxError):
        s.set_time(0.0, -1)
    with pytest.raises(cgx.CgxError):
        s.set_time(float("nan"), 3)
    s.set_time(1.5, 12)  # before init: accepted, kept
    rho, u, p = cases.tgv_state(np.array(m.x_cv[: m.ncv]), cases.tgv_params())
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    t, dt, st = s.time()
    assert (t, st) == (1.5, 12)
    assert s.step(3) == 0 and s.time()[2] == 15
    s.close()
