"""LIMIT_ASGS in the oracle (limitAsgs, IdealGasSolverSgs.cpp:4-48).

With the flag set and the solver's dt > 0, computeSgsVreman's a_sgs (already
divided by sos^2) is capped at 1/(4 dt fax) / sos^2, fax = 1/(gamma-1) +
|u|^2/(2 sos^2).  The reference's dt is 0 at initComplete on a fresh start,
so the first properties are not capped; after a step they are, with that
step's dt.  The cap is recomputed here from the oracle's primitive state and
dt.
"""
import numpy as np

from nextgen_b200 import cases
from nextgen_b200.meshgen import PeriodicBoxMesh
from oracle import Oracle


def _run(m, prm, state, limit, steps):
    p2 = prm.copy()
    p2.limit_asgs = limit
    o = Oracle(m, p2)
    o.set_state_primitive(*state)
    o.init_complete()
    a0 = o.aux()[:, 2].copy()
    if steps:
        assert o.step(steps) == 0
    return o, a0


def _cap(o, prm):
    _, u, _ = o.get_state()
    _, _, sos = o.primitive()
    dt = o.time()[1]
    inv_sos2 = 1.0 / (sos * sos)
    fax = 1.0 / (prm.gamma - 1.0) + 0.5 * (u * u).sum(1) * inv_sos2
    return 1.0 / (dt * fax * 4.0) * inv_sos2, dt


def test_limit_asgs_caps_after_a_step_only(built):
    n = 10
    m = PeriodicBoxMesh(n, jitter=0.25, seed=99)
    prm = cases.hit_params(Mt=0.3)
    prm.a_sgs_coeff = 3.0  # large enough that part of the mesh reaches the ceiling
    state = cases.hit_state(n, prm, Mt=0.3, k0=2.0)
    on, a0_on = _run(m, prm, state, 1, 0)
    off, a0_off = _run(m, prm, state, 0, 0)
    # initComplete on a fresh start: dt is 0, nothing is capped
    assert on.time()[1] == 0.0
    assert np.array_equal(a0_on, a0_off)
    on.close()
    off.close()

    on, _ = _run(m, prm, state, 1, 2)
    off, _ = _run(m, prm, state, 0, 2)
    cap, dt = _cap(on, prm)
    assert dt > 0.0
    a_on = on.aux()[:, 2]
    assert np.all(a_on <= cap * (1 + 1e-14))
    hit = np.isclose(a_on, cap, rtol=1e-14, atol=0.0)
    assert 0 < hit.sum() < m.ncv, hit.sum()
    # the unlimited run crosses its own ceiling somewhere; the two runs differ
    cap_off, _ = _cap(off, prm)
    assert np.any(off.aux()[:, 2] > cap_off * (1 + 1e-12))
    assert not np.array_equal(on.get_state()[1], off.get_state()[1])
    on.close()
    off.close()
