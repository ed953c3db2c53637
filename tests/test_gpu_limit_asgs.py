"""LIMIT_ASGS on the GPU against the oracle (limitAsgs,
IdealGasSolverSgs.cpp:4-48).

A jittered 10^3 HIT state with A_SGS_COEFF 3, so that part of the mesh
reaches the a_sgs ceiling once dt > 0:

* initComplete (dt 0 on a fresh start: nothing capped), then 3 steps: the
  state within 1e-12 and a_sgs within 1e-11 of the oracle, with the ceiling
  active in some cells and not in others;
* a NaN in the state: advanceSolution restores the stored state and
  recomputes the properties with the failed step's dt, as restoreData does
  (IdealGasSolver.hpp:377-405): a_sgs within 1e-11 of the oracle's;
* the mixed-precision form respects the ceiling to FP32 rounding.
"""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import PeriodicBoxMesh
from oracle import Oracle

pytestmark = pytest.mark.gpu

N = 10


@pytest.fixture(scope="module")
def setup(built):
    m = PeriodicBoxMesh(N, jitter=0.25, seed=99)
    prm = cases.hit_params(Mt=0.3)
    prm.a_sgs_coeff = 3.0
    prm.limit_asgs = 1
    state = cases.hit_state(N, prm, Mt=0.3, k0=2.0)
    return m, prm, state, cgx.Mesh(m, device=0)


def _pair(setup, prec=cgx.CGX_FP64):
    m, prm, state, gm = setup
    s = cgx.Solver(gm, prm, prec)
    s.set_state_primitive(*state)
    s.initComplete()
    o = Oracle(m, prm)
    o.set_state_primitive(*state)
    o.init_complete()
    return s, o


def _asgs_close(s, o):
    a, ra = s.aux()[:, 2], o.aux()[:, 2]
    return np.abs(a - ra).max() / (np.abs(ra).max() + 1e-300)


def _cap(u, sos, dt, gamma):
    inv = 1.0 / (sos * sos)
    fax = 1.0 / (gamma - 1.0) + 0.5 * (u * u).sum(1) * inv
    return 1.0 / (dt * fax * 4.0) * inv


def test_limit_asgs_steps(setup):
    m, prm, state, gm = setup
    s, o = _pair(setup)
    assert _asgs_close(s, o) <= 1e-11
    assert s.step(3) == 0 and o.step(3) == 0
    r1, u1, e1 = s.get_state()
    r2, u2, e2 = o.get_state()
    assert np.abs(r1 - r2).max() / np.abs(r2).max() <= 1e-12
    assert np.abs(e1 - e2).max() / np.abs(e2).max() <= 1e-12
    assert np.abs(u1 - u2).max() / np.abs(u2).max() <= 1e-11
    assert _asgs_close(s, o) <= 1e-11
    # the ceiling is active in part of the mesh
    _, _, sos = o.primitive()
    cap = _cap(u2, sos, o.time()[1], prm.gamma)
    hit = np.isclose(o.aux()[:, 2], cap, rtol=1e-14, atol=0.0)
    assert 0 < hit.sum() < m.ncv
    s.close()
    o.close()


def test_limit_asgs_after_restore(setup):
    m, prm, state, gm = setup
    s, o = _pair(setup)
    assert s.step(2) == 0 and o.step(2) == 0
    # the GPU's advanceSolution takes the dt set at the end of the last step;
    # the oracle's takes the one set_dt computes from the same state
    o.set_dt()
    bad = [a.copy() for a in s.get_state()]
    bad[0][5] = np.nan
    s.set_state(*bad)
    s.updateConservativeAndPrimitiveData()
    o.poison(5)
    assert s.advanceSolution() == -1
    assert o.advance_solution() == -1
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max()
    # restoreData recomputed the properties with the failed step's dt > 0
    assert _asgs_close(s, o) <= 1e-11
    _, u, _ = o.get_state()
    _, _, sos = o.primitive()
    cap = _cap(u, sos, o.time()[1], prm.gamma)
    assert np.isclose(o.aux()[:, 2], cap, rtol=1e-14, atol=0.0).any()
    s.close()
    o.close()


def test_limit_asgs_mixed(setup):
    m, prm, state, gm = setup
    s = cgx.Solver(gm, prm, cgx.CGX_MIXED)
    s.set_state_primitive(*state)
    s.initComplete()
    assert s.step(3) == 0
    _, u, _ = s.get_state()
    _, _, sos = s.primitive()
    cap = _cap(u, sos, s.time()[1], prm.gamma)
    a = s.aux()[:, 2]
    assert np.all(a <= cap * (1 + 1e-5))
    assert np.isclose(a, cap, rtol=1e-5, atol=0.0).any()
    s.close()
