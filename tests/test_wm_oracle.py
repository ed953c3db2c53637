"""The wall-model zones in the oracle, on CPU: the algebraic WM_ALG_ADIABATIC,
WM_ALG_ISOTHERMAL and WM_ALG_CONDUCTIVE and the equilibrium WM_EQ_ADIABATIC
and WM_EQ_ISOTHERMAL (WmAdiabatic, WmIsothermal, WmAlgConductive,
IdealGasSolverBcs.cpp:996-1478, 2054-2262, 2411-2595; AlgebraicWM.hpp,
EquilibriumWM.hpp).

* The restated law-of-the-wall solve recovers u_tau = 0.123 to 1e-7 at the
  y+ values of the reference's own known-answer test
  (src/charles/tests/wm_test.cpp:49-87), and 0 at a separation point.
* The restated tau_wall, wall heat flux and near-wall resistance equal the
  reference header's own
  (AlgebraicWM.hpp compiled where it lies) bit for bit over random inputs,
  and so do whole solver runs with wall-model zones.
* The restated equilibrium solve equals EquilibriumWM::solve_qt bit for bit
  (status included), and gives the laminar stress in the viscous sublayer.
* WM_ALG_CONDUCTIVE starts without a heat flux, and behind layers lets in
  less heat than without them.
* After initComplete the wall stress is the laminar estimate mu |u| / y1, so
  for a flow along the walls WM_ALG_ADIABATIC gives WALL_ADIABATIC's rhs (a
  moving wall included), and WM_ALG_ISOTHERMAL gives WALL_ISOTHERMAL's
  momentum rhs with the energy term mu aod (cp (T - T_w) + |u|^2/2) in place
  of the conduction term.
"""
import numpy as np
import pytest

import oracle as orc_mod
from nextgen_b200 import cases
from nextgen_b200.meshgen import ChannelMesh
from oracle import Oracle

WALL, ISO, WM_AD, WM_ISO, WM_COND, WM_EQ_AD, WM_EQ_ISO = 2, 3, 15, 16, 17, 19, 20
need_ref = pytest.mark.skipif(not orc_mod.ref_available(), reason="reference-built oracle absent")

KAPPA, B, YSTAR = 0.41, 5.2, 23.3244
A1 = 0.5 * (1.0 / (KAPPA * YSTAR) - 1.0) / YSTAR


def _uplus(yp):
    return yp + A1 * yp * yp if yp <= YSTAR else np.log(yp) / KAPPA + B


def test_known_answers(built):
    u_tau, nu, rho = 0.123, 1.0e-05, 1.2333
    for yp in (2.0, 15.0, 20.0, 23.32, 40.0, 100.0, 1000.0, 10000.0):
        y1 = nu * yp / u_tau
        u1 = u_tau * _uplus(yp)
        tau = orc_mod.wm_solve_tau(u1, y1, rho, rho * nu)
        assert abs(np.sqrt(tau / rho) - u_tau) < 1e-7
        # from a guess as the solver gives it (the last step's u_tau)
        tau = orc_mod.wm_solve_tau(u1, y1, rho, rho * nu, 0.5 * u_tau)
        assert abs(np.sqrt(tau / rho) - u_tau) < 1e-7
    assert orc_mod.wm_solve_tau(0.0, 0.005, rho, rho * nu) == 0.0  # separation point


@need_ref
def test_restated_wall_model_bitwise_equals_reference(built):
    rng = np.random.default_rng(5)
    for _ in range(400):
        u1 = float(10.0 ** rng.uniform(-3, 1))
        y1 = float(10.0 ** rng.uniform(-4, -1))
        rho = float(rng.uniform(0.5, 2.0))
        mu = float(10.0 ** rng.uniform(-6, -3))
        g = float(rng.choice([-1.0, 0.0, 10.0 ** rng.uniform(-3, 0)]))
        a = orc_mod.wm_solve_tau(u1, y1, rho, mu, g)
        assert a == orc_mod.wm_solve_tau(u1, y1, rho, mu, g, reference=True)
        args = (float(rng.uniform(0.8, 1.5)), float(rng.uniform(0.8, 1.5)), a, rho, mu, mu / 0.7, 3.5, y1)
        assert orc_mod.wm_q_wall(*args) == orc_mod.wm_q_wall(*args, reference=True)
        args = (a, rho, mu, mu / 0.7, 3.5, y1)
        assert orc_mod.wm_r_approx(*args) == orc_mod.wm_r_approx(*args, reference=True)


@need_ref
def test_restated_equilibrium_model_bitwise_equals_reference(built):
    """EquilibriumWM::solve_qt restated: the same tau_w, q_w, wall
    temperature as the reference header's own, isothermal and adiabatic,
    from guesses as the zones pass them (over the inputs where the solve
    converges: on a diverging one the header's own assert stops the
    process)."""
    rng = np.random.default_rng(9)
    cp, Pr = 3.5, 0.7
    converged = 0
    for k in range(120):
        u1 = float(10.0 ** rng.uniform(-2, 0.5))
        y1 = float(10.0 ** rng.uniform(-4, -1))
        rho = float(rng.uniform(0.7, 1.5))
        mu = float(10.0 ** rng.uniform(-6, -3.5))
        T1 = float(rng.uniform(0.8, 1.3))
        tau0 = mu * u1 / y1 * float(rng.uniform(0.3, 3.0))
        Tw = float(rng.uniform(0.7, 1.6)) if k % 2 else -(T1 + 0.5 * u1 * u1 / cp)
        q0 = 0.0 if Tw < 0 else mu * cp * (T1 - Tw) / y1
        a = orc_mod.wm_eq_solve(tau0, q0, Tw, u1, T1, rho, y1, mu, Pr, cp)
        if a[0] != 0 or not np.isfinite(a[1:]).all():
            # diverged (a NaN march): the reference header asserts on it
            continue
        converged += 1
        assert a == orc_mod.wm_eq_solve(tau0, q0, Tw, u1, T1, rho, y1, mu, Pr, cp, reference=True)
        assert a[1] > 0.0
    assert converged >= 90


def test_equilibrium_model_laminar_limit(built):
    """Deep in the viscous sublayer (y+ about 0.45, little eddy viscosity left by
    the damping) the adiabatic equilibrium model gives the laminar stress
    mu u1 / y1 to within the model's own tolerance."""
    cp, Pr, rho, mu, T1, u1 = 3.5, 0.7, 1.0, 1e-3, 1.0, 0.01
    y1 = 0.02  # y+ = y1 sqrt(rho mu u1 / y1) / mu, about 0.45
    rc, tau, q, Tw = orc_mod.wm_eq_solve(mu * u1 / y1, 0.0, -(T1 + 0.5 * u1 * u1 / cp), u1, T1, rho, y1, mu, Pr, cp)
    assert rc == 0 and q == 0.0 and Tw < 0.0
    assert abs(tau / (mu * u1 / y1) - 1.0) < 1e-3


@pytest.fixture(scope="module")
def chan(built):
    return ChannelMesh(12, 8, 6, L=(3.0, 2.0, 1.5), jitter=0.25, seed=7)


def _along(m, prm, T=1.0):
    """A uniform flow along the walls at temperature T (p = p_ref)."""
    rho = np.full(m.ncv, prm.p_ref / (T * prm.p_ref / prm.rho_ref / prm.T_ref))
    u = np.tile([0.2, 0.0, 0.05], (m.ncv, 1))
    p = np.full(m.ncv, prm.p_ref)
    return rho, u, p


def _rhs(m, prm, zones, state):
    o = Oracle(m, prm)
    for z, (k, a) in enumerate(zones):
        o.set_bc_params(z, k, a)
    o.set_state_primitive(*state)
    o.init_complete()
    r, sc = o.calc_rhs(1)
    mu = o.aux()[:, 0]  # uniform flow: no SGS viscosity, mu_total = mu_lam
    o.close()
    return r, sc, mu


def test_initial_wall_model_is_the_laminar_wall(chan):
    m = chan
    prm = cases.tgv_params(Re=400.0)
    st = _along(m, prm)
    a, sa, _ = _rhs(m, prm, ((WM_AD, [0.05, 0.0, -0.1]), (WM_AD, [])), st)
    b, _, _ = _rhs(m, prm, ((WALL, [0.05, 0.0, -0.1]), (WALL, [])), st)
    assert (np.abs(a - b) / np.maximum(np.abs(b), sa)).max() <= 1e-12


def test_initial_isothermal_wall_model(chan):
    m = chan
    prm = cases.tgv_params(Re=400.0)
    gamma, R = prm.gamma, prm.p_ref / prm.rho_ref / prm.T_ref
    cp = R * gamma / (gamma - 1.0)
    st = _along(m, prm, T=1.1)
    Tw = (1.3, 0.9)
    a, sa, mu = _rhs(m, prm, ((WM_ISO, [Tw[0]]), (WM_ISO, [Tw[1]])), st)
    b, _, _ = _rhs(m, prm, ((ISO, [Tw[0]]), (ISO, [Tw[1]])), st)
    assert (np.abs(a[:, :4] - b[:, :4]) / np.maximum(np.abs(b[:, :4]), sa[:, :4])).max() <= 1e-12
    # energy: the model's mu aod (cp (T - T_w) + |u|^2/2) for the conduction term
    want = b[:, 4].copy()
    T = st[2] / (st[0] * R)
    usq = (st[1] ** 2).sum(1)
    for f in range(m.nbf):
        i, z = m.cvobf[f], m.zone_bf[f]
        aod = m.area_over_delta_bf[f]
        want[i] += mu[i] / prm.Pr_lam * aod * cp * (T[i] - Tw[z])
        want[i] -= mu[i] * aod * (cp * (T[i] - Tw[z]) + 0.5 * usq[i])
    assert (np.abs(a[:, 4] - want) / np.maximum(np.abs(want), sa[:, 4])).max() <= 1e-12


def test_conductive_wall_model(chan):
    """WM_ALG_CONDUCTIVE: no heat flux before the first step (its initial
    hook), so for a flow along the walls its first rhs is WALL_ADIABATIC's;
    over a step with hot walls the heat that enters is less behind layers
    than without them (series resistance), and positive."""
    m = chan
    prm = cases.tgv_params(Re=400.0)
    st = _along(m, prm)
    a, sa, _ = _rhs(m, prm, ((WM_COND, [1.3, 0.01, 0.5]), (WM_COND, [1.2])), st)
    b, _, _ = _rhs(m, prm, ((WALL, []), (WALL, [])), st)
    assert (np.abs(a - b) / np.maximum(np.abs(b), sa)).max() <= 1e-12
    E = []
    for zones in (((WM_COND, [1.3, 0.05, 0.2]), (WM_COND, [1.3, 0.05, 0.2])), ((WM_COND, [1.3]), (WM_COND, [1.3]))):
        o = Oracle(m, prm)
        for z, (k, p) in enumerate(zones):
            o.set_bc_params(z, k, p)
        o.set_state_primitive(*st)
        o.init_complete()
        E0 = o.totals()[4]
        assert o.step(2) == 0
        E.append(o.totals()[4] - E0)
        o.close()
    assert 0.0 < E[0] < E[1]


def test_wall_model_refusals(chan):
    o = Oracle(chan, cases.tgv_params())
    for kind, bad in ((WM_AD, [0.1]), (WM_AD, [0.1, 0.2]), (WM_ISO, []), (WM_ISO, [1.0, 2.0]), (WM_COND, []),
                      (WM_COND, [1.0, 0.1]), (WM_EQ_AD, [0.1]), (WM_EQ_AD, [0.0] * 4), (WM_EQ_ISO, []),
                      (WM_EQ_ISO, [1.0, 0.7])):
        with pytest.raises(ValueError):
            o.set_bc_params(0, kind, bad)
    o.close()


@need_ref
def test_wall_model_solver_bitwise_equals_reference(chan):
    m = chan
    prm = cases.tgv_params(Re=400.0)
    x, y, z = m.x_cv[: m.ncv].T
    u = np.stack([0.3 + 0.1 * np.cos(2 * np.pi * z / m.L[2]), 0.02 * np.sin(2 * np.pi * x / m.L[0]),
                  0.05 * np.sin(np.pi * y / m.L[1])], 1)
    rho = 1.0 + 0.02 * np.cos(2 * np.pi * x / m.L[0])
    p = np.full(m.ncv, prm.p_ref)
    out = []
    for reference in (False, True):
        o = Oracle(m, prm, reference=reference)
        o.set_bc_params(0, WM_AD, [0.0, 0.0, 0.05])
        o.set_bc_params(1, WM_ISO, [1.2])
        o.set_state_primitive(rho, u, p)
        o.init_complete()
        assert o.step(4) == 0
        out.append(np.concatenate([v.reshape(m.ncv, -1) for v in o.get_state()], 1))
        o.close()
        o = Oracle(m, prm, reference=reference)
        o.set_bc_params(0, WM_EQ_AD, [0.0, 0.0, 0.05])
        o.set_bc_params(1, WM_EQ_ISO, [1.2, 0.7, 1.0, 1e-5])
        o.set_state_primitive(rho, u, p)
        o.init_complete()
        assert o.step(3) == 0
        out.append(np.concatenate([v.reshape(m.ncv, -1) for v in o.get_state()], 1))
        o.close()
        o = Oracle(m, prm, reference=reference)
        o.set_bc_params(0, WM_COND, [1.3, 0.01, 0.5])
        o.set_bc_params(1, WM_ISO, [0.9])
        o.set_state_primitive(rho, u, p)
        o.init_complete()
        assert o.step(4) == 0
        out.append(np.concatenate([v.reshape(m.ncv, -1) for v in o.get_state()], 1))
        out.append(o.calc_rhs(1)[0])
        o.close()
    assert np.array_equal(out[0], out[4])
    assert np.array_equal(out[1], out[5])
    assert np.array_equal(out[2], out[6])
    assert np.array_equal(out[3], out[7])


WM_EX_AD, WM_EX_ISO = 22, 23


def test_exchange_wall_model_at_its_own_cell(chan):
    """WM_EXCHANGE_ADIABATIC with each exchange point at its face's own cell
    centroid and a distance ratio of 1, or with no point located, is the
    algebraic WM_ALG_ADIABATIC wall, bit for bit (WmExchange,
    IdealGasSolverBcs.cpp:500-990); an exchange zone refuses points for the
    wrong face count."""
    m = chan
    prm = cases.tgv_params(Re=400.0)
    x, y, z = m.x_cv[: m.ncv].T
    u = np.stack([0.3 + 0.1 * np.cos(2 * np.pi * z / m.L[2]), 0.02 * np.sin(2 * np.pi * x / m.L[0]),
                  0.05 * np.sin(np.pi * y / m.L[1])], 1)
    rho, p = 1.0 + 0.02 * np.cos(2 * np.pi * x / m.L[0]), np.full(m.ncv, prm.p_ref)
    cells = {zz: m.cvobf[m.zone_bf == zz] for zz in (0, 1)}

    def run(form):
        o = Oracle(m, prm)
        for zz in (0, 1):
            if form == "alg":
                o.set_bc_params(zz, WM_AD, [])
            else:
                o.set_bc_params(zz, WM_EX_AD, [1.0] if form == "own" else [])
                cv = cells[zz] if form == "own" else -np.ones(cells[zz].size, dtype=np.int32)
                o.set_bc_exchange(zz, cv, m.x_cv[cells[zz]])
        o.set_state_primitive(rho, u, p)
        o.init_complete()
        r = o.calc_rhs(1)[0]
        assert o.step(3) == 0
        st = np.concatenate([v.reshape(m.ncv, -1) for v in o.get_state()], 1)
        o.close()
        return r, st

    a = run("alg")
    for form in ("own", "unlocated"):
        b = run(form)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    o = Oracle(m, prm)
    o.set_bc_params(0, WM_EX_ISO, [1.2, 2.5])
    with pytest.raises(ValueError):
        o.set_bc_exchange(0, cells[0][:-1], m.x_cv[cells[0][:-1]])
    with pytest.raises(ValueError):
        o.set_bc_params(1, WM_EX_ISO, [])
    o.close()


@need_ref
def test_exchange_wall_model_bitwise_equals_reference(chan):
    m = chan
    prm = cases.tgv_params(Re=400.0)
    x, y, z = m.x_cv[: m.ncv].T
    u = np.stack([0.3 + 0.1 * np.cos(2 * np.pi * z / m.L[2]), 0.02 * np.sin(2 * np.pi * x / m.L[0]),
                  0.05 * np.sin(np.pi * y / m.L[1])], 1)
    rho, p = 1.0 + 0.02 * np.cos(2 * np.pi * x / m.L[0]), np.full(m.ncv, prm.p_ref)
    out = []
    for reference in (False, True):
        o = Oracle(m, prm, reference=reference)
        o.set_bc_params(0, WM_EX_AD, [])
        o.set_bc_params(1, WM_EX_ISO, [1.2])
        for zz in (0, 1):
            c = m.cvobf[m.zone_bf == zz]
            nb = m.n_bf[m.zone_bf == zz]
            xe = m.x_cv[c] - 0.3 * nb / np.linalg.norm(nb, axis=1)[:, None]
            o.set_bc_exchange(zz, c, xe)
        o.set_state_primitive(rho, u, p)
        o.init_complete()
        assert o.step(3) == 0
        out.append(np.concatenate([v.reshape(m.ncv, -1) for v in o.get_state()], 1))
        o.close()
    assert np.array_equal(out[0], out[1])
