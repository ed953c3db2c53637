"""The reference's inviscid-vortex harness (IdealGasEulerSolver,
src/charles/charles_ig.cpp:88-290) on the CPU oracle: an exact isentropic
vortex advected across a periodic box with no viscosity and no SGS model,
reported through the same volume-weighted L2/Linf norms as its temporalHook.

The reference ships no expected numbers for this case, so these pin what its
discretisation guarantees: the harness is exact at t = 0, the error falls with
resolution at the scheme's rate (about fourth order on a lattice, where the
Voronoi faces are exact planes midway between cells; at least first order on a
jittered mesh), and mass, momentum and energy totals are kept to round-off.
"""
import numpy as np
import pytest

from nextgen_b200 import cases
from nextgen_b200.meshgen import PeriodicBoxMesh
from oracle import Oracle

T_END = 2.0
HALF = 5.0  # the box is [-5, 5]^2 in x, y


def vortex_mesh(n, jitter, nz=6):
    """n x n x nz box of cubic cells, 10 wide in x and y."""
    return PeriodicBoxMesh(n, n, nz, L=(2 * HALF, 2 * HALF, 2 * HALF * nz / n), jitter=jitter, seed=1234)


def centred(m):
    return np.array(m.x_cv[: m.ncv]) - np.array([HALF, HALF, 0.0])


def run_oracle(n, jitter):
    m = vortex_mesh(n, jitter)
    x = centred(m)
    prm = cases.vortex_params()
    kw = dict(Lx=HALF, Ly=HALF)
    rho, u, p = cases.vortex_state(x, prm, **kw)
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    tot0 = o.totals()
    while o.time()[0] < T_END:
        assert o.step(1) == 0
    t = o.time()[0]
    r1, u1, e1 = o.get_state()
    l2, linf = cases.vortex_errors(x, m.vol_cv, r1, u1, e1, prm, t, **kw)
    return l2, linf, tot0, o.totals()


def test_harness_exact_at_start(built):
    m = vortex_mesh(16, 0.25)
    x = centred(m)
    prm = cases.vortex_params()
    rho, u, p = cases.vortex_state(x, prm, Lx=HALF, Ly=HALF)
    rhoE = p / (prm.gamma - 1.0) + 0.5 * rho * (u * u).sum(1)
    l2, linf = cases.vortex_errors(x, m.vol_cv, rho, u, rhoE, prm, 0.0, Lx=HALF, Ly=HALF)
    assert l2.max() == 0.0 and linf.max() == 0.0
    # the exact solution is periodic: along x at u_inf = 0.5 it returns after
    # one box length, 10 / 0.5 = 20 time units
    a = cases.vortex_state(x, prm, t=0.0, Lx=HALF, Ly=HALF, theta=0.0)
    b = cases.vortex_state(x, prm, t=20.0, Lx=HALF, Ly=HALF, theta=0.0)
    for fa, fb in zip(a, b):
        assert np.abs(fa - fb).max() < 1e-12


def test_lattice_convergence(built):
    errs = [run_oracle(n, 0.0)[0][0] for n in (16, 24, 32)]
    orders = [np.log(errs[i] / errs[i + 1]) / np.log(r) for i, r in enumerate((24 / 16, 32 / 24))]
    assert min(orders) > 3.0, (errs, orders)


def test_jittered_convergence_and_conservation(built):
    res = {n: run_oracle(n, 0.25) for n in (16, 32)}
    e16, e32 = res[16][0][0], res[32][0][0]
    assert e32 < 0.4 * e16, (e16, e32)
    for n, (l2, linf, t0, t1) in res.items():
        assert np.all(np.isfinite(l2)) and linf[0] < 0.05
        # mass, x/y-momentum and energy: periodic box, no sources
        for k in (0, 1, 2, 4):
            assert abs(t1[k] - t0[k]) <= 1e-12 * max(abs(t0[k]), 1.0), (n, k, t0, t1)
