"""GPU path (libcgx.so through the C ABI) against the CPU oracle.

Per-cell criterion for face sums: |r_gpu - r_ref| / max(|r_ref|, sum_f |F_f|)
<= 1e-12, the denominator being the conditioning scale of a reordered sum.
Cell-wise quantities that are not sums compare relatively at 1e-12 (1e-11
where a transcendental from CUDA's libm enters).
"""
import os

import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import PeriodicBoxMesh
from oracle import Oracle
from oracle_weights import ERK3

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-12


def rel(a, ref, scale=None):
    den = np.abs(ref)
    if scale is not None:
        den = np.maximum(den, scale)
    den = np.maximum(den, 1e-300)
    return (np.abs(a - ref) / den).max()


def setup(n, jitter, kind="tgv", seed=1234, sfc=True, **kw):
    m = PeriodicBoxMesh(n, jitter=jitter, seed=seed)
    if kind == "tgv":
        prm = cases.tgv_params(**kw)
        rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    else:
        prm = cases.hit_params()
        rho, u, p = cases.hit_state(n, prm, k0=min(4.0, n / 4))
    gm = cgx.Mesh(m, device=0, sfc=sfc)
    s = cgx.Solver(gm, prm)
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    return m, prm, s, o


CASES = [
    (32, 0.0, "tgv"),    # the reference's CPU-runnable TGV configuration (32^3 lattice)
    (16, 0.25, "tgv"),
    (16, 0.25, "hit"),
    (12, 0.25, "tgv"),
]


@pytest.fixture(scope="module", params=CASES, ids=lambda c: "%s%d_j%g" % (c[2], c[0], c[1]))
def case(request, built):
    n, jit, kind = request.param
    return setup(n, jit, kind)


def test_calc_rhs(case):
    m, prm, s, o = case
    ref, scale = o.calc_rhs(1)
    got = s.calcRhs(1)
    assert rel(got, ref, scale) <= TOL


def test_primitive_grad_aux(case):
    m, prm, s, o = case
    p, T, sos = s.primitive()
    rp, rT, rs = o.primitive()
    assert rel(p, rp) <= TOL and rel(T, rT) <= TOL and rel(sos, rs) <= TOL
    g = s.grad().reshape(-1, 9)
    rg = o.grad().reshape(-1, 9)
    gs = np.abs(rg).max(axis=1, keepdims=True) + 1e-300
    assert (np.abs(g - rg) / gs).max() <= 1e-11
    a = s.aux()
    ra = o.aux()
    # mu_total, loc_total, a_sgs, fgr, symh, symp (log/exp/expm1 from CUDA's libm)
    for k in range(6):
        sc = np.abs(ra[:, k]).max() + 1e-300
        assert np.abs(a[:, k] - ra[:, k]).max() / sc <= 1e-11, k


def test_calc_cfl(case):
    m, prm, s, o = case
    mx, cfl = s.calcCfl(0.37, want_cells=True)
    rmx, rcfl = o.calc_cfl(0.37)
    assert rel(cfl, rcfl) <= TOL and abs(mx / rmx - 1) <= TOL


def test_rk3_stages(case):
    """calcRhs + rk3Step + updateConservativeAndPrimitiveData, stage by stage."""
    m, prm, s, o = case
    dt = 0.5 * prm.dt_data[0] / o.calc_cfl(1.0)[0]
    for st in range(3):
        s.calcRhs(st + 1, copy_out=False)
        o.calc_rhs(st + 1, want_scale=False)
        s.rk3Step(ERK3[st], dt, st + 1)
        o.rk3_step(ERK3[st], dt, st + 1)
        s.updateConservativeAndPrimitiveData()
        o.update_primitive()
    r1, u1, e1 = s.get_state()
    r2, u2, e2 = o.get_state()
    assert rel(r1, r2) <= 1e-13 and rel(e1, e2) <= 1e-13
    assert np.abs(u1 - u2).max() / np.abs(u2).max() <= 1e-12


def test_steps_match_oracle(built):
    m, prm, s, o = setup(12, 0.25, "tgv", seed=77)
    assert s.step(5) == 0
    assert o.step(5) == 0
    r1, u1, e1 = s.get_state()
    r2, u2, e2 = o.get_state()
    assert rel(r1, r2) <= 1e-12 and rel(e1, e2) <= 1e-12
    assert np.abs(u1 - u2).max() / np.abs(u2).max() <= 1e-11
    t1, dt1, st1 = s.time()
    t2, dt2, st2 = o.time()
    assert st1 == st2 == 5 and abs(t1 / t2 - 1) <= 1e-12 and abs(dt1 / dt2 - 1) <= 1e-12


def test_golden_fixtures(built):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden as mg
    for name in mg.CASES:
        g = np.load(os.path.join(HERE, "golden", name + ".npz"))
        m, prm, rho, u, p = mg.case_setup(name)
        assert mg.mesh_fingerprint(m) == str(g["fingerprint"])
        s = cgx.Solver(cgx.Mesh(m), prm)
        s.set_state_primitive(rho, u, p)
        s.initComplete()
        assert rel(s.calcRhs(1), g["rhs"], g["scale"]) <= TOL, name
        assert s.step(2) == 0
        r2, u2, e2 = s.get_state()
        assert rel(r2, g["rho2"]) <= 1e-12 and rel(e2, g["rhoE2"]) <= 1e-12, name


def test_tgv32_100_steps_conservation_and_oracle(built):
    """Config 0: TGV 32^3 lattice, CFL 0.8, 100 steps: conserved totals to
    round-off, and the GPU trajectory matches the oracle's."""
    m, prm, s, o = setup(32, 0.0, "tgv")
    t0 = s.totals()
    r0, u0, e0 = s.get_state()
    mom = (r0 * np.sqrt((u0 * u0).sum(1)) * m.vol_cv).sum()
    norm = np.array([np.abs(r0 * m.vol_cv).sum(), mom, mom, mom, np.abs(e0 * m.vol_cv).sum()])
    assert s.step(100) == 0
    assert o.step(100) == 0
    t1 = s.totals()
    assert (np.abs(t1 - t0) / norm).max() < 1e-13
    assert np.abs(t1 - o.totals()).max() / norm.max() < 1e-13
    r1, u1, e1 = s.get_state()
    r2, u2, e2 = o.get_state()
    assert rel(r1, r2) <= 1e-10 and rel(e1, e2) <= 1e-10
    assert np.abs(u1 - u2).max() / np.abs(u2).max() <= 1e-9


def test_deterministic(built):
    m = PeriodicBoxMesh(10, jitter=0.25, seed=8)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    outs = []
    for _ in range(2):
        s = cgx.Solver(cgx.Mesh(m), prm)
        s.set_state_primitive(rho, u, p)
        s.initComplete()
        s.step(3)
        outs.append(s.get_state())
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_sfc_renumbering_is_transparent(built):
    m = PeriodicBoxMesh(10, jitter=0.25, seed=9)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    out = []
    for sfc in (False, True):
        s = cgx.Solver(cgx.Mesh(m, sfc=sfc), prm)
        s.set_state_primitive(rho, u, p)
        s.initComplete()
        out.append(s.calcRhs(1))
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    ref, scale = o.calc_rhs(1)
    assert rel(out[0], ref, scale) <= TOL and rel(out[1], ref, scale) <= TOL


def test_nan_restores_state(built):
    """A NaN written into the state on the host: advanceSolution reports it,
    restores the stored state and scales the CFL target by 0.8."""
    m = PeriodicBoxMesh(8, jitter=0.25, seed=3)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    s = cgx.Solver(cgx.Mesh(m), prm)
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    s0 = s.get_state()
    bad = [a.copy() for a in s0]
    bad[0][5] = np.nan
    s.set_state(*bad)
    s.updateConservativeAndPrimitiveData()
    assert s.advanceSolution() == -1
    for a, b in zip(s.get_state(), s0):
        assert np.array_equal(a, b)
    t, dt, st = s.time()
    assert st == 0 and t == 0.0
    # the next step runs at 0.8 x the CFL target
    assert s.step(1) == 0
    ref = cgx.Solver(cgx.Mesh(m), prm)
    ref.set_state_primitive(rho, u, p)
    ref.initComplete()
    assert ref.step(1) == 0
    assert abs(s.time()[1] / ref.time()[1] - 0.8) <= 1e-12


def test_mesh_stats(built):
    m = PeriodicBoxMesh(12, jitter=0.25, seed=1)
    st = cgx.Mesh(m).stats()
    assert st.ncv == m.ncv
    assert abs(st.e_per_cell - m.e_per_cell) < 1e-12 and abs(st.f_per_cell - m.f_per_cell) < 1e-12
    assert st.n_ef_dir == 2 * m.nef_i + (m.nef - m.nef_i)
