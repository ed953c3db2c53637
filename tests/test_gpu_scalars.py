"""Passive transport scalars on the GPU (cgx_set_scalars: calcRhsScalars,
IdealGasSolver.cpp:537-693; advanceScalars, IdealGasSolver.cpp:874-892)
against the CPU oracle, through the C ABI.

rhs_sc is a face sum: per cell and scalar |r_gpu - r_ref| / max(|r_ref|,
sum_f |F_f|) <= 1e-12, as for the flow rhs.  States after RK3 steps compare
relatively at 1e-10, the tolerance the flow-state tests use.
"""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import PeriodicBoxMesh
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _scalars(x):
    return np.stack([np.ones(len(x)),
                     1.0 + 0.5 * np.sin(x[:, 0]) * np.cos(x[:, 1]),
                     np.cos(x[:, 2]) ** 2], axis=1)


@pytest.fixture(scope="module")
def pair(built):
    m = PeriodicBoxMesh(12, jitter=0.25, seed=1234)
    prm = cases.tgv_params()
    x = np.array(m.x_cv[: m.ncv])
    rho, u, p = cases.tgv_state(x, prm)
    sc = _scalars(x)
    gm = cgx.Mesh(m, device=0)
    s = cgx.Solver(gm, prm)
    s.set_state_primitive(rho, u, p)
    s.set_scalars(sc)
    s.initComplete()
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.set_scalars(sc)
    o.init_complete()
    return m, prm, (rho, u, p, sc), gm, s, o


def test_rhs_sc_matches_oracle(pair):
    m, prm, _, _, s, o = pair
    rhs = s.calcRhs(2)
    ref, scale = o.calc_rhs(2)
    assert (np.abs(rhs - ref) / np.maximum(np.abs(ref), scale)).max() <= TOL
    r = s.rhs_sc(2)
    rref, sscale = o.rhs_sc(2)
    err = np.abs(r - rref) / np.maximum(np.maximum(np.abs(rref), sscale), 1e-300)
    assert err.max() <= TOL, err.max()


def test_scalars_do_not_change_the_flow(pair):
    m, prm, (rho, u, p, sc), gm, s, _ = pair
    plain = cgx.Solver(gm, prm)
    plain.set_state_primitive(rho, u, p)
    plain.initComplete()
    a = plain.calcRhs(1)
    s.set_state_primitive(rho, u, p)
    s.set_scalars(sc)
    s.initComplete()
    b = s.calcRhs(1)
    assert np.array_equal(a, b)
    plain.close()


def test_steps_match_oracle(pair):
    m, prm, (rho, u, p, sc), gm, _, _ = pair
    s = cgx.Solver(gm, prm)
    s.set_state_primitive(rho, u, p)
    s.set_scalars(sc)
    s.initComplete()
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.set_scalars(sc)
    o.init_complete()
    n0 = s.launch_count()
    assert s.step(20) == 0 and o.step(20) == 0
    assert s.launch_count() - n0 >= 20 * 16  # 13 flow kernels + 3 scalar rhs per step
    g, r = s.get_scalars(), o.get_scalars()
    assert (np.abs(g - r) / np.abs(r)).max() <= 1e-10
    r1, u1, e1 = s.get_state()
    r2, u2, e2 = o.get_state()
    assert (np.abs(r1 - r2) / np.abs(r2)).max() <= 1e-10
    # the unit scalar follows continuity; sum(rho sc V) is conserved
    assert np.abs(g[:, 0] - 1.0).max() < 1e-13
    vol = np.array(m.vol_cv)
    t0 = (rho[:, None] * sc * vol[:, None]).sum(0)
    t1 = (r1[:, None] * g * vol[:, None]).sum(0)
    assert (np.abs(t1 - t0) / np.abs(t0)).max() < 1e-13
    s.close()


def test_scalar_arguments_checked(pair):
    m, prm, (rho, u, p, sc), gm, _, _ = pair
    s = cgx.Solver(gm, prm)
    with pytest.raises(cgx.CgxError):
        s.set_scalars(np.ones((m.ncv, 9)))  # more than 8 scalars
    with pytest.raises(cgx.CgxError):
        s.get_scalars()  # none set
    s.set_state_primitive(rho, u, p)
    s.set_scalars(sc)
    s.set_scalars(np.zeros((m.ncv, 0)))  # removed again
    s.initComplete()
    assert s.step(2) == 0
    s.close()


def test_mixed_precision_scalars(pair):
    """The mixed form advances scalars from its FP32 mass fluxes: rhs_sc
    within the mixed form's flux tolerance of the FP64 oracle, the unit scalar
    still follows continuity and sum(rho sc V) is still conserved (scalar
    sums and updates are FP64)."""
    m, prm, (rho, u, p, sc), gm, _, o = pair
    s = cgx.Solver(gm, prm, cgx.CGX_MIXED)
    s.set_state_primitive(rho, u, p)
    s.set_scalars(sc)
    s.initComplete()
    s.calcRhs(1)
    o.set_state_primitive(rho, u, p)
    o.set_scalars(sc)
    o.init_complete()
    o.calc_rhs(1)
    r = s.rhs_sc(1)
    rref, sscale = o.rhs_sc(1)
    err = np.abs(r - rref) / np.maximum(np.maximum(np.abs(rref), sscale), 1e-300)
    assert err.max() < 2e-5, err.max()  # FP32 flux arithmetic, as for the flow rhs
    assert s.step(20) == 0
    g = s.get_scalars()
    assert np.abs(g[:, 0] - 1.0).max() < 1e-12
    r1, _, _ = s.get_state()
    vol = np.array(m.vol_cv)
    t0 = (rho[:, None] * sc * vol[:, None]).sum(0)
    t1 = (r1[:, None] * g * vol[:, None]).sum(0)
    assert (np.abs(t1 - t0) / np.abs(t0)).max() < 1e-13
    s.close()
