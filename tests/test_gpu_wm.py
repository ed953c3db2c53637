"""The algebraic wall-model zones on the GPU against the oracle, on a channel
(periodic in x and z, walls at y = 0 and y = Ly): WM_ALG_ADIABATIC with a
moving wall, WM_ALG_ISOTHERMAL, WM_ALG_CONDUCTIVE behind two layers, and the
equilibrium WM_EQ_ADIABATIC and WM_EQ_ISOTHERMAL (WmAdiabatic, WmIsothermal,
WmAlgConductive, IdealGasSolverBcs.cpp:996-1478, 2054-2262, 2411-2595;
EquilibriumWM.hpp).

* calcRhs after initComplete (the laminar wall stress) within 1e-12 of the
  face-sum scale;
* 10 RK3 steps, each solving the law of the wall for every face at its first
  stage from the last step's tau_wall: state within 1e-10 of the oracle's;
* a NaN restores tau_wall with the state, and 3 more steps still match;
* the mixed-precision form within its flux tolerance of the FP64 path.
"""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import ChannelMesh
from oracle import Oracle

pytestmark = pytest.mark.gpu

WM_AD, WM_ISO = cgx.CGX_BC_WM_ALG_ADIABATIC, cgx.CGX_BC_WM_ALG_ISOTHERMAL
WM_COND = cgx.CGX_BC_WM_ALG_CONDUCTIVE
ZONES = ((WM_AD, (0.0, 0.0, 0.05)), (WM_ISO, (1.2,)))
ZONES_COND = ((WM_COND, (1.3, 0.01, 0.5, 0.02, 1.0)), (WM_AD, ()))
WM_EQ_AD, WM_EQ_ISO = cgx.CGX_BC_WM_EQ_ADIABATIC, cgx.CGX_BC_WM_EQ_ISOTHERMAL
ZONES_EQ = ((WM_EQ_AD, (0.0, 0.0, 0.05)), (WM_EQ_ISO, (1.2, 0.7, 1.0, 1e-5)))


@pytest.fixture(scope="module")
def chan(built):
    m = ChannelMesh(16, 12, 8, L=(4.0, 3.0, 2.0), jitter=0.25, seed=11)
    return m, cgx.Mesh(m, device=0)


def _state(m, prm):
    x, y, z = m.x_cv[: m.ncv].T
    Lx, Ly, Lz = m.L
    u = np.stack([0.3 + 0.1 * np.cos(2 * np.pi * z / Lz), 0.02 * np.sin(2 * np.pi * x / Lx),
                  0.05 * np.sin(np.pi * y / Ly)], 1)
    rho = 1.0 + 0.02 * np.cos(2 * np.pi * x / Lx)
    p = prm.p_ref * (1.0 + 0.01 * np.sin(2 * np.pi * z / Lz))
    return rho, u, p


def _make(m, gm, prm, prec=cgx.CGX_FP64, zones=ZONES):
    s = cgx.Solver(gm, prm, prec)
    o = Oracle(m, prm)
    for z, (k, a) in enumerate(zones):
        s.set_bc_params(z, k, a)
        o.set_bc_params(z, k, a)
    st = _state(m, prm)
    s.set_state_primitive(*st)
    s.initComplete()
    o.set_state_primitive(*st)
    o.init_complete()
    return s, o


@pytest.mark.parametrize("zones", [ZONES, ZONES_COND, ZONES_EQ], ids=["adiabatic_isothermal", "conductive",
                                                                     "equilibrium"])
def test_wall_models_match_oracle(chan, zones):
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    s, o = _make(m, gm, prm, zones=zones)
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    # a NaN in a cell on the zone-0 wall: both restore the stored state with
    # its tau_wall (the equilibrium isothermal zone 1 keeps its own, so the
    # NaN stays away from it)
    o.set_dt()
    icv = int(m.cvobf[m.zone_bf == 0][0])
    assert icv not in set(m.cvobf[m.zone_bf == 1].tolist())
    bad = [a.copy() for a in s.get_state()]
    bad[0][icv] = np.nan
    s.set_state(*bad)
    s.updateConservativeAndPrimitiveData()
    o.poison(icv)
    assert s.advanceSolution() == -1 and o.advance_solution() == -1
    assert s.step(3) == 0 and o.step(3) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    s.close()
    o.close()


def test_wall_models_mixed_close_to_fp64(chan):
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    res = {}
    for prec in (cgx.CGX_FP64, cgx.CGX_MIXED):
        s, o = _make(m, gm, prm, prec)
        o.close()
        assert s.step(10) == 0
        res[prec] = s.get_state()
        s.close()
    for a64, a32 in zip(res[cgx.CGX_FP64], res[cgx.CGX_MIXED]):
        assert np.sqrt(((a32 - a64) ** 2).mean() / (a64 ** 2).mean()) <= 1e-5


def test_wall_model_refusals(chan):
    m, gm = chan
    s = cgx.Solver(gm, cases.tgv_params())
    for kind, bad in ((WM_AD, (0.1,)), (WM_ISO, ()), (WM_ISO, (1.0, 2.0)), (WM_COND, (1.0, 0.1)),
                      (WM_EQ_AD, (0.1,)), (WM_EQ_ISO, (1.0, 0.7))):
        with pytest.raises(cgx.CgxError):
            s.set_bc_params(0, kind, bad)
    s.close()


WM_EX_AD, WM_EX_ISO = cgx.CGX_BC_WM_EXCHANGE_ADIABATIC, cgx.CGX_BC_WM_EXCHANGE_ISOTHERMAL


def test_exchange_wall_models_match_oracle(chan):
    """WM_EXCHANGE_ADIABATIC and WM_EXCHANGE_ISOTHERMAL (WmExchange,
    IdealGasSolverBcs.cpp:500-990): each face's velocity reconstructed at its
    exchange point x_bf - ratio delta n_hat in a nearby cell (every fifth face
    left unlocated); calcRhs within 1e-12, 10 steps within 1e-10 of the
    oracle, and a NaN restores tau_wall; an exchange zone without its points
    is refused."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    zones = ((WM_EX_AD, ()), (WM_EX_ISO, (1.2, 2.0)))
    ratios = (3.0, 2.0)
    xc = m.x_cv[: m.ncv]
    pts = {}
    for z in (0, 1):
        sel = m.zone_bf == z
        nb, xb = m.n_bf[sel], m.x_bf[sel]
        area = np.linalg.norm(nb, axis=1)
        delta = area / m.area_over_delta_bf[sel]
        xe = xb - ratios[z] * (delta / area)[:, None] * nb
        cv = np.array([int(np.argmin(((xc - q) ** 2).sum(1))) for q in xe], dtype=np.int32)
        cv[::5] = -1
        pts[z] = (cv, xe)
    s = cgx.Solver(gm, prm)
    o = Oracle(m, prm)
    for z, (k, a) in enumerate(zones):
        s.set_bc_params(z, k, a)
        o.set_bc_params(z, k, a)
    s2 = cgx.Solver(gm, prm)
    for z, (k, a) in enumerate(zones):
        s2.set_bc_params(z, k, a)
    for z in (0, 1):
        s.set_bc_exchange(z, *pts[z])
        o.set_bc_exchange(z, *pts[z])
    st = _state(m, prm)
    for h in (s, o):
        h.set_state_primitive(*st)
    s.initComplete()
    o.init_complete()
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    o.set_dt()
    icv = int(m.cvobf[m.zone_bf == 0][0])
    bad = [a.copy() for a in s.get_state()]
    bad[0][icv] = np.nan
    s.set_state(*bad)
    s.updateConservativeAndPrimitiveData()
    o.poison(icv)
    assert s.advanceSolution() == -1 and o.advance_solution() == -1
    assert s.step(3) == 0 and o.step(3) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    s2.set_state_primitive(*st)
    with pytest.raises(cgx.CgxError, match="exchange points"):
        s2.initComplete()
    for h in (s, o, s2):
        h.close()
