"""WALL_ISOTHERMAL and the characteristic boundary zones on the GPU against
the oracle, on a channel (periodic in x and z, zones at y = 0 and y = Ly):
CBC_UPT, CBC_RUNP and CBC_MPT add the HLLC Riemann flux between the cell
and the zone's boundary state (Cbc::addBoundaryFlux, IdealGasSolverBcs.cpp:
2960-2976; calcRiemannFlux, IdealGasSolverFlux.hpp:218-306); WALL_ISOTHERMAL
adds the wall's viscous and heat fluxes (IdealGasSolverBcs.cpp:1485-1510).

* calcRhs per cell within 1e-12 of the face-sum scale and calcCfl within
  1e-12, for an inflow/outflow pair of each kind and a hot isothermal wall;
  CBC_TOTAL_PT and CBC_EXTRAPOLATE set their boundary states after
  initComplete and renew them in each step (rk3Step of the zone);
* 10 RK3 steps: state within 1e-10 of the oracle's;
* a uniform flow through the channel stays uniform (rhs = 0 to round-off);
* the mixed-precision form within its flux tolerance of the FP64 path;
* CBC zones and transport scalars are refused together; wrong parameter
  counts are refused;
* the NSCBC zones, the zone-wide forms, CBC_RUP and WALL_CONDUCTIVE, the
  sponge layer, a profile zone and a HOOK zone against the oracle (or, for
  the hook, against the zone it reproduces), the mixed form of the zones
  with their own state, and STATIONARY_FRAME walls and a CBC_TOTAL_PT inlet
  in a rotating frame.
"""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import ChannelMesh
from oracle import Oracle

pytestmark = pytest.mark.gpu

UPT, RUNP, MPT, ISO = cgx.CGX_BC_CBC_UPT, cgx.CGX_BC_CBC_RUNP, cgx.CGX_BC_CBC_MPT, cgx.CGX_BC_WALL_ISOTHERMAL
EXTRAP, TOTAL_PT = cgx.CGX_BC_CBC_EXTRAPOLATE, cgx.CGX_BC_CBC_TOTAL_PT
P0 = cases.tgv_params(Re=400.0).p_ref  # T_ref = rho_ref = 1
# inflow at y = 0, outflow through the 4 x 2 zone at y = Ly
ZONES = {
    "upt_runp": ((UPT, (0.1, 0.4, 0.0, 1.01 * P0, 1.02)), (RUNP, (1.0, -0.3, 0.99 * P0))),
    "upt_mpt": ((UPT, (0.0, 0.35, 0.05, P0, 1.0)), (MPT, (-2.4, P0, 1.0))),
    "iso_mpt": ((ISO, (1.2,)), (MPT, (-2.4, P0, 1.0))),
    # boundary states that follow the flow: renewed each step / each stage
    "totalpt_extrap": ((TOTAL_PT, (1.02 * P0, 1.02, 0.05)), (EXTRAP, ())),
}


@pytest.fixture(scope="module")
def chan(built):
    m = ChannelMesh(16, 12, 8, L=(4.0, 3.0, 2.0), jitter=0.25, seed=11)
    return m, cgx.Mesh(m, device=0)


def _state(m, prm):
    x, y, z = m.x_cv[: m.ncv].T
    Lx, Ly, Lz = m.L
    xs, zs = 2 * np.pi * x / Lx, 2 * np.pi * z / Lz
    u = np.stack([0.2 * np.cos(zs) + 0.1, 0.3 + 0.05 * np.sin(xs), 0.1 * np.cos(xs)], 1)
    p = prm.p_ref * (1.0 + 0.02 * np.cos(xs) * np.sin(np.pi * y / Ly))
    rho = 1.0 + 0.03 * np.sin(zs)
    return rho, u, p


def _make(m, gm, prm, zones, prec=cgx.CGX_FP64, state=None):
    st = _state(m, prm) if state is None else state
    s = cgx.Solver(gm, prm, prec)
    o = Oracle(m, prm)
    for z, (k, a) in enumerate(zones):
        s.set_bc_params(z, k, a)
        o.set_bc_params(z, k, a)
    s.set_state_primitive(*st)
    s.initComplete()
    o.set_state_primitive(*st)
    o.init_complete()
    return s, o


@pytest.mark.parametrize("name", list(ZONES))
def test_cbc_rhs_and_cfl_match_oracle(chan, name):
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    s, o = _make(m, gm, prm, ZONES[name])
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    cg, cells = s.calcCfl(0.01, want_cells=True)
    co, ocells = o.calc_cfl(0.01)
    assert abs(cg - co) <= 1e-12 * co and (np.abs(cells - ocells) / ocells.max()).max() <= 1e-12
    s.close()
    o.close()


@pytest.mark.parametrize("name", ["upt_runp", "iso_mpt", "totalpt_extrap"])
def test_cbc_steps_match_oracle(chan, name):
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    s, o = _make(m, gm, prm, ZONES[name])
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    assert abs(s.time()[0] - o.time()[0]) <= 1e-13 * o.time()[0]
    s.close()
    o.close()


def test_uniform_flow_stays_uniform(chan):
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    u0 = np.array([0.1, 0.25, -0.05])
    rho = np.ones(m.ncv)
    u = np.tile(u0, (m.ncv, 1))
    p = np.full(m.ncv, prm.p_ref)
    T0 = prm.T_ref
    zones = ((UPT, (u0[0], u0[1], u0[2], prm.p_ref, T0)), (RUNP, (1.0, -u0[1], prm.p_ref)))
    s, o = _make(m, gm, prm, zones, state=(rho, u, p))
    r = s.calcRhs(1)
    ref = (u0 @ u0 + prm.p_ref) * np.linalg.norm(m.n_bf, axis=1).max()
    assert np.abs(r).max() <= 1e-12 * ref
    s.close()
    o.close()


def test_cbc_mixed_close_to_fp64(chan):
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    res = {}
    for prec in (cgx.CGX_FP64, cgx.CGX_MIXED):
        s, o = _make(m, gm, prm, ZONES["upt_runp"], prec)
        o.close()
        assert s.step(10) == 0
        res[prec] = s.get_state()
        s.close()
    for a64, a32 in zip(res[cgx.CGX_FP64], res[cgx.CGX_MIXED]):
        assert np.sqrt(((a32 - a64) ** 2).mean() / (a64 ** 2).mean()) <= 1e-5


def test_cbc_refusals(chan):
    m, gm = chan
    prm = cases.tgv_params()
    s = cgx.Solver(gm, prm)
    with pytest.raises(cgx.CgxError):
        s.set_bc_params(0, UPT, (0.1, 0.2))
    with pytest.raises(cgx.CgxError):
        s.set_bc_params(0, 9, ())
    with pytest.raises(cgx.CgxError):
        s.set_bc(0, UPT)  # the parameterised kinds go through set_bc_params
    s.set_bc_params(0, UPT, ZONES["upt_runp"][0][1])
    s.set_bc_params(1, RUNP, ZONES["upt_runp"][1][1])
    s.set_state_primitive(*_state(m, prm))
    s.initComplete()
    with pytest.raises(cgx.CgxError):
        s.set_scalars(np.zeros((m.ncv, 1)))
    s.close()


NSCBC_MT, NSCBC_OUT = cgx.CGX_BC_NSCBC_MT, cgx.CGX_BC_NSCBC_OUTLET_P


def test_nscbc_steps_and_restore_match_oracle(chan):
    """NSCBC_MT inflow and a partially reflecting NSCBC_OUTLET_P outlet: the
    faces' own rho, p, u advance with the zones' characteristic equations;
    10 steps match the oracle to 1e-10, and a NaN restores the state and the
    faces' states (Nscbc::storeData/restoreData) as the oracle does."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    zones = ((NSCBC_MT, (2.4, 1.0)), (NSCBC_OUT, (P0, 0.25, 3.0)))
    s, o = _make(m, gm, prm, zones)
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    # a NaN: both restore the stored state (step 0) with the faces' states
    o.set_dt()
    bad = [a.copy() for a in s.get_state()]
    bad[0][5] = np.nan
    s.set_state(*bad)
    s.updateConservativeAndPrimitiveData()
    o.poison(5)
    assert s.advanceSolution() == -1 and o.advance_solution() == -1
    assert s.step(3) == 0 and o.step(3) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    s.close()
    o.close()


NSCBC_MDOT = cgx.CGX_BC_NSCBC_OUTLET_MDOT


@pytest.mark.parametrize("zones", [((TOTAL_PT, (1.02 * P0, 1.02, 0.05, 1.0)), (EXTRAP, ())),
                                   ((NSCBC_MT, (2.4, -1.05)), (NSCBC_MDOT, (2.3, 0.05)))],
                         ids=["totalpt_use_avg", "mt_ttotal_outlet_mdot"])
def test_zone_wide_forms_match_oracle(chan, zones):
    """Zone means summed on the device in a fixed order: CBC_TOTAL_PT USE_AVG,
    NSCBC_MT T_TOTAL and NSCBC_OUTLET_MDOT over 10 steps against the oracle."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    s, o = _make(m, gm, prm, zones)
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    s.close()
    o.close()


RUP, COND = cgx.CGX_BC_CBC_RUP, cgx.CGX_BC_WALL_CONDUCTIVE


def test_rup_and_conductive_match_oracle(chan):
    """CBC_RUP inflow and a WALL_CONDUCTIVE wall behind two layers: calcRhs to
    1e-12 of the face-sum scale and 10 steps to 1e-10 against the oracle."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    zones = ((RUP, (1.0, 0.1, 0.4, 0.0, 1.01 * P0)), (COND, (1.1, 0.01, 0.5, 0.02, 1.0)))
    s, o = _make(m, gm, prm, zones)
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    with pytest.raises(cgx.CgxError):
        s.set_bc_params(1, COND, (1.0, 0.1))
    s.close()
    o.close()


SPONGE = cgx.CGX_BC_SPONGE


@pytest.mark.parametrize("kind", [1, 3], ids=["y", "rx"])
def test_sponge_matches_oracle(chan, kind):
    """SPONGE (Sponge, IdealGasSolverBcs.cpp:4080-4346) at y = Ly behind a
    CBC_UPT inflow: the flow set to a second state after initComplete so
    that the layer's volume term is live; calcRhs to 1e-12 of the face-sum
    scale, 10 steps (the sponge state relaxing at stage 1) to 1e-10, and a
    NaN restores the sponge state with the flow's, as the oracle does."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    x, y, z = m.x_cv[: m.ncv].T
    dist = (x, y, z, np.sqrt(y * y + z * z), np.sqrt(x * x + y * y))[kind]
    Lmax = dist.max() + 0.05
    length = 0.45 * (Lmax - dist.min())
    zones = ((UPT, (0.1, 0.4, 0.0, 1.01 * P0, 1.02)), (SPONGE, (kind, 3.0, 0.05, length, 1.01 * P0, Lmax)))
    s, o = _make(m, gm, prm, zones)
    rho, u, p = _state(m, prm)
    B = (2.0 - rho, u[:, [1, 2, 0]], prm.p_ref + 0.5 * (p - prm.p_ref))
    s.set_state_primitive(*B)
    s.updateConservativeAndPrimitiveData()
    s.calcSgsAndMaterialProperties()
    o.set_state_primitive(*B)
    o.update_primitive()
    o.calc_sgs_props()
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    o.set_dt()
    bad = [a.copy() for a in s.get_state()]
    bad[0][5] = np.nan
    s.set_state(*bad)
    s.updateConservativeAndPrimitiveData()
    o.poison(5)
    assert s.advanceSolution() == -1 and o.advance_solution() == -1
    assert s.step(3) == 0 and o.step(3) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    s.close()
    o.close()


def test_sponge_refusals(chan, built):
    m, gm = chan
    prm = cases.tgv_params()
    good = (1, 2.0, 0.5, 0.8, prm.p_ref, m.L[1])
    s = cgx.Solver(gm, prm)
    for bad in ((5,) + good[1:], (1.5,) + good[1:], good[:3] + (0.0,) + good[4:], good[:5]):
        with pytest.raises(cgx.CgxError):
            s.set_bc_params(1, SPONGE, bad)
    s.set_bc_params(1, SPONGE, good)
    with pytest.raises(cgx.CgxError):
        s.set_bc_params(0, SPONGE, good)  # one sponge zone
    with pytest.raises(cgx.CgxError):
        s.set_scalars(np.zeros((m.ncv, 1)))  # no transport scalars with CBC zones
    s.close()
    # the layer's cells come from the mesh's x_cv
    gm2 = cgx.Mesh(m, device=0, sfc=False)
    s2 = cgx.Solver(gm2, prm)
    with pytest.raises(cgx.CgxError):
        s2.set_bc_params(1, SPONGE, good)
    s2.close()
    gm2.close()


def test_profile_zone_matches_oracle(chan):
    """CBC_PROFILE (CbcProfile, IdealGasSolverBcs.cpp:3024-3180): an inflow
    whose state varies face by face (a parabolic normal speed, p and T
    varying along the zone) behind a CBC_RUNP outflow; calcRhs to 1e-12 and
    10 steps to 1e-10 against the oracle.  The kind is refused through
    cgx_set_bc_params and with a wrong face count."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    R, g = prm.p_ref / prm.rho_ref / prm.T_ref, prm.gamma
    faces = np.flatnonzero(m.zone_bf == 0)
    xf = m.x_cv[m.cvobf[faces]]
    T = 1.0 + 0.02 * xf[:, 2]
    p = P0 * (1.0 + 0.01 * xf[:, 0])
    st = np.column_stack([0.05 * np.cos(xf[:, 2]), 0.4 * (1.0 - ((xf[:, 0] - 2.0) / 2.0) ** 2), 0.0 * T,
                          R * T / p, p, R * T * g / (g - 1.0)])
    s = cgx.Solver(gm, prm)
    o = Oracle(m, prm)
    s.set_bc_profile(0, st)
    o.set_bc_profile(0, st)
    for h in (s, o):
        h.set_bc_params(1, RUNP, (1.0, -0.3, 0.99 * P0))
    st0 = _state(m, prm)
    s.set_state_primitive(*st0)
    s.initComplete()
    o.set_state_primitive(*st0)
    o.init_complete()
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    with pytest.raises(cgx.CgxError):
        s.set_bc_params(0, cgx.CGX_BC_CBC_PROFILE, ())
    with pytest.raises(cgx.CgxError):
        s.set_bc_profile(0, st[:-1])
    s.close()
    o.close()


def test_hook_zone_through_the_source_hook(chan):
    """HOOK (initHookBc): a zone whose flux is the caller's own code, added by
    the host hook of cgx_set_source_hook.  A hook that adds SlipWallBc's
    -p n_bf (IdealGasSolverBcs.cpp:14-23) to the zone's cells reproduces a
    SLIP zone: calcRhs within 1e-12 and 5 steps within 1e-10.  Transport
    scalars are refused with the hook zone."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    g = prm.gamma
    faces = np.flatnonzero(m.zone_bf == 0)
    cells, nb = m.cvobf[faces], m.n_bf[faces]

    def slip(rho, u, rhoE, rhs, time, stage):
        p = (g - 1.0) * (rhoE - 0.5 * rho * (u * u).sum(1))
        np.subtract.at(rhs[:, 1:4], cells, p[cells, None] * nb)

    st = _state(m, prm)
    out = []
    for hook in (True, False):
        s = cgx.Solver(gm, prm)
        s.set_bc_params(0, cgx.CGX_BC_HOOK if hook else cgx.CGX_BC_SLIP, ())
        s.set_bc_params(1, cgx.CGX_BC_SLIP, ())
        if hook:
            s.set_source_hook(slip)
        s.set_state_primitive(*st)
        s.initComplete()
        out.append(s.calcRhs(1))
        assert s.step(5) == 0
        out.append(np.concatenate([a.reshape(m.ncv, -1) for a in s.get_state()], 1))
        if hook:
            with pytest.raises(cgx.CgxError):
                s.set_scalars(np.zeros((m.ncv, 1)))
        s.close()
    scale = np.abs(out[2]).max(0)
    assert (np.abs(out[0] - out[2]) / scale).max() <= 1e-12
    assert np.abs(out[1] - out[3]).max() / np.abs(out[3]).max() <= 1e-10


@pytest.mark.parametrize("zones", [
    ((NSCBC_MT, (2.4, 1.0)), (NSCBC_OUT, (P0, 0.25, 3.0))),
    ((RUP, (1.0, 0.1, 0.4, 0.0, 1.01 * P0)), (COND, (1.1, 0.01, 0.5, 0.02, 1.0))),
    ((UPT, (0.1, 0.4, 0.0, 1.01 * P0, 1.02)), (SPONGE, (1, 3.0, 0.05, 1.5, 1.01 * P0, 3.0))),
], ids=["nscbc", "rup_conductive", "sponge"])
def test_zone_kinds_mixed_close_to_fp64(chan, zones):
    """The mixed-precision form with the zones that keep their own state (the
    NSCBC faces, the sponge state) and the other flux forms: 10 steps within
    the form's flux tolerance of the FP64 path."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    res = {}
    for prec in (cgx.CGX_FP64, cgx.CGX_MIXED):
        s, o = _make(m, gm, prm, zones, prec)
        o.close()
        assert s.step(10) == 0
        res[prec] = s.get_state()
        s.close()
    for a64, a32 in zip(res[cgx.CGX_FP64], res[cgx.CGX_MIXED]):
        assert np.sqrt(((a32 - a64) ** 2).mean() / (a64 ** 2).mean()) <= 1e-5


def test_stationary_walls_in_a_rotating_frame(chan):
    """STATIONARY_FRAME walls in a rotating frame: each wall face moves at
    -w x x_bf (WallAdiabatic/WmAdiabatic::initData, IdealGasSolverBcs.cpp:
    477-493, 1024-1040), given face by face, with the frame's own source terms:
    calcRhs within 1e-12, 10 steps within 1e-10 of the oracle."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    rev = np.array([0.0, 0.03, 0.0])
    w = rev * 2.0 * np.pi
    s = cgx.Solver(gm, prm)
    o = Oracle(m, prm)
    for h in (s, o):
        h.set_bc_params(0, cgx.CGX_BC_WALL_ADIABATIC, ())
        h.set_bc_params(1, cgx.CGX_BC_WM_ALG_ADIABATIC, ())
    for zone in (0, 1):
        ub = -np.cross(w, m.x_bf[m.zone_bf == zone])
        s.set_bc_face_velocity(zone, ub)
        o.set_bc_face_velocity(zone, ub)
    s.set_frame_rotation(rev, m.x_cv[: m.ncv])
    o.set_frame_rotation(rev)
    st = _state(m, prm)
    s.set_state_primitive(*st)
    s.initComplete()
    o.set_state_primitive(*st)
    o.init_complete()
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    with pytest.raises(cgx.CgxError):
        s.set_bc_face_velocity(0, np.zeros((3, 3)))  # wrong face count
    s.close()
    o.close()


def test_total_pt_inlet_in_a_rotating_frame(chan):
    """CBC_TOTAL_PT with STATIONARY_FRAME (CbcTotalPt, IdealGasSolverBcs.cpp:
    3372-3434): the frame velocity -w x x_bf of each face, given face by
    face, adds its part along the face to the boundary state; with the
    frame's source terms and an extrapolated outlet, calcRhs within 1e-12 and
    10 steps within 1e-10 of the oracle."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    rev = np.array([0.02, 0.05, -0.01])
    w = rev * 2.0 * np.pi
    s = cgx.Solver(gm, prm)
    o = Oracle(m, prm)
    for h in (s, o):
        h.set_bc_params(0, TOTAL_PT, (1.02 * P0, 1.02, 0.05))
        h.set_bc_params(1, EXTRAP, ())
    ufr = -np.cross(w, m.x_bf[m.zone_bf == 0])
    s.set_bc_face_velocity(0, ufr)
    o.set_bc_face_velocity(0, ufr)
    s.set_frame_rotation(rev, m.x_cv[: m.ncv])
    o.set_frame_rotation(rev)
    st = _state(m, prm)
    s.set_state_primitive(*st)
    s.initComplete()
    o.set_state_primitive(*st)
    o.init_complete()
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    with pytest.raises(cgx.CgxError):
        s.set_bc_face_velocity(1, np.zeros((int((m.zone_bf == 1).sum()), 3)))  # not for EXTRAPOLATE
    s.close()
    o.close()


def test_nscbc_zones_in_a_rotating_frame(chan):
    """NSCBC_MT and NSCBC_OUTLET_P in a rotating frame (NscbcMt::initData and
    calcRhs, NscbcOutletP::calcRhsPressure, IdealGasSolverBcs.cpp:3752-3830,
    3975-3996): the inflow's u_bc takes the frame velocity's part along the
    face and the outlet's u rhs the centrifugal and Coriolis accelerations;
    10 steps within 1e-10 of the oracle; without the faces' frame velocities
    the zones are refused."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    rev = np.array([0.01, 0.04, -0.02])
    w = rev * 2.0 * np.pi
    zones = ((NSCBC_MT, (2.4, 1.0)), (NSCBC_OUT, (P0, 0.25, 3.0)))
    s = cgx.Solver(gm, prm)
    o = Oracle(m, prm)
    for z, (k, a) in enumerate(zones):
        s.set_bc_params(z, k, a)
        o.set_bc_params(z, k, a)
        ufr = -np.cross(w, m.x_bf[m.zone_bf == z])
        s.set_bc_face_velocity(z, ufr)
        o.set_bc_face_velocity(z, ufr)
    s.set_frame_rotation(rev, m.x_cv[: m.ncv])
    o.set_frame_rotation(rev)
    st = _state(m, prm)
    s.set_state_primitive(*st)
    s.initComplete()
    o.set_state_primitive(*st)
    o.init_complete()
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    s.close()
    o.close()
    # without the faces' frame velocities the zones are refused in a rotating frame
    s = cgx.Solver(gm, prm)
    for z, (k, a) in enumerate(zones):
        s.set_bc_params(z, k, a)
    s.set_frame_rotation(rev, m.x_cv[: m.ncv])
    s.set_state_primitive(*st)
    with pytest.raises(cgx.CgxError, match="frame velocity"):
        s.initComplete()
    s.close()


def test_rup_inflow_in_a_rotating_frame(chan):
    """CBC_RUP with STATIONARY_FRAME (CbcRup, IdealGasSolverBcs.cpp:
    3297-3358): an inflow velocity off the rotation axis turns by -|w| t
    each stage (Rodrigues' formula) and adds the face's frame velocity;
    10 steps within 1e-10 of the oracle."""
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    rev = np.array([0.0, 0.05, 0.0])
    w = rev * 2.0 * np.pi
    s = cgx.Solver(gm, prm)
    o = Oracle(m, prm)
    for h in (s, o):
        h.set_bc_params(0, RUP, (1.0, 0.1, 0.4, 0.05, 1.01 * P0))
        h.set_bc_params(1, RUNP, (1.0, -0.3, 0.99 * P0))
    ufr = -np.cross(w, m.x_bf[m.zone_bf == 0])
    s.set_bc_face_velocity(0, ufr)
    o.set_bc_face_velocity(0, ufr)
    s.set_frame_rotation(rev, m.x_cv[: m.ncv])
    o.set_frame_rotation(rev)
    st = _state(m, prm)
    s.set_state_primitive(*st)
    s.initComplete()
    o.set_state_primitive(*st)
    o.init_complete()
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    s.close()
    o.close()
