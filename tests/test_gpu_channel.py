"""Boundary conditions on the GPU: a channel (periodic in x and z, walls at
y = 0 and y = Ly) with SLIP and WALL_ADIABATIC zones (addBoundaryFlux,
IdealGasSolverBcs.cpp:14-48; calcCfl's boundary faces, IdealGasSolver.cpp:
1068-1074), against the oracle.

* calcRhs per cell within 1e-12 of the face-sum scale, for slip walls, walls
  at rest, a moving wall (TRANSLATE) and one of each;
* calcCfl per cell within 1e-12;
* 20 RK3 steps: state within 1e-10 of the oracle's, mass and energy
  conserved to 1e-13;
* the mixed-precision form within its flux tolerance of the FP64 path;
* the GPU operator build from the mesher's compact channel equals the host
  generator's bit for bit (the boundary faces' Gij term included);
* a zone without a boundary condition is refused, and a batch refuses the
  mesh."""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import ChannelMesh, DeviceOperatorMesh
from oracle import Oracle

pytestmark = pytest.mark.gpu

SLIP, WALL = cgx.CGX_BC_SLIP, cgx.CGX_BC_WALL_ADIABATIC
L = (3.0, 2.0, 1.5)
BCS = {"slip": ((SLIP, None), (SLIP, None)), "wall": ((WALL, None), (WALL, None)),
       "moving": ((WALL, None), (WALL, (0.3, 0.0, -0.1))), "mixed_kinds": ((SLIP, None), (WALL, None))}


@pytest.fixture(scope="module")
def chan(built):
    m = ChannelMesh(16, 12, 8, L=(4.0, 3.0, 2.0), jitter=0.25, seed=11)
    return m, cgx.Mesh(m, device=0)


def _state(m, prm):
    x, y, z = m.x_cv[: m.ncv].T
    Lx, Ly, Lz = m.L
    xs, zs = 2 * np.pi * x / Lx, 2 * np.pi * z / Lz
    s = np.sin(np.pi * y / Ly)
    u = np.stack([s * np.cos(zs) + 0.2, 0.3 * np.sin(xs) * s * s, 0.2 * np.cos(xs)], 1)
    p = prm.p_ref * (1.0 + 0.01 * np.cos(xs) * s)
    return np.ones(m.ncv), u, p


def _make(m, gm, prm, bcs, prec=cgx.CGX_FP64):
    st = _state(m, prm)
    s = cgx.Solver(gm, prm, prec)
    o = Oracle(m, prm)
    for z, (k, uw) in enumerate(bcs):
        s.set_bc(z, k, uw)
        o.set_bc(z, k, uw)
    s.set_state_primitive(*st)
    s.initComplete()
    o.set_state_primitive(*st)
    o.init_complete()
    return s, o


@pytest.mark.parametrize("name", list(BCS))
def test_channel_rhs_and_cfl_match_oracle(chan, name):
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    s, o = _make(m, gm, prm, BCS[name])
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    cg, cells = s.calcCfl(0.01, want_cells=True)
    co, ocells = o.calc_cfl(0.01)
    assert abs(cg - co) <= 1e-12 * co and (np.abs(cells - ocells) / ocells.max()).max() <= 1e-12
    s.close()


@pytest.mark.parametrize("name", ["slip", "moving"])
def test_channel_steps_match_oracle(chan, name):
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    s, o = _make(m, gm, prm, BCS[name])
    t0 = s.totals()
    assert s.step(20) == 0 and o.step(20) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    t1 = s.totals()
    assert abs(t1[0] - t0[0]) <= 1e-13 * t0[0]
    if name == "slip":
        assert abs(t1[4] - t0[4]) <= 1e-13 * t0[4]
    assert abs(s.time()[0] - o.time()[0]) <= 1e-13 * o.time()[0]
    s.close()


def test_channel_mixed_close_to_fp64(chan):
    m, gm = chan
    prm = cases.tgv_params(Re=400.0)
    res = {}
    for prec in (cgx.CGX_FP64, cgx.CGX_MIXED):
        s, _ = _make(m, gm, prm, BCS["wall"], prec)
        assert s.step(20) == 0
        res[prec] = s.get_state()
        s.close()
    u64, u32 = res[cgx.CGX_FP64][1], res[cgx.CGX_MIXED][1]
    assert np.sqrt(((u32 - u64) ** 2).mean() / (u64 ** 2).mean()) <= 1e-5


def test_channel_device_operator_build_bit_identical(built):
    host = ChannelMesh(14, 10, 8, L=(3.5, 2.5, 2.0), jitter=0.3, seed=5)
    compact = ChannelMesh(14, 10, 8, L=(3.5, 2.5, 2.0), jitter=0.3, seed=5, compact_only=True)
    dev = DeviceOperatorMesh(compact)
    for f in ("cvocv_i", "cvocv_v", "cvocv_grad_coeff", "cvoef", "n_ef", "c_ef", "area_over_delta_fa", "cmag_cv",
              "dcmag_hat_cv", "sa_to_vol_ratio", "x_cv", "icv_owner_g", "shift_g", "cvobf", "zone_bf", "n_bf",
              "area_over_delta_bf", "Gij_bf"):
        assert np.array_equal(getattr(dev, f), getattr(host, f)), f
    assert (dev.nef, dev.nbf, dev.n_threshold) == (host.nef, host.nbf, host.n_threshold)
    dev.close()


def test_channel_refusals(chan):
    m, gm = chan
    prm = cases.tgv_params()
    s = cgx.Solver(gm, prm)
    s.set_state_primitive(*_state(m, prm))
    s.set_bc(0, SLIP)
    with pytest.raises(cgx.CgxError) as e:
        s.initComplete()  # zone 1 has no boundary condition
    assert e.value.code == -6
    with pytest.raises(cgx.CgxError):
        s.set_bc(2, SLIP)
    with pytest.raises(cgx.CgxError):
        s.set_bc(1, 7)
    s.close()
    b = cgx.Batch(0, cgx.CGX_FP64, max_cases=2, hbm_budget=1 << 30)
    st = _state(m, prm)
    with pytest.raises(cgx.CgxError):
        b.add(gm, prm, *st, 5)
    b.close()
