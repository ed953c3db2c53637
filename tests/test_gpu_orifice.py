"""The reference's own mesher output on the GPU: the orifice pipe of
src/core/common/tests/assets/orifice.mles (1056 cells, 693 boundary faces in
6 zones), read by this project's .mles reader into tests/golden/
orifice_compact.npz (tests/golden/make_orifice.py).  Its operators are built
on the GPU (cgx_operators_build, the file's Gij_bf in the gradient
coefficients), the walls run as WALL_ADIABATIC and the inlet, outlet and
orifice faces as SLIP, and:

* calcRhs matches the oracle on the same operators per cell within 1e-12 of
  the face-sum scale;
* 10 RK3 steps match the oracle's within 1e-10; mass and energy (closed
  box, adiabatic walls at rest) are conserved to 1e-13;
* the state written to a .sles file and read back into a new solver is bit
  for bit the same, with its step and time;
* with a CBC_UPT inlet and a CBC_RUNP outlet (through-flow), calcRhs within
  1e-12 and 10 steps within 1e-10 of the oracle."""
import os

import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import DeviceOperatorMesh
from nextgen_b200.mles import CompactMesh
from oracle import Oracle

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "orifice_compact.npz")


@pytest.fixture(scope="module")
def orifice(built):
    c = CompactMesh.load(FIXTURE)
    m = DeviceOperatorMesh(c)
    assert m.nbf == c.nbf and m.nef > 0
    prm = cases.tgv_params(Ma=0.2, Re=500.0, L=0.0326)
    x, y, z = m.x_cv[: m.ncv].T
    R2 = (y * y + z * z) / 0.01625797 ** 2
    Lx = 0.52
    u = np.stack([(0.5 + 0.5 * np.cos(2 * np.pi * x / Lx)) * (1.0 - R2), 0.05 * np.sin(2 * np.pi * x / Lx),
                  0.05 * np.cos(2 * np.pi * x / Lx) * y / 0.0163], 1)
    p = prm.p_ref * (1.0 + 0.01 * np.sin(2 * np.pi * x / Lx))
    rho = np.ones(m.ncv)
    kinds = [cgx.CGX_BC_WALL_ADIABATIC if "wall" in name and "oriface-wall" not in name else cgx.CGX_BC_SLIP
             for name in c.zone_names]
    return m, cgx.Mesh(m, device=0), prm, (rho, u, p), kinds


def _pair(orifice, through=False):
    m, gm, prm, st, kinds = orifice
    s = cgx.Solver(gm, prm)
    o = Oracle(m, prm)
    for z, k in enumerate(kinds):
        s.set_bc(z, k)
        o.set_bc(z, k)
    if through:
        # inflow at the inlet (u p T), outflow at the outlet (rho, speed, p)
        for z, k, a in ((0, cgx.CGX_BC_CBC_UPT, (0.3, 0.0, 0.0, prm.p_ref, prm.T_ref)),
                        (1, cgx.CGX_BC_CBC_RUNP, (prm.rho_ref, -0.3, prm.p_ref))):
            s.set_bc_params(z, k, a)
            o.set_bc_params(z, k, a)
    s.set_state_primitive(*st)
    s.initComplete()
    o.set_state_primitive(*st)
    o.init_complete()
    return s, o


def test_orifice_rhs_matches_oracle(orifice):
    s, o = _pair(orifice)
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    s.close()


def test_orifice_steps_and_sles(orifice, tmp_path):
    m = orifice[0]
    s, o = _pair(orifice)
    t0 = s.totals()
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    t1 = s.totals()
    assert abs(t1[0] - t0[0]) <= 1e-13 * t0[0] and abs(t1[4] - t0[4]) <= 1e-13 * t0[4]
    path = tmp_path / "orifice.00000010.sles"
    s.write_sles(path, params="ORIFICE WALL_ADIABATIC SLIP")
    s2 = cgx.Solver(orifice[1], orifice[2])
    for z, k in enumerate(orifice[4]):
        s2.set_bc(z, k)
    s2.read_sles(path)
    for a, b in zip(s2.get_state(), s.get_state()):
        assert np.array_equal(a, b)
    assert s2.time()[0] == s.time()[0] and s2.time()[2] == 10
    s.close()
    s2.close()


def test_orifice_through_flow_matches_oracle(orifice):
    s, o = _pair(orifice, through=True)
    r = s.calcRhs(1)
    ref, scale = o.calc_rhs(1)
    assert (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max() <= 1e-12
    assert s.step(10) == 0 and o.step(10) == 0
    for a, b in zip(s.get_state(), o.get_state()):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-10
    s.close()
    o.close()
