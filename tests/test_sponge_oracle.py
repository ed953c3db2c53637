"""The SPONGE zone in the oracle, on CPU, on a channel (periodic in x and z,
zones at y = 0 and y = Ly): Sponge (IdealGasSolverBcs.cpp:4080-4346).

* A uniform flow whose sponge state is its own (initialHook) and whose
  sponge pressure is its pressure is an exact solution (rhs = 0 to
  round-off).
* The layer's volume term, for each layer direction (x, y, z, the radius
  about x, the radius about z): with the sponge state taken from one state
  and the flow set to another, calcRhs minus calcRhs at zero strength is
  -vol strength x_sp^2 (U - U_sponge) on the cells past L_max - length and
  zero elsewhere, against a numpy restatement.
* With a sponge state that never relaxes and a layer over the whole channel,
  the velocity of a disturbed flow is held nearer its initial value than
  without one.
* The sponge's flux and volume term through the reference's own Riemann
  flux header, bit for bit.
"""
import numpy as np
import pytest

import oracle as orc_mod
from nextgen_b200 import cases
from nextgen_b200.meshgen import ChannelMesh
from oracle import Oracle

UPT, SPONGE = 4, 14
need_ref = pytest.mark.skipif(not orc_mod.ref_available(), reason="reference-built oracle absent")


@pytest.fixture(scope="module")
def chan(built):
    return ChannelMesh(12, 8, 6, L=(3.0, 2.0, 1.5), jitter=0.25, seed=7)


def _state(m, prm, amp=1.0):
    x, y, z = m.x_cv[: m.ncv].T
    Lx, Ly, Lz = m.L
    xs, zs = 2 * np.pi * x / Lx, 2 * np.pi * z / Lz
    u = np.stack([0.2 * amp * np.cos(zs) + 0.1, 0.3 + 0.05 * amp * np.sin(xs), 0.1 * amp * np.cos(xs)], 1)
    p = prm.p_ref * (1.0 + 0.02 * amp * np.cos(xs) * np.sin(np.pi * y / Ly))
    rho = 1.0 + 0.03 * amp * np.sin(zs)
    return rho, u, p


def _distance(m, kind):
    x, y, z = m.x_cv[: m.ncv].T
    return (x, y, z, np.sqrt(y * y + z * z), np.sqrt(x * x + y * y))[kind]


def test_uniform_flow_through_a_sponge(chan):
    m = chan
    prm = cases.tgv_params(Re=400.0)
    u0 = np.array([0.1, 0.25, -0.05])
    rho = np.ones(m.ncv)
    u = np.tile(u0, (m.ncv, 1))
    p = np.full(m.ncv, prm.p_ref)
    o = Oracle(m, prm)
    o.set_bc_params(0, UPT, [u0[0], u0[1], u0[2], prm.p_ref, prm.T_ref])
    o.set_bc_params(1, SPONGE, [1, 2.0, 0.5, 0.8, prm.p_ref, m.L[1]])
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    r, _ = o.calc_rhs(1)
    ref = (u0 @ u0 + prm.p_ref) * np.linalg.norm(m.n_bf, axis=1).max()
    assert np.abs(r).max() <= 1e-13 * ref
    o.close()


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4], ids=["x", "y", "z", "rx", "rz"])
def test_layer_volume_term(chan, kind):
    m = chan
    prm = cases.tgv_params(Re=400.0)
    gamma = prm.gamma
    R = prm.p_ref / prm.rho_ref / prm.T_ref
    s = _distance(m, kind)
    Lmax = s.max() + 0.05
    length = 0.45 * (Lmax - s.min())
    p_sp = 1.01 * prm.p_ref
    A = _state(m, prm, 1.0)
    B = _state(m, prm, -0.7)

    def rhs(strength):
        o = Oracle(m, prm)
        o.set_bc_params(0, UPT, [0.1, 0.3, 0.0, prm.p_ref, prm.T_ref])
        o.set_bc_params(1, SPONGE, [kind, strength, 0.5, length, p_sp, Lmax])
        o.set_state_primitive(*A)
        o.init_complete()  # the sponge state: A's T and u
        o.set_state_primitive(*B)
        o.update_primitive()
        o.calc_sgs_props()
        r, sc = o.calc_rhs(1)
        o.close()
        return r, sc

    strength = 3.0
    a, sa = rhs(strength)
    b, _ = rhs(0.0)
    # numpy restatement of the volume term
    rhoA, uA, pA = A
    T_sp = pA / (rhoA * R)
    rho_sp = p_sp / (T_sp * R)
    rhoB, uB, pB = B
    rhoEB = pB / (gamma - 1.0) + 0.5 * rhoB * (uB * uB).sum(1)
    rhoE_sp = p_sp / (gamma - 1.0) + 0.5 * rho_sp * (uA * uA).sum(1)
    layer = s > Lmax - length
    assert 0 < layer.sum() < m.ncv
    x_sp = np.where(layer, (s - (Lmax - length)) / length, 0.0)
    w = m.vol_cv[: m.ncv] * strength * x_sp * x_sp
    want = -w[:, None] * np.column_stack([rhoB - rho_sp, rhoB[:, None] * uB - rho_sp[:, None] * uA, rhoEB - rhoE_sp])
    got = a - b
    assert np.array_equal(got[~layer], np.zeros_like(got[~layer]))
    assert (np.abs(got - want) / np.maximum(np.abs(want), sa)).max() <= 1e-12


def test_sponge_holds_the_initial_state(chan):
    m = chan
    prm = cases.tgv_params(Re=400.0)
    A = _state(m, prm, 1.0)
    s = _distance(m, 1)
    out = {}
    for strength in (0.0, 200.0):
        o = Oracle(m, prm)
        o.set_bc_params(0, UPT, [0.1, 0.3, 0.0, prm.p_ref, prm.T_ref])
        # a layer over the whole channel whose state never relaxes
        o.set_bc_params(1, SPONGE, [1, strength, 1e30, s.max() - s.min() + 1.0, prm.p_ref, s.max() + 0.5])
        o.set_state_primitive(*A)
        o.init_complete()
        u0 = o.get_state()[1]
        assert o.step(10) == 0
        out[strength] = np.sqrt(((o.get_state()[1] - u0) ** 2).mean())
        o.close()
    assert out[200.0] < 0.5 * out[0.0]


def test_sponge_refusals(chan):
    m = chan
    prm = cases.tgv_params()
    o = Oracle(m, prm)
    good = [1, 2.0, 0.5, 0.8, prm.p_ref, m.L[1]]
    for bad in ([5] + good[1:], [1.5] + good[1:], good[:3] + [0.0] + good[4:], good[:5]):
        with pytest.raises(ValueError):
            o.set_bc_params(1, SPONGE, bad)
    o.set_bc_params(1, SPONGE, good)
    with pytest.raises(ValueError):
        o.set_bc_params(0, SPONGE, good)  # one sponge zone
    o.close()


@need_ref
def test_sponge_bitwise_equals_reference_flux(chan):
    m = chan
    prm = cases.tgv_params(Re=400.0)
    A = _state(m, prm, 1.0)
    B = _state(m, prm, -0.7)
    out = []
    for reference in (False, True):
        o = Oracle(m, prm, reference=reference)
        o.set_bc_params(0, UPT, [0.1, 0.3, 0.0, prm.p_ref, prm.T_ref])
        o.set_bc_params(1, SPONGE, [1, 3.0, 0.05, 1.0, 1.01 * prm.p_ref, m.L[1]])
        o.set_state_primitive(*A)
        o.init_complete()
        o.set_state_primitive(*B)
        o.update_primitive()
        o.calc_sgs_props()
        out.append(o.calc_rhs(1)[0])
        assert o.step(3) == 0
        out.append(np.concatenate([v.reshape(m.ncv, -1) for v in o.get_state()], 1))
        o.close()
    assert np.array_equal(out[0], out[2])
    assert np.array_equal(out[1], out[3])
