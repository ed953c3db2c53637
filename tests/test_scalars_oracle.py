"""Passive transport scalars in the CPU oracle (calcRhsScalars,
IdealGasSolver.cpp:537-693; advanceScalars, IdealGasSolver.cpp:874-892).

CPU only.  The reference has no scalar fixtures, so these pin the oracle's
scalar path by properties the reference's formulation guarantees exactly or
to round-off:
  * a scalar identically 1 has rhs_sc equal to the continuity rhs bit for bit
    (its convective flux is 0.5 (1 + 1) mf = mf and its diffusion is zero), and
    stays 1 to round-off through RK3 steps (advanceScalars divides by the new
    density);
  * sum(rho sc V) is conserved on a periodic box (every face flux enters the
    two cells with opposite signs);
  * the restated flux header and the reference's own header give the same
    scalars bit for bit; rank-partitioned face loops agree to round-off.
"""
import numpy as np
import pytest

from nextgen_b200 import cases
from nextgen_b200.meshgen import PeriodicBoxMesh
from oracle import Oracle, ref_available


def _scalars(x):
    return np.stack([np.ones(len(x)),
                     1.0 + 0.5 * np.sin(x[:, 0]) * np.cos(x[:, 1]),
                     np.cos(x[:, 2]) ** 2], axis=1)


@pytest.fixture(scope="module")
def box(built):
    m = PeriodicBoxMesh(10, jitter=0.25, seed=1234)
    prm = cases.tgv_params()
    x = np.array(m.x_cv[: m.ncv])
    rho, u, p = cases.tgv_state(x, prm)
    return m, prm, rho, u, p, _scalars(x)


def _oracle(box, nparts=1, reference=False):
    m, prm, rho, u, p, sc = box
    o = Oracle(m, prm, nparts=nparts, reference=reference)
    o.set_state_primitive(rho, u, p)
    o.set_scalars(sc)
    o.init_complete()
    return o


def test_unit_scalar_matches_continuity(box):
    o = _oracle(box)
    rhs, _ = o.calc_rhs(1)
    rs, _ = o.rhs_sc(1)
    assert np.array_equal(rs[:, 0], rhs[:, 0])
    assert o.step(10) == 0
    assert np.abs(o.get_scalars()[:, 0] - 1.0).max() < 1e-13


def test_scalar_mass_conserved(box):
    m = box[0]
    o = _oracle(box)
    vol = np.array(m.vol_cv)
    r0, _, _ = o.get_state()
    t0 = (r0[:, None] * o.get_scalars() * vol[:, None]).sum(0)
    assert o.step(20) == 0
    r1, _, _ = o.get_state()
    t1 = (r1[:, None] * o.get_scalars() * vol[:, None]).sum(0)
    assert (np.abs(t1 - t0) / np.abs(t0)).max() < 1e-13


def test_scalar_diffusion_smooths(box):
    # a scalar variance decays (convection is skew, diffusion dissipates)
    m = box[0]
    o = _oracle(box)
    vol = np.array(m.vol_cv)
    r0, _, _ = o.get_state()
    s0 = o.get_scalars()[:, 2]
    mean0 = (r0 * s0 * vol).sum() / (r0 * vol).sum()
    var0 = (r0 * (s0 - mean0) ** 2 * vol).sum()
    assert o.step(20) == 0
    r1, _, _ = o.get_state()
    s1 = o.get_scalars()[:, 2]
    mean1 = (r1 * s1 * vol).sum() / (r1 * vol).sum()
    var1 = (r1 * (s1 - mean1) ** 2 * vol).sum()
    assert var1 < var0


@pytest.mark.skipif(not ref_available(), reason="reference-header oracle not built")
def test_restated_equals_reference_header(box):
    a, b = _oracle(box), _oracle(box, reference=True)
    a.calc_rhs(1)
    b.calc_rhs(1)
    assert np.array_equal(a.rhs_sc(1, want_scale=False), b.rhs_sc(1, want_scale=False))
    assert a.step(5) == 0 and b.step(5) == 0
    assert np.array_equal(a.get_scalars(), b.get_scalars())


def test_ranks_agree_to_roundoff(box):
    a, b = _oracle(box), _oracle(box, nparts=4)
    a.calc_rhs(1)
    b.calc_rhs(1)
    ra, sa = a.rhs_sc(1)
    rb, _ = b.rhs_sc(1)
    err = np.abs(ra - rb) / np.maximum(np.abs(ra), sa)
    assert err.max() <= 1e-12
