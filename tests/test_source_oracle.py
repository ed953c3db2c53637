"""The oracle's source terms (a subclass's addSourceHook, added by calcRhs
after the face sums, IdealGasSolver.hpp:697-705), checked by properties on
CPU: on a periodic box the face sums of momentum cancel, so the momentum rhs
summed over cells is the body force g sum(rho V); a per-cell field is added
as is."""
import numpy as np

from nextgen_b200 import cases
from nextgen_b200.meshgen import PeriodicBoxMesh
from oracle import Oracle


def _oracle(m, prm, st):
    o = Oracle(m, prm)
    o.set_state_primitive(*st)
    o.init_complete()
    return o


def test_body_force_and_field(built):
    m = PeriodicBoxMesh(8, jitter=0.25, seed=3)
    prm = cases.tgv_params()
    st = cases.tgv_state(m.x_cv[: m.ncv], prm)
    vol = np.array(m.vol_cv)
    g = np.array([0.3, -1.1, 0.6])
    o0 = _oracle(m, prm, st)
    r0, scale = o0.calc_rhs(1)
    o = _oracle(m, prm, st)
    o.set_source(g=g)
    r1, _ = o.calc_rhs(1)
    rho, u = st[0], st[1]
    mass = (rho * vol).sum()
    assert np.abs(r1[:, 1:4].sum(0) - g * mass).max() <= 1e-12 * np.abs(g * mass).max()
    f = (rho * vol)[:, None] * g[None, :]
    assert np.abs(r1[:, 1:4] - r0[:, 1:4] - f).max() <= 1e-13 * np.abs(r0).max()
    assert np.abs(r1[:, 4] - r0[:, 4] - (f * u).sum(1)).max() <= 1e-13 * np.abs(r0).max()
    rng = np.random.default_rng(1)
    field = rng.normal(size=(m.ncv, 5))
    o.set_source(field=field)
    r2, _ = o.calc_rhs(1)
    assert np.abs(r2 - r0 - field).max() <= 1e-13 * (np.abs(r0).max() + 1.0)
    o.set_source()
    r3, _ = o.calc_rhs(1)
    assert np.array_equal(r3, r0)
