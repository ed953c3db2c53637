"""ROTATING_REFERENCE_FRAME in the oracle, on CPU: addRotationSourceTerms
(IdealGasSolver.cpp:695-733) with the rate turned from revolutions into
radians per unit time (IdealGasSolver.hpp:126-142).

* calcRhs with the frame minus calcRhs without it is, per cell, the
  centrifugal -rho vol w x (w x x) plus the Coriolis -2 rho vol w x u in the
  momentum and their dot product with u in the energy, against a numpy
  restatement, on a jittered periodic box and a channel;
* the Coriolis force does no work: the energy term is the centrifugal
  force's work alone;
* a rotating frame without the cell centroids is refused.
"""
import numpy as np
import pytest

from nextgen_b200 import cases
from nextgen_b200.cgx import mesh_desc
from nextgen_b200.meshgen import ChannelMesh, PeriodicBoxMesh
from oracle import Oracle

REV = np.array([0.05, -0.02, 0.11])


def _rhs(m, prm, st, rev=None, zones=()):
    o = Oracle(m, prm)
    for z, (k, a) in enumerate(zones):
        o.set_bc_params(z, k, a)
    if rev is not None:
        o.set_frame_rotation(rev)
    o.set_state_primitive(*st)
    o.init_complete()
    r, sc = o.calc_rhs(1)
    o.close()
    return r, sc


@pytest.mark.parametrize("kind", ["box", "channel"])
def test_rotation_terms(built, kind):
    if kind == "box":
        m = PeriodicBoxMesh(10, jitter=0.25, seed=4)
        zones = ()
    else:
        m = ChannelMesh(10, 6, 5, L=(3.0, 2.0, 1.5), jitter=0.25, seed=8)
        zones = ((1, []), (1, []))  # slip walls
    prm = cases.tgv_params(Re=400.0)
    x = m.x_cv[: m.ncv]
    rng = np.random.default_rng(2)
    rho = 1.0 + 0.05 * rng.standard_normal(m.ncv)
    u = 0.2 * rng.standard_normal((m.ncv, 3))
    p = prm.p_ref * (1.0 + 0.01 * rng.standard_normal(m.ncv))
    a, sa = _rhs(m, prm, (rho, u, p), REV, zones)
    b, _ = _rhs(m, prm, (rho, u, p), None, zones)
    w = REV * (2.0 * np.pi)
    rv = (rho * m.vol_cv[: m.ncv])[:, None]
    cent = -rv * np.cross(w, np.cross(w, x))
    cor = -2.0 * rv * np.cross(w, u)
    ms = cent + cor
    want = np.column_stack([np.zeros(m.ncv), ms, (ms * u).sum(1)])
    got = a - b
    scale = np.maximum(np.abs(want), sa)
    assert np.array_equal(got[:, 0], np.zeros(m.ncv))
    assert (np.abs(got - want) / scale).max() <= 1e-12
    # the Coriolis force does no work
    assert np.abs((cor * u).sum(1)).max() <= 1e-14 * np.abs(rv).max() * (np.abs(w).max() * (u * u).sum(1).max())
    assert (np.abs(got[:, 4] - (cent * u).sum(1)) / scale[:, 4]).max() <= 1e-12


def test_rotation_needs_the_centroids(built):
    import ctypes

    import oracle as orc
    m = PeriodicBoxMesh(6, jitter=0.25, seed=4)
    prm = cases.tgv_params()
    d = mesh_desc(m, with_x=False)
    L = orc._load(orc.LIB_PATH)
    h = L.orc_create(ctypes.byref(d), ctypes.byref(prm), 1)
    rev = np.ascontiguousarray(REV)
    assert L.orc_set_frame_rotation(h, rev.ctypes.data_as(orc.c_dbl_p)) == -1
    L.orc_destroy(h)
