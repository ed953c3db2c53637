"""Every lane-count variant the autotuner can choose gives calcRhs within
the face-sum tolerance of the oracle, so the variant picked on any mesh is
a correct one.  Lane counts per kernel are forced through CGX_TUNE
(extended faces, compact closures, gradient, once-per-step)."""
import os

import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import PeriodicBoxMesh
from oracle import Oracle

pytestmark = pytest.mark.gpu

TUNES = [(4, 16, 1, 1), (8, 8, 2, 4), (16, 4, 8, 8), (32, 2, 16, 16)]


@pytest.fixture(scope="module")
def case(built):
    m = PeriodicBoxMesh(14, jitter=0.25, seed=1234)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    ref, scale = o.calc_rhs(2)
    return m, prm, (rho, u, p), cgx.Mesh(m, device=0), ref, scale


@pytest.mark.parametrize("tune", TUNES, ids=lambda t: "%d-%d-%d-%d" % t)
@pytest.mark.parametrize("prec", [cgx.CGX_FP64, cgx.CGX_MIXED], ids=["fp64", "mixed"])
def test_lane_variant(case, tune, prec):
    m, prm, (rho, u, p), gm, ref, scale = case
    old = os.environ.get("CGX_TUNE")
    os.environ["CGX_TUNE"] = "%d,%d,%d,%d" % tune
    try:
        s = cgx.Solver(gm, prm, prec)
        s.set_state_primitive(rho, u, p)
        s.initComplete()
    finally:
        if old is None:
            os.environ.pop("CGX_TUNE", None)
        else:
            os.environ["CGX_TUNE"] = old
    t = s.tuning()
    assert (t["ext"], t["comp"], t["grad"], t["step_end"]) == tune
    r = s.calcRhs(2)
    err = (np.abs(r - ref) / np.maximum(np.abs(ref), scale)).max()
    tol = 1e-12 if prec == cgx.CGX_FP64 else 2e-5  # FP32 flux arithmetic in the mixed form
    assert err <= tol, err
    # the mass flux each variant leaves for the scalars: a unit scalar's
    # rhs_sc is the continuity rhs (-sum of the entries' mass fluxes)
    s.set_scalars(np.ones((m.ncv, 1)))
    r = s.calcRhs(2)
    rsc = s.rhs_sc(2)[:, 0]
    assert (np.abs(rsc - r[:, 0]) / np.maximum(np.abs(ref[:, 0]), scale[:, 0])).max() <= 1e-12
    s.set_scalars(np.zeros((m.ncv, 0)))
    assert s.step(3) == 0
    s.close()
