"""Mixed-precision form (FP32 flux/gradient/SGS arithmetic, FP64 face sums,
state, pressure recovery, dt and totals) against the FP64 path and the
oracle.  Tolerances are stated per quantity: face sums relative to their
conditioning scale, trajectories as the relative L2/Linf error of velocity
and pressure fluctuations and the relative kinetic-energy error.
"""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import PeriodicBoxMesh
from oracle import Oracle

pytestmark = pytest.mark.gpu


def solver(m, prm, rho, u, p, prec):
    s = cgx.Solver(cgx.Mesh(m), prm, prec)
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    return s


def ke(m, rho, u):
    return 0.5 * (rho * (u * u).sum(1) * m.vol_cv).sum()


@pytest.mark.parametrize("n,jit", [(32, 0.0), (16, 0.25)])
def test_mixed_rhs_close_to_fp64(built, n, jit):
    m = PeriodicBoxMesh(n, jitter=jit, seed=1234)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    ref, scale = o.calc_rhs(1)
    got = solver(m, prm, rho, u, p, cgx.CGX_MIXED).calcRhs(1)
    # FP32 flux arithmetic: ~1e-6 of the per-cell face-sum scale
    err = np.abs(got - ref) / np.maximum(np.abs(ref), scale)
    assert err.max() < 2e-5, err.max()
    assert np.median(err) < 2e-6


def test_mixed_trajectory_tgv32(built):
    """TGV Ma 0.1 on the 32^3 lattice, 100 steps: mixed vs FP64 GPU vs oracle."""
    m = PeriodicBoxMesh(32, jitter=0.0)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    s64 = solver(m, prm, rho, u, p, cgx.CGX_FP64)
    s32 = solver(m, prm, rho, u, p, cgx.CGX_MIXED)
    ke0 = ke(m, rho, u)
    assert s64.step(100) == 0 and s32.step(100) == 0
    r64, u64, e64 = s64.get_state()
    r32, u32, e32 = s32.get_state()
    p64 = s64.primitive()[0]
    p32 = s32.primitive()[0]
    ke64, ke32 = ke(m, r64, u64), ke(m, r32, u32)
    # kinetic-energy decay error relative to the FP64 decay and to KE itself
    assert abs(ke32 - ke64) / ke64 <= 1e-5
    assert np.sqrt(((u32 - u64) ** 2).mean()) / np.sqrt((u64 ** 2).mean()) <= 1e-5
    pf = p64 - p64.mean()
    assert np.sqrt(((p32 - p64) ** 2).mean()) / np.sqrt((pf ** 2).mean()) <= 1e-4
    # conservation is FP64 in both forms
    t32 = s32.totals()
    r0 = (rho * m.vol_cv).sum()
    assert abs(t32[0] - r0) / r0 < 1e-13
    # the FP64 path is the oracle's to round-off
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    assert o.step(100) == 0
    ro, uo, eo = o.get_state()
    assert abs(ke(m, ro, uo) - ke64) / ke64 < 1e-11
    assert ke64 < ke0


def test_mixed_jittered_hit(built):
    """Decaying turbulence (Mt 0.3) on a jittered 16^3 mesh, 50 steps."""
    n = 16
    m = PeriodicBoxMesh(n, jitter=0.25, seed=1235)
    prm = cases.hit_params()
    rho, u, p = cases.hit_state(n, prm, k0=4.0)
    s64 = solver(m, prm, rho, u, p, cgx.CGX_FP64)
    s32 = solver(m, prm, rho, u, p, cgx.CGX_MIXED)
    assert s64.step(50) == 0 and s32.step(50) == 0
    r64, u64, _ = s64.get_state()
    r32, u32, _ = s32.get_state()
    assert abs(ke(m, r32, u32) - ke(m, r64, u64)) / ke(m, r64, u64) <= 1e-5
    assert np.abs(u32 - u64).max() / np.abs(u64).max() <= 1e-4


def test_mixed_deterministic_and_launches(built):
    m = PeriodicBoxMesh(10, jitter=0.25, seed=8)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    outs = []
    for _ in range(2):
        s = solver(m, prm, rho, u, p, cgx.CGX_MIXED)
        n0 = s.launch_count()
        s.step(3)
        assert s.launch_count() - n0 == 3 * 13
        outs.append(s.get_state())
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
