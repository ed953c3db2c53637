"""Full-size checks: decaying isotropic turbulence on the jittered 128^3
lattice (about 2.1M cells, Mt 0.3): calcRhs against the oracle at 1e-12 per
cell, and size-independent properties of a few steps (conservation to
round-off, determinism, NaN-free, mixed within its tolerance)."""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import PeriodicBoxMesh
from oracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hit128(built):
    n = 128
    m = PeriodicBoxMesh(n, jitter=0.25, seed=1234)
    prm = cases.hit_params(Mt=0.3)
    rho, u, p = cases.hit_state(n, prm, Mt=0.3, k0=4.0, seed=4321)
    return m, cgx.Mesh(m), prm, rho, u, p


def test_hit128_calc_rhs_matches_oracle(hit128):
    m, gm, prm, rho, u, p = hit128
    s = cgx.Solver(gm, prm)
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    got = s.calcRhs(1)
    o = Oracle(m, prm, nparts=1)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    ref, scale = o.calc_rhs(1)
    err = np.abs(got - ref) / np.maximum(np.abs(ref), scale)
    assert err.max() <= 1e-12, err.max()


def test_hit128_steps_conserve_and_repeat(hit128):
    m, gm, prm, rho, u, p = hit128
    outs = []
    for _ in range(2):
        s = cgx.Solver(gm, prm)
        s.set_state_primitive(rho, u, p)
        s.initComplete()
        t0 = s.totals()
        assert s.step(10) == 0
        t1 = s.totals()
        outs.append(s.get_state())
    r0 = rho * m.vol_cv
    e_norm = (outs[0][2] * m.vol_cv).sum()
    mom = (rho * np.sqrt((u * u).sum(1)) * m.vol_cv).sum()
    assert abs(t1[0] - t0[0]) / r0.sum() < 1e-13
    assert np.abs(t1[1:4] - t0[1:4]).max() / mom < 1e-13
    assert abs(t1[4] - t0[4]) / e_norm < 1e-13
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_hit128_mixed_close_to_fp64(hit128):
    m, gm, prm, rho, u, p = hit128
    res = {}
    for prec in (cgx.CGX_FP64, cgx.CGX_MIXED):
        s = cgx.Solver(gm, prm, prec)
        s.set_state_primitive(rho, u, p)
        s.initComplete()
        assert s.step(20) == 0
        res[prec] = s.get_state()
    r64, u64, _ = res[cgx.CGX_FP64]
    r32, u32, _ = res[cgx.CGX_MIXED]
    ke64 = 0.5 * (r64 * (u64 * u64).sum(1) * m.vol_cv).sum()
    ke32 = 0.5 * (r32 * (u32 * u32).sum(1) * m.vol_cv).sum()
    assert abs(ke32 - ke64) / ke64 <= 1e-5
    assert np.sqrt(((u32 - u64) ** 2).mean() / (u64 ** 2).mean()) <= 1e-5


def test_hit128_200_step_trajectory_matches_oracle(hit128):
    """The decaying-turbulence configuration end to end: 200 RK3 steps at
    CFL 0.8 by the GPU path and by the oracle (on all host threads, cell
    ranges like MPI ranks) from the same state.  The state stays within
    1e-12 of the oracle's (relative L-inf), the conserved totals within 1e-13
    of their scale and the simulated time within 1e-14."""
    import os
    m, gm, prm, rho, u, p = hit128
    K = 200
    s = cgx.Solver(gm, prm)
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    assert s.step(K) == 0
    o = Oracle(m, prm, nparts=os.cpu_count() or 1)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    assert o.step(K) == 0
    g, r = s.get_state(), o.get_state()
    for a, b in zip(g, r):
        assert np.abs(a - b).max() / np.abs(b).max() <= 1e-12
    vol = np.array(m.vol_cv)
    scale = np.array([(r[0] * vol).sum()] + [np.abs(r[0] * r[1][:, k] * vol).sum() for k in range(3)] +
                     [(r[2] * vol).sum()])
    assert (np.abs(s.totals() - o.totals()) / scale).max() <= 1e-13
    ts, to = s.time(), o.time()
    assert ts[2] == to[2] == K
    assert abs(ts[0] - to[0]) / to[0] <= 1e-14
