"""The reference's inviscid-vortex harness (IdealGasEulerSolver,
src/charles/charles_ig.cpp:88-290) on the GPU, through the C ABI.

At a size the oracle runs in seconds the GPU's state after the advection
matches the oracle's at the flow-state tolerance (1e-10 relative) and so do
the harness's error norms.  At sizes above that the GPU alone is checked by
what the discretisation guarantees: the error against the exact vortex falls
with resolution (about fourth order on a lattice, at least first order on a
jittered mesh) and the totals are kept; the mixed form's errors stay within a
few percent of the FP64 form's, far below the truncation error they measure.
"""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from oracle import Oracle
from test_vortex_oracle import HALF, T_END, centred, vortex_mesh

pytestmark = pytest.mark.gpu

KW = dict(Lx=HALF, Ly=HALF)


def run_gpu(m, mode=cgx.CGX_FP64):
    x = centred(m)
    prm = cases.vortex_params()
    rho, u, p = cases.vortex_state(x, prm, **KW)
    gm = cgx.Mesh(m, device=0)
    s = cgx.Solver(gm, prm, mode)
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    tot0 = s.totals()
    while s.time()[0] < T_END:
        assert s.step(1) == 0
    t = s.time()[0]
    state = s.get_state()
    l2, linf = cases.vortex_errors(x, m.vol_cv, *state, prm, t, **KW)
    tot1 = s.totals()
    s.close()
    return l2, linf, tot0, tot1, state, t


def test_gpu_matches_oracle(built):
    m = vortex_mesh(32, 0.25)
    l2, linf, _, _, (r1, u1, e1), t = run_gpu(m)
    x = centred(m)
    prm = cases.vortex_params()
    rho, u, p = cases.vortex_state(x, prm, **KW)
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    while o.time()[0] < T_END:
        assert o.step(1) == 0
    assert o.time()[0] == pytest.approx(t, rel=1e-12)
    r2, u2, e2 = o.get_state()
    assert (np.abs(r1 - r2) / np.abs(r2)).max() <= 1e-10
    assert (np.abs(e1 - e2) / np.abs(e2)).max() <= 1e-10
    assert np.abs(u1 - u2).max() <= 1e-10 * np.abs(u2).max()
    l2o, _ = cases.vortex_errors(x, m.vol_cv, r2, u2, e2, prm, t, **KW)
    assert np.allclose(l2, l2o, rtol=1e-6, atol=0.0)


@pytest.mark.parametrize("jitter", [0.0, 0.25])
def test_gpu_convergence(built, jitter):
    res = {n: run_gpu(vortex_mesh(n, jitter)) for n in (64, 128)}
    e64, e128 = res[64][0][0], res[128][0][0]
    if jitter == 0.0:
        assert np.log2(e64 / e128) > 2.5, (e64, e128)
    else:
        assert e128 < 0.6 * e64, (e64, e128)
    for n, (l2, linf, t0, t1, _, _) in res.items():
        for k in (0, 1, 2, 4):
            assert abs(t1[k] - t0[k]) <= 1e-12 * max(abs(t0[k]), 1.0), (n, k, t0, t1)


def test_mixed_errors_track_fp64(built):
    m = vortex_mesh(64, 0.25)
    a = run_gpu(m)[0]
    b = run_gpu(m, cgx.CGX_MIXED)[0]
    assert np.all(np.abs(b - a) <= 0.05 * a + 1e-6), (a, b)
