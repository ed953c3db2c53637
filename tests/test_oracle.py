"""The CPU oracle: pinned to the reference's own flux code and to the golden
fixtures, conservation, rank decomposition and the NaN-recovery path.
"""
import os

import numpy as np
import pytest

from nextgen_b200 import cases
from nextgen_b200.meshgen import PeriodicBoxMesh

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")

import oracle as orc_mod  # noqa: E402
from oracle import Oracle  # noqa: E402

need_ref = pytest.mark.skipif(not orc_mod.ref_available(), reason="reference-built oracle absent")


def golden_cases():
    import sys
    sys.path.insert(0, GOLD)
    import make_golden
    return make_golden


def rel_err(a, ref, scale):
    return (np.abs(a - ref) / np.maximum(np.abs(ref), np.maximum(scale, 1e-300))).max()


@pytest.mark.parametrize("name", ["tgv8_lattice", "tgv6_jitter", "hit8_jitter"])
def test_oracle_matches_golden_fixture(built, name):
    mg = golden_cases()
    g = np.load(os.path.join(GOLD, name + ".npz"))
    m, prm, rho, u, p = mg.case_setup(name)
    assert mg.mesh_fingerprint(m) == str(g["fingerprint"]), "generated mesh differs from the fixture's"
    assert np.array_equal(rho, g["rho"]) and np.array_equal(u, g["u"]) and np.array_equal(p, g["p"])
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    rhs, scale = o.calc_rhs(1)
    # restated flux arithmetic in the reference's operation order: bit-identical
    assert np.array_equal(rhs, g["rhs"])
    assert np.array_equal(o.aux(), g["aux"])
    assert np.array_equal(o.grad(), g["grad"])
    assert o.step(2) == 0
    r2, u2, e2 = o.get_state()
    assert np.array_equal(r2, g["rho2"]) and np.array_equal(u2, g["u2"]) and np.array_equal(e2, g["rhoE2"])
    assert o.time()[0] == float(g["time2"])


@need_ref
@pytest.mark.parametrize("n,jit,kind", [(8, 0.0, "tgv"), (9, 0.25, "tgv"), (8, 0.25, "hit")])
def test_restatement_bitwise_equals_reference_flux_build(built, n, jit, kind):
    m = PeriodicBoxMesh(n, jitter=jit, seed=321)
    if kind == "tgv":
        prm = cases.tgv_params()
        rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    else:
        prm = cases.hit_params()
        rho, u, p = cases.hit_state(n, prm, k0=2.0)
    outs = []
    for ref in (False, True):
        o = Oracle(m, prm, reference=ref)
        assert o.uses_reference_flux == ref
        o.set_state_primitive(rho, u, p)
        o.init_complete()
        rhs, _ = o.calc_rhs(1)
        o.step(3)
        outs.append((rhs, o.get_state(), o.totals()))
    assert np.array_equal(outs[0][0], outs[1][0])
    for a, b in zip(outs[0][1], outs[1][1]):
        assert np.array_equal(a, b)
    assert np.array_equal(outs[0][2], outs[1][2])


def test_rank_decomposition_agrees(built):
    """nparts contiguous ranges (the reference's MPI layout) vs one rank."""
    m = PeriodicBoxMesh(10, jitter=0.25, seed=5)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    res = []
    for nparts in (1, 3, 8):
        o = Oracle(m, prm, nparts=nparts)
        o.set_state_primitive(rho, u, p)
        o.init_complete()
        rhs, scale = o.calc_rhs(1)
        res.append((rhs, scale))
        o.step(2)
        res[-1] += (o.get_state()[0],)
    for rhs, _, r in res[1:]:
        assert rel_err(rhs, res[0][0], res[0][1]) < 1e-14
        assert np.allclose(r, res[0][2], rtol=1e-13, atol=0)


def test_conservation_over_steps(built):
    m = PeriodicBoxMesh(10, jitter=0.25, seed=11)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    r0, u0, e0 = o.get_state()
    t0 = o.totals()
    mom = (r0 * np.sqrt((u0 * u0).sum(1)) * m.vol_cv).sum()
    norm = np.array([np.abs(r0 * m.vol_cv).sum(), mom, mom, mom, np.abs(e0 * m.vol_cv).sum()])
    assert o.step(20) == 0
    t1 = o.totals()
    assert (np.abs(t1 - t0) / norm).max() < 1e-13


def test_nan_restores_stored_state(built):
    m = PeriodicBoxMesh(6, jitter=0.25, seed=3)
    prm = cases.tgv_params()
    prm.check_interval = 1
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    s0 = o.get_state()
    assert o.step(1) == 0
    o.poison(5)
    assert o.step(1) == -1
    t, dt, st = o.time()
    assert st == 0 and t == 0.0  # back to the state stored by initComplete
    for a, b in zip(o.get_state(), s0):
        assert np.array_equal(a, b)
    # the next step uses 0.8 x the CFL target
    o.step(1)
    _, dt1, _ = o.time()
    o2 = Oracle(m, prm)
    o2.set_state_primitive(rho, u, p)
    o2.init_complete()
    o2.step(1)
    assert abs(dt1 / o2.time()[1] - 0.8) < 1e-12


def test_tgv_initial_rhs_symmetry(built):
    """On the unjittered lattice the TGV rhs inherits the flow's symmetry:
    the mass rhs is even under x -> -x about the box centre."""
    n = 8
    m = PeriodicBoxMesh(n, jitter=0.0)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    rhs, scale = o.calc_rhs(1)
    idx = np.arange(m.ncv)
    i, j, k = idx % n, (idx // n) % n, idx // (n * n)
    mirror = (n - 1 - i) + n * (j + n * k)
    assert rel_err(rhs[mirror, 0], rhs[:, 0], scale[:, 0]) < 1e-12
