"""Channel meshes (periodic in x and z, walls at y = 0 and y = Ly) and the
oracle's boundary conditions, on CPU.

Generator: cells close with their boundary faces; wall areas and the volume
are exact; area_over_delta_bf and Gij_bf are the reference's formulas
(src/core/common/StripedMesh.hpp:2781-2794), recomputed here in numpy; the
extended faces satisfy the geometric conservation law with the boundary faces
(sum of n_ef + sum of n_bf = 0 per cell, FlowSolver.hpp:1596-1630); the
gradient coefficients are exact for linear fields in cells away from the
walls.

Oracle: a fluid at rest is an exact solution (rhs = 0 to round-off) with slip
and with no-slip walls; with slip walls mass and the wall-parallel momentum
stay constant over RK3 steps, with adiabatic walls mass and energy do."""
import numpy as np
import pytest

from nextgen_b200 import cases
from nextgen_b200.meshgen import ChannelMesh
from oracle import Oracle

SLIP, WALL = 1, 2
L = (3.0, 2.0, 1.5)


@pytest.fixture(scope="module")
def chan(built):
    return ChannelMesh(12, 8, 6, L=L, jitter=0.25, seed=7)


def _area_sum(m):
    """Sum of |n| over each cell's compact and boundary faces."""
    a = np.linalg.norm(m.n_fa, axis=1)
    area = np.zeros(m.ncv)
    np.add.at(area, m.cvofa[:, 0], a)
    own = m.cvofa[:, 1] < m.ncv
    np.add.at(area, m.cvofa[own, 1], a[own])
    np.add.at(area, m.cvobf, m.area_bf)
    return area


def test_anisotropic_lattice_refused(built):
    # hy much smaller than hx: cells would reach beyond the candidate
    # neighbourhood, so the generator refuses the mesh
    with pytest.raises(RuntimeError, match="do not close"):
        ChannelMesh(10, 8, 6, L=(2.0 * np.pi, 2.0, np.pi), jitter=0.25, seed=7)


def test_geometry(chan):
    m = chan
    assert m.nbf > 0 and m.nbf_zones == 2
    S = np.zeros((m.ncv, 3))
    np.add.at(S, m.cvofa[:, 0], m.n_fa)
    own = m.cvofa[:, 1] < m.ncv
    np.add.at(S, m.cvofa[own, 1], -m.n_fa[own])
    np.add.at(S, m.cvobf, m.n_bf)
    assert (np.linalg.norm(S, axis=1) / _area_sum(m)).max() < 1e-12
    assert abs(m.vol_cv.sum() - np.prod(L)) < 1e-12 * np.prod(L)
    for z, sgn in ((0, -1.0), (1, 1.0)):
        sel = m.zone_bf == z
        assert abs(m.area_bf[sel].sum() - L[0] * L[2]) < 1e-12 * L[0] * L[2]
        assert (np.sign(m.n_bf[sel, 1]) == sgn).all()
        assert np.abs(m.n_bf[sel][:, [0, 2]]).max() < 1e-12 * m.area_bf[sel].max()
        assert np.abs(m.x_bf[sel, 1] - (0.0 if z == 0 else L[1])).max() < 1e-12
    # no periodic ghost in y
    assert (m.shift_g[:, 1] == 0).all()


def test_boundary_face_formulas(chan):
    m = chan
    dx = m.x_bf - m.x_vv[m.cvobf]
    area = np.linalg.norm(m.n_bf, axis=1)
    assert np.array_equal(area, m.area_bf)
    un = m.n_bf / np.maximum(area, 1e-20)[:, None]
    dp = (dx * un).sum(1)
    vol = m.vol_cv[m.cvobf]
    clip = np.minimum(0.25 * vol ** (1.0 / 3.0), 0.25 * vol / np.maximum(area, 1e-20))
    aod = np.where(dp < clip, area / clip, area / dp)
    assert np.allclose(m.area_over_delta_bf, aod, rtol=1e-14, atol=0)
    assert np.allclose(m.Gij_bf, -m.n_bf[:, :, None] * dx[:, None, :], rtol=1e-15, atol=1e-300)


def test_extended_gcl_and_gradient(chan):
    m = chan
    S = np.zeros((m.ncv, 3))
    np.add.at(S, m.cvoef[:, 0], m.n_ef)
    own = m.cvoef[:, 1] < m.ncv
    np.add.at(S, m.cvoef[own, 1], -m.n_ef[own])
    np.add.at(S, m.cvobf, m.n_bf)
    assert (np.linalg.norm(S, axis=1) / _area_sum(m)).max() < 1e-12
    # gradient of a linear field through cvocv: exact in cells whose compact
    # stencil touches no wall (the zero-gradient wall term biases the others)
    g = np.array([1.1234, -1.3243, 1.5321])
    phi = m.x_cv @ g
    grad = np.zeros((m.ncv, 3))
    for c in range(m.ncv):
        b, e = m.cvocv_i[c], m.cvocv_i[c + 1]
        grad[c] = (m.cvocv_grad_coeff[b + 1:e] * (phi[m.cvocv_v[b + 1:e]] - phi[c])[:, None]).sum(0)
    wall = np.zeros(m.ncv, bool)
    wall[m.cvobf] = True
    near = wall.copy()
    for c in np.nonzero(wall)[0]:
        near[m.owner(m.cvocv_v[m.cvocv_i[c]:m.cvocv_i[c + 1]])] = True
    far = ~near
    assert far.sum() > m.ncv // 3
    assert np.abs(grad[far] - g).max() < 1e-12


def _oracle(m, prm, st, kinds):
    o = Oracle(m, prm)
    for z, k in enumerate(kinds):
        o.set_bc(z, k)
    o.set_state_primitive(*st)
    o.init_complete()
    return o


@pytest.mark.parametrize("kinds", [(SLIP, SLIP), (WALL, WALL), (SLIP, WALL)])
def test_rest_is_a_solution(chan, kinds):
    m = chan
    prm = cases.tgv_params()
    rho = np.ones(m.ncv)
    p = np.full(m.ncv, prm.p_ref)
    o = _oracle(m, prm, (rho, np.zeros((m.ncv, 3)), p), kinds)
    r, scale = o.calc_rhs(1)
    assert np.abs(r).max() <= 1e-12 * prm.p_ref * np.abs(m.n_fa).max()


def _channel_state(m, prm, Ma=0.2):
    """A wall-bounded vortex field: u = U sin(pi y/Ly) cos z', v = 0.3 U sin x'
    sin(pi y/Ly)^2, w = 0.2 U cos x' (x', z' scaled to 2 pi over the box);
    uniform rho and p."""
    x, y, z = m.x_cv[: m.ncv].T
    x = x * (2.0 * np.pi / L[0])
    z = z * (2.0 * np.pi / L[2])
    U = 1.0
    s = np.sin(np.pi * y / L[1])
    u = np.stack([U * s * np.cos(z), 0.3 * U * np.sin(x) * s * s, 0.2 * U * np.cos(x)], 1)
    return np.ones(m.ncv), u, np.full(m.ncv, prm.p_ref)


def test_channel_conservation(chan):
    m = chan
    prm = cases.tgv_params(Re=400.0)
    st = _channel_state(m, prm)
    vol = np.array(m.vol_cv)
    for kinds in ((SLIP, SLIP), (WALL, WALL)):
        o = _oracle(m, prm, st, kinds)
        t0 = o.totals()
        assert o.step(20) == 0
        t1 = o.totals()
        r, u, e = o.get_state()
        mom = (r * np.abs(u).sum(1) * vol).sum()
        assert abs(t1[0] - t0[0]) <= 1e-13 * t0[0]
        assert abs(t1[4] - t0[4]) <= 1e-13 * t0[4]  # no work, no heat at the walls
        if kinds == (SLIP, SLIP):
            assert abs(t1[1] - t0[1]) <= 1e-13 * mom and abs(t1[3] - t0[3]) <= 1e-13 * mom


def test_wall_momentum_balance(chan):
    """The face sums telescope, so the momentum rhs summed over the cells is
    the walls' force: -sum over boundary faces of (p n_bf + tau), with
    tau = mu_lam area_over_delta_bf u at a wall at rest."""
    m = chan
    prm = cases.tgv_params(Re=400.0)
    o = _oracle(m, prm, _channel_state(m, prm), (WALL, WALL))
    r, _ = o.calc_rhs(1)
    p, T, _ = o.primitive()
    _, u, _ = o.get_state()
    mu_lam = prm.mu_ref * (1.0 + np.expm1(prm.mu_power_law * np.log(T / prm.T_ref)))
    c = m.cvobf
    f = -(p[c, None] * m.n_bf + (mu_lam[c] * m.area_over_delta_bf)[:, None] * u[c])
    want = f.sum(0)
    scale = np.abs(f).sum(0) + np.abs(r[:, 1:4]).sum(0) * 1e-3
    assert (np.abs(r[:, 1:4].sum(0) - want) / scale).max() <= 1e-11
