"""Mesh and operator generator: the reference's own operator self-checks.

GCL of compact and extended faces (FlowSolver.hpp:1596-1666), linear-field
gradient exactness through cvocv_grad_coeff (StaticSolver.cpp:5559-5596) and
through the extended operator (StripedMesh.hpp:6880-6960), and the gradient
coefficients rebuilt with the reference's own calcSvd33 (SvdNew.hpp:24).
"""
import ctypes
import os

import numpy as np
import pytest

from nextgen_b200.meshgen import PeriodicBoxMesh

L = 2 * np.pi


def gcl(m, n, cv, nint):
    g = np.zeros((m.ncv, 3))
    np.add.at(g, cv[:, 0], n)
    np.add.at(g, cv[:nint, 1], -n[:nint])
    return np.abs(g).max() / m.h ** 2


@pytest.fixture(scope="module", params=[(8, 0.0), (10, 0.25), (12, 0.25)])
def mesh(request, built):
    n, jit = request.param
    return PeriodicBoxMesh(n, jitter=jit, seed=1234)


def test_lattice_counts(built):
    m = PeriodicBoxMesh(32, jitter=0.0)
    assert m.ncv == 32768
    assert m.f_per_cell == 3.0  # 6 compact faces per hex cell
    assert m.e_per_cell == 12.0  # 24 extended neighbours per cell
    assert m.n_threshold == 0
    assert np.allclose(m.vol_cv, (L / 32) ** 3, rtol=1e-12)


def test_volume_and_ghosts(mesh):
    m = mesh
    assert abs(m.vol_cv.sum() - L ** 3) < 1e-10 * L ** 3
    assert (m.vol_cv > 0).all()
    # ghosts are translated copies of their owners
    g = np.arange(m.ncv, m.ncv_g2)
    own = m.icv_owner_g
    assert ((own >= 0) & (own < m.ncv)).all()
    assert np.allclose(m.x_cv[g], m.x_cv[own] + m.shift_g * L, atol=1e-12)
    # internal faces: both cells owned; periodic faces: second cell a ghost
    assert (m.cvofa[: m.nfa_i] < m.ncv).all() and (m.cvofa[m.nfa_i:, 1] >= m.ncv).all()
    assert (m.cvoef[: m.nef_i] < m.ncv).all() and (m.cvoef[m.nef_i:, 1] >= m.ncv).all()
    assert (m.cvofa[m.nfa_i:, 1] < m.ncv_g).all()  # compact faces reach level-1 ghosts only


def test_gcl(mesh):
    m = mesh
    assert gcl(m, m.n_fa, m.cvofa, m.nfa_i) < 1e-13
    assert gcl(m, m.n_ef, m.cvoef, m.nef_i) < 1e-13


def test_linear_gradient_exactness(mesh):
    m = mesh
    G = np.array([1.1234, -1.3243, 1.5321])
    phi = m.x_cv @ G
    gp = np.zeros((m.ncv, 3))
    for icv in range(m.ncv):
        s, e = m.cvocv_i[icv], m.cvocv_i[icv + 1]
        assert m.cvocv_v[s] == icv  # diagonal first
        nb = m.cvocv_v[s + 1:e]
        gp[icv] = (m.cvocv_grad_coeff[s + 1:e] * (phi[nb] - phi[icv])[:, None]).sum(0)
    assert np.abs(gp / G - 1).max() < 1e-12
    # extended operator: sum 0.5 (n + c) (phi1 - phi0) = vol grad(phi)
    gp = np.zeros((m.ncv, 3))
    c0, c1 = m.cvoef[:, 0], m.cvoef[:, 1]
    d = (phi[c1] - phi[c0])[:, None]
    np.add.at(gp, c0, 0.5 * m.n_ef * d + 0.5 * m.c_ef * d)
    ii = slice(0, m.nef_i)
    np.add.at(gp, c1[ii], -(0.5 * m.n_ef[ii] * (-d[ii]) + 0.5 * m.c_ef[ii] * d[ii]))
    assert np.abs(gp / (m.vol_cv[:, None] * G) - 1).max() < 1e-12


def test_compact_faces_are_extended_faces(mesh):
    m = mesh
    ef = set(map(tuple, m.cvoef.tolist()))
    for a, b in m.cvofa.tolist():
        assert (a, b) in ef or (b, a) in ef


def test_area_over_delta(mesh):
    m = mesh
    c0, c1 = m.cvofa[:, 0], m.cvofa[:, 1]
    dx = m.x_cv[c1] - m.x_cv[c0]
    a2 = (m.n_fa ** 2).sum(1)
    ref = a2 / (dx * m.n_fa).sum(1)
    assert np.allclose(m.area_over_delta_fa, ref, rtol=1e-14)


def test_deterministic_across_thread_counts(built):
    a = PeriodicBoxMesh(9, jitter=0.25, seed=7, nthreads=1)
    b = PeriodicBoxMesh(9, jitter=0.25, seed=7, nthreads=4)
    for k in ("cvofa", "n_fa", "cvoef", "n_ef", "c_ef", "cvocv_grad_coeff", "vol_cv", "icv_owner_g"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_jittered_stencil_sizes(built):
    m = PeriodicBoxMesh(12, jitter=0.25, seed=1234)
    assert 6.5 < m.f_per_cell < 9.0
    assert 30.0 < m.e_per_cell < 50.0


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                                    "libref.so")), reason="reference-built oracle absent")
def test_grad_coeff_with_reference_svd(built):
    """Rebuild cvocv_grad_coeff (StaticSolver.cpp:5598-5765) with the
    reference's calcSvd33 and compare with the generator's own SVD."""
    from oracle import REF_LIB_PATH
    R = ctypes.CDLL(REF_LIB_PATH)
    dp = ctypes.POINTER(ctypes.c_double)
    R.orc_ref_svd33.argtypes = [dp, dp, dp, dp]
    m = PeriodicBoxMesh(7, jitter=0.25, seed=99)
    fa_of = {}
    for ifa, (a, b) in enumerate(m.cvofa.tolist()):
        fa_of.setdefault(a, []).append((ifa, 1.0, b))
        if ifa < m.nfa_i:
            fa_of.setdefault(b, []).append((ifa, -1.0, a))
    worst = 0.0
    for icv in range(m.ncv):
        s, e = m.cvocv_i[icv], m.cvocv_i[icv + 1]
        faces = sorted(fa_of[icv])
        gc = np.zeros((e - s, 3))
        A = np.zeros(9)
        for i in range(3):
            A[i * 3 + i] = m.vol_cv[icv]
        for k, (ifa, sg, nbr) in enumerate(faces):
            assert m.cvocv_v[s + 1 + k] == nbr
            r = m.x_fa[ifa] - 0.5 * (m.x_cv[icv] + m.x_cv[nbr])
            for j in range(3):
                for i in range(3):
                    A[j * 3 + i] -= r[j] * m.n_fa[ifa][i] * sg
            gc[k + 1] += 0.5 * m.n_fa[ifa] * sg
            gc[0] -= 0.5 * m.n_fa[ifa] * sg
        A /= m.vol_cv[icv]
        gc /= m.vol_cv[icv]
        U, V, sig = np.zeros(9), np.zeros(9), np.zeros(3)
        R.orc_ref_svd33(A.ctypes.data_as(dp), U.ctypes.data_as(dp), V.ctypes.data_as(dp), sig.ctypes.data_as(dp))
        sinv = np.where(sig < 0.45, 0.0, 1.0 / np.where(sig == 0, 1, sig))
        Vm = V.reshape(3, 3) * sinv[:, None]  # row j = column j of V
        Um = U.reshape(3, 3)
        Am = A.reshape(3, 3)  # Am[j][i] = A(i, j)
        for k in range(e - s):
            g = gc[k]
            b = Am.T @ g
            tmp = Um @ (g - b)
            gc[k] = g + Vm.T @ tmp
        worst = max(worst, np.abs(gc - m.cvocv_grad_coeff[s:e]).max() / np.abs(gc).max())
    assert worst < 1e-12, worst


def test_compact_only_is_the_generators_compact_part(built):
    """cgx_meshgen_periodic_box_compact returns the full generator's cells,
    compact faces and level-1 ghosts unchanged, and no operator arrays."""
    a = PeriodicBoxMesh(10, 9, 8, L=(1.0, 0.9, 0.8), jitter=0.3, seed=11)
    b = PeriodicBoxMesh(10, 9, 8, L=(1.0, 0.9, 0.8), jitter=0.3, seed=11, compact_only=True)
    assert (b.ncv, b.ncv_g, b.ncv_g2, b.nfa, b.nfa_i, b.nef) == (a.ncv, a.ncv_g, a.ncv_g, a.nfa, a.nfa_i, 0)
    for f in ("cvofa", "n_fa", "x_fa", "vol_cv", "x_vv"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    ng1 = a.ncv_g - a.ncv
    assert np.array_equal(a.x_cv[: a.ncv_g], b.x_cv)
    assert np.array_equal(a.icv_owner_g[:ng1], b.icv_owner_g)
    assert np.array_equal(a.shift_g[:ng1], b.shift_g)
    for f in ("cvocv_i", "cvocv_grad_coeff", "cvoef", "n_ef", "c_ef", "area_over_delta_fa", "dcmag_hat_cv"):
        assert getattr(b, f) is None, f


def test_compact_only_checks_arguments(built):
    for kw in (dict(nx=3), dict(nx=8, jitter=0.5), dict(nx=8, L=(1.0, 0.0, 1.0))):
        with pytest.raises(RuntimeError):
            PeriodicBoxMesh(compact_only=True, **kw)
