"""Caller host arrays of both kinds through the C ABI.  Page-locked arrays
are copied directly; pageable ones (a host solver's new[] arrays) of 4 MiB or
more go through the library's pinned staging chunks.  Both must give the
same bits, in and out, for the state, the rhs and the scalars.

A 96^3 box (884,736 cells) makes every state array large enough to be
staged, and several 64 MiB chunks long.
"""
import numpy as np
import pytest
import torch

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import PeriodicBoxMesh

pytestmark = pytest.mark.gpu


def _pinned(shape):
    return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()


def test_pageable_and_pinned_agree(built):
    m = PeriodicBoxMesh(96, jitter=0.25, seed=17)
    N = m.ncv
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(np.array(m.x_cv[:N]), prm)
    s = cgx.Solver(cgx.Mesh(m, device=0), prm)
    s.set_state_primitive(rho, u, p)  # pageable in
    s.initComplete()
    r0, u0, e0 = s.get_state()  # pageable out
    rp, up, ep = _pinned(N), _pinned((N, 3)), _pinned(N)
    s.get_state_ptr(rp.ctypes.data, up.ctypes.data, ep.ctypes.data)  # pinned out
    assert np.array_equal(r0, rp) and np.array_equal(u0, up) and np.array_equal(e0, ep)
    assert np.array_equal(r0, rho)
    # pinned in, pageable out: the round trip is exact
    s.set_state_ptr(rp.ctypes.data, up.ctypes.data, ep.ctypes.data)
    r1, u1, e1 = s.get_state()
    assert np.array_equal(r1, r0) and np.array_equal(u1, u0) and np.array_equal(e1, e0)
    # pageable in again, after a step: same as pinned in
    assert s.step(2) == 0
    r2, u2, e2 = s.get_state()
    s.set_state(r2, u2, e2)
    r3, u3, e3 = s.get_state()
    assert np.array_equal(r3, r2) and np.array_equal(u3, u2) and np.array_equal(e3, e2)
    # the rhs (5N doubles, several chunks) into pageable memory
    s.initComplete()
    rhs = s.calcRhs(1)
    assert rhs.shape == (N, 5) and np.isfinite(rhs).all()
    s.close()
