"""cgx_step_out: steps, then the state in the caller's host arrays, the copy
of page-locked arrays running beside the last step's gradient and step-end
kernels.  The arrays must equal cgx_step + cgx_get_state bit for bit, for
page-locked and pageable arrays, over one and several steps, and after a
NaN they hold the restored state with the NaN code returned.
"""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import PeriodicBoxMesh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(built):
    m = PeriodicBoxMesh(20, jitter=0.25, seed=21)
    prm = cases.tgv_params()
    st = cases.tgv_state(m.x_cv[: m.ncv], prm)
    return m, prm, st, cgx.Mesh(m, device=0)


def _solver(setup):
    m, prm, st, gm = setup
    s = cgx.Solver(gm, prm)
    s.set_state_primitive(*st)
    s.initComplete()
    return s


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("nsteps", [1, 3])
def test_step_out_equals_step_then_get_state(setup, pinned, nsteps):
    import torch
    m = setup[0]
    n = m.ncv
    a, b = _solver(setup), _solver(setup)
    for _ in range(2):
        assert a.step(nsteps) == 0
        want = a.get_state()
        if pinned:
            bufs = [torch.empty(k, dtype=torch.float64, pin_memory=True) for k in (n, 3 * n, n)]
            ptrs = [t.data_ptr() for t in bufs]
        else:
            bufs = [np.empty(k) for k in (n, 3 * n, n)]
            ptrs = [x.ctypes.data for x in bufs]
        assert b.step_out_ptr(nsteps, *ptrs) == 0
        got = [np.asarray(t.numpy() if pinned else t) for t in bufs]
        assert np.array_equal(got[0], want[0])
        assert np.array_equal(got[1].reshape(n, 3), want[1])
        assert np.array_equal(got[2], want[2])
        assert a.time() == b.time()
    a.close()
    b.close()


def test_step_out_after_a_nan_holds_the_restored_state(setup):
    import torch
    m = setup[0]
    n = m.ncv
    s = _solver(setup)
    bad = [x.copy() for x in s.get_state()]
    bad[0][7] = np.nan
    s.set_state(*bad)
    s.updateConservativeAndPrimitiveData()
    bufs = [torch.empty(k, dtype=torch.float64, pin_memory=True) for k in (n, 3 * n, n)]
    assert s.step_out_ptr(1, *[t.data_ptr() for t in bufs]) == -1
    want = s.get_state()
    assert np.isfinite(bufs[0].numpy()).all()
    assert np.array_equal(bufs[0].numpy(), want[0])
    assert np.array_equal(bufs[2].numpy(), want[2])
    s.close()
