"""The operator build on the GPU (cgx_operators_build, include/cgx_ops.h)
against the host generator, through the C ABI.

Both builds restate the same reference functions (calcCvGradCoeff,
StaticSolver.cpp:5598-5765; buildExtendedFaces with EF_OPS DEFAULT,
StripedMesh.hpp:5269-6960; the FlowSolver.hpp:702-760, 859-878 factors) and
evaluate them in the same order without multiply-add contraction, so every
array must agree bit for bit: the index arrays and the ghost numbering
exactly, the coefficients to the last bit.  A solver on the device-built mesh
then gives the same rhs as one on the host-built mesh.
"""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import DeviceOperatorMesh, PeriodicBoxMesh, compact_desc

pytestmark = pytest.mark.gpu

FIELDS = ["cvocv_i", "cvocv_v", "cvocv_grad_coeff", "cvoef", "n_ef", "c_ef", "area_over_delta_fa",
          "cmag_cv", "dcmag_hat_cv", "sa_to_vol_ratio", "x_cv", "icv_owner_g", "shift_g",
          "cvofa", "n_fa", "x_fa", "vol_cv", "x_vv"]

MESHES = [
    dict(nx=12, jitter=0.25, seed=1234),
    dict(nx=16, ny=12, nz=10, L=(1.0, 0.8, 0.7), jitter=0.3, seed=99),
    dict(nx=20, jitter=0.0),
    dict(nx=32, ny=32, nz=6, L=(10.0, 10.0, 1.875), jitter=0.25, seed=1234),
    dict(nx=24, jitter=0.3, seed=7, interp_factor=0.25, sigma_thresh=0.9),  # 9111 cells thresholded
    dict(nx=8, ny=8, nz=4, L=(1.0, 1.0, 0.5), jitter=0.25, seed=3),  # thinnest box the generator makes
    dict(nx=4, jitter=0.2, seed=5),  # 64 cells: most faces periodic
]


def _id(kw):
    return "-".join("%s%s" % (k, v) for k, v in kw.items())


@pytest.mark.parametrize("kw", MESHES, ids=_id)
def test_device_build_equals_host(built, kw):
    opts = {k: kw[k] for k in ("interp_factor", "sigma_thresh") if k in kw}
    host = PeriodicBoxMesh(**kw)
    dev = DeviceOperatorMesh(host, device=0, **opts)
    for a in ("ncv", "ncv_g", "ncv_g2", "nfa", "nfa_i", "nef", "nef_i", "n_threshold"):
        assert getattr(dev, a) == getattr(host, a), a
    for f in FIELDS:
        a, b = getattr(dev, f), getattr(host, f)
        assert a.shape == b.shape, f
        assert np.array_equal(a, b), (f, int((a != b).sum()), float(np.abs(a - b).max()))
    assert dev.device_ms > 0.0
    dev.close()


def test_from_the_mesher_alone(built):
    """The pipeline a served mesh takes: the mesher's compact output
    (cgx_meshgen_periodic_box_compact) -> cgx_operators_build gives the full
    host generator's mesh."""
    kw = dict(nx=18, ny=14, nz=12, L=(1.2, 0.9, 0.8), jitter=0.25, seed=21)
    full = PeriodicBoxMesh(**kw)
    dev = DeviceOperatorMesh(PeriodicBoxMesh(compact_only=True, **kw))
    assert (dev.ncv_g2, dev.nef, dev.nef_i) == (full.ncv_g2, full.nef, full.nef_i)
    for f in FIELDS:
        assert np.array_equal(getattr(dev, f), getattr(full, f)), f


def test_solver_on_device_built_mesh(built):
    host = PeriodicBoxMesh(14, jitter=0.25, seed=5)
    dev = DeviceOperatorMesh(host)
    prm = cases.tgv_params()
    x = np.array(host.x_cv[: host.ncv])
    rho, u, p = cases.tgv_state(x, prm)
    out = []
    for m in (host, dev):
        s = cgx.Solver(cgx.Mesh(m, device=0), prm)
        s.set_state_primitive(rho, u, p)
        s.initComplete()
        r = s.calcRhs(1)
        assert s.step(5) == 0
        out.append((r, s.get_state()))
        s.close()
    assert np.array_equal(out[0][0], out[1][0])
    for a, b in zip(out[0][1], out[1][1]):
        assert np.array_equal(a, b)


def test_inconsistent_compact_mesh_rejected(built):
    """Out-of-range cells in the compact faces are caught by the build's own
    range checks (no kernel indexes with them) and reported as CGX_E_ARG."""
    import ctypes
    from nextgen_b200.meshgen import _ops_lib, MeshgenOut
    host = PeriodicBoxMesh(8, jitter=0.2)
    d = compact_desc(host)
    bad = np.array(host.cvofa, copy=True)
    bad[3, 1] = host.ncv + 10 ** 6  # an internal face pointing past every cell
    d.cvofa = bad.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    L = _ops_lib()
    out = ctypes.POINTER(MeshgenOut)()
    rc = L.cgx_operators_build(ctypes.byref(d), 1.0 / 3.0, 0.45, 0, ctypes.byref(out), None)
    assert rc == -1 and not out  # CGX_E_ARG
    assert b"inconsistent" in L.cgx_last_error()
