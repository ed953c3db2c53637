"""The device reciprocal of the flux kernels (Newton-Raphson iteration from
the hardware approximation) against IEEE 1.0/x, over the arguments the
kernels give it: sums of two specific volumes 1/rho (the face density
2/(v0+v1) of calcInternalFluxNew, IdealGasSolverFlux.hpp:23) and mean sound
speeds (the face Mach number of calcInternalCompactFluxNewGrad,
IdealGasSolverFlux.hpp:146).  Bound: 1 ulp."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ulps(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def test_rcp_within_one_ulp(built):
    from nextgen_b200 import cgx
    L = cgx.lib()
    f = L.cgx_selftest_rcp
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    rng = np.random.default_rng(11)
    # densities 1e-3 .. 1e3 (sums of two specific volumes) and sound speeds
    # 1e-2 .. 1e4, log-uniform, plus powers of two and their neighbours
    rho = np.exp(rng.uniform(np.log(1e-3), np.log(1e3), (200000, 2)))
    v_sum = (1.0 / rho).sum(1)
    sos = np.exp(rng.uniform(np.log(1e-2), np.log(1e4), 200000))
    p2 = 2.0 ** np.arange(-20, 21, dtype=np.float64)
    edges = np.concatenate([p2, np.nextafter(p2, 0), np.nextafter(p2, np.inf)])
    x = np.ascontiguousarray(np.concatenate([v_sum, sos, edges]))
    out = np.empty_like(x)
    assert f(0, x.ctypes.data, out.ctypes.data, x.size) == 0, L.cgx_last_error()
    ref = 1.0 / x
    u = _ulps(out, ref)
    assert u.max() <= 1, "max %d ulp at x=%r" % (u.max(), x[u.argmax()])
