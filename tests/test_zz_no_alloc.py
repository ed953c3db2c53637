"""cgx_totals_noalloc: the report() totals for callers that cannot allocate
device memory (their buffers come from another allocator), with the
reduction's scratch in a static device array instead of an allocation.

Checked through the C ABI against the allocating entry point cgx_totals on
the same state, twice in a row (the second call reuses the static scratch
the first one left behind), at the 1e-13 relative tolerance the totals
tests use elsewhere (the two reductions group the sums differently).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_totals_noalloc_matches_allocating_totals(built):
    import torch
    from nextgen_b200 import cases, cgx
    from nextgen_b200.meshgen import PeriodicBoxMesh

    L = cgx.lib()
    f = L.cgx_totals_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]

    m = PeriodicBoxMesh(24, jitter=0.25, seed=5)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    s = cgx.Solver(cgx.Mesh(m), prm)
    s.set_state_primitive(rho, u, p)
    s.initComplete()
    assert s.step(3) == 0
    ref = s.totals()  # allocating path (solver's own partials buffer)
    r, uu, e = s.get_state()

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    d_rho = torch.tensor(r, device=dev)
    d_u = torch.tensor(uu.reshape(-1), device=dev)
    d_e = torch.tensor(e, device=dev)
    d_v = torch.tensor(np.array(m.vol_cv), device=dev)
    out = torch.zeros(5, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    norm = np.array([np.abs(r * m.vol_cv).sum()] + [(r * np.abs(uu).sum(1) * m.vol_cv).sum()] * 3 +
                    [np.abs(e * m.vol_cv).sum()])
    for _ in range(2):
        out.zero_()
        rc = f(m.ncv, d_rho.data_ptr(), d_u.data_ptr(), d_e.data_ptr(), d_v.data_ptr(), out.data_ptr(),
               ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.cgx_last_error()
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy()
        assert (np.abs(got - ref) / norm).max() <= 1e-13

    # sizes beyond the stated maximum are refused before any GPU work
    rc = f(16_777_217, d_rho.data_ptr(), d_u.data_ptr(), d_e.data_ptr(), d_v.data_ptr(), out.data_ptr(), None)
    assert rc == -1 and b"exceed the maximum" in L.cgx_last_error()
    # a null array is refused too
    rc = f(m.ncv, None, d_u.data_ptr(), d_e.data_ptr(), d_v.data_ptr(), out.data_ptr(), None)
    assert rc == -1 and b"null" in L.cgx_last_error()

    # n = 0: one block of zero partials, totals zero (the scratch still holds
    # the previous call's partials, which must not leak into the result)
    out.fill_(7.0)
    assert f(0, None, None, None, None, out.data_ptr(), ctypes.c_void_p(stream.cuda_stream)) == 0
    torch.cuda.synchronize(dev)
    assert (out.cpu().numpy() == 0.0).all()

    # n = 2049: one cell past a whole block of 2048, against a numpy sum
    n = 2049
    rng = np.random.default_rng(3)
    hr, hu, he, hv = rng.uniform(0.5, 2, n), rng.uniform(-1, 1, (n, 3)), rng.uniform(1, 3, n), rng.uniform(0.1, 1, n)
    tr, tu, te, tv = (torch.tensor(a.reshape(-1), device=dev) for a in (hr, hu, he, hv))
    want = np.array([(hr * hv).sum()] + [(hr * hu[:, k] * hv).sum() for k in range(3)] + [(he * hv).sum()])
    wnorm = np.array([(hr * hv).sum()] + [(hr * np.abs(hu[:, k]) * hv).sum() for k in range(3)] + [(he * hv).sum()])
    for _ in range(2):
        out.zero_()
        assert f(n, tr.data_ptr(), tu.data_ptr(), te.data_ptr(), tv.data_ptr(), out.data_ptr(),
                 ctypes.c_void_p(stream.cuda_stream)) == 0
        torch.cuda.synchronize(dev)
        assert (np.abs(out.cpu().numpy() - want) / wnorm).max() <= 1e-13
