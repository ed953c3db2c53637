"""cgx_step_profiled advances exactly as cgx_step does (the timing events
recorded in its step graph change nothing) and reports positive face-kernel
times, the pair's being the sum of the two kernels'."""
import numpy as np
import pytest

from nextgen_b200 import cases, cgx
from nextgen_b200.meshgen import PeriodicBoxMesh

pytestmark = pytest.mark.gpu


def test_profiled_steps_equal_plain_steps(built):
    m = PeriodicBoxMesh(12, jitter=0.25, seed=1234)
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    gm = cgx.Mesh(m, device=0)
    out = []
    for profiled in (False, True):
        s = cgx.Solver(gm, prm)
        s.set_state_primitive(rho, u, p)
        s.initComplete()
        if profiled:
            ms, face = s.step_profiled(4)
            assert ms > 0 and face["ext"] > 0 and face["comp"] > 0
            assert abs(face["rhs"] - face["ext"] - face["comp"]) <= 1e-9 * face["rhs"] + 1e-12
        else:
            assert s.step(4) == 0
        out.append(s.get_state())
        assert s.time()[2] == 4
        s.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)
