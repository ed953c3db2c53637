"""Generate the golden fixtures of tests/golden/ from the reference-built oracle.

The expected values come from oracle/_ref/libref.so: the oracle compiled with
the reference's own IdealGasSolverFlux.hpp, States.hpp and RkWeights.hpp (from
the reference source tree, in place).  Run from the repository root after
`make -C oracle ref`:

    python tests/golden/make_golden.py

Each fixture stores a fingerprint of the generated mesh, the initial
primitive state, calcRhs of stage 1 after initComplete with its conditioning
scale, the state after two RK3 steps at CFL 0.8 and the conserved totals.
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from nextgen_b200 import cases  # noqa: E402
from nextgen_b200.meshgen import PeriodicBoxMesh  # noqa: E402

CASES = {
    # name: (n, jitter, seed, kind)
    "tgv8_lattice": (8, 0.0, 1234, "tgv"),
    "tgv6_jitter": (6, 0.25, 1234, "tgv"),
    "hit8_jitter": (8, 0.25, 1235, "hit"),
}


def mesh_fingerprint(m):
    h = hashlib.sha256()
    for a in (m.cvofa, m.n_fa, m.area_over_delta_fa, m.vol_cv, m.cvocv_i, m.cvocv_v,
              m.cvocv_grad_coeff, m.cvoef, m.n_ef, m.c_ef, m.dcmag_hat_cv, m.sa_to_vol_ratio,
              m.icv_owner_g):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def case_setup(name):
    n, jit, seed, kind = CASES[name]
    m = PeriodicBoxMesh(n, jitter=jit, seed=seed)
    if kind == "tgv":
        prm = cases.tgv_params()
        rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    else:
        prm = cases.hit_params()
        rho, u, p = cases.hit_state(n, prm, k0=2.0, seed=4321)
    return m, prm, rho, u, p


def main():
    from oracle import Oracle, ref_available
    if not ref_available():
        sys.exit("oracle/_ref/libref.so not built: make -C oracle ref")
    for name in CASES:
        m, prm, rho, u, p = case_setup(name)
        o = Oracle(m, prm, nparts=1, reference=True)
        assert o.uses_reference_flux
        o.set_state_primitive(rho, u, p)
        o.init_complete()
        rhs, scale = o.calc_rhs(1)
        aux = o.aux()
        grad = o.grad()
        assert o.step(2) == 0
        r2, u2, e2 = o.get_state()
        t, dt, st = o.time()
        np.savez_compressed(os.path.join(HERE, name + ".npz"),
                            fingerprint=np.array(mesh_fingerprint(m)),
                            rho=rho, u=u, p=p, rhs=rhs, scale=scale, aux=aux, grad=grad,
                            rho2=r2, u2=u2, rhoE2=e2, time2=t, dt2=dt, totals2=o.totals())
        print(name, m.ncv, "cells, max|rhs|", np.abs(rhs).max(), "time", t)


if __name__ == "__main__":
    main()
