"""ctypes access to the CPU oracle (oracle.h).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the package.

`Oracle(mesh, params, nparts, reference=False)` wraps liboracle.so (restated
face fluxes); reference=True wraps _ref/libref.so (the reference's own
IdealGasSolverFlux.hpp compiled in place), when it has been built.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libref.so")

c_dbl_p = ctypes.POINTER(ctypes.c_double)
c_int_p = ctypes.POINTER(ctypes.c_int)

_libs = {}


def ref_available():
    return os.path.exists(REF_LIB_PATH)


def _load(path):
    if path in _libs:
        return _libs[path]
    from nextgen_b200.cgx import MeshDesc, Params
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    sig = {
        "orc_create": (vp, [ctypes.POINTER(MeshDesc), ctypes.POINTER(Params), ctypes.c_int]),
        "orc_destroy": (None, [vp]),
        "orc_set_state": (None, [vp, c_dbl_p, c_dbl_p, c_dbl_p]),
        "orc_set_state_primitive": (None, [vp, c_dbl_p, c_dbl_p, c_dbl_p]),
        "orc_get_state": (None, [vp, c_dbl_p, c_dbl_p, c_dbl_p]),
        "orc_init_complete": (None, [vp]),
        "orc_update_primitive": (None, [vp]),
        "orc_calc_sgs_props": (None, [vp]),
        "orc_calc_rhs": (None, [vp, ctypes.c_int, c_dbl_p, c_dbl_p]),
        "orc_rk3_step": (None, [vp, c_dbl_p, ctypes.c_double, ctypes.c_int]),
        "orc_set_scalars": (ctypes.c_int, [vp, ctypes.c_int, c_dbl_p]),
        "orc_get_scalars": (None, [vp, c_dbl_p]),
        "orc_get_rhs_sc": (None, [vp, ctypes.c_int, c_dbl_p, c_dbl_p]),
        "orc_calc_cfl": (ctypes.c_double, [vp, ctypes.c_double, c_dbl_p]),
        "orc_set_dt": (ctypes.c_double, [vp]),
        "orc_advance_solution": (ctypes.c_int, [vp]),
        "orc_step": (ctypes.c_int, [vp, ctypes.c_int]),
        "orc_totals": (None, [vp, c_dbl_p]),
        "orc_get_time": (None, [vp, c_dbl_p, c_dbl_p, c_int_p]),
        "orc_get_primitive": (None, [vp, c_dbl_p, c_dbl_p, c_dbl_p]),
        "orc_get_grad": (None, [vp, c_dbl_p]),
        "orc_get_aux": (None, [vp, c_dbl_p]),
        "orc_poison": (None, [vp, ctypes.c_int]),
        "orc_set_source": (None, [vp, ctypes.c_double, c_dbl_p, c_dbl_p]),
        "orc_set_bc": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, c_dbl_p]),
        "orc_set_bc_params": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, c_dbl_p, ctypes.c_int]),
        "orc_uses_reference_flux": (ctypes.c_int, []),
        "orc_wm_solve_tau": (ctypes.c_double, [ctypes.c_double] * 5),
        "orc_wm_q_wall": (ctypes.c_double, [ctypes.c_double] * 8),
        "orc_wm_r_approx": (ctypes.c_double, [ctypes.c_double] * 6),
        "orc_set_bc_profile": (ctypes.c_int, [vp, ctypes.c_int, c_dbl_p, ctypes.c_int]),
        "orc_wm_eq_solve": (ctypes.c_int, [c_dbl_p] + [ctypes.c_double] * 10),
        "orc_set_frame_rotation": (ctypes.c_int, [vp, c_dbl_p]),
        "orc_set_bc_face_velocity": (ctypes.c_int, [vp, ctypes.c_int, c_dbl_p, ctypes.c_int]),
        "orc_set_bc_exchange": (ctypes.c_int, [vp, ctypes.c_int, c_int_p, c_dbl_p, ctypes.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _libs[path] = L
    return L


def wm_solve_tau(u1, y1, rho, mu, ut_guess=-1.0, reference=False):
    """The algebraic wall model's tau_wall (AlgebraicWM::solve_tau): the
    restatement, or the reference header's own with reference=True."""
    return _load(REF_LIB_PATH if reference else LIB_PATH).orc_wm_solve_tau(u1, y1, rho, mu, ut_guess)


def wm_q_wall(T1, Tw, tau, rho, mu, locp, cp, y1, reference=False):
    """The algebraic wall model's wall heat flux (compute_q_wall_approx)."""
    return _load(REF_LIB_PATH if reference else LIB_PATH).orc_wm_q_wall(T1, Tw, tau, rho, mu, locp, cp, y1)


def wm_r_approx(tau, rho, mu, locp, cp, y1, reference=False):
    """The algebraic wall model's near-wall thermal resistance (compute_R_approx)."""
    return _load(REF_LIB_PATH if reference else LIB_PATH).orc_wm_r_approx(tau, rho, mu, locp, cp, y1)


def wm_eq_solve(tau, q, T_w, u1, T1, rho1, y1, mu1, Pr_lam, cp, relax=0.7, y_plus0=1.0, tol=1e-4,
                reference=False):
    """The equilibrium wall model (EquilibriumWM::solve_qt with its guesses):
    returns (status, tau, q, T_w); T_w < 0 asks for the adiabatic form."""
    a = np.array([tau, q, T_w], dtype=np.float64)
    rc = _load(REF_LIB_PATH if reference else LIB_PATH).orc_wm_eq_solve(
        _dp(a), u1, T1, rho1, y1, mu1, Pr_lam, cp, relax, y_plus0, tol)
    return rc, a[0], a[1], a[2]


def _dp(a):
    return None if a is None else a.ctypes.data_as(c_dbl_p)


class Oracle:
    def __init__(self, mesh, params, nparts=1, reference=False):
        from nextgen_b200.cgx import mesh_desc
        path = REF_LIB_PATH if reference else LIB_PATH
        if not os.path.exists(path):
            raise OSError("%s not built (make -C oracle%s)" % (path, " ref" if reference else ""))
        self.L = _load(path)
        self.desc = mesh_desc(mesh)  # x_cv: for a sponge layer's cells
        self.params = params
        self.ncv = mesh.ncv
        self.h = self.L.orc_create(ctypes.byref(self.desc), ctypes.byref(params), int(nparts))
        if not self.h:
            raise RuntimeError("orc_create failed")
        self.uses_reference_flux = bool(self.L.orc_uses_reference_flux())

    def set_state(self, rho, u, rhoE):
        rho, u, rhoE = (np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, rhoE))
        self.L.orc_set_state(self.h, _dp(rho), _dp(u), _dp(rhoE))

    def set_state_primitive(self, rho, u, p):
        rho, u, p = (np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, p))
        self.L.orc_set_state_primitive(self.h, _dp(rho), _dp(u), _dp(p))

    def get_state(self):
        n = self.ncv
        rho, u, rhoE = np.empty(n), np.empty((n, 3)), np.empty(n)
        self.L.orc_get_state(self.h, _dp(rho), _dp(u), _dp(rhoE))
        return rho, u, rhoE

    def init_complete(self):
        self.L.orc_init_complete(self.h)

    def update_primitive(self):
        self.L.orc_update_primitive(self.h)

    def calc_sgs_props(self):
        self.L.orc_calc_sgs_props(self.h)

    def calc_rhs(self, rk_stage=1, want_scale=True):
        rhs = np.empty((self.ncv, 5))
        scale = np.empty((self.ncv, 5)) if want_scale else None
        self.L.orc_calc_rhs(self.h, int(rk_stage), _dp(rhs), _dp(scale))
        return (rhs, scale) if want_scale else rhs

    def set_scalars(self, sc):
        """Transport scalars sc[ncv][nsc] (calcRhsScalars / advanceScalars)."""
        sc = np.ascontiguousarray(sc, dtype=np.float64).reshape(self.ncv, -1)
        self.nsc = sc.shape[1]
        if self.L.orc_set_scalars(self.h, int(self.nsc), _dp(sc)) != 0:
            raise ValueError("orc_set_scalars failed")

    def get_scalars(self):
        sc = np.empty((self.ncv, getattr(self, "nsc", 0)))
        if sc.size:
            self.L.orc_get_scalars(self.h, _dp(sc))
        return sc

    def rhs_sc(self, rk_stage=1, want_scale=True):
        """rhs_sc[ncv][nsc] (and its conditioning scale) of the last calc_rhs."""
        nsc = getattr(self, "nsc", 0)
        r = np.empty((self.ncv, nsc))
        sc = np.empty((self.ncv, nsc)) if want_scale else None
        self.L.orc_get_rhs_sc(self.h, int(rk_stage), _dp(r), _dp(sc))
        return (r, sc) if want_scale else r

    def rk3_step(self, w, dt, stage):
        w = np.ascontiguousarray(w, dtype=np.float64)
        self.L.orc_rk3_step(self.h, _dp(w), float(dt), int(stage))

    def calc_cfl(self, dt=1.0):
        cfl = np.empty(self.ncv)
        mx = self.L.orc_calc_cfl(self.h, float(dt), _dp(cfl))
        return mx, cfl

    def set_dt(self):
        return self.L.orc_set_dt(self.h)

    def advance_solution(self):
        return self.L.orc_advance_solution(self.h)

    def step(self, n):
        return self.L.orc_step(self.h, int(n))

    def totals(self):
        out = np.empty(5)
        self.L.orc_totals(self.h, _dp(out))
        return out

    def time(self):
        t, dt, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self.L.orc_get_time(self.h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st))
        return t.value, dt.value, st.value

    def primitive(self):
        n = self.ncv
        p, T, sos = np.empty(n), np.empty(n), np.empty(n)
        self.L.orc_get_primitive(self.h, _dp(p), _dp(T), _dp(sos))
        return p, T, sos

    def grad(self):
        g = np.empty((self.ncv, 3, 3))
        self.L.orc_get_grad(self.h, _dp(g))
        return g

    def aux(self):
        a = np.empty((self.ncv, 6))
        self.L.orc_get_aux(self.h, _dp(a))
        return a

    def set_source(self, A=0.0, g=(0.0, 0.0, 0.0), field=None):
        """Source terms after the face sums (a subclass's addSourceHook):
        f = vol rho (A u + g) into rhou, f.u into rhoE, plus field[ncv][5]."""
        gg = np.ascontiguousarray(g, dtype=np.float64)
        f = None if field is None else np.ascontiguousarray(field, dtype=np.float64).reshape(self.ncv, 5)
        self.L.orc_set_source(self.h, float(A), _dp(gg), _dp(f))

    def set_bc(self, zone, kind, u_wall=None):
        """Boundary condition of a boundary zone (CGX_BC_SLIP = 1,
        CGX_BC_WALL_ADIABATIC = 2; u_wall zero if None)."""
        uw = None if u_wall is None else np.ascontiguousarray(u_wall, dtype=np.float64)
        if self.L.orc_set_bc(self.h, int(zone), int(kind), _dp(uw)) != 0:
            raise ValueError("orc_set_bc: bad zone or kind")

    def set_bc_params(self, zone, kind, params=()):
        """Boundary condition with the reference's zone parameters:
        WALL_ISOTHERMAL (T) = 3, CBC_UPT (u0 u1 u2 p T) = 4, CBC_RUNP
        (rho un p) = 5, CBC_MPT (mdot p T) = 6."""
        a = np.ascontiguousarray(params, dtype=np.float64).reshape(-1)
        if self.L.orc_set_bc_params(self.h, int(zone), int(kind), _dp(a) if a.size else None, int(a.size)) != 0:
            raise ValueError("orc_set_bc_params: bad zone, kind or parameters")

    def set_bc_profile(self, zone, states):
        """CBC_PROFILE: states[nz][6] = u0 u1 u2 sp_vol p h of the zone's faces."""
        a = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 6)
        if self.L.orc_set_bc_profile(self.h, int(zone), _dp(a), int(a.shape[0])) != 0:
            raise ValueError("orc_set_bc_profile: bad zone or face count")

    def set_bc_face_velocity(self, zone, u):
        """A velocity face by face, u[nz][3]: an adiabatic wall's or
        CBC_TOTAL_PT's frame velocity."""
        a = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 3)
        if self.L.orc_set_bc_face_velocity(self.h, int(zone), _dp(a), int(a.shape[0])) != 0:
            raise ValueError("orc_set_bc_face_velocity: bad zone, kind or face count")

    def set_bc_exchange(self, zone, cv, x):
        """A WM_EXCHANGE zone's exchange points: cells cv[nz] (-1: not located), points x[nz][3]."""
        c = np.ascontiguousarray(cv, dtype=np.int32).reshape(-1)
        a = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        if self.L.orc_set_bc_exchange(self.h, int(zone), c.ctypes.data_as(c_int_p), _dp(a), int(c.size)) != 0:
            raise ValueError("orc_set_bc_exchange: bad zone, kind, cells or face count")

    def set_frame_rotation(self, rev):
        """ROTATING_REFERENCE_FRAME: the rate in revolutions per unit time."""
        a = np.ascontiguousarray(rev, dtype=np.float64).reshape(3)
        if self.L.orc_set_frame_rotation(self.h, _dp(a)) != 0:
            raise ValueError("orc_set_frame_rotation: the mesh's x_cv is needed")

    def poison(self, icv):
        self.L.orc_poison(self.h, int(icv))

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
