"""Host-side mirror of the reference solver interface over the C ABI
(include/cgx.h).

`Solver` exposes the reference's IdealGasSolver hot-path calls under their
reference names (calcRhs, rk3Step, updateConservativeAndPrimitiveData,
calcSgsAndMaterialProperties, calcCfl, advanceSolution, setDt-driven stepping,
report() totals) on top of libcgx.so, with host numpy arrays in the caller's
cell order.  Errors from the library raise `CgxError` carrying the library's
message; there is no fallback path: without libcgx.so or a GPU the calls fail.
"""
import ctypes

import numpy as np

from . import _lib

c_int_p = ctypes.POINTER(ctypes.c_int)
c_dbl_p = ctypes.POINTER(ctypes.c_double)

CGX_FP64 = 0
CGX_MIXED = 1

ERRORS = {-1: "CGX_E_ARG", -2: "CGX_E_OOM", -3: "CGX_E_CUDA", -4: "CGX_E_NAN",
          -5: "CGX_E_TIMEOUT", -6: "CGX_E_STATE"}


class CgxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "?"), code, msg))
        self.code = code


class Params(ctypes.Structure):
    """cgx_params: solver parameters named after the reference's input keys."""
    _fields_ = [
        ("gamma", ctypes.c_double), ("p_ref", ctypes.c_double), ("rho_ref", ctypes.c_double),
        ("T_ref", ctypes.c_double), ("mu_ref", ctypes.c_double),
        ("mu_power_law", ctypes.c_double), ("Pr_lam", ctypes.c_double),
        ("sgs_model", ctypes.c_int),
        ("vreman_coeff", ctypes.c_double), ("a_sgs_coeff", ctypes.c_double),
        ("a_sgs_coeff2", ctypes.c_double), ("lambda_dil_coeff", ctypes.c_double),
        ("Pr_t", ctypes.c_double),
        ("coeff_p", ctypes.c_double), ("coeff_h", ctypes.c_double), ("gr_nrm", ctypes.c_double),
        ("diss_mode", ctypes.c_int), ("dt_mode", ctypes.c_int),
        ("dt_data", ctypes.c_double * 2), ("check_interval", ctypes.c_int),
        ("limit_asgs", ctypes.c_int),
    ]

    def __init__(self, **kw):
        super().__init__()
        # reference defaults (IdealGasSolver.hpp:147-155, IdealGasSolverSgs.cpp:209-213,
        # IdealGasSolver.cpp:202-203,904)
        self.gamma = 1.4
        self.p_ref = 1.0
        self.rho_ref = 1.0
        self.T_ref = 1.0
        self.mu_ref = 1.0
        self.mu_power_law = 0.75
        self.Pr_lam = 0.7
        self.sgs_model = 0
        self.vreman_coeff = 0.07
        self.a_sgs_coeff = 0.05
        self.a_sgs_coeff2 = 0.0015
        self.lambda_dil_coeff = 0.0
        self.Pr_t = 0.9
        self.coeff_p = 0.5
        self.coeff_h = 0.1
        self.gr_nrm = 0.03
        self.diss_mode = 0
        self.dt_mode = 1
        self.dt_data[0] = 0.8
        self.dt_data[1] = 0.0
        self.check_interval = 1
        self.limit_asgs = 0
        for k, v in kw.items():
            setattr(self, k, v)

    def copy(self):
        p = Params()
        ctypes.pointer(p)[0] = self
        return p


class MeshDesc(ctypes.Structure):
    """cgx_mesh_desc: the reference's single-rank mesh arrays."""
    _fields_ = [
        ("ncv", ctypes.c_int), ("ncv_g2", ctypes.c_int), ("nfa", ctypes.c_int), ("nef", ctypes.c_int),
        ("cvofa", c_int_p), ("n_fa", c_dbl_p), ("area_over_delta_fa", c_dbl_p),
        ("vol_cv", c_dbl_p), ("cvocv_i", c_int_p), ("cvocv_v", c_int_p),
        ("cvocv_grad_coeff", c_dbl_p), ("cvoef", c_int_p), ("n_ef", c_dbl_p), ("c_ef", c_dbl_p),
        ("dcmag_hat_cv", c_dbl_p), ("sa_to_vol_ratio", c_dbl_p), ("icv_owner_g", c_int_p),
        ("x_cv", c_dbl_p),
        ("nbf", ctypes.c_int), ("nbf_zones", ctypes.c_int), ("cvobf", c_int_p), ("n_bf", c_dbl_p),
        ("area_over_delta_bf", c_dbl_p), ("zone_bf", c_int_p),
    ]


def _p(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def mesh_desc(mesh, with_x=True):
    """cgx_mesh_desc over the arrays of a PeriodicBoxMesh (or any object with
    the same attribute names).  The arrays must outlive the descriptor."""
    d = MeshDesc()
    d.ncv, d.ncv_g2, d.nfa, d.nef = mesh.ncv, mesh.ncv_g2, mesh.nfa, mesh.nef
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a
    d.cvofa = _p(arr(mesh.cvofa, np.int32), ctypes.c_int)
    d.n_fa = _p(arr(mesh.n_fa, np.float64), ctypes.c_double)
    d.area_over_delta_fa = _p(arr(mesh.area_over_delta_fa, np.float64), ctypes.c_double)
    d.vol_cv = _p(arr(mesh.vol_cv, np.float64), ctypes.c_double)
    d.cvocv_i = _p(arr(mesh.cvocv_i, np.int32), ctypes.c_int)
    d.cvocv_v = _p(arr(mesh.cvocv_v, np.int32), ctypes.c_int)
    d.cvocv_grad_coeff = _p(arr(mesh.cvocv_grad_coeff, np.float64), ctypes.c_double)
    d.cvoef = _p(arr(mesh.cvoef, np.int32), ctypes.c_int)
    d.n_ef = _p(arr(mesh.n_ef, np.float64), ctypes.c_double)
    d.c_ef = _p(arr(mesh.c_ef, np.float64), ctypes.c_double)
    d.dcmag_hat_cv = _p(arr(mesh.dcmag_hat_cv, np.float64), ctypes.c_double)
    d.sa_to_vol_ratio = _p(arr(mesh.sa_to_vol_ratio, np.float64), ctypes.c_double)
    d.icv_owner_g = _p(arr(mesh.icv_owner_g, np.int32), ctypes.c_int)
    d.x_cv = _p(arr(mesh.x_cv[: mesh.ncv], np.float64), ctypes.c_double) if with_x else None
    nbf = int(getattr(mesh, "nbf", 0) or 0)
    if nbf > 0:
        d.nbf, d.nbf_zones = nbf, int(mesh.nbf_zones)
        d.cvobf = _p(arr(mesh.cvobf, np.int32), ctypes.c_int)
        d.n_bf = _p(arr(mesh.n_bf, np.float64), ctypes.c_double)
        d.area_over_delta_bf = _p(arr(mesh.area_over_delta_bf, np.float64), ctypes.c_double)
        d.zone_bf = _p(arr(mesh.zone_bf, np.int32), ctypes.c_int)
    d._keep = keep
    return d


class MeshStats(ctypes.Structure):
    _fields_ = [("ncv", ctypes.c_int), ("n_ef_dir", ctypes.c_longlong),
                ("n_cf_dir", ctypes.c_longlong), ("e_per_cell", ctypes.c_double),
                ("f_per_cell", ctypes.c_double), ("device_bytes", ctypes.c_size_t)]


EXPORTS = [
    "cgx_params_default", "cgx_mesh_create", "cgx_mesh_stats_get", "cgx_mesh_destroy",
    "cgx_solver_create", "cgx_solver_destroy", "cgx_set_state", "cgx_set_state_primitive",
    "cgx_get_state", "cgx_init_complete", "cgx_update_primitive", "cgx_calc_sgs_props",
    "cgx_calc_rhs", "cgx_rk3_step", "cgx_calc_cfl", "cgx_advance_solution", "cgx_step",
    "cgx_get_time", "cgx_totals", "cgx_get_primitive", "cgx_get_grad", "cgx_get_aux",
    "cgx_synchronize", "cgx_launch_count", "cgx_last_error", "cgx_step_timed", "cgx_kernel_times", "cgx_get_tuning",
    "cgx_set_scalars", "cgx_get_scalars", "cgx_get_rhs_sc", "cgx_step_profiled", "cgx_set_time",
    "cgx_set_source", "cgx_set_source_hook", "cgx_set_bc", "cgx_set_bc_params", "cgx_set_host_threads",
    "cgx_set_bc_profile", "cgx_set_frame_rotation", "cgx_step_out", "cgx_set_bc_face_velocity",
    "cgx_set_bc_exchange",
]

CGX_BC_SLIP = 1
CGX_BC_WALL_ADIABATIC = 2
CGX_BC_WALL_ISOTHERMAL = 3
CGX_BC_CBC_UPT = 4
CGX_BC_CBC_RUNP = 5
CGX_BC_CBC_MPT = 6
CGX_BC_CBC_EXTRAPOLATE = 7
CGX_BC_CBC_TOTAL_PT = 8
CGX_BC_NSCBC_MT = 9
CGX_BC_NSCBC_OUTLET_P = 10
CGX_BC_NSCBC_OUTLET_MDOT = 11
CGX_BC_CBC_RUP = 12
CGX_BC_WALL_CONDUCTIVE = 13
CGX_BC_SPONGE = 14
CGX_BC_WM_ALG_ADIABATIC = 15
CGX_BC_WM_ALG_ISOTHERMAL = 16
CGX_BC_WM_ALG_CONDUCTIVE = 17
CGX_BC_CBC_PROFILE = 18
CGX_BC_WM_EQ_ADIABATIC = 19
CGX_BC_WM_EQ_ISOTHERMAL = 20
CGX_BC_HOOK = 21
CGX_BC_WM_EXCHANGE_ADIABATIC = 22
CGX_BC_WM_EXCHANGE_ISOTHERMAL = 23


class Source(ctypes.Structure):
    """cgx_source: per-cell force f = vol rho (A u + g) and an optional field."""
    _fields_ = [("A", ctypes.c_double), ("g", ctypes.c_double * 3), ("field", ctypes.POINTER(ctypes.c_double))]


# cgx_source_hook: (user, ncv, rho, u, rhoE, rhs, time, rk_stage)
SOURCE_HOOK = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.c_int)

_LIB = None


def lib():
    """libcgx.so with argument types declared."""
    global _LIB
    if _LIB is not None:
        return _LIB
    L = _lib.load("libcgx.so")
    vp = ctypes.c_void_p
    sig = {
        "cgx_params_default": (None, [ctypes.POINTER(Params)]),
        "cgx_mesh_create": (ctypes.c_int, [ctypes.POINTER(MeshDesc), ctypes.c_int, ctypes.POINTER(vp)]),
        "cgx_mesh_stats_get": (ctypes.c_int, [vp, ctypes.POINTER(MeshStats)]),
        "cgx_mesh_destroy": (ctypes.c_int, [vp]),
        "cgx_solver_create": (ctypes.c_int, [vp, ctypes.POINTER(Params), ctypes.c_int, ctypes.POINTER(vp)]),
        "cgx_solver_destroy": (ctypes.c_int, [vp]),
        "cgx_set_state": (ctypes.c_int, [vp, c_dbl_p, c_dbl_p, c_dbl_p]),
        "cgx_set_state_primitive": (ctypes.c_int, [vp, c_dbl_p, c_dbl_p, c_dbl_p]),
        "cgx_get_state": (ctypes.c_int, [vp, c_dbl_p, c_dbl_p, c_dbl_p]),
        "cgx_init_complete": (ctypes.c_int, [vp]),
        "cgx_update_primitive": (ctypes.c_int, [vp]),
        "cgx_calc_sgs_props": (ctypes.c_int, [vp]),
        "cgx_calc_rhs": (ctypes.c_int, [vp, c_dbl_p, ctypes.c_double, ctypes.c_int]),
        "cgx_rk3_step": (ctypes.c_int, [vp, c_dbl_p, ctypes.c_double, ctypes.c_int]),
        "cgx_calc_cfl": (ctypes.c_int, [vp, ctypes.c_double, c_dbl_p, c_dbl_p]),
        "cgx_advance_solution": (ctypes.c_int, [vp]),
        "cgx_step": (ctypes.c_int, [vp, ctypes.c_int]),
        "cgx_get_time": (ctypes.c_int, [vp, c_dbl_p, c_dbl_p, c_int_p]),
        "cgx_set_time": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int]),
        "cgx_totals": (ctypes.c_int, [vp, c_dbl_p]),
        "cgx_get_primitive": (ctypes.c_int, [vp, c_dbl_p, c_dbl_p, c_dbl_p]),
        "cgx_get_grad": (ctypes.c_int, [vp, c_dbl_p]),
        "cgx_get_aux": (ctypes.c_int, [vp, c_dbl_p]),
        "cgx_synchronize": (ctypes.c_int, [vp]),
        "cgx_launch_count": (ctypes.c_longlong, [vp]),
        "cgx_last_error": (ctypes.c_char_p, []),
        "cgx_step_timed": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
        "cgx_kernel_times": (ctypes.c_int, [vp, ctypes.c_int, c_dbl_p]),
        "cgx_step_profiled": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float), c_dbl_p]),
        "cgx_get_tuning": (ctypes.c_int, [vp, c_int_p]),
        "cgx_set_scalars": (ctypes.c_int, [vp, ctypes.c_int, c_dbl_p]),
        "cgx_set_source": (ctypes.c_int, [vp, ctypes.POINTER(Source)]),
        "cgx_set_bc": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, c_dbl_p]),
        "cgx_set_bc_params": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, c_dbl_p, ctypes.c_int]),
        "cgx_set_bc_profile": (ctypes.c_int, [vp, ctypes.c_int, c_dbl_p, ctypes.c_int]),
        "cgx_set_frame_rotation": (ctypes.c_int, [vp, c_dbl_p, c_dbl_p]),
        "cgx_step_out": (ctypes.c_int, [vp, ctypes.c_int, c_dbl_p, c_dbl_p, c_dbl_p]),
        "cgx_set_bc_face_velocity": (ctypes.c_int, [vp, ctypes.c_int, c_dbl_p, ctypes.c_int]),
        "cgx_set_bc_exchange": (ctypes.c_int, [vp, ctypes.c_int, c_int_p, c_dbl_p, ctypes.c_int]),
        "cgx_set_host_threads": (ctypes.c_int, [ctypes.c_int]),
        "cgx_set_source_hook": (ctypes.c_int, [vp, SOURCE_HOOK, vp]),
        "cgx_get_scalars": (ctypes.c_int, [vp, c_dbl_p]),
        "cgx_get_rhs_sc": (ctypes.c_int, [vp, ctypes.c_int, c_dbl_p]),
        "cgx_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_size_t,
                                             ctypes.POINTER(vp)]),
        "cgx_batch_destroy": (ctypes.c_int, [vp]),
        "cgx_batch_add": (ctypes.c_int, [vp, vp, ctypes.POINTER(Params), c_dbl_p, c_dbl_p, c_dbl_p,
                                          ctypes.c_int, c_int_p]),
        "cgx_batch_step": (ctypes.c_int, [vp, ctypes.c_int, c_int_p]),
        "cgx_batch_prepare": (ctypes.c_int, [vp, vp, ctypes.POINTER(Params), c_dbl_p, c_dbl_p, c_dbl_p,
                                              ctypes.c_int, ctypes.POINTER(vp)]),
        "cgx_batch_admit": (ctypes.c_int, [vp, vp, c_int_p]),
        "cgx_batch_case_release": (ctypes.c_int, [vp]),
        "cgx_batch_done": (ctypes.c_int, [vp, c_int_p, ctypes.c_int, c_int_p]),
        "cgx_batch_get_state": (ctypes.c_int, [vp, ctypes.c_int, c_dbl_p, c_dbl_p, c_dbl_p]),
        "cgx_batch_get_time": (ctypes.c_int, [vp, ctypes.c_int, c_dbl_p, c_dbl_p, c_int_p]),
        "cgx_batch_remove": (ctypes.c_int, [vp, ctypes.c_int]),
        "cgx_batch_bytes": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
        "cgx_batch_launch_count": (ctypes.c_longlong, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _LIB = L
    return L


def _check(rc):
    if rc != 0:
        raise CgxError(rc, lib().cgx_last_error().decode())
    return rc


def set_host_threads(n):
    """Host threads for the calling thread's later parallel host phases
    (mesh set-up); n <= 0 restores all cores.  Other threads are unaffected."""
    _check(lib().cgx_set_host_threads(int(n)))


def _out(n, *shape):
    return np.empty((n,) + shape, dtype=np.float64)


def _dp(a):
    return None if a is None else a.ctypes.data_as(c_dbl_p)


class Mesh:
    """Device copy of a mesh (cgx_mesh_create)."""

    def __init__(self, mesh, device=0, sfc=True):
        self.desc = mesh_desc(mesh, with_x=sfc)
        self.ncv = mesh.ncv
        h = ctypes.c_void_p()
        _check(lib().cgx_mesh_create(ctypes.byref(self.desc), int(device), ctypes.byref(h)))
        self.h = h

    def stats(self):
        st = MeshStats()
        _check(lib().cgx_mesh_stats_get(self.h, ctypes.byref(st)))
        return st

    def close(self):
        if self.h:
            lib().cgx_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """IdealGasSolver hot path on the GPU (cgx_solver_*)."""

    def __init__(self, mesh, params, precision=CGX_FP64):
        self.mesh = mesh
        self.ncv = mesh.ncv
        self.params = params
        h = ctypes.c_void_p()
        _check(lib().cgx_solver_create(mesh.h, ctypes.byref(params), int(precision), ctypes.byref(h)))
        self.h = h

    # -- state ------------------------------------------------------------
    def set_state(self, rho, u, rhoE):
        rho, u, rhoE = (np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, rhoE))
        _check(lib().cgx_set_state(self.h, _dp(rho), _dp(u), _dp(rhoE)))

    def set_state_primitive(self, rho, u, p):
        rho, u, p = (np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, p))
        _check(lib().cgx_set_state_primitive(self.h, _dp(rho), _dp(u), _dp(p)))

    def get_state(self):
        rho, u, rhoE = _out(self.ncv), _out(self.ncv, 3), _out(self.ncv)
        _check(lib().cgx_get_state(self.h, _dp(rho), _dp(u), _dp(rhoE)))
        return rho, u, rhoE

    # -- passive transport scalars (transport_scalar_vec) ---------------------
    def set_scalars(self, sc):
        """Transport scalars sc[ncv][nsc] (nsc <= 8, both precisions); from now
        on calcRhs forms rhs_sc (calcRhsScalars) and the steps advance them
        (advanceScalars).  An empty second axis removes them."""
        sc = np.ascontiguousarray(sc, dtype=np.float64).reshape(self.ncv, -1)
        _check(lib().cgx_set_scalars(self.h, int(sc.shape[1]), _dp(sc) if sc.size else None))
        self.nsc = sc.shape[1]

    def get_scalars(self):
        sc = _out(self.ncv, getattr(self, "nsc", 0))
        _check(lib().cgx_get_scalars(self.h, _dp(sc)))
        return sc

    def rhs_sc(self, rk_stage=1):
        """rhs_sc[ncv][nsc] of a stage (unscaled face sums)."""
        out = _out(self.ncv, getattr(self, "nsc", 0))
        _check(lib().cgx_get_rhs_sc(self.h, int(rk_stage), _dp(out)))
        return out

    # -- boundary conditions (registerBoundaryConditions) ----------------------
    def set_bc(self, zone, kind, u_wall=None):
        """Boundary condition of boundary zone `zone`: CGX_BC_SLIP or
        CGX_BC_WALL_ADIABATIC (u_wall: the wall velocity, zero if None)."""
        uw = None if u_wall is None else np.ascontiguousarray(u_wall, dtype=np.float64)
        _check(lib().cgx_set_bc(self.h, int(zone), int(kind), _dp(uw)))

    def set_bc_params(self, zone, kind, params=()):
        """Boundary condition with the reference's zone parameters in input
        order: WALL_ISOTHERMAL (T), CBC_UPT (u0 u1 u2 p T), CBC_RUNP
        (rho un p), CBC_MPT (mdot p T), CBC_EXTRAPOLATE (none), CBC_TOTAL_PT
        (p_total T_total t_relax [use_avg]), NSCBC_MT (mdot T; T < 0: the
        total temperature -T), NSCBC_OUTLET_P (p_ref sigma L_ref),
        NSCBC_OUTLET_MDOT (mdot t_relax), CBC_RUP (rho u0 u1 u2 p),
        WALL_CONDUCTIVE (T_end [L k]...), SPONGE (type strength t_relax
        length p_sponge L_max; the mesh needs x_cv), WM_ALG_ADIABATIC
        ([u_wall]), WM_ALG_ISOTHERMAL (T), WM_ALG_CONDUCTIVE (T_end [L k]...),
        WM_EQ_ADIABATIC ([u_wall [relax y_plus0 tol]]), WM_EQ_ISOTHERMAL (T
        [relax y_plus0 tol]), HOOK (none: the flux comes from the source
        hook);
        SLIP and
        WALL_ADIABATIC as set_bc."""
        a = np.ascontiguousarray(params, dtype=np.float64).reshape(-1)
        _check(lib().cgx_set_bc_params(self.h, int(zone), int(kind), _dp(a) if a.size else None, int(a.size)))

    def set_bc_profile(self, zone, states):
        """CBC_PROFILE zone: states[nz][6] = u0 u1 u2 sp_vol p h of each of the
        zone's faces, in the order the mesh lists them (the reference's
        bf_state after CbcProfile::initData)."""
        a = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 6)
        _check(lib().cgx_set_bc_profile(self.h, int(zone), _dp(a), int(a.shape[0])))

    def set_bc_face_velocity(self, zone, u):
        """A velocity face by face, u[nz][3], the zone's faces in the order
        the mesh lists them: an adiabatic wall's velocity, or CBC_TOTAL_PT's
        frame velocity (STATIONARY_FRAME: -w x x_bf)."""
        a = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 3)
        _check(lib().cgx_set_bc_face_velocity(self.h, int(zone), _dp(a), int(a.shape[0])))

    def set_bc_exchange(self, zone, cv, x):
        """A WM_EXCHANGE zone's exchange points: the cells that hold them
        cv[nz] (reference numbering, -1 where not located) and the points
        x[nz][3], the zone's faces in the order the mesh lists them."""
        c = np.ascontiguousarray(cv, dtype=np.int32).reshape(-1)
        a = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        _check(lib().cgx_set_bc_exchange(self.h, int(zone), c.ctypes.data_as(c_int_p), _dp(a), int(c.size)))

    def set_frame_rotation(self, rev, x_cv):
        """ROTATING_REFERENCE_FRAME: rev[3] in revolutions per unit time, the
        cell centroids x_cv[ncv][3] in reference order; zeros remove it."""
        r = np.ascontiguousarray(rev, dtype=np.float64).reshape(3)
        x = np.ascontiguousarray(np.asarray(x_cv)[: self.ncv], dtype=np.float64).reshape(self.ncv, 3)
        _check(lib().cgx_set_frame_rotation(self.h, _dp(r), _dp(x)))

    # -- source terms (addSourceHook) ----------------------------------------
    def set_source(self, A=0.0, g=(0.0, 0.0, 0.0), field=None):
        """Device-side source of every stage: f = vol rho (A u + g) into rhou,
        f.u into rhoE, plus field[ncv][5] (reference order) if given.  All
        zero / None removes it."""
        src = Source()
        src.A = float(A)
        src.g = (ctypes.c_double * 3)(*[float(x) for x in g])
        f = None
        if field is not None:
            f = np.ascontiguousarray(field, dtype=np.float64).reshape(self.ncv, 5)
            src.field = _dp(f)
        _check(lib().cgx_set_source(self.h, ctypes.byref(src)))

    def set_source_hook(self, fn):
        """Host hook of every stage with addSourceHook's contract:
        fn(rho[ncv], u[ncv,3], rhoE[ncv], rhs[ncv,5], time, rk_stage) adds to
        rhs (zero on entry); the arrays are views of the library's
        page-locked copies, valid during the call.  fn runs on a CUDA host
        thread and must not call the library.  None removes it."""
        if fn is None:
            _check(lib().cgx_set_source_hook(self.h, SOURCE_HOOK(), None))
            self._hook = None
            return

        def thunk(user, ncv, rho, u, rhoE, rhs, time, stage):
            n = int(ncv)
            fn(np.ctypeslib.as_array(rho, (n,)), np.ctypeslib.as_array(u, (n, 3)),
               np.ctypeslib.as_array(rhoE, (n,)), np.ctypeslib.as_array(rhs, (n, 5)), float(time), int(stage))
        cb = SOURCE_HOOK(thunk)
        _check(lib().cgx_set_source_hook(self.h, cb, None))
        self._hook = cb  # the callback must outlive the solver's use of it

    # -- reference calls ----------------------------------------------------
    def initComplete(self):
        _check(lib().cgx_init_complete(self.h))

    def updateConservativeAndPrimitiveData(self):
        _check(lib().cgx_update_primitive(self.h))

    def calcSgsAndMaterialProperties(self):
        _check(lib().cgx_calc_sgs_props(self.h))

    def calcRhs(self, rk_stage=1, time=0.0, copy_out=True):
        out = _out(self.ncv, 5) if copy_out else None
        _check(lib().cgx_calc_rhs(self.h, _dp(out), float(time), int(rk_stage)))
        return out

    def rk3Step(self, rk_wgt, dt, rk_stage):
        w = np.ascontiguousarray(rk_wgt, dtype=np.float64)
        _check(lib().cgx_rk3_step(self.h, _dp(w), float(dt), int(rk_stage)))

    def calcCfl(self, dt=1.0, want_cells=False):
        mx = ctypes.c_double()
        cfl = _out(self.ncv) if want_cells else None
        _check(lib().cgx_calc_cfl(self.h, float(dt), ctypes.byref(mx), _dp(cfl)))
        return (mx.value, cfl) if want_cells else mx.value

    def advanceSolution(self):
        """0, or -1 after a NaN (state restored, dt_data[0] scaled by 0.8)."""
        rc = lib().cgx_advance_solution(self.h)
        if rc == -4:
            return -1
        _check(rc)
        return 0

    def step(self, nsteps):
        """nsteps of setDt + advanceSolution; 0 or -1 after a NaN."""
        rc = lib().cgx_step(self.h, int(nsteps))
        if rc == -4:
            return -1
        _check(rc)
        return 0

    def time(self):
        t, dt, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _check(lib().cgx_get_time(self.h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st)))
        return t.value, dt.value, st.value

    def set_time(self, time, step):
        """Restart at (time, step): cgx_set_time."""
        _check(lib().cgx_set_time(self.h, float(time), int(step)))

    def write_sles(self, path, params=""):
        """The current state, step and time as a .sles result file
        (writeSles, StaticSolver.hpp:2311-2321), cells in the mesh's order."""
        from .mles import write_sles
        rho, u, rhoE = self.get_state()
        t, _, step = self.time()
        write_sles(path, rho, u, rhoE, step, t, params)

    def read_sles(self, path):
        """Restart from a .sles file: its state, then its time and step."""
        from .mles import read_sles
        rho, u, rhoE, step, t = read_sles(path, self.ncv)
        self.set_state(rho, u, rhoE)
        self.set_time(t, step)

    def totals(self):
        out = np.empty(5)
        _check(lib().cgx_totals(self.h, _dp(out)))
        return out

    def primitive(self):
        p, T, sos = _out(self.ncv), _out(self.ncv), _out(self.ncv)
        _check(lib().cgx_get_primitive(self.h, _dp(p), _dp(T), _dp(sos)))
        return p, T, sos

    def grad(self):
        g = _out(self.ncv, 3, 3)
        _check(lib().cgx_get_grad(self.h, _dp(g)))
        return g

    def aux(self):
        a = _out(self.ncv, 6)
        _check(lib().cgx_get_aux(self.h, _dp(a)))
        return a

    def step_timed(self, nsteps):
        """Run nsteps; return their device time in ms (CUDA events on the
        solver's stream)."""
        ms = ctypes.c_float()
        _check(lib().cgx_step_timed(self.h, int(nsteps), ctypes.byref(ms)))
        return float(ms.value)

    def step_profiled(self, nsteps):
        """Run nsteps; return (device ms of the steps, {rhs, ext, comp}: the
        face kernels' average launch time in ms, timed inside the steps)."""
        ms = ctypes.c_float()
        f = np.zeros(3)
        _check(lib().cgx_step_profiled(self.h, int(nsteps), ctypes.byref(ms), _dp(f)))
        return float(ms.value), dict(zip(("rhs", "ext", "comp"), f.tolist()))

    def kernel_times(self, reps=5):
        """Average ms per launch of {rhs (both face kernels), rk+prim, grad,
        step_end, ext (extended-face kernel), comp (compact closures)}."""
        ms = np.zeros(6)
        _check(lib().cgx_kernel_times(self.h, int(reps), _dp(ms)))
        return dict(zip(("rhs", "rk_prim", "grad", "step_end", "ext", "comp"), ms.tolist()))

    def tuning(self):
        """Lanes per cell picked by the autotuner: ext, comp, grad, step_end."""
        t = (ctypes.c_int * 4)()
        _check(lib().cgx_get_tuning(self.h, t))
        return dict(zip(("ext", "comp", "grad", "step_end"), list(t)))

    def set_state_ptr(self, rho_ptr, u_ptr, rhoE_ptr):
        """cgx_set_state from raw host pointers (e.g. pinned buffers)."""
        _check(lib().cgx_set_state(self.h, ctypes.cast(rho_ptr, c_dbl_p), ctypes.cast(u_ptr, c_dbl_p),
                                   ctypes.cast(rhoE_ptr, c_dbl_p)))

    def get_state_ptr(self, rho_ptr, u_ptr, rhoE_ptr):
        _check(lib().cgx_get_state(self.h, ctypes.cast(rho_ptr, c_dbl_p), ctypes.cast(u_ptr, c_dbl_p),
                                   ctypes.cast(rhoE_ptr, c_dbl_p)))

    def step_out_ptr(self, nsteps, rho_ptr, u_ptr, rhoE_ptr):
        """cgx_step_out: nsteps, then the state into the host arrays at these
        addresses, its copy beside the step's last kernels (pageable arrays
        through the library's pinned chunks).  Returns 0, or -1 after a NaN
        (state restored)."""
        rc = lib().cgx_step_out(self.h, int(nsteps), ctypes.cast(rho_ptr, c_dbl_p), ctypes.cast(u_ptr, c_dbl_p),
                                ctypes.cast(rhoE_ptr, c_dbl_p))
        if rc == -4:
            return -1
        _check(rc)
        return 0

    def synchronize(self):
        _check(lib().cgx_synchronize(self.h))

    def launch_count(self):
        return int(lib().cgx_launch_count(self.h))

    def close(self):
        if self.h:
            lib().cgx_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PreparedCase:
    """A case built by Batch.prepare(), not yet admitted."""

    def __init__(self, h, mesh):
        self.h = h
        self.mesh = mesh

    def release(self):
        if self.h:
            lib().cgx_batch_case_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class Batch:
    """Resident cases advanced together (cgx_batch_*): continuous batching.

    add() admits a case (returns its id, or None when the HBM budget is
    full), step() advances every active case, done() lists finished cases,
    get_state()/remove() retire them."""

    def __init__(self, device=0, precision=CGX_FP64, max_cases=256, hbm_budget=64 << 30):
        h = ctypes.c_void_p()
        _check(lib().cgx_batch_create(int(device), int(precision), int(max_cases), int(hbm_budget),
                                      ctypes.byref(h)))
        self.h = h
        self.precision = precision
        self.ncv = {}
        self._meshes = {}

    def add(self, mesh, params, rho, u, p, nsteps):
        rho, u, p = (np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, p))
        cid = ctypes.c_int()
        rc = lib().cgx_batch_add(self.h, mesh.h, ctypes.byref(params), _dp(rho), _dp(u), _dp(p),
                                 int(nsteps), ctypes.byref(cid))
        if rc == -2:
            return None
        _check(rc)
        self.ncv[cid.value] = mesh.ncv
        self._meshes[cid.value] = mesh
        return cid.value

    def prepare(self, mesh, params, rho, u, p, nsteps):
        """A case built for this batch but not in it yet (cgx_batch_prepare):
        safe to call from another thread while the batch steps.  Returns a
        handle for admit()."""
        rho, u, p = (np.ascontiguousarray(a, dtype=np.float64) for a in (rho, u, p))
        h = ctypes.c_void_p()
        _check(lib().cgx_batch_prepare(self.h, mesh.h, ctypes.byref(params), _dp(rho), _dp(u), _dp(p),
                                       int(nsteps), ctypes.byref(h)))
        return PreparedCase(h, mesh)

    def admit(self, case):
        """Join a prepared case between steps; its id, or None (and the case
        stays prepared) when the HBM budget or the slots are full."""
        cid = ctypes.c_int()
        rc = lib().cgx_batch_admit(self.h, case.h, ctypes.byref(cid))
        if rc == -2:
            return None
        _check(rc)
        case.h = None  # owned by the batch now
        self.ncv[cid.value] = case.mesh.ncv
        self._meshes[cid.value] = case.mesh
        return cid.value

    def step(self, nsteps):
        n = ctypes.c_int()
        _check(lib().cgx_batch_step(self.h, int(nsteps), ctypes.byref(n)))
        return n.value

    def done(self):
        n = ctypes.c_int()
        _check(lib().cgx_batch_done(self.h, None, 0, ctypes.byref(n)))
        ids = (ctypes.c_int * max(n.value, 1))()
        _check(lib().cgx_batch_done(self.h, ids, n.value, ctypes.byref(n)))
        return list(ids)[: n.value]

    def get_state(self, cid):
        n = self.ncv[cid]
        rho, u, rhoE = _out(n), _out(n, 3), _out(n)
        _check(lib().cgx_batch_get_state(self.h, int(cid), _dp(rho), _dp(u), _dp(rhoE)))
        return rho, u, rhoE

    def time(self, cid):
        t, dt, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _check(lib().cgx_batch_get_time(self.h, int(cid), ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st)))
        return t.value, dt.value, st.value

    def remove(self, cid):
        _check(lib().cgx_batch_remove(self.h, int(cid)))
        self.ncv.pop(cid, None)
        self._meshes.pop(cid, None)

    def bytes(self):
        u, b = ctypes.c_size_t(), ctypes.c_size_t()
        _check(lib().cgx_batch_bytes(self.h, ctypes.byref(u), ctypes.byref(b)))
        return u.value, b.value

    def launch_count(self):
        return int(lib().cgx_batch_launch_count(self.h))

    def close(self):
        if self.h:
            lib().cgx_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
