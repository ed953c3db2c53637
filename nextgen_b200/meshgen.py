"""Python access to the host mesh/operator generator (include/cgx_meshgen.h).

`PeriodicBoxMesh` owns one generated mesh.  Arrays are exposed as numpy views
on the generator's own buffers (no copies) for as long as the object lives;
`.ptr` is the raw `cgx_meshgen_out*` that the GPU library and the oracle take.
"""
import ctypes
import os

import numpy as np

from . import _lib

c_int_p = ctypes.POINTER(ctypes.c_int)
c_dbl_p = ctypes.POINTER(ctypes.c_double)


class MeshgenOut(ctypes.Structure):
    _fields_ = [
        ("ncv", ctypes.c_int), ("ncv_g", ctypes.c_int), ("ncv_g2", ctypes.c_int),
        ("nfa", ctypes.c_int), ("nfa_i", ctypes.c_int),
        ("nef", ctypes.c_int), ("nef_i", ctypes.c_int),
        ("n_threshold", ctypes.c_int),
        ("h", ctypes.c_double),
        ("cvofa", c_int_p), ("n_fa", c_dbl_p), ("x_fa", c_dbl_p),
        ("area_over_delta_fa", c_dbl_p),
        ("vol_cv", c_dbl_p), ("x_cv", c_dbl_p), ("x_vv", c_dbl_p),
        ("cvocv_i", c_int_p), ("cvocv_v", c_int_p), ("cvocv_grad_coeff", c_dbl_p),
        ("cvoef", c_int_p), ("n_ef", c_dbl_p), ("c_ef", c_dbl_p),
        ("cmag_cv", c_dbl_p), ("dcmag_hat_cv", c_dbl_p), ("sa_to_vol_ratio", c_dbl_p),
        ("icv_owner_g", c_int_p), ("shift_g", c_int_p),
        ("nbf", ctypes.c_int), ("nbf_zones", ctypes.c_int),
        ("cvobf", c_int_p), ("zone_bf", c_int_p), ("n_bf", c_dbl_p), ("x_bf", c_dbl_p),
        ("area_bf", c_dbl_p), ("area_over_delta_bf", c_dbl_p), ("Gij_bf", c_dbl_p),
    ]


def _load():
    lib = _lib.load("libcgx_meshgen.so")
    lib.cgx_meshgen_periodic_box.restype = ctypes.c_int
    lib.cgx_meshgen_periodic_box.argtypes = [
        ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_double, ctypes.c_double, ctypes.c_double,
        ctypes.c_double, ctypes.c_ulonglong, ctypes.c_double, ctypes.c_double,
        ctypes.c_int, ctypes.POINTER(ctypes.POINTER(MeshgenOut))]
    lib.cgx_meshgen_periodic_box_compact.restype = ctypes.c_int
    lib.cgx_meshgen_periodic_box_compact.argtypes = [
        ctypes.c_int, ctypes.c_int, ctypes.c_int,
        ctypes.c_double, ctypes.c_double, ctypes.c_double,
        ctypes.c_double, ctypes.c_ulonglong, ctypes.c_int, ctypes.POINTER(ctypes.POINTER(MeshgenOut))]
    for name in ("cgx_meshgen_channel", "cgx_meshgen_channel_compact"):
        f = getattr(lib, name)
        f.restype = ctypes.c_int
        f.argtypes = ([ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                       ctypes.c_double, ctypes.c_ulonglong] +
                      ([] if name.endswith("compact") else [ctypes.c_double, ctypes.c_double]) +
                      [ctypes.c_int, ctypes.POINTER(ctypes.POINTER(MeshgenOut))])
    lib.cgx_meshgen_free.restype = None
    lib.cgx_meshgen_free.argtypes = [ctypes.POINTER(MeshgenOut)]
    lib.cgx_meshgen_last_error.restype = ctypes.c_char_p
    lib.cgx_meshgen_last_error.argtypes = []
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _load()
    return _LIB


def _view(ptr, shape, dtype):
    if not ptr:
        return None
    n = int(np.prod(shape))
    if n == 0:
        return np.zeros(shape, dtype=dtype)
    ct = ctypes.c_int if dtype == np.int32 else ctypes.c_double
    buf = (ct * n).from_address(ctypes.addressof(ptr.contents))
    return np.frombuffer(buf, dtype=dtype).reshape(shape)


class PeriodicBoxMesh:
    """Voronoi mesh of an n^3 (jittered) lattice in a periodic box.

    Mirrors what the reference holds after StaticSolver::init() +
    FlowSolver::init() on one rank (see include/cgx_meshgen.h for the layout).
    """

    def __init__(self, nx, ny=None, nz=None, L=2.0 * np.pi, jitter=0.0, seed=1234,
                 interp_factor=1.0 / 3.0, sigma_thresh=0.45, nthreads=0, compact_only=False):
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        Ls = (L, L, L) if np.isscalar(L) else tuple(L)
        out = ctypes.POINTER(MeshgenOut)()
        if compact_only:
            # the mesher's part only (operators None): input of DeviceOperatorMesh
            rc = lib().cgx_meshgen_periodic_box_compact(int(nx), int(ny), int(nz), Ls[0], Ls[1], Ls[2],
                                                        float(jitter), int(seed), int(nthreads),
                                                        ctypes.byref(out))
        else:
            rc = lib().cgx_meshgen_periodic_box(int(nx), int(ny), int(nz), Ls[0], Ls[1], Ls[2],
                                                float(jitter), int(seed), float(interp_factor),
                                                float(sigma_thresh), int(nthreads),
                                                ctypes.byref(out))
        if rc != 0:
            raise RuntimeError("meshgen failed (%d): %s" % (rc, lib().cgx_meshgen_last_error().decode()))
        self._free = lib().cgx_meshgen_free
        self._attach(out, (int(nx), int(ny), int(nz)), Ls, float(jitter), int(seed))

    def _attach(self, out, dims, Ls, jitter, seed):
        self.ptr = out
        self.dims = dims
        self.L = Ls
        self.jitter = jitter
        self.seed = seed
        m = out.contents
        self.ncv, self.ncv_g, self.ncv_g2 = m.ncv, m.ncv_g, m.ncv_g2
        self.nfa, self.nfa_i, self.nef, self.nef_i = m.nfa, m.nfa_i, m.nef, m.nef_i
        self.n_threshold = m.n_threshold
        self.h = m.h
        ng = self.ncv_g2 - self.ncv
        self.cvofa = _view(m.cvofa, (self.nfa, 2), np.int32)
        self.n_fa = _view(m.n_fa, (self.nfa, 3), np.float64)
        self.x_fa = _view(m.x_fa, (self.nfa, 3), np.float64)
        self.area_over_delta_fa = _view(m.area_over_delta_fa, (self.nfa,), np.float64)
        self.vol_cv = _view(m.vol_cv, (self.ncv,), np.float64)
        self.x_cv = _view(m.x_cv, (self.ncv_g2, 3), np.float64)
        self.x_vv = _view(m.x_vv, (self.ncv, 3), np.float64) if m.x_vv else None
        self.cvocv_i = _view(m.cvocv_i, (self.ncv + 1,), np.int32)
        ncoc = int(self.cvocv_i[-1]) if self.cvocv_i is not None else 0
        self.cvocv_v = _view(m.cvocv_v, (ncoc,), np.int32)
        self.cvocv_grad_coeff = _view(m.cvocv_grad_coeff, (ncoc, 3), np.float64)
        self.cvoef = _view(m.cvoef, (self.nef, 2), np.int32)
        self.n_ef = _view(m.n_ef, (self.nef, 3), np.float64)
        self.c_ef = _view(m.c_ef, (self.nef, 3), np.float64)
        self.cmag_cv = _view(m.cmag_cv, (self.ncv,), np.float64)
        self.dcmag_hat_cv = _view(m.dcmag_hat_cv, (self.ncv,), np.float64)
        self.sa_to_vol_ratio = _view(m.sa_to_vol_ratio, (self.ncv,), np.float64)
        self.icv_owner_g = _view(m.icv_owner_g, (ng,), np.int32)
        self.shift_g = _view(m.shift_g, (ng, 3), np.int32)
        self.nbf, self.nbf_zones = m.nbf, m.nbf_zones
        self.cvobf = _view(m.cvobf, (self.nbf,), np.int32)
        self.zone_bf = _view(m.zone_bf, (self.nbf,), np.int32)
        self.n_bf = _view(m.n_bf, (self.nbf, 3), np.float64)
        self.x_bf = _view(m.x_bf, (self.nbf, 3), np.float64)
        self.area_bf = _view(m.area_bf, (self.nbf,), np.float64)
        self.area_over_delta_bf = _view(m.area_over_delta_bf, (self.nbf,), np.float64)
        self.Gij_bf = _view(m.Gij_bf, (self.nbf, 3, 3), np.float64)

    def owner(self, idx):
        """Owned cell of a cell-or-ghost index array."""
        idx = np.asarray(idx)
        out = idx.copy()
        g = idx >= self.ncv
        out[g] = self.icv_owner_g[idx[g] - self.ncv]
        return out

    @property
    def e_per_cell(self):
        """Extended faces per cell (each face counted once)."""
        return (self.nef_i + 0.5 * (self.nef - self.nef_i)) / self.ncv

    @property
    def f_per_cell(self):
        """Compact faces per cell (each face counted once)."""
        return (self.nfa_i + 0.5 * (self.nfa - self.nfa_i)) / self.ncv

    def close(self):
        if getattr(self, "ptr", None):
            self._free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ChannelMesh(PeriodicBoxMesh):
    """Voronoi mesh of an nx*ny*nz (jittered) lattice in a channel: periodic
    in x and z, walls at y = 0 (boundary zone 0) and y = Ly (zone 1)."""

    def __init__(self, nx, ny=None, nz=None, L=(2.0 * np.pi, 2.0, np.pi), jitter=0.0, seed=1234,
                 interp_factor=1.0 / 3.0, sigma_thresh=0.45, nthreads=0, compact_only=False):
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        Ls = (L, L, L) if np.isscalar(L) else tuple(float(v) for v in L)
        out = ctypes.POINTER(MeshgenOut)()
        if compact_only:
            rc = lib().cgx_meshgen_channel_compact(int(nx), int(ny), int(nz), Ls[0], Ls[1], Ls[2], float(jitter),
                                                   int(seed), int(nthreads), ctypes.byref(out))
        else:
            rc = lib().cgx_meshgen_channel(int(nx), int(ny), int(nz), Ls[0], Ls[1], Ls[2], float(jitter), int(seed),
                                           float(interp_factor), float(sigma_thresh), int(nthreads),
                                           ctypes.byref(out))
        if rc != 0:
            raise RuntimeError("meshgen failed (%d): %s" % (rc, lib().cgx_meshgen_last_error().decode()))
        self._free = lib().cgx_meshgen_free
        self._attach(out, (int(nx), int(ny), int(nz)), Ls, float(jitter), int(seed))


class CompactDesc(ctypes.Structure):
    """cgx_compact_desc (include/cgx_ops.h)."""
    _fields_ = [
        ("ncv", ctypes.c_int), ("ncv_g", ctypes.c_int), ("nfa", ctypes.c_int), ("nfa_i", ctypes.c_int),
        ("L", ctypes.c_double * 3), ("h", ctypes.c_double),
        ("cvofa", c_int_p), ("n_fa", c_dbl_p), ("x_fa", c_dbl_p), ("vol_cv", c_dbl_p),
        ("x_cv", c_dbl_p), ("x_vv", c_dbl_p), ("icv_owner_g", c_int_p), ("shift_g", c_int_p),
        ("nbf", ctypes.c_int), ("nbf_zones", ctypes.c_int),
        ("cvobf", c_int_p), ("zone_bf", c_int_p), ("n_bf", c_dbl_p), ("x_bf", c_dbl_p),
        ("area_bf", c_dbl_p), ("area_over_delta_bf", c_dbl_p), ("Gij_bf", c_dbl_p),
    ]


def _ops_lib():
    from . import cgx
    L = cgx.lib()
    if not getattr(L, "_ops_bound", False):
        L.cgx_operators_build.restype = ctypes.c_int
        L.cgx_operators_build.argtypes = [ctypes.POINTER(CompactDesc), ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, ctypes.POINTER(ctypes.POINTER(MeshgenOut)),
                                          ctypes.POINTER(ctypes.c_float)]
        L.cgx_operators_free.restype = None
        L.cgx_operators_free.argtypes = [ctypes.POINTER(MeshgenOut)]
        L._ops_bound = True
    return L


def compact_desc(mesh):
    """The compact part of a mesh (cells, compact faces, level-1 ghosts) as a
    cgx_compact_desc.  The arrays stay owned by `mesh`."""
    ng1 = mesh.ncv_g - mesh.ncv
    d = CompactDesc()
    d.ncv, d.ncv_g, d.nfa, d.nfa_i = mesh.ncv, mesh.ncv_g, mesh.nfa, mesh.nfa_i
    d.L[:] = [float(v) for v in mesh.L]
    d.h = mesh.h
    keep = []

    def ptr(a, ct, n=None):
        a = np.ascontiguousarray(a if n is None else a[:n])
        keep.append(a)
        return a.ctypes.data_as(ctypes.POINTER(ct))
    d.cvofa = ptr(mesh.cvofa, ctypes.c_int)
    d.n_fa = ptr(mesh.n_fa, ctypes.c_double)
    d.x_fa = ptr(mesh.x_fa, ctypes.c_double)
    d.vol_cv = ptr(mesh.vol_cv, ctypes.c_double)
    d.x_cv = ptr(mesh.x_cv, ctypes.c_double, mesh.ncv)
    d.x_vv = ptr(mesh.x_vv, ctypes.c_double) if mesh.x_vv is not None else None
    d.icv_owner_g = ptr(mesh.icv_owner_g, ctypes.c_int, ng1)
    d.shift_g = ptr(mesh.shift_g, ctypes.c_int, ng1)
    d.nbf = getattr(mesh, "nbf", 0) or 0
    d.nbf_zones = getattr(mesh, "nbf_zones", 0) or 0
    if d.nbf > 0:
        d.cvobf = ptr(mesh.cvobf, ctypes.c_int)
        d.Gij_bf = ptr(mesh.Gij_bf, ctypes.c_double)
        for f, ct in (("zone_bf", ctypes.c_int), ("n_bf", ctypes.c_double), ("x_bf", ctypes.c_double),
                      ("area_bf", ctypes.c_double), ("area_over_delta_bf", ctypes.c_double)):
            a = getattr(mesh, f, None)
            if a is not None:
                setattr(d, f, ptr(a, ct))
    d._keep = keep
    return d


class DeviceOperatorMesh(PeriodicBoxMesh):
    """A mesh whose operators (gradient coefficients, extended faces, level-2
    ghosts, per-cell factors) were built on the GPU by cgx_operators_build
    from another mesh's compact part.  Same attributes as PeriodicBoxMesh;
    `device_ms` is the device time of the build."""

    def __init__(self, source, device=0, interp_factor=1.0 / 3.0, sigma_thresh=0.45):
        L = _ops_lib()
        desc = compact_desc(source)
        out = ctypes.POINTER(MeshgenOut)()
        ms = ctypes.c_float()
        rc = L.cgx_operators_build(ctypes.byref(desc), float(interp_factor), float(sigma_thresh), int(device),
                                   ctypes.byref(out), ctypes.byref(ms))
        if rc != 0:
            from . import cgx
            raise cgx.CgxError(rc, L.cgx_last_error().decode())
        self.device_ms = ms.value
        self._free = L.cgx_operators_free
        self._attach(out, source.dims, source.L, source.jitter, source.seed)
