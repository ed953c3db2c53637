"""Python access to the .mles reader (include/cgx_mles.h).

`MlesMesh(path)` holds one file's mesh; its arrays are numpy views on the
reader's buffers (None where the file has no such record) for as long as the
object lives.  Names follow the reference's StripedMesh members
(src/core/common/StripedMesh.hpp): x_no, cvofa, noofa_i/v, n_fa, x_fa, cvobf,
noobf_i/v, n_bf, x_bf, area_bf, area_over_delta_bf, Gij_bf, vol_cv, r_vv,
x_vv, x_cv, and the boundary zones.
"""
import ctypes

import numpy as np

from .meshgen import lib as _meshgen_lib

c_int_p = ctypes.POINTER(ctypes.c_int)
c_dbl_p = ctypes.POINTER(ctypes.c_double)

ERRORS = {-1: "CGX_MLES_E_IO", -2: "CGX_MLES_E_FORMAT", -3: "CGX_MLES_E_UNSUPPORTED", -4: "CGX_MLES_E_OOM"}


class BfZone(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 52), ("nbf", ctypes.c_longlong), ("ibf_f", ctypes.c_longlong),
                ("area", ctypes.c_double), ("area_over_delta", ctypes.c_double),
                ("n", ctypes.c_double * 3), ("x", ctypes.c_double * 3)]


class Mles(ctypes.Structure):
    _fields_ = [
        ("io_version", ctypes.c_int),
        ("nno", ctypes.c_longlong), ("nbf", ctypes.c_longlong), ("nfa", ctypes.c_longlong),
        ("ncv", ctypes.c_longlong), ("nno_p", ctypes.c_longlong), ("nno_pb", ctypes.c_longlong),
        ("nfa_p", ctypes.c_longlong), ("nfa_zone", ctypes.c_longlong * 27),
        ("x_no", c_dbl_p), ("cvofa", c_int_p), ("noofa_i", c_int_p), ("noofa_v", c_int_p),
        ("n_fa", c_dbl_p), ("x_fa", c_dbl_p),
        ("cvobf", c_int_p), ("noobf_i", c_int_p), ("noobf_v", c_int_p),
        ("n_bf", c_dbl_p), ("x_bf", c_dbl_p), ("area_bf", c_dbl_p), ("area_over_delta_bf", c_dbl_p),
        ("Gij_bf", c_dbl_p),
        ("vol_cv", c_dbl_p), ("r_vv", c_dbl_p), ("x_vv", c_dbl_p), ("x_cv", c_dbl_p),
        ("nbf_zones", ctypes.c_int), ("bf_zones", ctypes.POINTER(BfZone)),
        ("ncv_zones", ctypes.c_int), ("cv_zone_ncv", ctypes.c_longlong * 16),
    ]


class MlesError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "?"), code, msg))
        self.code = code


def _lib():
    L = _meshgen_lib()
    if not getattr(L, "_mles_bound", False):
        L.cgx_sles_write.restype = ctypes.c_int
        L.cgx_sles_write.argtypes = [ctypes.c_char_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_double, c_dbl_p,
                                     c_dbl_p, c_dbl_p, ctypes.c_char_p]
        L.cgx_sles_read.restype = ctypes.c_int
        L.cgx_sles_read.argtypes = [ctypes.c_char_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_double), c_dbl_p, c_dbl_p, c_dbl_p]
        L.cgx_mles_read.restype = ctypes.c_int
        L.cgx_mles_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.POINTER(Mles))]
        L.cgx_mles_free.restype = None
        L.cgx_mles_free.argtypes = [ctypes.POINTER(Mles)]
        L.cgx_mles_last_error.restype = ctypes.c_char_p
        L.cgx_mles_last_error.argtypes = []
        L._mles_bound = True
    return L


def _view(ptr, shape, dtype):
    if not ptr:
        return None
    n = int(np.prod(shape))
    if n == 0:
        return np.zeros(shape, dtype=dtype)
    ct = ctypes.c_int if dtype == np.int32 else ctypes.c_double
    buf = (ct * n).from_address(ctypes.addressof(ptr.contents))
    return np.frombuffer(buf, dtype=dtype).reshape(shape)


class MlesMesh:
    """One .mles file read by cgx_mles_read."""

    def __init__(self, path):
        L = _lib()
        out = ctypes.POINTER(Mles)()
        rc = L.cgx_mles_read(str(path).encode(), ctypes.byref(out))
        if rc != 0:
            raise MlesError(rc, L.cgx_mles_last_error().decode())
        self.ptr = out
        m = out.contents
        self.io_version = m.io_version
        for k in ("nno", "nbf", "nfa", "ncv", "nno_p", "nno_pb", "nfa_p"):
            setattr(self, k, int(getattr(m, k)))
        self.nfa_zone = np.array(m.nfa_zone[:], dtype=np.int64)
        nno, nbf, nfa, ncv = self.nno, self.nbf, self.nfa, self.ncv
        self.x_no = _view(m.x_no, (nno, 3), np.float64)
        self.cvofa = _view(m.cvofa, (nfa, 2), np.int32)
        self.noofa_i = _view(m.noofa_i, (nfa + 1,), np.int32)
        self.noofa_v = _view(m.noofa_v, (int(self.noofa_i[-1]),), np.int32) if self.noofa_i is not None else None
        self.n_fa = _view(m.n_fa, (nfa, 3), np.float64)
        self.x_fa = _view(m.x_fa, (nfa, 3), np.float64)
        self.cvobf = _view(m.cvobf, (nbf,), np.int32)
        self.noobf_i = _view(m.noobf_i, (nbf + 1,), np.int32)
        self.noobf_v = _view(m.noobf_v, (int(self.noobf_i[-1]),), np.int32) if self.noobf_i is not None else None
        self.n_bf = _view(m.n_bf, (nbf, 3), np.float64)
        self.x_bf = _view(m.x_bf, (nbf, 3), np.float64)
        self.area_bf = _view(m.area_bf, (nbf,), np.float64)
        self.area_over_delta_bf = _view(m.area_over_delta_bf, (nbf,), np.float64)
        self.Gij_bf = _view(m.Gij_bf, (nbf, 3, 3), np.float64)
        self.vol_cv = _view(m.vol_cv, (ncv,), np.float64)
        self.r_vv = _view(m.r_vv, (ncv,), np.float64)
        self.x_vv = _view(m.x_vv, (ncv, 3), np.float64)
        self.x_cv = _view(m.x_cv, (ncv, 3), np.float64)
        self.bf_zones = [dict(name=z.name.decode(), nbf=int(z.nbf), ibf_f=int(z.ibf_f), area=z.area,
                              area_over_delta=z.area_over_delta, n=np.array(z.n[:]), x=np.array(z.x[:]))
                         for z in (m.bf_zones[i] for i in range(m.nbf_zones))]
        self.cv_zone_ncv = [int(m.cv_zone_ncv[i]) for i in range(min(m.ncv_zones, 16))]

    def close(self):
        if getattr(self, "ptr", None):
            _lib().cgx_mles_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_sles(path, rho, u, rhoE, step=0, time=0.0, params=""):
    """Write a .sles result file (cgx_sles_write): rho[ncv], u[ncv][3],
    rhoE[ncv] in the mesh's cell order, the step and the time."""
    rho, rhoE = (np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (rho, rhoE))
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 3)
    dp = lambda a: a.ctypes.data_as(c_dbl_p)
    rc = _lib().cgx_sles_write(str(path).encode(), rho.size, int(step), float(time), dp(rho), dp(u), dp(rhoE),
                               (params or "").encode())
    if rc != 0:
        raise MlesError(rc, _lib().cgx_mles_last_error().decode())


def read_sles(path, ncv):
    """(rho, u, rhoE, step, time) of a .sles result file of ncv cells."""
    rho, u, rhoE = np.empty(ncv), np.empty((ncv, 3)), np.empty(ncv)
    st, t = ctypes.c_int(), ctypes.c_double()
    dp = lambda a: a.ctypes.data_as(c_dbl_p)
    rc = _lib().cgx_sles_read(str(path).encode(), int(ncv), ctypes.byref(st), ctypes.byref(t), dp(rho), dp(u),
                              dp(rhoE))
    if rc != 0:
        raise MlesError(rc, _lib().cgx_mles_last_error().decode())
    return rho, u, rhoE, st.value, t.value


class CompactMesh:
    """The mesher's part of a non-periodic mesh -- cells, internal faces and
    boundary faces with their zones -- in the form the GPU operator build
    takes (meshgen.compact_desc): from an MlesMesh (`from_mles`) or from the
    arrays saved by `save` (`load`).  Internal faces are ordered by their
    first cell (cvofa[:,0] < cvofa[:,1]); boundary faces keep the file's
    order, each with the index of its zone in `zone_names`."""

    FIELDS = ("cvofa", "n_fa", "x_fa", "vol_cv", "x_cv", "x_vv", "cvobf", "zone_bf", "n_bf", "x_bf", "area_bf",
              "area_over_delta_bf", "Gij_bf")

    def __init__(self, arrays, zone_names):
        for k in self.FIELDS:
            setattr(self, k, np.ascontiguousarray(arrays[k]))
        self.zone_names = list(zone_names)
        self.ncv = self.ncv_g = self.ncv_g2 = int(self.vol_cv.size)
        self.nfa = self.nfa_i = int(self.cvofa.shape[0])
        self.nbf = int(self.cvobf.size)
        self.nbf_zones = len(self.zone_names)
        self.nef = self.nef_i = 0
        self.icv_owner_g = np.zeros(0, np.int32)
        self.shift_g = np.zeros((0, 3), np.int32)
        # no periodic images: the box lengths only have to be positive
        self.L = (1.0, 1.0, 1.0)
        self.h = float(np.cbrt(self.vol_cv.mean()))
        self.dims, self.jitter, self.seed = (self.ncv, 1, 1), 0.0, 0

    @classmethod
    def from_mles(cls, m):
        if m.nfa_p != 0 or m.nno_p != 0:
            raise ValueError("periodic meshes are not handled")
        c = np.asarray(m.cvofa)
        n, x = np.asarray(m.n_fa), np.asarray(m.x_fa)
        # each face from its lower cell, faces ordered by (lower cell, upper)
        flip = c[:, 0] > c[:, 1]
        c = np.where(flip[:, None], c[:, ::-1], c)
        n = np.where(flip[:, None], -n, n)
        order = np.lexsort((c[:, 1], c[:, 0]))
        zone = np.zeros(m.nbf, np.int32)
        for k, z in enumerate(m.bf_zones):
            zone[z["ibf_f"]:z["ibf_f"] + z["nbf"]] = k
        arrays = dict(cvofa=c[order].astype(np.int32), n_fa=n[order], x_fa=x[order], vol_cv=m.vol_cv,
                      x_cv=m.x_cv, x_vv=m.x_vv if m.x_vv is not None else m.x_cv, cvobf=m.cvobf, zone_bf=zone,
                      n_bf=m.n_bf, x_bf=m.x_bf, area_bf=m.area_bf, area_over_delta_bf=m.area_over_delta_bf,
                      Gij_bf=m.Gij_bf)
        return cls({k: np.array(v) for k, v in arrays.items()}, [z["name"] for z in m.bf_zones])

    def save(self, path):
        np.savez_compressed(path, zone_names=np.array(self.zone_names), **{k: getattr(self, k) for k in self.FIELDS})

    @classmethod
    def load(cls, path):
        d = np.load(path)
        return cls({k: d[k] for k in cls.FIELDS}, [str(s) for s in d["zone_names"]])
