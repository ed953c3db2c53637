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
