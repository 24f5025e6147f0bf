"""ctypes loader for the C oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates original/nemolite2d.f90 in plain C (oracle/nemolite2d_oracle.c).
Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this module,
and only as the checker or the timed CPU baseline; the product never does.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "liboracle.so")

SSHN, UN, VN, SSHA, UA, VA, SSHN_U, SSHN_V, HT, HU, HV, XT, YT = range(13)
T_FIELDS = (SSHN, SSHA, HT, XT, YT)
U_FIELDS = (UN, UA, SSHN_U, HU)
V_FIELDS = (VN, VA, SSHN_V, HV)


class Params(ctypes.Structure):
    _fields_ = [
        ("jpi", ctypes.c_int), ("jpj", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dep_const", ctypes.c_double),
        ("nit000", ctypes.c_int), ("nitend", ctypes.c_int), ("irecord", ctypes.c_int),
        ("rdt", ctypes.c_double), ("cbfr", ctypes.c_double), ("visc", ctypes.c_double),
        ("amp_tide", ctypes.c_double), ("tide_phase", ctypes.c_double), ("lat", ctypes.c_double),
        ("nbump", ctypes.c_int), ("seed", ctypes.c_uint64),
        ("bump_amp", ctypes.c_double), ("bump_wmin", ctypes.c_double),
        ("bump_wmax", ctypes.c_double), ("hmin", ctypes.c_double), ("hmax", ctypes.c_double),
    ]


def build():
    """Compile the oracle with its Makefile (strict IEEE flags)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        vp = ctypes.c_void_p
        dp = P(ctypes.c_double)
        L.oracle_default_params.argtypes = [P(Params)]
        L.oracle_create.argtypes = [P(Params)]
        L.oracle_create.restype = vp
        L.oracle_destroy.argtypes = [vp]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        for name in ("oracle_continuity", "oracle_momentum", "oracle_momentum_u",
                     "oracle_momentum_v", "oracle_bc_solid_u", "oracle_bc_solid_v",
                     "oracle_bc_flather_u", "oracle_bc_flather_v", "oracle_next"):
            getattr(L, name).argtypes = [vp]
        L.oracle_bc.argtypes = [vp, ctypes.c_double]
        L.oracle_bc_ssh.argtypes = [vp, ctypes.c_double]
        L.oracle_step.argtypes = [vp, ctypes.c_int]
        L.oracle_run.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.oracle_get_field.argtypes = [vp, ctypes.c_int, dp]
        L.oracle_get_field.restype = ctypes.c_long
        L.oracle_set_state.argtypes = [vp, dp, dp, dp]
        L.oracle_set_grid.argtypes = [vp, ctypes.POINTER(ctypes.c_int)] + [dp] * 11
        L.oracle_checksum_seq.argtypes = [vp, ctypes.c_int]
        L.oracle_checksum_seq.restype = ctypes.c_double
        L.oracle_checksum_tree.argtypes = [vp, ctypes.c_int]
        L.oracle_checksum_tree.restype = ctypes.c_double
        L.oracle_tree_sum_abs.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_tree_sum_abs.restype = ctypes.c_double
        _lib = L
    return _lib


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def default_params(**kw):
    p = Params()
    lib().oracle_default_params(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def set_threads(n):
    lib().oracle_set_threads(int(n))


def field_shape(field, jpi, jpj):
    """(ny, nx) of the dense Fortran-bounded region, C-order view of column-major."""
    if field in T_FIELDS:
        return (jpj, jpi)
    if field in U_FIELDS:
        return (jpj, jpi + 1)
    return (jpj + 1, jpi)


class Model:
    """One oracle instance (grid + initialisation of original/nemolite2d.f90)."""

    def __init__(self, params=None, **kw):
        self.p = params if params is not None else default_params(**kw)
        self.h = lib().oracle_create(ctypes.byref(self.p))
        if not self.h:
            raise ValueError("oracle_create rejected the parameters")
        self.jpi, self.jpj = self.p.jpi, self.p.jpj

    def close(self):
        if self.h:
            lib().oracle_destroy(self.h)
            self.h = None

    __del__ = close

    def step(self, istp):
        lib().oracle_step(self.h, istp)

    def run(self, istp0, n):
        lib().oracle_run(self.h, istp0, n)

    def continuity(self):
        lib().oracle_continuity(self.h)

    def momentum_u(self):
        lib().oracle_momentum_u(self.h)

    def momentum_v(self):
        lib().oracle_momentum_v(self.h)

    def bc_ssh(self, rtime):
        lib().oracle_bc_ssh(self.h, rtime)

    def bc_solid_u(self):
        lib().oracle_bc_solid_u(self.h)

    def bc_solid_v(self):
        lib().oracle_bc_solid_v(self.h)

    def bc_flather_u(self):
        lib().oracle_bc_flather_u(self.h)

    def bc_flather_v(self):
        lib().oracle_bc_flather_v(self.h)

    def next(self):
        lib().oracle_next(self.h)

    def field(self, f):
        out = np.empty(field_shape(f, self.jpi, self.jpj), dtype=np.float64)
        n = lib().oracle_get_field(self.h, f, _dptr(out))
        assert n == out.size
        return out

    def set_state(self, sshn, un, vn):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (sshn, un, vn)]
        lib().oracle_set_state(self.h, *[_dptr(x) for x in a])

    def set_grid(self, pt, e1t, e2t, e1u, e2u, e1v, e2v, gphiu, gphiv, ht=None, hu=None, hv=None):
        """General grid (oracle_set_grid): arrays of shape (jpj+2, jpi+2) over
        (0:jpi+1, 0:jpj+1); depths None keep the current ones."""
        shape = (self.jpj + 2, self.jpi + 2)
        p = np.ascontiguousarray(pt, dtype=np.int32)
        assert p.shape == shape
        a = [None if x is None else np.ascontiguousarray(x, dtype=np.float64)
             for x in (e1t, e2t, e1u, e2u, e1v, e2v, gphiu, gphiv, ht, hu, hv)]
        assert all(x is None or x.shape == shape for x in a)
        ptrs = [ctypes.POINTER(ctypes.c_double)() if x is None else _dptr(x) for x in a]
        rc = lib().oracle_set_grid(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), *ptrs)
        if rc != 0:
            raise ValueError("oracle_set_grid: mask values must be -1, 0 or 1")

    def checksum(self, f, order="seq"):
        if order == "seq":
            return lib().oracle_checksum_seq(self.h, f)
        return lib().oracle_checksum_tree(self.h, f)


def tree_sum_abs(a2d):
    """Device-order sum of |a| over a (ny, nx) C-order array."""
    a = np.ascontiguousarray(a2d, dtype=np.float64)
    ny, nx = a.shape
    return lib().oracle_tree_sum_abs(_dptr(a), nx, ny, nx)
