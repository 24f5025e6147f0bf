"""Python host side of the B200 NEMOLite2D stepper, over its C ABI.

Mirrors the reference's routine boundary (original/nemolite2d.f90:375-386:
continuity, momentum, bc, next) and the drop-in CUDA-library symbols of
cuda/cuda_nemolite2d.cu:234-270, through ctypes bindings of
lib/libnemo_b200.so (or lib/libnemo_b200_strict.so, the -fmad=false build).

There is no CPU fallback: if the shared library is missing or cannot load,
importing or constructing anything raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.dirname(_HERE)
LIB_DIR = os.path.join(PKG_DIR, "lib")

SSHN, UN, VN, SSHA, UA, VA, SSHN_U, SSHN_V, HT, HU, HV, XT, YT = range(13)
FIELD_NAMES = {SSHN: "sshn", UN: "un", VN: "vn", SSHA: "ssha", UA: "ua", VA: "va",
               SSHN_U: "sshn_u", SSHN_V: "sshn_v", HT: "ht", HU: "hu", HV: "hv",
               XT: "xt", YT: "yt"}
T_FIELDS = (SSHN, SSHA, HT, XT, YT)
U_FIELDS = (UN, UA, SSHN_U, HU)
V_FIELDS = (VN, VA, SSHN_V, HV)

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA runtime error", 3: "allocation failed",
          4: "invalid state", 5: "device wait timed out", 6: "unsupported"}

# Every symbol include/nemo_b200.h declares.
EXPORTED = [
    "nemo_default_params", "nemo_create", "nemo_destroy", "nemo_continuity", "nemo_momentum",
    "nemo_momentum_u", "nemo_momentum_v", "nemo_bc", "nemo_bc_ssh", "nemo_bc_solid_u",
    "nemo_bc_solid_v", "nemo_bc_flather_u", "nemo_bc_flather_v", "nemo_next", "nemo_step",
    "nemo_step_n", "nemo_checksums", "nemo_checksum", "nemo_retrieve", "nemo_record",
    "nemo_record_wait", "nemo_host_alloc", "nemo_host_free", "nemo_set_state", "nemo_set_grid",
    "nemo_sync", "nemo_get_dims", "nemo_device_field", "nemo_set_schedule", "nemo_get_schedule",
    "nemo_status_string", "nemo_build_is_strict", "nemo_checksums_noalloc", "nemo_autotune",
    "nemo_ens_generate", "nemo_ens_create", "nemo_ens_destroy", "nemo_ens_step_n",
    "nemo_ens_checksums", "nemo_ens_retrieve", "nemo_ens_set_state", "nemo_ens_set_schedule",
    "nemo_ens_get_schedule", "nemo_ens_use_graph", "nemo_ens_info", "nemo_ens_autotune",
    "nemo_sur_default_config", "nemo_sur_create", "nemo_sur_destroy", "nemo_sur_info",
    "nemo_sur_get_params", "nemo_sur_set_params", "nemo_sur_get_grads", "nemo_sur_set_norm",
    "nemo_sur_get_norm", "nemo_sur_predict", "nemo_sur_loss_grad", "nemo_sur_adamw",
    "nemo_sur_train_step", "nemo_sur_pack_ens", "nemo_sur_advance_ens", "nemo_ens_compare",
    "nemo_hyb_default_config", "nemo_hyb_run", "nemo_conv3x3_fwd", "nemo_conv3x3_wgrad",
    "nemo_conv3x3_fwd_variant", "nemo_conv3x3_wgrad_variant", "nemo_debug_fail_alloc",
    "nemo_debug_conv_wait",
    "cuda_setup_model_params_", "cuda_initialise_grid_", "cuda_continuity_", "cuda_momentum_",
    "cuda_boundary_conditions_", "cuda_next_", "cuda_retrieve_grid_constants_",
    "cuda_retrieve_results_", "cuda_finalise_", "nemo_compat_last_status", "nemo_compat_context",
]


class NemoError(RuntimeError):
    def __init__(self, status, where):
        super().__init__("%s failed: %s (status %d)" % (where, STATUS.get(status, "?"), status))
        self.status = status


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
        ("stream", ctypes.c_void_p), ("device", ctypes.c_int),
    ]


class Schedule(ctypes.Structure):
    _fields_ = [("warps", ctypes.c_int), ("occupancy", ctypes.c_int), ("rows", ctypes.c_int)]


class Member(ctypes.Structure):
    _fields_ = [("jpi", ctypes.c_int), ("jpj", ctypes.c_int),
                ("amp_tide", ctypes.c_double), ("tide_phase", ctypes.c_double),
                ("dep_const", ctypes.c_double), ("nbump", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("bump_amp", ctypes.c_double), ("bump_wmin", ctypes.c_double),
                ("bump_wmax", ctypes.c_double), ("hmin", ctypes.c_double), ("hmax", ctypes.c_double)]


class EnsSchedule(ctypes.Structure):
    _fields_ = [("warps", ctypes.c_int), ("occupancy", ctypes.c_int), ("rows", ctypes.c_int),
                ("order", ctypes.c_int), ("ctas", ctypes.c_int)]


def lib_path(strict=False):
    return os.path.join(LIB_DIR, "libnemo_b200_strict.so" if strict else "libnemo_b200.so")


_libs = {}


def load(strict=False):
    """Load (once) and type the shared library.  Raises if it is missing."""
    if strict in _libs:
        return _libs[strict]
    path = lib_path(strict)
    if not os.path.exists(path):
        raise ImportError("nemo_b200: %s is not built (run `make -C %s`); no fallback exists"
                          % (path, PKG_DIR))
    L = ctypes.CDLL(path)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    P = ctypes.POINTER
    L.nemo_default_params.argtypes = [P(Params)]
    L.nemo_create.argtypes = [P(Params), P(vp)]
    for n in ("nemo_destroy", "nemo_continuity", "nemo_momentum", "nemo_momentum_u",
              "nemo_momentum_v", "nemo_bc_solid_u", "nemo_bc_solid_v", "nemo_bc_flather_u",
              "nemo_bc_flather_v", "nemo_next", "nemo_sync"):
        getattr(L, n).argtypes = [vp]
    L.nemo_bc.argtypes = [vp, dp]
    L.nemo_bc_ssh.argtypes = [vp, dp]
    L.nemo_step.argtypes = [vp, ip]
    L.nemo_step_n.argtypes = [vp, ip, ip]
    L.nemo_checksums.argtypes = [vp, P(dp)]
    L.nemo_checksum.argtypes = [vp, ip, P(dp)]
    L.nemo_retrieve.argtypes = [vp, ip, P(dp), ctypes.c_long]
    L.nemo_record.argtypes = [vp, P(dp)]
    L.nemo_record_wait.argtypes = [vp]
    L.nemo_set_state.argtypes = [vp, P(dp), P(dp), P(dp)]
    L.nemo_set_grid.argtypes = [vp, P(Grid)]
    L.nemo_get_dims.argtypes = [vp, P(ip), P(ip)]
    L.nemo_device_field.argtypes = [vp, ip, P(P(dp)), P(ctypes.c_long)]
    L.nemo_set_schedule.argtypes = [vp, P(Schedule)]
    L.nemo_get_schedule.argtypes = [vp, P(Schedule)]
    L.nemo_status_string.argtypes = [ip]
    L.nemo_status_string.restype = ctypes.c_char_p
    L.nemo_build_is_strict.restype = ip
    L.cuda_setup_model_params_.argtypes = [ip, ip, dp, dp, dp, ip, ip, ip, dp, dp, dp]
    L.cuda_setup_model_params_.restype = None
    for n in ("cuda_initialise_grid_", "cuda_continuity_", "cuda_momentum_", "cuda_next_",
              "cuda_finalise_"):
        getattr(L, n).argtypes = []
        getattr(L, n).restype = None
    L.cuda_boundary_conditions_.argtypes = [dp]
    L.cuda_boundary_conditions_.restype = None
    L.cuda_retrieve_grid_constants_.argtypes = [P(dp), P(dp), P(dp), ip, ip]
    L.cuda_retrieve_grid_constants_.restype = None
    L.cuda_retrieve_results_.argtypes = [P(dp)] * 5 + [ip, ip]
    L.cuda_retrieve_results_.restype = None
    L.nemo_compat_context.restype = vp
    L.nemo_checksums_noalloc.argtypes = [P(ctypes.c_void_p), ip, ip, ip, ctypes.c_long,
                                         ctypes.c_void_p, ctypes.c_void_p]
    L.nemo_autotune.argtypes = [vp, ip, P(Schedule), P(dp)]
    L.nemo_debug_fail_alloc.argtypes = [ip]
    L.nemo_debug_conv_wait.argtypes = [ctypes.c_ulonglong, ip]
    L.nemo_ens_generate.argtypes = [ctypes.c_uint64, ip, ip, ip, dp, P(Member)]
    L.nemo_ens_create.argtypes = [P(Params), P(Member), ip, P(vp)]
    L.nemo_ens_destroy.argtypes = [vp]
    L.nemo_ens_step_n.argtypes = [vp, ip, ip]
    L.nemo_ens_checksums.argtypes = [vp, P(dp)]
    L.nemo_ens_retrieve.argtypes = [vp, ip, ip, P(dp), ctypes.c_long]
    L.nemo_ens_set_state.argtypes = [vp, ip, P(dp), P(dp), P(dp)]
    L.nemo_ens_set_schedule.argtypes = [vp, P(EnsSchedule)]
    L.nemo_ens_get_schedule.argtypes = [vp, P(EnsSchedule)]
    L.nemo_ens_use_graph.argtypes = [vp, ip]
    L.nemo_ens_info.argtypes = [vp, P(ip), P(ctypes.c_longlong)]
    L.nemo_ens_autotune.argtypes = [vp, ip, P(EnsSchedule), P(dp)]
    from . import surrogate as _sur
    _sur.declare(L)
    _libs[strict] = L
    return L


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def check(status, where):
    if status != 0:
        raise NemoError(status, where)


def default_params(strict=False, **kw):
    p = Params()
    load(strict).nemo_default_params(ctypes.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError("unknown parameter %r" % k)
        setattr(p, k, v)
    return p


def field_shape(field, jpi, jpj):
    """(ny, nx): C-order view of the field's Fortran-bounded column-major block."""
    if field in T_FIELDS:
        return (jpj, jpi)
    if field in U_FIELDS:
        return (jpj, jpi + 1)
    if field in V_FIELDS:
        return (jpj + 1, jpi)
    raise ValueError("unknown field %r" % field)


class Grid(ctypes.Structure):
    """nemo_grid: host arrays over (0:jpi+1, 0:jpj+1), column-major."""
    _fields_ = [("pt", ctypes.POINTER(ctypes.c_int))] + [
        (n, ctypes.POINTER(ctypes.c_double))
        for n in ("e1t", "e2t", "e1u", "e2u", "e1v", "e2v", "gphiu", "gphiv", "ht", "hu", "hv")]


class Model:
    """One model instance on one GPU (a nemo_ctx)."""

    def __init__(self, params=None, strict=False, **kw):
        self.lib = load(strict)
        self.strict = strict
        self.p = params if params is not None else default_params(strict, **kw)
        h = ctypes.c_void_p()
        check(self.lib.nemo_create(ctypes.byref(self.p), ctypes.byref(h)), "nemo_create")
        self.h = h
        self.jpi, self.jpj = self.p.jpi, self.p.jpj

    def close(self):
        if getattr(self, "h", None):
            self.lib.nemo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # per-routine boundary
    def continuity(self):
        check(self.lib.nemo_continuity(self.h), "nemo_continuity")

    def momentum(self):
        check(self.lib.nemo_momentum(self.h), "nemo_momentum")

    def momentum_u(self):
        check(self.lib.nemo_momentum_u(self.h), "nemo_momentum_u")

    def momentum_v(self):
        check(self.lib.nemo_momentum_v(self.h), "nemo_momentum_v")

    def bc(self, rtime):
        check(self.lib.nemo_bc(self.h, rtime), "nemo_bc")

    def bc_ssh(self, rtime):
        check(self.lib.nemo_bc_ssh(self.h, rtime), "nemo_bc_ssh")

    def bc_solid_u(self):
        check(self.lib.nemo_bc_solid_u(self.h), "nemo_bc_solid_u")

    def bc_solid_v(self):
        check(self.lib.nemo_bc_solid_v(self.h), "nemo_bc_solid_v")

    def bc_flather_u(self):
        check(self.lib.nemo_bc_flather_u(self.h), "nemo_bc_flather_u")

    def bc_flather_v(self):
        check(self.lib.nemo_bc_flather_v(self.h), "nemo_bc_flather_v")

    def next(self):
        check(self.lib.nemo_next(self.h), "nemo_next")

    def step(self, istp):
        check(self.lib.nemo_step(self.h, istp), "nemo_step")

    # fused path
    def step_n(self, istp0, n):
        check(self.lib.nemo_step_n(self.h, istp0, n), "nemo_step_n")

    def set_schedule(self, warps=2, occupancy=None, rows=32):
        """occupancy None: the context's default staging (216 when the in-kernel
        reciprocal depths passed their check, else 116).  After set_grid the
        general grid's kernel takes warps 2, occupancy 3 or 4 (ring slots) or 0
        (rows loaded where used), rows >= 1."""
        if occupancy is None:
            occupancy = 216 if self.recip_in_kernel() else 116
        s = Schedule(warps, occupancy, rows)
        check(self.lib.nemo_set_schedule(self.h, ctypes.byref(s)), "nemo_set_schedule")

    def get_schedule(self):
        s = Schedule()
        check(self.lib.nemo_get_schedule(self.h, ctypes.byref(s)), "nemo_get_schedule")
        return (s.warps, s.occupancy, s.rows)

    def recip_in_kernel(self):
        """True when the schedules that form the reciprocal depths in the
        kernel (occupancy 216, 220) are available for this grid."""
        s = Schedule(2, 216, 32)
        keep = Schedule()
        check(self.lib.nemo_get_schedule(self.h, ctypes.byref(keep)), "nemo_get_schedule")
        ok = self.lib.nemo_set_schedule(self.h, ctypes.byref(s)) == 0
        check(self.lib.nemo_set_schedule(self.h, ctypes.byref(keep)), "nemo_set_schedule")
        return ok

    def sync(self):
        check(self.lib.nemo_sync(self.h), "nemo_sync")

    def checksums(self):
        out = np.zeros(3, dtype=np.float64)
        check(self.lib.nemo_checksums(self.h, _dptr(out)), "nemo_checksums")
        return out

    def checksum(self, field):
        out = np.zeros(1, dtype=np.float64)
        check(self.lib.nemo_checksum(self.h, field, _dptr(out)), "nemo_checksum")
        return float(out[0])

    def field(self, f, out=None):
        shape = field_shape(f, self.jpi, self.jpj)
        if out is None:
            out = np.empty(shape, dtype=np.float64)
        assert out.shape == shape and out.dtype == np.float64 and out.flags.c_contiguous
        check(self.lib.nemo_retrieve(self.h, f, _dptr(out), shape[1]), "nemo_retrieve")
        return out

    def record(self, out):
        """Start an output record of the current state into `out` (float64
        [3][jpj][jpi], C-contiguous; pinned memory lets the copy overlap later
        steps): sshn and the cell-centred u, v.  record_wait() blocks until it
        has landed."""
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == 3 * self.jpi * self.jpj
        check(self.lib.nemo_record(self.h, _dptr(out)), "nemo_record")

    def record_wait(self):
        check(self.lib.nemo_record_wait(self.h), "nemo_record_wait")

    def set_state(self, sshn, un, vn):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (sshn, un, vn)]
        for f, x in zip((SSHN, UN, VN), a):
            assert x.shape == field_shape(f, self.jpi, self.jpj), (f, x.shape)
        check(self.lib.nemo_set_state(self.h, *[_dptr(x) for x in a]), "nemo_set_state")

    # parameters that change the arithmetic of a step; a checkpoint records
    # them and a restart into a model that differs in any of them is refused
    _CHECKPOINT_PARAMS = ("dx", "dy", "dep_const", "rdt", "cbfr", "visc", "amp_tide",
                          "tide_phase", "lat", "nbump", "seed", "bump_amp", "bump_wmin",
                          "bump_wmax", "hmin", "hmax")

    def _geometry_digest(self):
        """SHA-256 over the device depths ht, hu, hv and the arrays of the last
        set_grid call (mask, scale factors, latitudes), if any."""
        import hashlib
        h = hashlib.sha256()
        for f in (HT, HU, HV):
            h.update(np.ascontiguousarray(self.field(f)).tobytes())
        h.update(getattr(self, "_grid_digest", b""))
        return h.hexdigest()

    def save_checkpoint(self, path, istp):
        """Write the state after step istp (sshn, un, vn in Fortran bounds,
        FP64) to an .npz file, with the model parameters and a digest of the
        geometry (depths and any set_grid arrays).  Every step derives the rest
        of the state from these three fields, so load_checkpoint followed by
        steps istp+1... gives the uninterrupted run bit for bit (the reference
        writes no restart files; this is the build's own format).  The file is
        written beside `path` first and renamed over it, so a crash during the
        write leaves any previous checkpoint at `path` intact."""
        params = np.array([float(getattr(self.p, k)) for k in self._CHECKPOINT_PARAMS])
        tmp = path + ".tmp"
        with open(tmp, "wb") as fh:
            np.savez(fh, istp=np.int64(istp), jpi=np.int64(self.jpi), jpj=np.int64(self.jpj),
                     params=params, param_names=np.array(self._CHECKPOINT_PARAMS),
                     geometry=np.array(self._geometry_digest()),
                     sshn=self.field(SSHN), un=self.field(UN), vn=self.field(VN))
            fh.flush()
            os.fsync(fh.fileno())
        os.replace(tmp, path)

    def load_checkpoint(self, path):
        """Restore a save_checkpoint file; returns the step it was taken after.
        Raises ValueError when the file was written by a model with another
        grid size, other parameters or another geometry."""
        with np.load(path) as z:
            if int(z["jpi"]) != self.jpi or int(z["jpj"]) != self.jpj:
                raise ValueError("checkpoint is for a %dx%d grid" % (int(z["jpi"]), int(z["jpj"])))
            names = [str(x) for x in z["param_names"]]
            mine = {k: float(getattr(self.p, k)) for k in self._CHECKPOINT_PARAMS}
            for k, v in zip(names, z["params"]):
                if k not in mine or mine[k] != float(v):
                    raise ValueError("checkpoint parameter %s = %r, this model has %r"
                                     % (k, float(v), mine.get(k)))
            if str(z["geometry"]) != self._geometry_digest():
                raise ValueError("checkpoint was written on another geometry (depths or grid arrays)")
            self.set_state(z["sshn"], z["un"], z["vn"])
            return int(z["istp"])

    def set_grid(self, pt, e1t, e2t, e1u, e2u, e1v, e2v, gphiu, gphiv, ht=None, hu=None, hv=None):
        """General grid (nemo_set_grid): arrays of shape (jpj+2, jpi+2) over
        (0:jpi+1, 0:jpj+1); depths None keep the current ones.  Steps then
        run the per-routine kernels."""
        shape = (self.jpj + 2, self.jpi + 2)
        p = np.ascontiguousarray(pt, dtype=np.int32)
        assert p.shape == shape
        a = [None if x is None else np.ascontiguousarray(x, dtype=np.float64)
             for x in (e1t, e2t, e1u, e2u, e1v, e2v, gphiu, gphiv, ht, hu, hv)]
        assert all(x is None or x.shape == shape for x in a)
        g = Grid(p.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                 *[ctypes.POINTER(ctypes.c_double)() if x is None else _dptr(x) for x in a])
        check(self.lib.nemo_set_grid(self.h, ctypes.byref(g)), "nemo_set_grid")
        import hashlib
        h = hashlib.sha256(p.tobytes())
        for x in a[:8]:
            h.update(x.tobytes())
        self._grid_digest = h.digest()

    def autotune(self, steps=5):
        sch = Schedule()
        ms = ctypes.c_double()
        check(self.lib.nemo_autotune(self.h, steps, ctypes.byref(sch), ctypes.byref(ms)),
              "nemo_autotune")
        return (sch.warps, sch.occupancy, sch.rows), ms.value

    def device_field(self, f):
        ptr = ctypes.POINTER(ctypes.c_double)()
        pitch = ctypes.c_long()
        check(self.lib.nemo_device_field(self.h, f, ctypes.byref(ptr), ctypes.byref(pitch)),
              "nemo_device_field")
        return ctypes.cast(ptr, ctypes.c_void_p).value, pitch.value


def is_strict_build(strict):
    return bool(load(strict).nemo_build_is_strict())


def generate_members(seed, n, side_min=64, side_max=1024, amp_scale=1.0, strict=False):
    """Member recipe of the batched configuration (see nemo_ens_generate)."""
    arr = (Member * n)()
    check(load(strict).nemo_ens_generate(seed, n, side_min, side_max, amp_scale, arr),
          "nemo_ens_generate")
    return list(arr)


def member_params(common, m):
    """Single-grid parameters equal to ensemble member m (for comparisons)."""
    p = Params()
    ctypes.pointer(p)[0] = common
    p.jpi, p.jpj = m.jpi, m.jpj
    p.amp_tide, p.tide_phase = m.amp_tide, m.tide_phase
    p.dep_const, p.nbump, p.seed = m.dep_const, m.nbump, m.seed
    p.bump_amp, p.bump_wmin, p.bump_wmax = m.bump_amp, m.bump_wmin, m.bump_wmax
    p.hmin, p.hmax = m.hmin, m.hmax
    return p


class Ensemble:
    """Many members of uneven size advanced together (a nemo_ens)."""

    def __init__(self, members, strict=False, common=None, **kw):
        self.lib = load(strict)
        self.common = common if common is not None else default_params(strict, **kw)
        self.members = list(members)
        arr = (Member * len(self.members))(*self.members)
        h = ctypes.c_void_p()
        check(self.lib.nemo_ens_create(ctypes.byref(self.common), arr, len(self.members),
                                       ctypes.byref(h)), "nemo_ens_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.nemo_ens_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step_n(self, istp0, n):
        check(self.lib.nemo_ens_step_n(self.h, istp0, n), "nemo_ens_step_n")

    def checksums(self):
        out = np.zeros(3 * len(self.members), dtype=np.float64)
        check(self.lib.nemo_ens_checksums(self.h, _dptr(out)), "nemo_ens_checksums")
        return out.reshape(-1, 3)

    def field(self, member, f):
        m = self.members[member]
        shape = field_shape(f, m.jpi, m.jpj)
        out = np.empty(shape, dtype=np.float64)
        check(self.lib.nemo_ens_retrieve(self.h, member, f, _dptr(out), shape[1]),
              "nemo_ens_retrieve")
        return out

    def set_state(self, member, sshn, un, vn):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (sshn, un, vn)]
        check(self.lib.nemo_ens_set_state(self.h, member, *[_dptr(x) for x in a]),
              "nemo_ens_set_state")

    def set_schedule(self, warps=2, occupancy=None, rows=16, order=1, ctas=0):
        """occupancy None: 216 when every member's in-kernel reciprocal depths
        passed their check, else 116."""
        if occupancy is None:
            s = EnsSchedule(2, 216, rows, order, ctas)
            occupancy = 216 if self.lib.nemo_ens_set_schedule(self.h, ctypes.byref(s)) == 0 else 116
        s = EnsSchedule(warps, occupancy, rows, order, ctas)
        check(self.lib.nemo_ens_set_schedule(self.h, ctypes.byref(s)), "nemo_ens_set_schedule")

    def get_schedule(self):
        s = EnsSchedule()
        check(self.lib.nemo_ens_get_schedule(self.h, ctypes.byref(s)), "nemo_ens_get_schedule")
        return (s.warps, s.occupancy, s.rows, s.order, s.ctas)

    def use_graph(self, on):
        check(self.lib.nemo_ens_use_graph(self.h, 1 if on else 0), "nemo_ens_use_graph")

    def info(self):
        n = ctypes.c_int()
        c = ctypes.c_longlong()
        check(self.lib.nemo_ens_info(self.h, ctypes.byref(n), ctypes.byref(c)), "nemo_ens_info")
        return n.value, c.value

    def autotune(self, steps=5):
        s = EnsSchedule()
        ms = ctypes.c_double()
        check(self.lib.nemo_ens_autotune(self.h, steps, ctypes.byref(s), ctypes.byref(ms)),
              "nemo_ens_autotune")
        return (s.warps, s.occupancy, s.rows, s.order, s.ctas), ms.value
