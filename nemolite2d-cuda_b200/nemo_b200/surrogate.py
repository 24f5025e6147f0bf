"""BF16 convolutional surrogate, hybrid controller and single-convolution
entry points of the C ABI (nemo_sur_*, nemo_hyb_*, nemo_conv3x3_*).

Device buffers are passed as integer addresses (for instance a torch
tensor's data_ptr()); the surrogate orders its work on its own stream unless
given one, and every call that returns host data has finished on the device.
"""
import ctypes

import numpy as np

from . import check, load


class SurConfig(ctypes.Structure):
    _fields_ = [("nblocks", ctypes.c_int), ("batch", ctypes.c_int), ("height", ctypes.c_int),
                ("width", ctypes.c_int), ("train", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("stream", ctypes.c_void_p), ("device", ctypes.c_int), ("patch", ctypes.c_int)]


class AdamW(ctypes.Structure):
    _fields_ = [("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float),
                ("eps", ctypes.c_float), ("weight_decay", ctypes.c_float)]


class HybConfig(ctypes.Structure):
    _fields_ = [("k", ctypes.c_int), ("anchor", ctypes.c_int), ("tol", ctypes.c_double),
                ("per_member", ctypes.c_int), ("quarantine", ctypes.c_double), ("rewind", ctypes.c_int),
                ("correct", ctypes.c_int)]


class HybStats(ctypes.Structure):
    _fields_ = [("sur_calls", ctypes.c_longlong), ("sur_steps", ctypes.c_longlong),
                ("solver_steps", ctypes.c_longlong), ("fallbacks", ctypes.c_longlong),
                ("windows", ctypes.c_longlong),
                ("max_shadow_err", ctypes.c_double), ("last_shadow_err", ctypes.c_double),
                ("seconds", ctypes.c_double), ("launches", ctypes.c_longlong),
                ("quarantined", ctypes.c_longlong), ("rewound", ctypes.c_longlong)]


def declare(L):
    vp, ip, dp, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_float
    P = ctypes.POINTER
    L.nemo_sur_default_config.argtypes = [P(SurConfig)]
    L.nemo_sur_create.argtypes = [P(SurConfig), P(vp)]
    L.nemo_sur_destroy.argtypes = [vp]
    L.nemo_sur_info.argtypes = [vp, P(ctypes.c_longlong), P(ctypes.c_longlong)]
    for n in ("nemo_sur_get_params", "nemo_sur_set_params", "nemo_sur_get_grads",
              "nemo_sur_set_norm", "nemo_sur_get_norm"):
        getattr(L, n).argtypes = [vp, P(fp)]
    L.nemo_sur_predict.argtypes = [vp, vp, vp, ip, vp]
    L.nemo_sur_loss_grad.argtypes = [vp, vp, vp, vp, ip, P(dp)]
    L.nemo_sur_adamw.argtypes = [vp, P(AdamW)]
    L.nemo_sur_train_step.argtypes = [vp, vp, vp, vp, ip, P(AdamW), P(dp)]
    L.nemo_sur_pack_ens.argtypes = [vp, vp, vp]
    L.nemo_sur_advance_ens.argtypes = [vp, vp, ip]
    L.nemo_ens_compare.argtypes = [vp, vp, P(dp)]
    L.nemo_hyb_default_config.argtypes = [P(HybConfig)]
    L.nemo_hyb_run.argtypes = [vp, vp, P(HybConfig), ip, ip, P(HybStats)]
    L.nemo_conv3x3_fwd.argtypes = [vp, vp, vp, vp, vp, ip, vp, vp, ip, ip, ip, vp, vp]
    L.nemo_conv3x3_wgrad.argtypes = [vp, vp, vp, vp, ip, ip, ip, ip, vp, vp]
    L.nemo_conv3x3_fwd_variant.argtypes = [ip, ip]
    L.nemo_conv3x3_wgrad_variant.argtypes = [ip]


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def adamw(lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=1e-4):
    return AdamW(lr, beta1, beta2, eps, weight_decay)


class Surrogate:
    """A nemo_sur: the residual CNN with its FP32 master parameters."""

    def __init__(self, nblocks=8, batch=64, height=256, width=256, train=True, seed=1234,
                 stream=None, device=-1, strict=False, patch=1):
        self.lib = load(strict)
        c = SurConfig()
        check(self.lib.nemo_sur_default_config(ctypes.byref(c)), "nemo_sur_default_config")
        c.nblocks, c.batch, c.height, c.width = nblocks, batch, height, width
        c.train, c.seed, c.stream, c.device = int(bool(train)), seed, stream, device
        c.patch = patch
        self.cfg = c
        h = ctypes.c_void_p()
        check(self.lib.nemo_sur_create(ctypes.byref(c), ctypes.byref(h)), "nemo_sur_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.nemo_sur_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        n, f = ctypes.c_longlong(), ctypes.c_longlong()
        check(self.lib.nemo_sur_info(self.h, ctypes.byref(n), ctypes.byref(f)), "nemo_sur_info")
        return n.value, f.value

    @property
    def patch(self):
        return self.cfg.patch

    def out_shape(self, n):
        """Shape of predict's FP32 output for n images."""
        P = self.cfg.patch
        if P == 1:
            return (n, self.cfg.height, self.cfg.width, 4)
        return (n, self.cfg.height // P, self.cfg.width // P, 3 * P * P)

    @property
    def nlayers(self):
        return 2 * self.cfg.nblocks + 2

    def params(self):
        out = np.empty(self.info()[0], dtype=np.float32)
        check(self.lib.nemo_sur_get_params(self.h, _fptr(out)), "nemo_sur_get_params")
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.info()[0]
        check(self.lib.nemo_sur_set_params(self.h, _fptr(p)), "nemo_sur_set_params")

    def grads(self):
        out = np.empty(self.info()[0], dtype=np.float32)
        check(self.lib.nemo_sur_get_grads(self.h, _fptr(out)), "nemo_sur_get_grads")
        return out

    def split(self, flat):
        """(weights [L][9][64][64], biases [L][64]) views of a flat parameter array."""
        L = self.nlayers
        nw = L * 9 * 64 * 64
        return flat[:nw].reshape(L, 9, 64, 64), flat[nw:].reshape(L, 64)

    def set_norm(self, in_scale, in_shift, out_scale):
        a = np.array(list(in_scale) + list(in_shift) + list(out_scale), dtype=np.float32)
        assert a.size == 11
        check(self.lib.nemo_sur_set_norm(self.h, _fptr(a)), "nemo_sur_set_norm")

    def get_norm(self):
        a = np.empty(11, dtype=np.float32)
        check(self.lib.nemo_sur_get_norm(self.h, _fptr(a)), "nemo_sur_get_norm")
        return a[:4].copy(), a[4:8].copy(), a[8:].copy()

    def predict(self, snap, tide, n, out=None):
        check(self.lib.nemo_sur_predict(self.h, snap, tide, n, out), "nemo_sur_predict")

    def loss_grad(self, snap0, snap1, tide, n):
        loss = ctypes.c_double()
        check(self.lib.nemo_sur_loss_grad(self.h, snap0, snap1, tide, n, ctypes.byref(loss)),
              "nemo_sur_loss_grad")
        return loss.value

    def adamw(self, hp):
        check(self.lib.nemo_sur_adamw(self.h, ctypes.byref(hp)), "nemo_sur_adamw")

    def train_step(self, snap0, snap1, tide, n, hp):
        loss = ctypes.c_double()
        check(self.lib.nemo_sur_train_step(self.h, snap0, snap1, tide, n, ctypes.byref(hp),
                                           ctypes.byref(loss)), "nemo_sur_train_step")
        return loss.value

    def pack_ens(self, ens, snap):
        check(self.lib.nemo_sur_pack_ens(self.h, ens.h, snap), "nemo_sur_pack_ens")

    def advance_ens(self, ens, istp_end):
        check(self.lib.nemo_sur_advance_ens(self.h, ens.h, istp_end), "nemo_sur_advance_ens")

    def save(self, path):
        sc, sh, osc = self.get_norm()
        np.savez(path, params=self.params(), in_scale=sc, in_shift=sh, out_scale=osc,
                 nblocks=self.cfg.nblocks, patch=self.cfg.patch)

    def load_file(self, path):
        z = np.load(path)
        assert int(z["nblocks"]) == self.cfg.nblocks
        assert int(z["patch"]) == self.cfg.patch if "patch" in z else self.cfg.patch == 1
        self.set_params(z["params"])
        self.set_norm(z["in_scale"], z["in_shift"], z["out_scale"])


def ens_compare(a, ref):
    """Relative L2 difference per member of a against ref: array (nmem, 3) for ssh, u, v."""
    out = np.empty(3 * len(a.members), dtype=np.float64)
    check(a.lib.nemo_ens_compare(a.h, ref.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
          "nemo_ens_compare")
    return out.reshape(-1, 3)


def hyb_run(sur, ens, istp0, nsteps, k=10, anchor=100, tol=0.01, per_member=True, quarantine=0.05,
            rewind=True, correct=False):
    """Hybrid run (nemo_hyb_run); returns the statistics as a dict (counts of
    member-windows and member-steps).  quarantine: shadow error beyond which a
    member stays on the FP64 solver (0: never); rewind: such a member (and,
    after the last window, a diverged one) restarts from its FP64 state at the
    start of the latest recent window the surrogate advanced it in; correct:
    the calls of an accepted window add the shadow step's correction of the
    window's first prediction."""
    c = HybConfig(k, anchor, tol, int(bool(per_member)), quarantine, int(bool(rewind)),
                  int(bool(correct)))
    st = HybStats()
    check(sur.lib.nemo_hyb_run(sur.h, ens.h, ctypes.byref(c), istp0, nsteps, ctypes.byref(st)),
          "nemo_hyb_run")
    return {f: getattr(st, f) for f, _ in HybStats._fields_}


def conv3x3_fwd(lib, x, w, n, h, wd, err, bias=None, residual=None, mask=None, relu=False,
                out=None, out32=None, stream=None):
    check(lib.nemo_conv3x3_fwd(x, w, bias, residual, mask, int(bool(relu)), out, out32, n, h, wd,
                               err, stream), "nemo_conv3x3_fwd")


def conv3x3_fwd_variant(lib, variant, rows=0):
    """Select the forward kernel process-wide (4, the default: three output
    rows per MMA with TMA stores of the outputs; 2: the same with per-thread
    stores; 3: 2 with two CTAs per SM; 1: row ring; 0: window per tap) and the
    rows per strip (default 32) of the
    ring kernels; returns the previous variant."""
    return lib.nemo_conv3x3_fwd_variant(variant, rows)


def conv3x3_wgrad_variant(lib, variant):
    """Select the weight-gradient kernel process-wide (2: all taps per CTA with
    a fixed-order sum of the CTAs' partials; 3, the default: the same with
    128-pixel column chunks where the width allows; 1: three vertical
    taps per MMA; 0: tap pairs); returns the previous variant (-1 only
    queries)."""
    return lib.nemo_conv3x3_wgrad_variant(variant)


def conv3x3_wgrad(lib, x, dz, dw, n, h, wd, err, db=None, ctas=0, stream=None):
    check(lib.nemo_conv3x3_wgrad(x, dz, dw, db, n, h, wd, ctas, err, stream), "nemo_conv3x3_wgrad")
