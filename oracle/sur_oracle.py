"""CPU FP64 restatement of the surrogate network (test infrastructure only).

Checks the B200 surrogate's tcgen05 convolution kernels (forward, data
gradient, weight and bias gradients), its loss, its AdamW update and its
whole-network gradients.  The surrogate has no counterpart in the reference,
so parity here is against this restatement, which is pinned by central
finite differences of its own FP64 backward pass (tests/test_sur_oracle.py).

Conventions match the library: NHWC tensors with 64 channels, weights
w[tap][co][ci] with tap = 3*(dy+1) + (dx+1), zero padding,
out[n, y, x, co] = sum_{tap, ci} x[n, y+dy, x+dx, ci] * w[tap, co, ci].
With `bf16=True` the forward and backward round every stored activation and
gradient tensor to BF16 where the device stores BF16, so that only the
accumulation precision (FP32 on the device) differs.
"""
import numpy as np

CH = 64


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(a):
    """BF16 bit patterns (uint16) of bf16(a)."""
    return (bf16(a).astype(np.float32).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(u):
    return (np.asarray(u, dtype=np.uint32) << 16).view(np.float32).astype(np.float64)


def _shifted(x, dy, dx):
    """x[n, y+dy, x+dx, :] with zeros outside the image."""
    N, H, W, C = x.shape
    out = np.zeros_like(x)
    ys, ye = max(0, -dy), min(H, H - dy)
    xs, xe = max(0, -dx), min(W, W - dx)
    out[:, ys:ye, xs:xe] = x[:, ys + dy:ye + dy, xs + dx:xe + dx]
    return out


def conv3x3(x, w):
    """Raw 3x3 convolution accumulator (FP64)."""
    acc = np.zeros(x.shape[:3] + (w.shape[1],), dtype=np.float64)
    for tap in range(9):
        dy, dx = tap // 3 - 1, tap % 3 - 1
        acc += _shifted(x, dy, dx) @ w[tap].T
    return acc


def epilogue(acc, bias=None, residual=None, mask=None, relu=False):
    v = acc.copy()
    if bias is not None:
        v += bias
    if residual is not None:
        v += residual
    if mask is not None:
        v = np.where(mask > 0, v, 0.0)
    if relu:
        v = np.maximum(v, 0.0)
    return v


def wgrad(x, dz):
    """dw[tap, co, ci] = sum_p dz[p, co] x[p + off(tap), ci]; db[co] = sum_p dz[p, co]."""
    dw = np.zeros((9, dz.shape[-1], x.shape[-1]))
    dzf = dz.reshape(-1, dz.shape[-1])
    for tap in range(9):
        dy, dx = tap // 3 - 1, tap % 3 - 1
        dw[tap] = dzf.T @ _shifted(x, dy, dx).reshape(-1, x.shape[-1])
    return dw, dzf.sum(axis=0)


def flip_transpose(w):
    """Weights of the data gradient: wt[tap, ci, co] = w[8 - tap, co, ci]."""
    return np.ascontiguousarray(w[::-1].transpose(0, 2, 1))


# ---- network ---------------------------------------------------------------------
def split_params(flat, nblocks):
    L = 2 * nblocks + 2
    nw = L * 9 * CH * CH
    return flat[:nw].reshape(L, 9, CH, CH), flat[nw:].reshape(L, CH)


def out_channels(patch):
    """FP32 output channels per network pixel."""
    return 4 if patch == 1 else 3 * patch * patch


def to_patches(f, patch):
    """(N, H, W, F) per T-cell -> (N, H/P, W/P, F*P*P), channel f*P*P + P*sy + sx."""
    N, H, W, F = f.shape
    P = patch
    g = f.reshape(N, H // P, P, W // P, P, F)            # n, Y, sy, X, sx, f
    return g.transpose(0, 1, 3, 5, 2, 4).reshape(N, H // P, W // P, F * P * P)


def from_patches(g, patch, nf):
    """Inverse of to_patches for the first nf*P*P channels."""
    N, Hn, Wn, _ = g.shape
    P = patch
    h = g[..., :nf * P * P].reshape(N, Hn, Wn, nf, P, P)  # n, Y, X, f, sy, sx
    return h.transpose(0, 1, 4, 2, 5, 3).reshape(N, Hn * P, Wn * P, nf)


def make_input(snap, tide, in_scale, in_shift, patch=1):
    """x0 (N, H/P, W/P, 64) from snapshots (N, H, W, 4) and tides (N,), in
    float32 arithmetic as the device does it.  Channels: ssh, u, v of the
    patch's T-cells (P*P each), depth (one channel for P = 1, else the means
    of the four P/2 x P/2 quadrants), the open-boundary row flag and the tide
    on network row 0."""
    snap = np.asarray(snap, dtype=np.float32)
    N, H, W, _ = snap.shape
    P = patch
    sc = np.asarray(in_scale, dtype=np.float32)
    sh = np.asarray(in_shift, dtype=np.float32)
    f = (snap - sh) * sc
    x = np.zeros((N, H // P, W // P, CH), dtype=np.float32)
    x[..., :3 * P * P] = to_patches(f[..., :3], P)
    if P == 1:
        x[..., 3] = f[..., 3]
        fc = 4
    else:
        d = f[..., 3].reshape(N, H // P, 2, P // 2, W // P, 2, P // 2)  # n Y qy sy X qx sx
        acc = np.zeros((N, H // P, 2, W // P, 2), dtype=np.float32)
        for sy in range(P // 2):                # the device's summation order
            for sx in range(P // 2):
                acc = acc + d[:, :, :, sy, :, :, sx]
        q = acc * np.float32(4.0 / (P * P))
        x[..., 3 * P * P:3 * P * P + 4] = q.transpose(0, 1, 3, 2, 4).reshape(N, H // P, W // P, 4)
        fc = 3 * P * P + 4
    x[:, 0, :, fc] = 1.0
    t = (np.asarray(tide, dtype=np.float32) - sh[0]) * sc[0]
    x[:, 0, :, fc + 1] = t[:, None]
    return x


def make_target(snap0, snap1, out_scale):
    """Normalised deltas per T-cell (N, H, W, 4), channel 3 zero."""
    d = (np.asarray(snap1, np.float32) - np.asarray(snap0, np.float32))[..., :3]
    t = np.zeros(d.shape[:-1] + (4,), dtype=np.float32)
    t[..., :3] = d * np.asarray(out_scale, np.float32)
    return t


def forward(x0, W, B, nblocks, bf16_acts=True):
    """Returns (y [N,Hn,Wn,64] FP64 network output, cache of activations)."""
    r = bf16 if bf16_acts else (lambda a: a)
    Wq = bf16(W) if bf16_acts else W
    x0 = r(x0)
    h = [r(epilogue(conv3x3(x0, Wq[0]), B[0], relu=True))]
    t = []
    for i in range(nblocks):
        ti = r(epilogue(conv3x3(h[i], Wq[1 + 2 * i]), B[1 + 2 * i], relu=True))
        t.append(ti)
        h.append(r(epilogue(conv3x3(ti, Wq[2 + 2 * i]), B[2 + 2 * i], residual=h[i])))
    y = epilogue(conv3x3(h[-1], Wq[-1]), B[-1])
    return y, dict(x0=x0, h=h, t=t, Wq=Wq)


def deltas(y, patch=1):
    """Per-T-cell deltas (N, H, W, 3) of a network output (N, Hn, Wn, 64)."""
    return y[..., :3] if patch == 1 else from_patches(y, patch, 3)


def loss_and_dout(y, target, bf16_acts=True, patch=1):
    d = deltas(y, patch) - np.asarray(target, dtype=np.float64)[..., :3]
    npix = d.shape[0] * d.shape[1] * d.shape[2]
    loss = float((d * d).sum() / (3.0 * npix))
    g = 2.0 * d / (3.0 * npix)
    if bf16_acts:
        # the device forms 2 * gscale * d in float32 before rounding
        gs = np.float32(1.0 / (3.0 * npix))
        g = (np.float32(2.0) * gs * d.astype(np.float32)).astype(np.float64)
        g = bf16(g)
    dout = np.zeros(y.shape[:3] + (CH,))
    if patch == 1:
        dout[..., :3] = g
    else:
        dout[..., :3 * patch * patch] = to_patches(g, patch)
    return loss, dout


def backward(dout, cache, nblocks, bf16_acts=True):
    """Gradients (dW [L,9,64,64], dB [L,64]) of the loss whose output gradient is dout."""
    r = bf16 if bf16_acts else (lambda a: a)
    Wq, h, t, x0 = cache["Wq"], cache["h"], cache["t"], cache["x0"]
    L = 2 * nblocks + 2
    dW = np.zeros((L, 9, CH, CH))
    dB = np.zeros((L, CH))
    dW[L - 1], dB[L - 1] = wgrad(h[-1], dout)
    g = conv3x3(dout, flip_transpose(Wq[L - 1]))
    if nblocks == 0:
        g = np.where(h[0] > 0, g, 0.0)
    g = r(g)
    for i in reversed(range(nblocks)):
        la, lb = 1 + 2 * i, 2 + 2 * i
        dW[lb], dB[lb] = wgrad(t[i], g)
        dt = r(epilogue(conv3x3(g, flip_transpose(Wq[lb])), mask=t[i]))
        dW[la], dB[la] = wgrad(h[i], dt)
        gn = epilogue(conv3x3(dt, flip_transpose(Wq[la])), residual=g, mask=h[0] if i == 0 else None)
        g = r(gn)
    dW[0], dB[0] = wgrad(x0, g)
    return dW, dB


def loss_grad(flat_params, nblocks, snap0, snap1, tide, norm, bf16_acts=True, patch=1):
    """Loss and flat gradient (weights then biases) as nemo_sur_loss_grad."""
    in_scale, in_shift, out_scale = norm
    W, B = split_params(np.asarray(flat_params, dtype=np.float64), nblocks)
    x0 = make_input(snap0, tide, in_scale, in_shift, patch).astype(np.float64)
    tgt = make_target(snap0, snap1, out_scale)
    y, cache = forward(x0, W, B, nblocks, bf16_acts)
    loss, dout = loss_and_dout(y, tgt, bf16_acts, patch)
    dW, dB = backward(dout, cache, nblocks, bf16_acts)
    return loss, np.concatenate([dW.ravel(), dB.ravel()])


def adamw(p, g, m, v, t, lr, b1, b2, eps, wd, nw):
    """One AdamW step in float32 (decoupled decay on the first nw entries)."""
    f = np.float32
    p, g, m, v = (np.asarray(a, dtype=np.float32).copy() for a in (p, g, m, v))
    m = f(b1) * m + (f(1) - f(b1)) * g
    v = f(b2) * v + (f(1) - f(b2)) * g * g
    # bias corrections from the float32 betas, in double, then rounded
    bc1 = f(1.0 - float(f(b1)) ** t)
    bc2 = f(1.0 - float(f(b2)) ** t)
    upd = (m / bc1) / (np.sqrt(v / bc2) + f(eps))
    upd[:nw] += f(wd) * p[:nw]
    p = p - f(lr) * upd
    return p, m, v
