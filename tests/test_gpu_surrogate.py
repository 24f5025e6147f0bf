"""tcgen05/TMA convolution kernels, the surrogate's training step and the
hybrid controller against the CPU FP64 oracle (oracle/sur_oracle.py).

Tolerances: BF16 outputs within 1 BF16 ulp of the oracle rounded to BF16
(FP32 device accumulation vs FP64 can flip a rounding); FP32 outputs within
1e-4 of the output's max-norm; whole-network gradients within 2e-2 normwise
per layer (BF16 activations and gradients in both, FP32 vs FP64 sums).
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from oracle import sur_oracle as so


@pytest.fixture(scope="module")
def env():
    import torch
    import nemo_b200
    from nemo_b200 import surrogate as sm
    return torch, nemo_b200, sm


def dev_bf16(torch, a):
    bits = so.bf16_bits(a).view(np.int16)
    return torch.from_numpy(bits.copy()).view(torch.bfloat16).cuda()


def host_bf16(torch, t):
    return so.from_bf16_bits(t.view(torch.int16).cpu().numpy().view(np.uint16))


def ulp_close(got, ref):
    """|got - ref| <= 1 BF16 ulp of ref (plus a tiny absolute floor)."""
    tol = np.abs(ref) * 2.0 ** -7 + 1e-30
    bad = np.abs(got - ref) > tol
    return bad.mean(), np.abs(got - ref).max()


@pytest.fixture(params=[(2, 16), (2, 2), (2, 1), (2, 5), (3, 16), (3, 2), (3, 1), (4, 16), (4, 1), (4, 5),
                        (1, 16), (1, 2), (0, 0)],
                ids=["tri16", "tri2", "tri1", "tri5", "tri2cta16", "tri2cta2", "tri2cta1", "tritma16",
                     "tritma1", "tritma5", "rows16", "rows2", "per-tap"])
def variant(request, env):
    """Each forward kernel variant (three output rows per MMA with 16, 2, 1 or
    5 rows per strip, the same two CTAs per SM, the same with TMA stores of
    the output, row ring with 16 or 2 rows per strip, window per tap),
    restored to the default afterwards."""
    torch, nb, sm = env
    lib = nb.load(False)
    prev = sm.conv3x3_fwd_variant(lib, *request.param)
    yield request.param
    sm.conv3x3_fwd_variant(lib, prev, 32)  # the default, restored


def run_fwd(torch, sm, lib, x, w, bias=None, residual=None, mask=None, relu=False, out32=False):
    N, H, W, _ = x.shape
    xd, wd = dev_bf16(torch, x), dev_bf16(torch, w)
    bd = torch.from_numpy(np.asarray(bias, np.float32)).cuda() if bias is not None else None
    rd = dev_bf16(torch, residual) if residual is not None else None
    md = dev_bf16(torch, mask) if mask is not None else None
    out = torch.empty((N, H, W, 64), dtype=torch.bfloat16, device="cuda")
    o32 = torch.empty((N, H, W, 4), dtype=torch.float32, device="cuda") if out32 else None
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ptr = lambda t: t.data_ptr() if t is not None else None
    sm.conv3x3_fwd(lib, xd.data_ptr(), wd.data_ptr(), N, H, W, err.data_ptr(), bias=ptr(bd),
                   residual=ptr(rd), mask=ptr(md), relu=relu, out=out.data_ptr(), out32=ptr(o32),
                   stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return host_bf16(torch, out), (o32.cpu().numpy().astype(np.float64) if out32 else None)


@pytest.mark.parametrize("tap", range(9))
def test_fwd_one_hot_tap_is_an_exact_shift(env, variant, tap):
    torch, nb, sm = env
    rng = np.random.default_rng(tap)
    x = so.bf16(rng.normal(size=(2, 5, 256, 64)))
    w = np.zeros((9, 64, 64))
    perm = rng.permutation(64)
    w[tap][np.arange(64), perm] = 1.0  # out channel co reads input channel perm[co]
    got, _ = run_fwd(torch, sm, nb.load(False), x, w)
    ref = so.conv3x3(x, w)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("shape", [(2, 6, 128), (1, 3, 384), (3, 1, 256), (2, 37, 128)])
def test_fwd_random_matches_oracle(env, variant, shape):
    torch, nb, sm = env
    N, H, W = shape
    rng = np.random.default_rng(N * 100 + H)
    x = so.bf16(rng.normal(size=(N, H, W, 64)))
    w = so.bf16(rng.normal(0, 0.1, size=(9, 64, 64)))
    b = rng.normal(size=64).astype(np.float32)
    res = so.bf16(rng.normal(size=(N, H, W, 64)))
    mask = so.bf16(rng.normal(size=(N, H, W, 64)))
    lib = nb.load(False)
    for kw in (dict(), dict(bias=b, relu=True), dict(bias=b, residual=res), dict(residual=res, mask=mask)):
        got, o32 = run_fwd(torch, sm, lib, x, w, out32=True, **kw)
        ref = so.epilogue(so.conv3x3(x, w), kw.get("bias"), kw.get("residual"), kw.get("mask"),
                          kw.get("relu", False))
        frac, _ = ulp_close(got, so.bf16(ref))
        assert frac < 2e-3, (kw.keys(), frac)
        assert np.abs(o32 - ref[..., :4]).max() <= 1e-4 * np.abs(ref[..., :4]).max()


def test_dgrad_with_flipped_weights_matches_oracle(env, variant):
    torch, nb, sm = env
    rng = np.random.default_rng(7)
    dz = so.bf16(rng.normal(size=(2, 4, 128, 64)))
    w = so.bf16(rng.normal(0, 0.1, size=(9, 64, 64)))
    t = so.bf16(np.maximum(rng.normal(size=(2, 4, 128, 64)), 0))
    got, o32 = run_fwd(torch, sm, nb.load(False), dz, so.flip_transpose(w), mask=t, out32=True)
    ref = so.epilogue(so.conv3x3(dz, so.flip_transpose(w)), mask=t)
    frac, _ = ulp_close(got, so.bf16(ref))
    assert frac < 2e-3
    assert np.abs(o32 - ref[..., :4]).max() <= 1e-4 * np.abs(ref[..., :4]).max()


@pytest.fixture(params=[2, 3, 1, 0], ids=["wg-strip", "wg-strip128", "wg-tri", "wg-pairs"])
def wvariant(request, env):
    """Each weight-gradient kernel (all taps per CTA with a fixed-order sum, in
    64- and 128-pixel column chunks; six taps per MMA; tap pairs), restored to
    the default afterwards."""
    torch, nb, sm = env
    lib = nb.load(False)
    prev = sm.conv3x3_wgrad_variant(lib, request.param)
    yield request.param
    sm.conv3x3_wgrad_variant(lib, prev)


@pytest.mark.parametrize("shape,ctas", [((2, 5, 128), 0), ((1, 7, 192), 3), ((3, 2, 64), 1), ((1, 1, 64), 0),
                                        ((2, 13, 256), 5), ((1, 3, 384), 0)])
def test_wgrad_and_bias_grad_match_oracle(env, wvariant, shape, ctas):
    torch, nb, sm = env
    N, H, W = shape
    rng = np.random.default_rng(H * W)
    x = so.bf16(rng.normal(size=(N, H, W, 64)))
    dz = so.bf16(rng.normal(size=(N, H, W, 64)))
    dw = torch.full((9, 64, 64), 0.5, dtype=torch.float32, device="cuda")  # accumulates
    db = torch.full((64,), -1.0, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    xd, dzd = dev_bf16(torch, x), dev_bf16(torch, dz)  # referenced until the kernel is done
    sm.conv3x3_wgrad(nb.load(False), xd.data_ptr(), dzd.data_ptr(), dw.data_ptr(), N, H, W,
                     err.data_ptr(), db=db.data_ptr(), ctas=ctas,
                     stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    rw, rb = so.wgrad(x, dz)
    gw = dw.cpu().numpy() - 0.5
    gb = db.cpu().numpy() + 1.0
    assert np.abs(gw - rw).max() <= 1e-4 * np.abs(rw).max()
    assert np.abs(gb - rb).max() <= 1e-4 * np.abs(rb).max()


@pytest.mark.parametrize("shape,ctas", [((4, 33, 256), 0), ((2, 9, 128), 7)])
def test_default_wgrad_is_bitwise_repeatable(env, shape, ctas):
    """The default weight gradient sums per-CTA partials in a fixed order: the
    same inputs give the same bits on every call (the atomic variants do not
    promise that)."""
    torch, nb, sm = env
    lib = nb.load(False)
    assert sm.conv3x3_wgrad_variant(lib, -1) == 3  # the default
    N, H, W = shape
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn((N, H, W, 64), device="cuda", generator=g).to(torch.bfloat16)
    dz = torch.randn((N, H, W, 64), device="cuda", generator=g).to(torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    outs = []
    for _ in range(3):
        dw = torch.zeros((9, 64, 64), dtype=torch.float32, device="cuda")
        db = torch.zeros(64, dtype=torch.float32, device="cuda")
        sm.conv3x3_wgrad(lib, x.data_ptr(), dz.data_ptr(), dw.data_ptr(), N, H, W, err.data_ptr(),
                         db=db.data_ptr(), ctas=ctas, stream=torch.cuda.current_stream().cuda_stream)
        outs.append((dw.cpu().numpy().view(np.int32), db.cpu().numpy().view(np.int32)))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    for dw, db in outs[1:]:
        np.testing.assert_array_equal(dw, outs[0][0])
        np.testing.assert_array_equal(db, outs[0][1])


def test_training_is_reproducible(env):
    """Two surrogates with the same seed trained on the same batches end with
    bit-identical parameters: every kernel of the training step, the weight
    gradient included, is free of order-dependent sums."""
    torch, nb, sm = env
    N, H, W = 4, 16, 128
    rng = np.random.default_rng(12)
    snap0, snap1, tide, norm, d = random_setup(rng, torch, N, H, W)
    hp = sm.adamw(lr=2e-3, weight_decay=1e-4)
    params = []
    for _ in range(2):
        s = sm.Surrogate(nblocks=2, batch=N, height=H, width=W, seed=31)
        s.set_norm(*norm)
        for _ in range(5):
            s.train_step(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), N, hp)
        torch.cuda.synchronize()
        params.append(s.params())
        s.close()
    np.testing.assert_array_equal(params[0].view(np.int32), params[1].view(np.int32))


def test_conv_rejects_unsupported_shapes(env):
    """Widths the kernels do not tile are refused before any launch (the
    buffers are sized for the request, so nothing could go out of bounds)."""
    torch, nb, sm = env
    lib = nb.load(False)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    x = torch.zeros((1, 2, 96, 64), dtype=torch.bfloat16, device="cuda")
    w = torch.zeros((9, 64, 64), dtype=torch.bfloat16, device="cuda")
    out = torch.zeros_like(x)
    dw = torch.zeros((9, 64, 64), dtype=torch.float32, device="cuda")
    with pytest.raises(nb.NemoError):  # 96 is not a multiple of 128
        sm.conv3x3_fwd(lib, x.data_ptr(), w.data_ptr(), 1, 2, 96, err.data_ptr(), out=out.data_ptr())
    with pytest.raises(nb.NemoError):  # 96 is not a multiple of 64
        sm.conv3x3_wgrad(lib, x.data_ptr(), x.data_ptr(), dw.data_ptr(), 1, 2, 96, err.data_ptr())
    torch.cuda.synchronize()
    assert not out.any() and not dw.any() and int(err.item()) == 0


def random_setup(rng, torch, N, H, W):
    snap0 = rng.normal(size=(N, H, W, 4)).astype(np.float32)
    snap1 = (snap0 + rng.normal(0, 0.5, size=snap0.shape)).astype(np.float32)
    tide = rng.normal(size=N).astype(np.float32)
    norm = ([1.0, 2.0, 0.5, 1.5], [0.0, 0.1, 0.0, 0.2], [1.0, 0.8, 1.2])
    d = [torch.from_numpy(a).cuda() for a in (snap0, snap1, tide)]
    return snap0, snap1, tide, norm, d


@pytest.mark.parametrize("nblocks", [1, 2])
def test_network_loss_and_gradients_match_oracle(env, nblocks):
    torch, nb, sm = env
    N, H, W = 2, 6, 128
    rng = np.random.default_rng(10 + nblocks)
    s = sm.Surrogate(nblocks=nblocks, batch=N, height=H, width=W, seed=5)
    p = s.params()
    Wt, Bs = s.split(p)
    Bs[:] = rng.normal(0, 0.05, size=Bs.shape)
    Wt[-1, :, :3, :] = rng.normal(0, 0.05, size=Wt[-1, :, :3, :].shape)  # a larger output layer
    s.set_params(p)
    snap0, snap1, tide, norm, d = random_setup(rng, torch, N, H, W)
    s.set_norm(*norm)
    torch.cuda.synchronize()
    loss = s.loss_grad(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), N)
    g = s.grads()
    rloss, rg = so.loss_grad(p.astype(np.float64), nblocks, snap0, snap1, tide, norm, bf16_acts=True)
    assert abs(loss - rloss) <= 1e-3 * rloss
    gw, gb = s.split(g)
    rw, rb = so.split_params(rg, nblocks)
    for l in range(2 * nblocks + 2):
        e_w = np.linalg.norm(gw[l] - rw[l]) / np.linalg.norm(rw[l])
        e_b = np.linalg.norm(gb[l] - rb[l]) / np.linalg.norm(rb[l])
        assert e_w < 2e-2 and e_b < 2e-2, (l, e_w, e_b)
    # the padded input channels and unused output channels get no gradient
    assert not gw[0][:, :, 6:].any()
    assert not gw[-1][:, 3:, :].any()


def test_adamw_matches_oracle(env):
    torch, nb, sm = env
    N, H, W = 1, 4, 128
    rng = np.random.default_rng(3)
    s = sm.Surrogate(nblocks=1, batch=N, height=H, width=W, seed=9)
    snap0, snap1, tide, norm, d = random_setup(rng, torch, N, H, W)
    s.set_norm(*norm)
    p0 = s.params()
    hp = sm.adamw(lr=3e-3, weight_decay=0.05)
    s.loss_grad(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), N)
    g = s.grads()
    s.adamw(hp)
    p1 = s.params()
    nw = s.nlayers * 9 * 64 * 64
    z = np.zeros_like(p0)
    rp, _, _ = so.adamw(p0, g, z, z, 1, 3e-3, 0.9, 0.999, 1e-8, 0.05, nw)
    np.testing.assert_allclose(p1, rp, rtol=2e-6, atol=1e-8)
    assert not s.grads().any()  # cleared for the next accumulation


def test_predict_matches_oracle_forward(env):
    torch, nb, sm = env
    N, H, W = 2, 5, 128
    rng = np.random.default_rng(4)
    s = sm.Surrogate(nblocks=2, batch=N, height=H, width=W, train=False, seed=2)
    p = s.params()
    Wt, Bs = s.split(p)
    Wt[-1, :, :3, :] = rng.normal(0, 0.05, size=Wt[-1, :, :3, :].shape)
    s.set_params(p)
    snap0, _, tide, norm, d = random_setup(rng, torch, N, H, W)
    s.set_norm(*norm)
    out = torch.empty((N, H, W, 4), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    s.predict(d[0].data_ptr(), d[2].data_ptr(), N, out.data_ptr())
    Wr, Br = so.split_params(p.astype(np.float64), 2)
    x0 = so.make_input(snap0, tide, norm[0], norm[1]).astype(np.float64)
    y, _ = so.forward(x0, Wr, Br, 2, bf16_acts=True)
    got = out.cpu().numpy()
    assert np.abs(got[..., :3] - y[..., :3]).max() <= 2e-2 * np.abs(y[..., :3]).max()


@pytest.mark.parametrize("patch", [2, 4])
def test_patch_predict_matches_oracle_forward(env, patch):
    """The patch network: inputs gathered from P x P T-cells, FP32 outputs
    in the [n][h/P][w/P][3 P^2] layout."""
    torch, nb, sm = env
    P = patch
    N, H, W = 2, 3 * P, 128 * P
    rng = np.random.default_rng(40 + P)
    s = sm.Surrogate(nblocks=1, batch=N, height=H, width=W, train=False, seed=6, patch=P)
    p = s.params()
    Wt, Bs = s.split(p)
    Wt[-1, :, :3 * P * P, :] = rng.normal(0, 0.05, size=Wt[-1, :, :3 * P * P, :].shape)
    Bs[-1, :3 * P * P] = rng.normal(0, 0.05, size=3 * P * P)
    s.set_params(p)
    snap0, _, tide, norm, d = random_setup(rng, torch, N, H, W)
    s.set_norm(*norm)
    out = torch.empty(s.out_shape(N), dtype=torch.float32, device="cuda")
    assert s.out_shape(N) == (N, H // P, W // P, 3 * P * P)
    torch.cuda.synchronize()
    s.predict(d[0].data_ptr(), d[2].data_ptr(), N, out.data_ptr())
    Wr, Br = so.split_params(p.astype(np.float64), 1)
    x0 = so.make_input(snap0, tide, norm[0], norm[1], patch=P).astype(np.float64)
    y, _ = so.forward(x0, Wr, Br, 1, bf16_acts=True)
    got = out.cpu().numpy()
    ref = y[..., :3 * P * P]
    assert np.abs(got - ref).max() <= 2e-2 * np.abs(ref).max()


def test_patch_loss_and_gradients_match_oracle(env):
    torch, nb, sm = env
    P, N, H, W, nblocks = 2, 2, 6, 256, 1
    rng = np.random.default_rng(77)
    s = sm.Surrogate(nblocks=nblocks, batch=N, height=H, width=W, seed=8, patch=P)
    p = s.params()
    Wt, Bs = s.split(p)
    Bs[:] = rng.normal(0, 0.05, size=Bs.shape)
    Wt[-1, :, :12, :] = rng.normal(0, 0.05, size=Wt[-1, :, :12, :].shape)
    s.set_params(p)
    snap0, snap1, tide, norm, d = random_setup(rng, torch, N, H, W)
    s.set_norm(*norm)
    torch.cuda.synchronize()
    loss = s.loss_grad(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), N)
    g = s.grads()
    rloss, rg = so.loss_grad(p.astype(np.float64), nblocks, snap0, snap1, tide, norm,
                             bf16_acts=True, patch=P)
    assert abs(loss - rloss) <= 1e-3 * rloss
    gw, gb = s.split(g)
    rw, rb = so.split_params(rg, nblocks)
    for l in range(2 * nblocks + 2):
        e_w = np.linalg.norm(gw[l] - rw[l]) / np.linalg.norm(rw[l])
        e_b = np.linalg.norm(gb[l] - rb[l]) / np.linalg.norm(rb[l])
        assert e_w < 2e-2 and e_b < 2e-2, (l, e_w, e_b)
    # input channels past the tide and output channels past 3 P^2 get no gradient
    assert not gw[0][:, :, 3 * P * P + 6:].any()
    assert not gw[-1][:, 3 * P * P:, :].any()


def assert_flather_row(nb, e, m, ssh, v):
    """v(ji, 0) after a surrogate call: the solver's open-boundary closure
    v(ji,1) + sqrt(g/hv(ji,0)) * (sshn_v(ji,0) - sshn_v(ji,1)), with the stored
    sshn_v(ji,0) zero for members started from rest."""
    hv0 = e.field(m, nb.HV)[0]
    sv1 = 0.5 * (ssh[0] + ssh[1])
    np.testing.assert_allclose(v[0], v[1] + np.sqrt(9.80665 / hv0) * (0.0 - sv1), rtol=1e-13, atol=1e-300)


def small_ensemble(nb, seed, n, side):
    from nemo_b200 import train as tr
    return nb.Ensemble(tr.square_members(seed, n, side, 0.2), **tr.COMMON)


def test_pack_and_advance_follow_the_grid_layout(env):
    torch, nb, sm = env
    side, n = 128, 3
    e = small_ensemble(nb, 21, n, side)
    e.step_n(1, 60)
    s = sm.Surrogate(nblocks=1, batch=n, height=side, width=side, train=False, seed=3)
    snap = torch.empty((n, side, side, 4), dtype=torch.float32, device="cuda")
    s.pack_ens(e, snap.data_ptr())
    sn = snap.cpu().numpy()
    before = [[e.field(m, f) for f in (nb.SSHN, nb.UN, nb.VN, nb.HT)] for m in range(n)]
    for m in range(n):
        ssh, u, v, ht = before[m]
        np.testing.assert_array_equal(sn[m, ..., 0], ssh.astype(np.float32))
        np.testing.assert_array_equal(sn[m, ..., 1], u[:, :side].astype(np.float32))
        np.testing.assert_array_equal(sn[m, ..., 2], v[:side, :].astype(np.float32))
        np.testing.assert_array_equal(sn[m, ..., 3], ht.astype(np.float32))
    # one surrogate call: compare with predict's deltas
    from nemo_b200 import train as tr
    out = torch.empty_like(snap)
    tide = torch.tensor([tr.tide_of(mb, 70) for mb in e.members], dtype=torch.float32).cuda()
    torch.cuda.synchronize()
    s.predict(snap.data_ptr(), tide.data_ptr(), n, out.data_ptr())
    o = out.cpu().numpy()
    s.advance_ens(e, 70)
    _, _, osc = s.get_norm()
    for m in range(n):
        ssh0, u0, v0, _ = before[m]
        ssh, u, v = (e.field(m, f) for f in (nb.SSHN, nb.UN, nb.VN))
        exp = ssh0 + (o[m, ..., 0] / osc[0]).astype(np.float64)
        exp[0, :] = tr.tide_of(e.members[m], 70)
        np.testing.assert_allclose(ssh, exp, rtol=1e-12, atol=0)
        assert not u[:, 0].any() and not u[:, side].any() and not v[side, :].any()
        np.testing.assert_allclose(u[:, 1:side], u0[:, 1:side] + (o[m, :, 1:, 1] / osc[1]), rtol=1e-12)
        np.testing.assert_allclose(v[1:side, :], v0[1:side, :] + (o[m, 1:, :, 2] / osc[2]), rtol=1e-12)
        assert_flather_row(nb, e, m, ssh, v)


def test_patch_advance_applies_each_cells_delta(env):
    """One patch-4 surrogate call moves every T-cell by its own channel of
    the patch output."""
    torch, nb, sm = env
    from nemo_b200 import train as tr
    P, side, n = 4, 512, 2
    e = small_ensemble(nb, 23, n, side)
    e.step_n(1, 40)
    s = sm.Surrogate(nblocks=1, batch=n, height=side, width=side, train=False, seed=3, patch=P)
    p = s.params()
    Wt, Bs = s.split(p)
    Bs[-1, :48] = np.random.default_rng(5).normal(0, 0.1, size=48)
    s.set_params(p)
    s.set_norm([1, 1, 1, 1], [0, 0, 0, 100], [1e3, 1e3, 1e3])
    snap = torch.empty((n, side, side, 4), dtype=torch.float32, device="cuda")
    s.pack_ens(e, snap.data_ptr())
    out = torch.empty(s.out_shape(n), dtype=torch.float32, device="cuda")
    tide = torch.tensor([tr.tide_of(mb, 50) for mb in e.members], dtype=torch.float32).cuda()
    torch.cuda.synchronize()
    s.predict(snap.data_ptr(), tide.data_ptr(), n, out.data_ptr())
    o = so.from_patches(out.cpu().numpy().astype(np.float64), P, 3)
    before = [[e.field(m, f) for f in (nb.SSHN, nb.UN, nb.VN)] for m in range(n)]
    s.advance_ens(e, 50)
    _, _, osc = s.get_norm()
    for m in range(n):
        ssh0, u0, v0 = before[m]
        ssh, u, v = (e.field(m, f) for f in (nb.SSHN, nb.UN, nb.VN))
        exp = ssh0 + (o[m, ..., 0].astype(np.float32) / osc[0]).astype(np.float64)
        exp[0, :] = tr.tide_of(e.members[m], 50)
        np.testing.assert_allclose(ssh, exp, rtol=1e-12, atol=0)
        np.testing.assert_allclose(u[:, 1:side], u0[:, 1:side] + (o[m, :, 1:, 1].astype(np.float32) / osc[1]),
                                   rtol=1e-12)
        np.testing.assert_allclose(v[1:side, :], v0[1:side, :] + (o[m, 1:, :, 2].astype(np.float32) / osc[2]),
                                   rtol=1e-12)
        assert_flather_row(nb, e, m, ssh, v)
        assert not u[:, 0].any() and not u[:, side].any() and not v[side, :].any()


def test_hybrid_with_zero_tolerance_reproduces_the_solver_bitwise(env):
    torch, nb, sm = env
    side, n = 128, 2
    a = small_ensemble(nb, 31, n, side)
    b = small_ensemble(nb, 31, n, side)
    s = sm.Surrogate(nblocks=1, batch=n, height=side, width=side, train=False, seed=4)
    st = sm.hyb_run(s, a, 0, 300, tol=1e-300)  # every window falls back
    b.step_n(1, 300)
    assert st["fallbacks"] == 3 * n and st["windows"] == 3 * n
    assert st["solver_steps"] == 300 * n and st["sur_steps"] == 0
    for m in range(n):
        for f in (nb.SSHN, nb.UN, nb.VN):
            np.testing.assert_array_equal(a.field(m, f), b.field(m, f))
    assert np.all(sm.ens_compare(a, b) == 0.0)


def test_hybrid_accepts_surrogate_windows_and_reports_errors(env):
    torch, nb, sm = env
    side, n = 128, 2
    a = small_ensemble(nb, 41, n, side)
    b = small_ensemble(nb, 41, n, side)
    s = sm.Surrogate(nblocks=1, batch=1, height=side, width=side, train=False, seed=4)  # 2 chunks
    st = sm.hyb_run(s, a, 0, 200, k=10, anchor=100, tol=1e300, quarantine=0.0)  # never falls back
    b.step_n(1, 200)
    assert st["fallbacks"] == 0 and st["sur_steps"] == 180 * n and st["solver_steps"] == 20 * n
    assert st["sur_calls"] == 20 and st["max_shadow_err"] > 0
    # 20 solver launches; a window's shadow prediction packs, builds the input
    # and runs the 4 convolutions per chunk of one member, then the error
    # kernel; each of the 9 calls per window adds apply and the boundary closure
    per_predict = 1 + 1 + 4
    assert st["launches"] == 20 + 2 * n * per_predict + 2 * 1 + 2 * 9 * n * (per_predict + 2)
    err = sm.ens_compare(a, b)
    assert err.shape == (n, 3) and np.all(np.isfinite(err)) and np.all(err > 0)


def test_hybrid_members_fall_back_on_their_own(env):
    """Per-member fallback: with a tolerance between two members' shadow
    errors, the failing member follows the FP64 solver bit for bit while the
    other advances by the surrogate; whole-ensemble fallback sends both back."""
    torch, nb, sm = env
    side, n = 128, 3
    s = sm.Surrogate(nblocks=1, batch=n, height=side, width=side, train=False, seed=4)
    # shadow errors of the first window, per member
    probe = small_ensemble(nb, 51, n, side)
    ref = small_ensemble(nb, 51, n, side)
    snap = torch.empty((n, side, side, 4), dtype=torch.float32, device="cuda")
    s.pack_ens(probe, snap.data_ptr())
    s.advance_ens(probe, 10)
    ref.step_n(1, 10)
    e0 = sm.ens_compare(probe, ref)[:, 0]
    order = np.argsort(e0)
    assert e0[order[0]] < e0[order[-1]]
    if e0[order[1]] - e0[order[0]] < 1e-3 * e0[order[1]]:
        pytest.skip("members' shadow errors too close to separate")
    tol = 0.5 * (e0[order[0]] + e0[order[1]])
    a = small_ensemble(nb, 51, n, side)
    b = small_ensemble(nb, 51, n, side)
    st = sm.hyb_run(s, a, 0, 100, tol=tol, quarantine=0.0)
    b.step_n(1, 100)
    assert st["windows"] == n and st["fallbacks"] == n - 1
    assert st["solver_steps"] == 10 * n + 90 * (n - 1) and st["sur_steps"] == 90
    err = sm.ens_compare(a, b)
    for m in range(n):
        if m == order[0]:
            assert err[m, 0] > 0  # advanced by the surrogate
        else:
            for f in (nb.SSHN, nb.UN, nb.VN):
                np.testing.assert_array_equal(a.field(m, f), b.field(m, f))
    c = small_ensemble(nb, 51, n, side)
    st = sm.hyb_run(s, c, 0, 100, tol=tol, per_member=False, quarantine=0.0)
    assert st["fallbacks"] == n and st["sur_steps"] == 0
    assert np.all(sm.ens_compare(c, b) == 0.0)


def test_quarantined_members_stay_on_the_solver(env):
    """A member whose shadow error passes the quarantine limit stays on the
    FP64 solver for the rest of the run, even where later errors would pass."""
    torch, nb, sm = env
    side, n = 128, 2
    a = small_ensemble(nb, 61, n, side)
    b = small_ensemble(nb, 61, n, side)
    s = sm.Surrogate(nblocks=1, batch=n, height=side, width=side, train=False, seed=4)
    st = sm.hyb_run(s, a, 0, 300, tol=1e300, quarantine=1e-300)
    b.step_n(1, 300)
    assert st["quarantined"] == n and st["fallbacks"] == 3 * n and st["sur_steps"] == 0
    for m in range(n):
        for f in (nb.SSHN, nb.UN, nb.VN):
            np.testing.assert_array_equal(a.field(m, f), b.field(m, f))
    c = small_ensemble(nb, 61, n, side)
    st = sm.hyb_run(s, c, 0, 100, tol=1e300, quarantine=0.0)  # never (one window: the
    assert st["quarantined"] == 0 and st["fallbacks"] == 0    # untrained network stays finite)


def test_rewound_member_follows_the_solver_exactly(env):
    """A member accepted in one window and quarantined in the next restarts
    from its FP64 state at the accepted window's start: the solver re-runs
    that window, so its trajectory is the plain solver's bit for bit.
    Without rewinding the surrogate's window stays in it.  The network adds
    1e30 to u and v at every call (a call adds its output divided by the
    output scale): the first shadow error is large but finite (accepted
    under a limit of 1e100); from the state nine calls leave, the solver's
    shadow steps overflow, so the second window's error is not finite and
    the member is quarantined."""
    torch, nb, sm = env
    side, n = 128, 1
    s = sm.Surrogate(nblocks=1, batch=n, height=side, width=side, train=False, seed=4)
    p = np.zeros_like(s.params())
    p[-64:] = 1.0  # the output layer's biases (the parameters end with the layers' biases)
    s.set_params(p)
    s.set_norm([1.0] * 4, [0.0] * 4, [1e38, 1e-30, 1e-30])

    def developed():  # 300 solver steps from rest
        e = small_ensemble(nb, 61, n, side)
        e.step_n(1, 300)
        return e

    r0 = sm.hyb_run(s, developed(), 300, 100, tol=1e300, quarantine=0.0)["last_shadow_err"]
    assert np.isfinite(r0) and r0 < 1e100, r0
    plain = developed()
    plain.step_n(301, 300)
    a = developed()
    st = sm.hyb_run(s, a, 300, 300, tol=1e300, quarantine=1e100)
    assert st["quarantined"] == 1 and st["rewound"] == 1 and st["fallbacks"] == 2
    # three shadow steps, the rewound window re-run with the next shadow step,
    # two fallen-back windows
    assert st["sur_steps"] == 90 and st["solver_steps"] == 3 * 10 + 110 + 2 * 90
    for f in (nb.SSHN, nb.UN, nb.VN):
        np.testing.assert_array_equal(a.field(0, f), plain.field(0, f))
    b = developed()
    st = sm.hyb_run(s, b, 300, 300, tol=1e300, quarantine=1e100, rewind=False)
    assert st["quarantined"] == 1 and st["rewound"] == 0
    assert not np.array_equal(b.field(0, nb.SSHN), plain.field(0, nb.SSHN))


def test_last_window_left_non_finite_is_rerun_by_the_solver(env):
    """The last window's surrogate calls meet no later shadow check: a member
    they leave non-finite goes back to that window's start and the solver
    runs the window.  The network (no residual blocks) maps the SSH's 3x3
    sums through a ReLU and a second 3x3 sum, and a call adds that over an
    output scale of 1e-30: from a normal state (|ssh| < 1) the addition is
    finite (an accepted, finite shadow prediction), from the state one call
    leaves the FP32 division overflows to inf."""
    torch, nb, sm = env
    side, n = 128, 1
    s = sm.Surrogate(nblocks=0, batch=n, height=side, width=side, train=False, seed=4)
    p = np.zeros_like(s.params())
    wl = 9 * 64 * 64  # weights per layer, [tap][out channel][in channel]
    for layer in (0, 1):
        for tap in range(9):
            p[layer * wl + tap * 64 * 64] = 1.0  # in channel 0 (ssh) -> out channel 0
    s.set_params(p)
    s.set_norm([1.0] * 4, [0.0] * 4, [1e-30, 1.0, 1.0])

    def developed():
        e = small_ensemble(nb, 61, n, side)
        e.step_n(1, 300)
        return e

    plain = developed()
    plain.step_n(301, 100)
    a = developed()
    st = sm.hyb_run(s, a, 300, 100, tol=1e300, quarantine=1e100)
    assert st["fallbacks"] == 0 and st["rewound"] == 1
    # work done: the discarded window's calls count, and so do its re-run steps
    assert st["sur_steps"] == 90 and st["solver_steps"] == 10 + 100
    for f in (nb.SSHN, nb.UN, nb.VN):
        np.testing.assert_array_equal(a.field(0, f), plain.field(0, f))
    b = developed()
    st = sm.hyb_run(s, b, 300, 100, tol=1e300, quarantine=1e100, rewind=False)
    assert st["rewound"] == 0 and not np.all(np.isfinite(b.field(0, nb.SSHN)))


def test_training_beats_persistence_on_held_out_runs(env):
    """The trained surrogate's one-call SSH error on unseen members is well
    below the error of the method without it (no change over 10 steps)."""
    torch, nb, sm = env
    from nemo_b200 import train as tr
    side = 128
    s = sm.Surrogate(nblocks=2, batch=16, height=side, width=side, seed=11)
    snaps, tides = tr.generate_runs(s, seed=100, nmem=16, side=side, steps=400)
    s.set_norm(*tr.compute_norm(snaps))
    before = tr.evaluate_one_call(s, seed=900, nmem=8, side=side, spin_up=250)
    losses = tr.train(s, tr.PairSampler(snaps, tides, seed=1), iters=400, batch=16, lr=2e-3)
    after = tr.evaluate_one_call(s, seed=900, nmem=8, side=side, spin_up=250)
    assert np.mean(losses[-20:]) < 0.2 * np.mean(losses[:5])
    pers = after["persistence"][:, 0].mean()
    trained = after["surrogate"][:, 0].mean()
    untrained = before["surrogate"][:, 0].mean()
    print("ssh rel err: persistence %.4f untrained %.4f trained %.4f" % (pers, untrained, trained))
    assert trained < 0.5 * pers
    assert trained < untrained


def test_chunked_data_set_holds_the_runs_of_one_ensemble(env):
    """generate_dataset (the 2048-run training set, generated a chunk of runs
    at a time) holds exactly the snapshots one ensemble of all the runs gives,
    and ChunkPairSampler draws (snapshot k, snapshot k+1) pairs of one run with
    the boundary SSH of the later one."""
    torch, nb, sm = env
    from nemo_b200 import train as tr
    side = 128
    s = sm.Surrogate(nblocks=1, batch=4, height=side, width=side, seed=2)
    chunks, dropped = tr.generate_dataset(s, seed=31, nruns=7, side=side, steps=60, chunk=3)
    whole, tides = tr.generate_runs(s, seed=31, nmem=7, side=side, steps=60)
    assert dropped == tr.generate_runs.dropped
    assert sum(c[0].shape[1] for c in chunks) == whole.shape[1] == 7 - dropped
    assert torch.equal(torch.cat([c[0] for c in chunks], 1), whole)
    assert torch.equal(torch.cat([c[1] for c in chunks], 1), tides)
    sampler = tr.ChunkPairSampler(chunks, seed=5)
    assert len(sampler) == (whole.shape[0] - 1) * whole.shape[1]
    s0, s1, t1 = sampler.batch(9)
    assert s0.shape == (9, side, side, 4) and s1.shape == s0.shape and t1.shape == (9,)
    S, M = whole.shape[0], whole.shape[1]
    for i in range(9):
        hits = [(k, m) for k in range(S - 1) for m in range(M)
                if torch.equal(whole[k, m], s0[i]) and torch.equal(whole[k + 1, m], s1[i])]
        assert hits, "sampled pair %d is not two consecutive snapshots of one run" % i
        assert any(float(tides[k + 1, m]) == float(t1[i]) for k, m in hits)


def test_rewind_from_the_fourth_window_restores_the_third_windows_start(env):
    """The window starts are kept in three slots (slot x mod 3 holds window
    x): a member accepted in window 2 and quarantined in window 3 restarts
    from window 2's start, so its run equals two hybrid windows followed by
    the plain solver, bit for bit.  The network (no residual blocks) passes
    only the boundary row's tide input, less a threshold set between the
    tides windows 2 and 3 predict (times the boundary flag), through a ReLU:
    windows 0-2 see a zero output (persistence, accepted), window 3's
    prediction adds inf to u (its FP32 quotient by an output scale of 1e-35
    overflows), so its shadow error is not finite.  The start step is the
    first at which the tide rises through the four windows."""
    torch, nb, sm = env
    from nemo_b200 import train as tr
    side, n = 128, 1
    member = tr.square_members(61, n, side, 0.2)[0]

    def tides(i0):
        return [tr.tide_of(member, i0 + 100 * w + 10) for w in range(4)]

    istp0 = next(i for i in range(0, 2300, 10)
                 if all(b - a > 0.05 * member.amp_tide for a, b in zip(tides(i), tides(i)[1:])))
    t = tides(istp0)
    theta = 0.5 * (t[2] + t[3])
    s = sm.Surrogate(nblocks=0, batch=n, height=side, width=side, train=False, seed=4)
    p = np.zeros_like(s.params())
    wl = 9 * 64 * 64
    big = 2.0 ** 33
    centre = 4 * 64 * 64                         # tap (0, 0), [out channel][in channel]
    p[0 * wl + centre + 0 * 64 + 5] = big        # tide input (channel 5) -> channel 0
    p[0 * wl + centre + 0 * 64 + 4] = -big * theta  # boundary flag (channel 4) -> channel 0
    p[1 * wl + centre + 1 * 64 + 0] = 1.0        # channel 0 -> u output
    s.set_params(p)
    s.set_norm([1.0] * 4, [0.0] * 4, [1.0, 1e-35, 1.0])

    def developed():
        e = small_ensemble(nb, 61, n, side)
        if istp0 > 0:
            e.step_n(1, istp0)
        return e

    ref = developed()
    st = sm.hyb_run(s, ref, istp0, 200, tol=1e300, quarantine=1e100)
    assert st["fallbacks"] == 0 and st["quarantined"] == 0 and st["sur_steps"] == 180, st
    ref.step_n(istp0 + 201, 200)
    a = developed()
    st = sm.hyb_run(s, a, istp0, 400, tol=1e300, quarantine=1e100)
    assert st["quarantined"] == 1 and st["rewound"] == 1 and st["fallbacks"] == 1, st
    assert st["sur_steps"] == 270 and st["solver_steps"] == 4 * 10 + 110 + 90, st
    for f in (nb.SSHN, nb.UN, nb.VN):
        np.testing.assert_array_equal(a.field(0, f), ref.field(0, f))


def test_shadow_correction_is_added_by_every_accepted_call(env):
    """With correct=True every surrogate call of an accepted window adds,
    per cell, the FP32 difference between the shadow state and the window's
    first prediction.  A network with a zero output predicts no change, so
    after the window each interior value is the shadow state plus nine times
    (shadow - window start), the boundary row holds the tide and the open
    boundary's v is the Flather value."""
    torch, nb, sm = env
    side, n = 128, 1
    s = sm.Surrogate(nblocks=0, batch=n, height=side, width=side, train=False, seed=4)
    s.set_params(np.zeros_like(s.params()))
    s.set_norm([1.0] * 4, [0.0] * 4, [1.0, 1.0, 1.0])

    def developed():
        e = small_ensemble(nb, 61, n, side)
        e.step_n(1, 300)
        return e

    ref = developed()
    start = [ref.field(0, f).copy() for f in (nb.SSHN, nb.UN, nb.VN)]
    ref.step_n(301, 10)  # the shadow step
    shadow = [ref.field(0, f).copy() for f in (nb.SSHN, nb.UN, nb.VN)]
    a = developed()
    st = sm.hyb_run(s, a, 300, 100, tol=1e300, quarantine=1e100, correct=True)
    assert st["fallbacks"] == 0 and st["sur_steps"] == 90, st
    got = [a.field(0, f) for f in (nb.SSHN, nb.UN, nb.VN)]
    want = []
    for x0, xf in zip(start, shadow):
        d = (xf - x0.astype(np.float32).astype(np.float64)).astype(np.float32).astype(np.float64)
        x = xf.copy()
        for _ in range(9):
            x = (x + 0.0) + d
        want.append(x)
    np.testing.assert_array_equal(got[0][1:], want[0][1:])          # ssh below the tide row
    np.testing.assert_array_equal(got[1][:, 1:-1], want[1][:, 1:-1])  # u between the walls
    np.testing.assert_array_equal(got[2][1:-1], want[2][1:-1])      # v between boundary and wall
    b = developed()
    sm.hyb_run(s, b, 300, 100, tol=1e300, quarantine=1e100)  # without: persistence from the shadow
    np.testing.assert_array_equal(b.field(0, nb.UN)[:, 1:-1], shadow[1][:, 1:-1])
