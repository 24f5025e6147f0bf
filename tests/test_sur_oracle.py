"""The surrogate's CPU FP64 oracle, pinned against finite differences (CPU only)."""
import numpy as np
import pytest

from oracle import sur_oracle as so


def test_bf16_rounding_ties_to_even():
    one = 1.0
    ulp = 2.0 ** -7
    vals = np.array([one, one + ulp / 2, one + 1.5 * ulp, one + ulp / 4, -3.0, 0.0])
    r = so.bf16(vals)
    assert list(r) == [1.0, 1.0, one + 2 * ulp, 1.0, -3.0, 0.0]
    assert so.from_bf16_bits(so.bf16_bits(vals)).tolist() == r.tolist()


def test_conv_matches_direct_sum_and_shift_taps():
    rng = np.random.default_rng(1)
    x = rng.normal(size=(2, 5, 7, 64))
    w = rng.normal(size=(9, 64, 64))
    acc = so.conv3x3(x, w)
    n, y, xx = 1, 0, 6  # a corner: taps reaching outside read zero
    ref = np.zeros(64)
    for tap in range(9):
        dy, dx = tap // 3 - 1, tap % 3 - 1
        if 0 <= y + dy < 5 and 0 <= xx + dx < 7:
            ref += w[tap] @ x[n, y + dy, xx + dx]
    np.testing.assert_allclose(acc[n, y, xx], ref, rtol=1e-12)
    # a one-hot tap shifts the image
    e = np.zeros((9, 64, 64))
    e[5] = np.eye(64)  # dy = 0, dx = +1
    np.testing.assert_array_equal(so.conv3x3(x, e)[:, :, :-1], x[:, :, 1:])
    assert not so.conv3x3(x, e)[:, :, -1].any()


def test_dgrad_and_wgrad_are_adjoints_of_conv():
    rng = np.random.default_rng(2)
    x = rng.normal(size=(2, 4, 6, 64))
    w = rng.normal(size=(9, 64, 64))
    dz = rng.normal(size=(2, 4, 6, 64))
    lhs = (so.conv3x3(x, w) * dz).sum()
    assert np.isclose(lhs, (x * so.conv3x3(dz, so.flip_transpose(w))).sum(), rtol=1e-11)
    dw, db = so.wgrad(x, dz)
    assert np.isclose(lhs, (dw * w).sum(), rtol=1e-11)
    np.testing.assert_allclose(db, dz.reshape(-1, 64).sum(0), rtol=1e-12)


@pytest.mark.parametrize("nblocks", [0, 1])
def test_network_gradient_matches_finite_differences(nblocks):
    rng = np.random.default_rng(3 + nblocks)
    N, H, W = 1, 4, 5
    L = 2 * nblocks + 2
    Wt = rng.normal(0, 0.15, size=(L, 9, 64, 64))
    Wt[0, :, :, 6:] = 0.0
    Bs = rng.normal(0, 0.1, size=(L, 64))
    flat = np.concatenate([Wt.ravel(), Bs.ravel()])
    snap0 = rng.normal(size=(N, H, W, 4))
    snap1 = snap0 + rng.normal(0, 0.3, size=(N, H, W, 4))
    tide = rng.normal(size=N)
    norm = (np.ones(4), np.zeros(4), np.ones(3))
    loss, g = so.loss_grad(flat, nblocks, snap0, snap1, tide, norm, bf16_acts=False)
    # central differences on a sample of coordinates in every layer and the biases
    nw = L * 9 * 64 * 64
    idx = []
    for l in range(L):
        base = l * 9 * 64 * 64
        idx += list(base + rng.choice(9 * 64 * (6 if l == 0 else 64), 4, replace=False) % (9 * 64 * 64))
        idx.append(nw + l * 64 + int(rng.integers(0, 3 if l == L - 1 else 64)))
    h = 1e-6
    for i in idx:
        fp, fm = flat.copy(), flat.copy()
        fp[i] += h
        fm[i] -= h
        lp, _ = so.loss_grad(fp, nblocks, snap0, snap1, tide, norm, bf16_acts=False)
        lm, _ = so.loss_grad(fm, nblocks, snap0, snap1, tide, norm, bf16_acts=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_adamw_restatement_single_step():
    p = np.array([1.0, -2.0, 0.5], dtype=np.float32)
    g = np.array([0.1, -0.2, 0.0], dtype=np.float32)
    z = np.zeros(3, dtype=np.float32)
    p1, m1, v1 = so.adamw(p, g, z, z, 1, lr=0.01, b1=0.9, b2=0.999, eps=1e-8, wd=0.1, nw=2)
    # first step: m_hat = g, v_hat = g^2 -> update = sign(g) (+ decay on weights)
    np.testing.assert_allclose(p1[:2], p[:2] - 0.01 * (np.sign(g[:2]) + 0.1 * p[:2]), rtol=1e-5)
    assert p1[2] == p[2]


@pytest.mark.parametrize("patch", [2, 4])
def test_patch_layout_round_trips_and_places_each_cell(patch):
    rng = np.random.default_rng(7)
    P = patch
    f = rng.normal(size=(2, 3 * P, 2 * P, 3))
    g = so.to_patches(f, P)
    assert g.shape == (2, 3, 2, 3 * P * P)
    np.testing.assert_array_equal(so.from_patches(g, P, 3), f)
    # network pixel (X, Y) = (1, 2), field 2, sub-cell (sx, sy) = (P-1, 1)
    assert g[1, 2, 1, 2 * P * P + P * 1 + (P - 1)] == f[1, 2 * P + 1, P + P - 1, 2]


@pytest.mark.parametrize("patch", [2, 4])
def test_patch_input_channels(patch):
    rng = np.random.default_rng(8)
    P = patch
    N, H, W = 2, 2 * P, 3 * P
    snap = rng.normal(size=(N, H, W, 4)).astype(np.float32)
    tide = np.array([0.3, -0.7], np.float32)
    sc, sh = [2.0, 1.0, 0.5, 0.25], [0.0, 0.0, 0.0, 1.0]
    x = so.make_input(snap, tide, sc, sh, patch=P)
    assert x.shape == (N, 2, 3, 64)
    # ssh of T-cell (x, y) = (P + 1, P) sits in network pixel (1, 1), sub-cell (1, 0)
    assert x[0, 1, 1, 1] == np.float32(snap[0, P, P + 1, 0] * 2.0)
    # depth quadrant means: quadrant (qy, qx) = (1, 0) of network pixel (0, 0)
    q = (snap[1, P // 2:P, 0:P // 2, 3] - 1.0) * 0.25
    assert np.isclose(x[1, 0, 0, 3 * P * P + 2], q.mean(), rtol=1e-6)
    fc = 3 * P * P + 4
    assert (x[:, 0, :, fc] == 1).all() and not x[:, 1:, :, fc].any()
    np.testing.assert_array_equal(x[:, 0, 0, fc + 1], tide * 2.0)
    assert not x[..., fc + 2:].any()


def test_patch_network_gradient_matches_finite_differences():
    rng = np.random.default_rng(11)
    P, N, H, W, nblocks = 2, 1, 4, 6, 1
    L = 2 * nblocks + 2
    Wt = rng.normal(0, 0.15, size=(L, 9, 64, 64))
    Bs = rng.normal(0, 0.1, size=(L, 64))
    flat = np.concatenate([Wt.ravel(), Bs.ravel()])
    snap0 = rng.normal(size=(N, H, W, 4))
    snap1 = snap0 + rng.normal(0, 0.3, size=(N, H, W, 4))
    tide = rng.normal(size=N)
    norm = (np.ones(4), np.zeros(4), np.ones(3))
    loss, g = so.loss_grad(flat, nblocks, snap0, snap1, tide, norm, bf16_acts=False, patch=P)
    nw = L * 9 * 64 * 64
    idx = list(rng.choice(nw, 12, replace=False)) + [nw + (L - 1) * 64 + 5, nw + 3]
    h = 1e-6
    for i in idx:
        fp, fm = flat.copy(), flat.copy()
        fp[i] += h
        fm[i] -= h
        lp, _ = so.loss_grad(fp, nblocks, snap0, snap1, tide, norm, bf16_acts=False, patch=P)
        lm, _ = so.loss_grad(fm, nblocks, snap0, snap1, tide, norm, bf16_acts=False, patch=P)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])
