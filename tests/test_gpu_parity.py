"""Parity of the CUDA stepper with the oracle and the reference's golden vectors.

Two builds of the same sources are checked:
  * lib/libnemo_b200_strict.so (-fmad=false): bit-for-bit equal (sign of zero
    included) to the oracle and to the golden vectors executed from
    original/nemolite2d.f90, through both the per-routine path and the fused
    path;
  * lib/libnemo_b200.so (default, FMA contraction on): relative max-norm
    error max|gpu - ref| / max|ref| <= 1e-12 per field after every record.
"""
import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES

pytestmark = pytest.mark.gpu

TOL = 1e-12
STATE = [("sshn", 0), ("un", 1), ("vn", 2)]
ALL = STATE + [("ssha", 3), ("ua", 4), ("va", 5), ("sshn_u", 6), ("sshn_v", 7)]


@pytest.fixture(scope="module")
def nb():
    import nemo_b200
    nemo_b200.load(False)
    nemo_b200.load(True)
    return nemo_b200


def bits(a):
    return np.ascontiguousarray(a).view(np.int64)


def relerr(a, b):
    d = np.max(np.abs(a - b)) if a.size else 0.0
    s = np.max(np.abs(b)) if b.size else 0.0
    return d / s if s > 0 else d


def golden_params(z):
    return dict(jpi=int(z["jpi"]), jpj=int(z["jpj"]), dx=float(z["nml_dx"]), dy=float(z["nml_dy"]),
                dep_const=float(z["nml_dep_const"]), rdt=float(z["nml_rdt"]),
                cbfr=float(z["nml_cbfr"]), visc=float(z["nml_visc"]))


@pytest.mark.parametrize("case", GOLDEN_CASES)
@pytest.mark.parametrize("path", ["routine", "fused"])
def test_strict_build_matches_golden_bitwise(nb, case, path):
    z = np.load("%s/%s.npz" % (GOLDEN, case))
    m = nb.Model(strict=True, **golden_params(z))
    fields = ALL if path == "routine" else ALL
    last = 0
    for r in z["records"]:
        r = int(r)
        if r > 0:
            if path == "routine":
                for istp in range(last + 1, r + 1):
                    m.step(istp)
            else:
                m.step_n(last + 1, r - last)
            last = r
        for name, fid in fields:
            np.testing.assert_array_equal(bits(m.field(fid)), bits(z["s%05d_%s" % (r, name)]),
                                          err_msg="%s %s step %d %s" % (case, path, r, name))


@pytest.mark.parametrize("jpi,jpj,tile", [(257, 131, (4, 0, 64)), (130, 300, (2, 20, 7)),
                                          (257, 131, (2, 116, 16)), (130, 300, (4, 116, 7)),
                                          (61, 29, (2, 120, 3)), (3, 5, (2, 116, 1)),
                                          (257, 131, (2, 216, 32)), (130, 300, (4, 220, 9)),
                                          (3, 5, (2, 216, 1)), (96, 33, (4, 216, 0)),
                                          (2, 2, (2, 0, 1)), (3, 5, (4, 16, 2)), (96, 33, (8, 16, 16)),
                                          (61, 29, (4, 24, 3)), (125, 40, (2, -16, 0)),
                                          (62, 9, (2, 0, 0)), (63, 12, (8, 24, 5)),
                                          (70, 21, (4, -20, 4))])
def test_strict_fused_matches_oracle_ragged_bathymetry(nb, oracle_mod, jpi, jpj, tile):
    kw = dict(jpi=jpi, jpj=jpj, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.5,
              tide_phase=0.3, nbump=12, seed=77, bump_amp=30.0, bump_wmin=3e3, bump_wmax=40e3,
              hmin=20.0)
    m = nb.Model(strict=True, **kw)
    m.set_schedule(*tile)
    o = oracle_mod.Model(**kw)
    for name, fid in [("ht", nb.HT), ("hu", nb.HU), ("hv", nb.HV)]:
        np.testing.assert_array_equal(bits(m.field(fid)), bits(o.field(fid)), err_msg=name)
    istp = 1
    for nsteps in (1, 7, 25):
        m.step_n(istp, nsteps)
        o.run(istp, nsteps)
        istp += nsteps
        for name, fid in STATE:
            np.testing.assert_array_equal(bits(m.field(fid)), bits(o.field(fid)),
                                          err_msg="%dx%d step %d %s" % (jpi, jpj, istp - 1, name))


def test_strict_routines_one_by_one_from_random_state(nb, oracle_mod):
    """Each routine of the per-routine boundary against the oracle's routine."""
    jpi, jpj = 70, 45
    kw = dict(jpi=jpi, jpj=jpj, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=1.0, nbump=5,
              seed=3, bump_amp=20.0, bump_wmin=5e3, bump_wmax=20e3)
    rng = np.random.default_rng(11)
    sshn = rng.normal(0, 0.1, (jpj, jpi))
    un = rng.normal(0, 0.2, (jpj, jpi + 1))
    vn = rng.normal(0, 0.2, (jpj + 1, jpi))
    m = nb.Model(strict=True, **kw)
    o = oracle_mod.Model(**kw)
    m.set_state(sshn, un, vn)
    o.set_state(sshn, un, vn)
    rtime = 37 * 20.0
    steps = [("continuity", lambda: (m.continuity(), o.continuity())),
             ("momentum_u", lambda: (m.momentum_u(), o.momentum_u())),
             ("momentum_v", lambda: (m.momentum_v(), o.momentum_v())),
             ("bc_ssh", lambda: (m.bc_ssh(rtime), o.bc_ssh(rtime))),
             ("bc_solid_u", lambda: (m.bc_solid_u(), o.bc_solid_u())),
             ("bc_solid_v", lambda: (m.bc_solid_v(), o.bc_solid_v())),
             ("bc_flather_u", lambda: (m.bc_flather_u(), o.bc_flather_u())),
             ("bc_flather_v", lambda: (m.bc_flather_v(), o.bc_flather_v())),
             ("next", lambda: (m.next(), o.next()))]
    for label, fn in steps:
        fn()
        for name, fid in ALL:
            np.testing.assert_array_equal(bits(m.field(fid)), bits(o.field(fid)),
                                          err_msg="after %s: %s" % (label, name))


@pytest.mark.parametrize("strict", [True, False])
@pytest.mark.parametrize("mags", [(-322, -280), (-322, 0), (-310, -290)])
@pytest.mark.parametrize("sched", [(2, 216, 32), (2, 116, 16), (2, -20, 16), (2, 20, 7)])
def test_tiny_values_take_the_exact_division_path(nb, oracle_mod, strict, mags, sched):
    """States whose values reach the subnormal range, alone or mixed with
    ordinary values and whole rows of zeros: rows holding nonzero values
    below 2^-300 (and their neighbours) are computed with IEEE division, so
    the strict build stays bit-identical to the oracle there too, for every
    way of staging rows."""
    jpi, jpj = 150, 90
    kw = dict(jpi=jpi, jpj=jpj, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.2)
    rng = np.random.default_rng(5)
    def tiny(shape):
        mag = 10.0 ** rng.uniform(mags[0], mags[1], shape)
        x = mag * rng.choice([-1.0, 1.0], shape)
        x[rng.random(shape) < 0.3] = 0.0
        x[rng.random(shape[0]) < 0.3] = 0.0
        return x
    st = (tiny((jpj, jpi)), tiny((jpj, jpi + 1)), tiny((jpj + 1, jpi)))
    m = nb.Model(strict=strict, **kw)
    m.set_schedule(*sched)
    o = oracle_mod.Model(**kw)
    m.set_state(*st)
    o.set_state(*st)
    m.step_n(1, 6)
    o.run(1, 6)
    for name, fid in STATE:
        a, b = m.field(fid), o.field(fid)
        if strict:
            np.testing.assert_array_equal(bits(a), bits(b), err_msg=name)
        else:
            assert relerr(a, b) <= TOL, name


def test_in_kernel_reciprocals_are_checked_and_default(nb):
    """The depths of a seeded grid pass the setup check of the in-kernel
    reciprocal depths (Newton steps from a single-precision seed, compared
    with RN(1/h) cell by cell), so the default schedule forms them in the
    kernel; with the stored reciprocals the strict results are identical."""
    kw = dict(jpi=300, jpj=200, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.4, nbump=16,
              seed=21, bump_amp=35.0, bump_wmin=4e3, bump_wmax=80e3, hmin=12.0)
    a = nb.Model(strict=True, **kw)
    b = nb.Model(strict=True, **kw)
    assert a.recip_in_kernel() and a.get_schedule() == (2, 216, 32)
    b.set_schedule(2, 116, 32)
    a.step_n(1, 60)
    b.step_n(1, 60)
    for name, fid in STATE:
        np.testing.assert_array_equal(bits(a.field(fid)), bits(b.field(fid)), err_msg=name)


def test_record_stages_the_output_fields_without_disturbing_the_run(nb):
    """nemo_record: sshn and the cell-centred u, v of the current state reach
    host memory (the go2d columns 4-6), and the steps launched while the
    record travels give the same state as a run that never recorded."""
    import torch
    kw = dict(jpi=150, jpj=97, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.3, nbump=6,
              seed=8, bump_amp=20.0, bump_wmin=5e3, bump_wmax=40e3)
    a = nb.Model(strict=True, **kw)
    b = nb.Model(strict=True, **kw)
    a.step_n(1, 40)
    b.step_n(1, 40)
    rec = [torch.zeros(3 * 97 * 150, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
    ssh, u, v = a.field(nb.SSHN), a.field(nb.UN), a.field(nb.VN)
    a.record(rec[0])
    a.step_n(41, 30)  # overlaps the copy
    a.record(rec[1])
    a.record_wait()
    b.step_n(41, 30)
    r0 = rec[0].reshape(3, 97, 150)
    np.testing.assert_array_equal(r0[0], ssh)
    np.testing.assert_array_equal(r0[1], 0.5 * (u[:, :-1] + u[:, 1:]))
    np.testing.assert_array_equal(r0[2], 0.5 * (v[:-1, :] + v[1:, :]))
    for name, fid in STATE:
        np.testing.assert_array_equal(bits(a.field(fid)), bits(b.field(fid)), err_msg=name)
    np.testing.assert_array_equal(rec[1].reshape(3, 97, 150)[0], b.field(nb.SSHN))


def test_strict_fused_equals_routine_path_from_random_state(nb):
    jpi, jpj = 200, 150
    kw = dict(jpi=jpi, jpj=jpj, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=1.0, nbump=8,
              seed=5, bump_amp=30.0, bump_wmin=5e3, bump_wmax=50e3)
    rng = np.random.default_rng(2)
    st = (rng.normal(0, 0.1, (jpj, jpi)), rng.normal(0, 0.3, (jpj, jpi + 1)),
          rng.normal(0, 0.3, (jpj + 1, jpi)))
    a = nb.Model(strict=True, **kw)
    b = nb.Model(strict=True, **kw)
    a.set_state(*st)
    b.set_state(*st)
    a.step_n(10, 15)
    for istp in range(10, 25):
        b.step(istp)
    for name, fid in ALL:
        np.testing.assert_array_equal(bits(a.field(fid)), bits(b.field(fid)), err_msg=name)


def test_default_build_config0_within_tolerance_every_record(nb, oracle_mod):
    """128^2, rdt 20, cbfr 1.5e-4, visc 0.1, 2000 steps, records every 100."""
    kw = dict(jpi=128, jpj=128, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.2)
    m = nb.Model(strict=False, **kw)
    o = oracle_mod.Model(**kw)
    for rec in range(20):
        m.step_n(1 + 100 * rec, 100)
        o.run(1 + 100 * rec, 100)
        for name, fid in STATE:
            e = relerr(m.field(fid), o.field(fid))
            assert e <= TOL, "step %d %s rel err %.3e" % (100 * (rec + 1), name, e)
        ck = m.checksums()
        ref = [o.checksum(f, "seq") for f in (oracle_mod.SSHN, oracle_mod.UA, oracle_mod.VA)]
        np.testing.assert_allclose(ck, ref, rtol=1e-11)


def test_strict_checksums_bitwise_tree_order(nb, oracle_mod):
    kw = dict(jpi=300, jpj=77, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.2)
    m = nb.Model(strict=True, **kw)
    o = oracle_mod.Model(**kw)
    m.step_n(1, 60)
    o.run(1, 60)
    ck = m.checksums()
    for k, f in enumerate((oracle_mod.SSHN, oracle_mod.UN, oracle_mod.VN)):
        assert ck[k] == o.checksum(f, "tree")
        assert abs(ck[k] - o.checksum(f, "seq")) <= 1e-13 * abs(ck[k])
    assert m.checksum(nb.UA) == ck[1] and m.checksum(nb.VA) == ck[2]


@pytest.mark.parametrize("sched", [(2, 0, 1), (2, 16, 16), (4, 0, 64), (4, 20, 5), (8, 16, 256),
                                   (8, 0, 33), (2, 24, 0), (2, -24, 16), (2, 116, 16), (2, 120, 1),
                                   (4, 116, 0), (4, 120, 9), (2, 216, 32), (2, 220, 5), (4, 216, 0),
                                   (4, 220, 11)])
def test_schedule_does_not_change_results(nb, sched):
    """Strict build: bit-identical for every schedule.  Default build: each
    register-budget variant is compiled separately and may contract multiply-
    adds differently, so schedules agree to the stated tolerance."""
    kw = dict(jpi=333, jpj=210, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.6, nbump=6,
              seed=9, bump_amp=25.0, bump_wmin=5e3, bump_wmax=60e3)
    for strict in (True, False):
        ref = nb.Model(strict=strict, **kw)
        ref.set_schedule(4, 0, 64)
        m = nb.Model(strict=strict, **kw)
        m.set_schedule(*sched)
        ref.step_n(1, 40)
        m.step_n(1, 40)
        for name, fid in STATE:
            a, b = m.field(fid), ref.field(fid)
            if strict:
                np.testing.assert_array_equal(bits(a), bits(b), err_msg=name)
            else:
                assert relerr(a, b) <= TOL, name


CONFIG1 = dict(jpi=4096, jpj=4096, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.2, nbump=32,
               seed=1234, bump_amp=40.0, bump_wmin=20e3, bump_wmax=200e3, hmin=10.0)


def test_config1_full_run_every_record_against_openmp_oracle(nb, oracle_mod):
    """The benchmarked configuration end to end: 4096^2, 32 seeded bumps
    (seed 1234), 1000 steps from rest, a record every 100 steps
    (original/nemolite2d.f90:74-85, :384).  At every record the full sshn,
    un and vn fields of the strict build equal the oracle's bit for bit and
    its checksums equal the oracle's tree-order sums; the default build, on
    the schedule the bench runs, stays within 1e-12 relative max-norm and its
    checksums within 1e-11 of the oracle's sequential sums."""
    import os
    oracle_mod.set_threads(max(1, len(os.sched_getaffinity(0))))
    o = oracle_mod.Model(**CONFIG1)
    s = nb.Model(strict=True, **CONFIG1)
    d = nb.Model(strict=False, **CONFIG1)
    worst = {}
    try:
        for rec in range(10):
            istp0 = 1 + 100 * rec
            s.step_n(istp0, 100)
            d.step_n(istp0, 100)
            o.run(istp0, 100)
            step = istp0 + 99
            for name, fid in STATE:
                ref = o.field(fid)
                np.testing.assert_array_equal(bits(s.field(fid)), bits(ref),
                                              err_msg="step %d %s" % (step, name))
                e = relerr(d.field(fid), ref)
                worst[name] = max(worst.get(name, 0.0), e)
                assert e <= TOL, "default build step %d %s rel err %.3e" % (step, name, e)
            cs, cd = s.checksums(), d.checksums()
            tree = [o.checksum(f, "tree") for f in (oracle_mod.SSHN, oracle_mod.UN, oracle_mod.VN)]
            seq = [o.checksum(f, "seq") for f in (oracle_mod.SSHN, oracle_mod.UN, oracle_mod.VN)]
            assert list(cs) == tree, "step %d strict checksums" % step
            np.testing.assert_allclose(cd, seq, rtol=1e-11, err_msg="step %d" % step)
            assert np.all(np.isfinite(cs)) and np.all(cs > 0)
    finally:
        oracle_mod.set_threads(1)
    print("config 1, 1000 steps: worst default-build relative max-norm error per field "
          + ", ".join("%s %.3e" % kv for kv in worst.items()))


def test_long_run_properties_at_4096(nb):
    """1000 fused steps at 4096^2: finite, walls exactly zero, clamped row exact."""
    m = nb.Model(strict=False, **CONFIG1)
    m.step_n(1, 1000)
    ck = m.checksums()
    assert np.all(np.isfinite(ck)) and np.all(ck > 0)
    u = m.field(nb.UN)
    v = m.field(nb.VN)
    s = m.field(nb.SSHN)
    assert not np.any(u[:, 0]) and not np.any(u[:, -1]) and not np.any(v[-1, :])
    om = 2.0 * 3.14159 / (12.42 * 3600.0)
    assert np.all(s[0] == 0.2 * np.sin(om * (1000 * 20.0)))


def test_compat_symbols_drive_the_reference_sequence(nb, oracle_mod):
    """cuda_setup_model_params_ / cuda_initialise_grid_ / per-step calls /
    cuda_retrieve_results_ as cuda/nemolite2d.f90 drives them."""
    import ctypes
    L = nb.load(True)
    jpi, jpj, rdt = 40, 30, 20.0
    L.cuda_setup_model_params_(jpi, jpj, 1000.0, 1000.0, 100.0, 1, 20, 5, rdt, 0.00015, 0.1)
    L.cuda_initialise_grid_()
    assert L.nemo_compat_last_status() == 0
    o = oracle_mod.Model(jpi=jpi, jpj=jpj, rdt=rdt, cbfr=0.00015, visc=0.1)
    P = ctypes.POINTER(ctypes.c_double)
    for istp in range(1, 21):
        rtime = istp * rdt
        L.cuda_continuity_()
        L.cuda_momentum_()
        L.cuda_boundary_conditions_(rtime)
        L.cuda_next_()
        o.step(istp)
    out = {k: np.empty(s) for k, s in [("sshn", (jpj, jpi)), ("un", (jpj, jpi + 1)),
                                       ("vn", (jpj + 1, jpi)), ("ua", (jpj, jpi + 1)),
                                       ("va", (jpj + 1, jpi))]}
    L.cuda_retrieve_results_(*[out[k].ctypes.data_as(P) for k in ("sshn", "un", "vn", "ua", "va")],
                             jpi, jpj)
    xt, yt, ht = (np.empty((jpj, jpi)) for _ in range(3))
    L.cuda_retrieve_grid_constants_(xt.ctypes.data_as(P), yt.ctypes.data_as(P),
                                    ht.ctypes.data_as(P), jpi, jpj)
    assert L.nemo_compat_last_status() == 0
    for k, fid in [("sshn", 0), ("un", 1), ("vn", 2), ("ua", 4), ("va", 5)]:
        np.testing.assert_array_equal(bits(out[k]), bits(o.field(fid)), err_msg=k)
    np.testing.assert_array_equal(xt, o.field(oracle_mod.XT))
    np.testing.assert_array_equal(yt, o.field(oracle_mod.YT))
    np.testing.assert_array_equal(ht, o.field(oracle_mod.HT))
    L.cuda_finalise_()
    assert not L.nemo_compat_context()


def test_invalid_arguments_fail_loudly(nb):
    with pytest.raises(nb.NemoError):
        nb.Model(jpi=1, jpj=10)
    with pytest.raises(nb.NemoError):
        nb.Model(jpi=10, jpj=0)
    m = nb.Model(jpi=10, jpj=10)
    with pytest.raises(nb.NemoError):
        m.set_schedule(3, 0, 4)
    with pytest.raises(nb.NemoError):
        m.set_schedule(8, 20, 4)
    with pytest.raises(nb.NemoError):
        m.step_n(1, -1)
    with pytest.raises(nb.NemoError):
        m.checksum(nb.XT)


def _general_models(nb, oracle_mod, strict, seed=3, jpi=150, jpj=97):
    from gridcases import NAMES, random_grid
    kw = dict(jpi=jpi, jpj=jpj, rdt=10.0, cbfr=0.00015, visc=0.1, amp_tide=0.3)
    pt, g = random_grid(seed, jpi, jpj)
    m = nb.Model(strict=strict, **kw)
    o = oracle_mod.Model(**kw)
    m.set_grid(pt, *[g[n] for n in NAMES])
    o.set_grid(pt, *[g[n] for n in NAMES])
    return m, o


def test_strict_general_grid_matches_oracle_routine_by_routine(nb, oracle_mod):
    """A general grid (open water on all four borders, islands, per-point
    scale factors, latitudes and depths): every routine of the strict build
    equals the oracle bit for bit, including the Flather condition on u."""
    m, o = _general_models(nb, oracle_mod, True)
    for name, fid in ALL:
        np.testing.assert_array_equal(bits(m.field(fid)), bits(o.field(fid)), err_msg="set_grid: " + name)
    for istp in range(1, 4):
        rtime = istp * 10.0
        for label, fn in [("continuity", lambda: (m.continuity(), o.continuity())),
                          ("momentum_u", lambda: (m.momentum_u(), o.momentum_u())),
                          ("momentum_v", lambda: (m.momentum_v(), o.momentum_v())),
                          ("bc_ssh", lambda: (m.bc_ssh(rtime), o.bc_ssh(rtime))),
                          ("bc_solid_u", lambda: (m.bc_solid_u(), o.bc_solid_u())),
                          ("bc_solid_v", lambda: (m.bc_solid_v(), o.bc_solid_v())),
                          ("bc_flather_u", lambda: (m.bc_flather_u(), o.bc_flather_u())),
                          ("bc_flather_v", lambda: (m.bc_flather_v(), o.bc_flather_v())),
                          ("next", lambda: (m.next(), o.next()))]:
            fn()
            for name, fid in ALL:
                np.testing.assert_array_equal(bits(m.field(fid)), bits(o.field(fid)),
                                              err_msg="step %d after %s: %s" % (istp, label, name))


def test_strict_general_grid_step_n_matches_oracle(nb, oracle_mod):
    """nemo_step_n on a general grid runs the routine sequence: bitwise with
    the oracle after 150 steps; the fused schedules' autotuner is refused."""
    m, o = _general_models(nb, oracle_mod, True, seed=11, jpi=131, jpj=140)
    m.step_n(1, 150)
    o.run(1, 150)
    for name, fid in ALL:
        np.testing.assert_array_equal(bits(m.field(fid)), bits(o.field(fid)), err_msg=name)
    ck = m.checksums()
    assert ck[1] == o.checksum(oracle_mod.UN, "tree")
    with pytest.raises(nb.NemoError):
        m.autotune(2)


def _channel_grid(seed, jpi, jpj):
    """random_grid plus open cells inside the domain that form one-cell water
    channels between two open cells along x and along y (the only places where
    the reference's in-place Flather sweeps chain two updates), and an open
    cell next to an island."""
    from gridcases import random_grid
    pt, g = random_grid(seed, jpi, jpj)
    for jj in (20, 21, 40):
        pt[jj, 30] = -1
        pt[jj, 31] = 1
        pt[jj, 32] = -1
    for ji in (60, 61):
        pt[50, ji] = -1
        pt[51, ji] = 1
        pt[52, ji] = -1
    pt[70, 90] = -1
    pt[70, 91] = 0
    return pt, g


@pytest.mark.parametrize("strict", [True, False])
@pytest.mark.parametrize("gsched", [None, (2, 0, 32), (2, 4, 7), (2, 3, 1), (2, 3, 200)])
def test_general_fused_step_equals_routines_with_flather_chains(nb, oracle_mod, strict, gsched):
    """The general grid's fused step (one kernel plus the Flather chains)
    against the per-routine kernels and the oracle, from a random state, on a
    mask with interior open cells and one-cell channels in both directions:
    bitwise in the strict build, within 1e-12 in the default build.  Every
    schedule of the general kernel (rows loaded where used, or staged through
    a ring of 3 or 4 slots; 1 row to the whole grid per CTA) gives these."""
    from gridcases import NAMES
    jpi, jpj = 150, 97
    kw = dict(jpi=jpi, jpj=jpj, rdt=10.0, cbfr=0.00015, visc=0.1, amp_tide=0.3)
    pt, g = _channel_grid(8, jpi, jpj)
    rng = np.random.default_rng(3)
    st = (rng.normal(0, 0.05, (jpj, jpi)), rng.normal(0, 0.1, (jpj, jpi + 1)),
          rng.normal(0, 0.1, (jpj + 1, jpi)))
    fused = nb.Model(strict=strict, **kw)
    routine = nb.Model(strict=strict, **kw)
    o = oracle_mod.Model(**kw)
    for m in (fused, routine, o):
        m.set_grid(pt, *[g[n] for n in NAMES])
        m.set_state(*st)
    if gsched is not None:
        fused.set_schedule(*gsched)
        assert fused.get_schedule() == gsched
    else:
        assert fused.get_schedule() == (2, 3, 32)
        for bad in ((2, 216, 32), (4, 3, 32), (2, 5, 32), (2, 3, 0)):
            with pytest.raises(nb.NemoError):
                fused.set_schedule(*bad)
    fused.step_n(1, 6)
    for istp in range(1, 7):
        routine.step(istp)
        o.step(istp)
    for name, fid in STATE:
        a, b, r = fused.field(fid), routine.field(fid), o.field(fid)
        if strict:
            np.testing.assert_array_equal(bits(a), bits(r), err_msg="fused " + name)
            np.testing.assert_array_equal(bits(b), bits(r), err_msg="routines " + name)
        else:
            assert relerr(a, r) <= TOL and relerr(b, r) <= TOL, name


def test_default_grid_through_set_grid_is_the_built_in_grid(nb):
    """The reference's grid passed as arrays gives, in the strict build, the
    same bits as the built-in grid (routine path and fused path)."""
    from gridcases import NAMES, default_grid
    kw = dict(jpi=77, jpj=64, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.4)
    pt, g = default_grid(77, 64)
    a = nb.Model(strict=True, **kw)
    b = nb.Model(strict=True, **kw)
    c = nb.Model(strict=True, **kw)
    b.set_grid(pt, *[g[n] for n in NAMES])
    for istp in range(1, 41):
        a.step(istp)
    b.step_n(1, 40)
    c.step_n(1, 40)
    for name, fid in STATE:
        np.testing.assert_array_equal(bits(a.field(fid)), bits(b.field(fid)), err_msg=name)
        np.testing.assert_array_equal(bits(c.field(fid)), bits(b.field(fid)), err_msg=name)


def test_default_build_general_grid_within_tolerance(nb, oracle_mod):
    m, o = _general_models(nb, oracle_mod, False, seed=5)
    for rec in range(4):
        m.step_n(1 + 100 * rec, 100)
        o.run(1 + 100 * rec, 100)
        for name, fid in STATE:
            assert relerr(m.field(fid), o.field(fid)) <= TOL, (rec, name)


def _advance(m, istp0, n, path):
    if path == "fused":
        m.step_n(istp0, n)
        return
    for istp in range(istp0, istp0 + n):
        m.continuity()
        m.momentum()
        m.bc(istp * m.p.rdt)
        m.next()


@pytest.mark.parametrize("strict", [True, False])
@pytest.mark.parametrize("path", ["fused", "routines"])
@pytest.mark.parametrize("grid", ["built-in", "set_grid"])
def test_checkpoint_restart_is_bit_exact(nb, tmp_path, strict, path, grid):
    """save_checkpoint after step 60, restart in a fresh context, steps 61..120:
    the same bits as the uninterrupted run, in both builds, through the fused
    path and through the continuity/momentum/bc/next calls, on the built-in
    grid and on a general grid."""
    from gridcases import NAMES, random_grid
    kw = dict(jpi=150, jpj=97, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.4, nbump=6,
              seed=8, bump_amp=20.0, bump_wmin=5e3, bump_wmax=40e3)
    if grid == "set_grid":
        kw["rdt"] = 10.0
        pt, g = random_grid(4, 150, 97)

    def make(**over):
        m = nb.Model(strict=strict, **dict(kw, **over))
        if grid == "set_grid":
            m.set_grid(pt, *[g[n] for n in NAMES])
        return m

    a = make()
    _advance(a, 1, 60, path)
    ck = str(tmp_path / "ck.npz")
    a.save_checkpoint(ck, 60)
    assert not (tmp_path / "ck.npz.tmp").exists()
    _advance(a, 61, 60, path)
    b = make()
    istp = b.load_checkpoint(ck)
    assert istp == 60
    _advance(b, istp + 1, 60, path)
    for name, fid in STATE:
        np.testing.assert_array_equal(bits(a.field(fid)), bits(b.field(fid)), err_msg=name)


def test_checkpoint_refuses_another_model(nb, tmp_path):
    """A checkpoint restarts only a model of the same size, parameters and
    geometry; anything else raises instead of silently computing another run."""
    from gridcases import NAMES, random_grid
    kw = dict(jpi=150, jpj=97, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.4, nbump=6,
              seed=8, bump_amp=20.0, bump_wmin=5e3, bump_wmax=40e3)
    a = nb.Model(**kw)
    a.step_n(1, 10)
    ck = str(tmp_path / "ck.npz")
    a.save_checkpoint(ck, 10)
    for over in (dict(jpi=151), dict(seed=9), dict(rdt=10.0), dict(visc=0.2), dict(amp_tide=0.3),
                 dict(cbfr=0.001), dict(tide_phase=0.1)):
        c = nb.Model(**dict(kw, **over))
        with pytest.raises(ValueError):
            c.load_checkpoint(ck)
    pt, g = random_grid(4, 150, 97)
    d = nb.Model(**kw)
    d.set_grid(pt, *[g[n] for n in NAMES])
    with pytest.raises(ValueError):
        d.load_checkpoint(ck)
    e = nb.Model(**kw)
    assert e.load_checkpoint(ck) == 10
