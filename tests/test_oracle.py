"""The CPU oracle against golden vectors executed from the reference source.

tests/golden/*.npz were produced by tests/golden/make_golden.py, which runs the
statements of original/nemolite2d.f90 (grid, initialisation, continuity,
momentum, bc, next) in IEEE double.  The oracle must reproduce every recorded
field bit for bit, sign of zero included.
"""
import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES

FIELDS = [("sshn", 0), ("un", 1), ("vn", 2), ("ssha", 3), ("ua", 4), ("va", 5),
          ("sshn_u", 6), ("sshn_v", 7)]


def load(name):
    return np.load("%s/%s.npz" % (GOLDEN, name))


def model_for(o, z, **kw):
    return o.Model(jpi=int(z["jpi"]), jpj=int(z["jpj"]), dx=float(z["nml_dx"]),
                   dy=float(z["nml_dy"]), dep_const=float(z["nml_dep_const"]),
                   rdt=float(z["nml_rdt"]), cbfr=float(z["nml_cbfr"]),
                   visc=float(z["nml_visc"]), **kw)


def bits(a):
    return np.ascontiguousarray(a).view(np.int64)


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_oracle_matches_reference_source(oracle_mod, case):
    z = load(case)
    m = model_for(oracle_mod, z)
    last = 0
    for r in z["records"]:
        if r > 0:
            m.run(last + 1, int(r) - last)
            last = int(r)
        for name, fid in FIELDS:
            np.testing.assert_array_equal(bits(m.field(fid)), bits(z["s%05d_%s" % (r, name)]),
                                          err_msg="%s step %d field %s" % (case, r, name))
    assert m.checksum(oracle_mod.UA) == float(z["ua_checksum"])
    assert m.checksum(oracle_mod.VA) == float(z["va_checksum"])


@pytest.mark.parametrize("case", ["g10x10_ref128phys", "g32x32_ref128phys"])
def test_oracle_grid_matches_reference(oracle_mod, case):
    z = load(case)
    m = model_for(oracle_mod, z)
    for name, fid in [("ht", oracle_mod.HT), ("hu", oracle_mod.HU), ("hv", oracle_mod.HV),
                      ("xt", oracle_mod.XT), ("yt", oracle_mod.YT)]:
        np.testing.assert_array_equal(m.field(fid), z["grid_" + name])


def test_openmp_is_bitwise_identical(oracle_mod):
    kw = dict(jpi=64, jpj=48, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.2)
    a = oracle_mod.Model(**kw)
    b = oracle_mod.Model(**kw)
    oracle_mod.set_threads(1)
    a.run(1, 60)
    oracle_mod.set_threads(4)
    b.run(1, 60)
    oracle_mod.set_threads(1)
    for fid in (oracle_mod.SSHN, oracle_mod.UN, oracle_mod.VN):
        np.testing.assert_array_equal(bits(a.field(fid)), bits(b.field(fid)))


def test_zero_amplitude_stays_at_rest(oracle_mod):
    m = oracle_mod.Model(jpi=20, jpj=16, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.0)
    m.run(1, 50)
    for fid in (oracle_mod.SSHN, oracle_mod.UN, oracle_mod.VN):
        assert not np.any(m.field(fid))


def test_clamped_row_follows_tide(oracle_mod):
    amp, rdt = 0.7, 20.0
    m = oracle_mod.Model(jpi=24, jpj=20, rdt=rdt, cbfr=0.00015, visc=0.1, amp_tide=amp)
    om = 2.0 * 3.14159 / (12.42 * 3600.0)
    for istp in range(1, 30):
        m.step(istp)
        row = m.field(oracle_mod.SSHN)[0]  # jj = 1
        assert np.all(row == amp * np.sin(om * (istp * rdt)))


def test_wall_velocities_are_zero(oracle_mod):
    m = oracle_mod.Model(jpi=24, jpj=20, rdt=20.0, cbfr=0.00015, visc=0.1)
    m.run(1, 40)
    u = m.field(oracle_mod.UN)
    v = m.field(oracle_mod.VN)
    assert not np.any(u[:, 0]) and not np.any(u[:, -1])   # ji = 0 and ji = jpi
    assert not np.any(v[-1, :])                            # jj = jpj
    assert np.any(v[0, :])                                 # Flather row jj = 0 is active


def test_tree_checksum_close_to_reference_order(oracle_mod):
    m = oracle_mod.Model(jpi=300, jpj=70, rdt=20.0, cbfr=0.00015, visc=0.1)
    m.run(1, 30)
    for fid in (oracle_mod.SSHN, oracle_mod.UA, oracle_mod.VA):
        s, t = m.checksum(fid, "seq"), m.checksum(fid, "tree")
        assert abs(s - t) <= 1e-13 * abs(s)


def test_bathymetry_is_seeded_and_bounded(oracle_mod):
    kw = dict(jpi=200, jpj=150, nbump=32, seed=1234, bump_amp=40.0,
              bump_wmin=20e3, bump_wmax=60e3, hmin=10.0)
    a = oracle_mod.Model(**kw)
    b = oracle_mod.Model(**kw)
    c = oracle_mod.Model(**dict(kw, seed=99))
    ht = a.field(oracle_mod.HT)
    np.testing.assert_array_equal(ht, b.field(oracle_mod.HT))
    assert not np.array_equal(ht, c.field(oracle_mod.HT))
    assert ht.min() >= 10.0 and ht.std() > 0.5
