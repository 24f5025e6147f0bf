"""General grids (masks with open water on every border, islands, per-point
scale factors and latitudes) in the oracle: the default grid passed as
arrays reproduces the built-in one bit for bit, and a general grid runs
finite with its walls closed.  The B200 parity on general grids is in
tests/test_gpu_parity.py."""
import numpy as np
import pytest

from gridcases import NAMES, default_grid, random_grid

FIELDS = ("SSHN", "UN", "VN", "SSHA", "UA", "VA", "SSHN_U", "SSHN_V")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def test_default_grid_as_arrays_is_the_built_in_grid(oracle_mod):
    kw = dict(jpi=41, jpj=29, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.2)
    a = oracle_mod.Model(**kw)
    b = oracle_mod.Model(**kw)
    pt, g = default_grid(41, 29)
    b.set_grid(pt, *[g[n] for n in NAMES])
    a.run(1, 60)
    b.run(1, 60)
    for f in FIELDS:
        fid = getattr(oracle_mod, f)
        np.testing.assert_array_equal(bits(a.field(fid)), bits(b.field(fid)), err_msg=f)


def test_general_grid_runs_with_open_borders_and_islands(oracle_mod):
    jpi, jpj = 48, 36
    kw = dict(jpi=jpi, jpj=jpj, rdt=10.0, cbfr=0.00015, visc=0.1, amp_tide=0.3)
    m = oracle_mod.Model(**kw)
    pt, g = random_grid(3, jpi, jpj)
    m.set_grid(pt, *[g[n] for n in NAMES])
    m.run(1, 200)
    ua, va = m.field(oracle_mod.UA), m.field(oracle_mod.VA)   # (jpj, jpi+1), (jpj+1, jpi)
    for f in (oracle_mod.SSHN, oracle_mod.UN, oracle_mod.VN):
        assert np.all(np.isfinite(m.field(f)))
    # u points between two land/wall cells stay at rest (solid, :648-652)
    for jj in range(1, jpj + 1):
        for ji in range(0, jpi + 1):
            if pt[jj, ji] == 0 and pt[jj, ji + 1] == 0:
                assert ua[jj - 1, ji] == 0.0
    # the open borders move water through: some boundary velocity is nonzero
    assert np.any(ua[:, 0] != 0.0) or np.any(ua[:, jpi] != 0.0)
    assert np.any(va[0, :] != 0.0) or np.any(va[jpj, :] != 0.0)


def test_mask_values_are_checked(oracle_mod):
    m = oracle_mod.Model(jpi=10, jpj=8)
    pt, g = default_grid(10, 8)
    pt[3, 3] = 2
    with pytest.raises(ValueError):
        m.set_grid(pt, *[g[n] for n in NAMES])
