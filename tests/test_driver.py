"""The C++ host driver keeps the reference program's I/O contract.

original/nemolite2d.f90 reads ./namelist (&namctl), echoes it, prints
'ua checksum = ' / 'va checksum = ' in E16.8 and a dl_timer report whose rows
tools/benchmark-extractor.py parses (JPIGLO/JPJGLO lines, checksum lines,
rows 'Time-stepping', 'Continuity', 'Momentum', 'BCs', 'Next' with counts,
total, average, avg/repeat, std err in columns 1-5).
"""
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG

DRIVER = os.path.join(PKG, "bin", "nemolite2d")

NAMELIST = """!-----------------------------------------------------------------------
&namctl     !   parameters for a example setup
!-----------------------------------------------------------------------
   jpiglo      =     {jpiglo}               !  number of columns of model grid
   jpjglo      =     {jpjglo}               !  number of rows of model grid
   jphgr_msh   =       {jphgr}               !  type of grid
   dx          =    1000.0             !  grid size in x direction (m)
   dy          =    1000.0             !  grid size in y direction (m)
   dep_const   =     100.0             !  constant depth (m)
   nit000      =       1               !  first time step
   nitend      =    {nitend}               !43200               !  end time step
   irecord     =     {irecord}               ! 180               !  intervals to save results
   rdt         =      20.0             !  size of time step (second)
   cbfr        =       0.00015          !  bottom friction coefficeint
   visc        =       0.1             !  horizontal kinematic viscosity coefficient
{extra}/
"""


def write_nl(d, jpiglo=34, jpjglo=34, nitend=100, irecord=25, jphgr=1, extra=""):
    p = os.path.join(d, "namelist")
    with open(p, "w") as fh:
        fh.write(NAMELIST.format(jpiglo=jpiglo, jpjglo=jpjglo, nitend=nitend, irecord=irecord,
                                 jphgr=jphgr, extra=extra))
    return p


@pytest.fixture(scope="module")
def driver():
    subprocess.run(["make", "-s", "-C", PKG], check=True)
    assert os.path.exists(DRIVER)
    return DRIVER


def run(driver, cwd, *args):
    return subprocess.run([driver, *args], cwd=cwd, capture_output=True, text=True, timeout=600)


def fortran_e(v, w, d):
    """Reference Ew.d rendering (0.ddddE+xx), used to check the driver's output."""
    if v == 0:
        s = "0." + "0" * d + "E+00"
    else:
        m = "%.*e" % (d - 1, abs(v))
        mant, ex = m.split("e")
        s = ("-" if v < 0 else "") + "0." + mant.replace(".", "") + "E%+03d" % (int(ex) + 1)
    return s.rjust(w)


def extractor_parse(text):
    """The parsing rules of tools/benchmark-extractor.py:144-195."""
    out = {}
    for line in text.splitlines():
        line = line.strip()
        if line.startswith("JPIGLO"):
            out["jpiglo"] = int(line.split("=")[-1].replace(",", "").strip())
        if line.startswith("JPJGLO"):
            out["jpjglo"] = int(line.split("=")[-1].replace(",", "").strip())
        if line.startswith("ua checksum"):
            out["ua"] = np.float64(line.split("=")[-1].replace(",", "").strip())
        if line.startswith("va checksum"):
            out["va"] = np.float64(line.split("=")[-1].replace(",", "").strip())
        for lab in ("Time-stepping", "Continuity", "Momentum", "BCs", "Next"):
            if line.startswith(lab):
                sp = line.split()
                out[lab] = [np.float64(x) for x in sp[1:6]]
    return out


def test_echo_namelist_parses_like_reference(driver, tmp_path):
    write_nl(str(tmp_path), jpiglo=130, jpjglo=66)
    r = run(driver, str(tmp_path), "--echo-namelist")
    assert r.returncode == 0, r.stderr
    p = extractor_parse(r.stdout)
    assert p["jpiglo"] == 130 and p["jpjglo"] == 66


def test_bad_namelist_stops_with_reference_message(driver, tmp_path):
    with open(tmp_path / "namelist", "w") as fh:
        fh.write("&namctl jpiglo = 34, bogus_key = 3 /\n")
    r = run(driver, str(tmp_path))
    assert r.returncode != 0
    assert "err found in reading namelist file" in r.stdout
    os.remove(tmp_path / "namelist")
    r = run(driver, str(tmp_path))
    assert r.returncode != 0 and "err found in reading namelist file" in r.stdout


@pytest.mark.parametrize("irecord", [0, -5])
def test_nonpositive_irecord_is_a_namelist_error(driver, tmp_path, irecord):
    """MOD(istp, irecord) has no value for irecord <= 0: the driver stops with
    a namelist error before touching the device instead of dividing by zero."""
    write_nl(str(tmp_path), irecord=irecord)
    r = run(driver, str(tmp_path))
    assert r.returncode not in (0, -8), r.stdout + r.stderr  # -8: SIGFPE
    assert "err found in reading namelist file" in r.stdout
    assert "irecord" in r.stderr


def test_grid_from_file_is_refused_like_reference(driver, tmp_path):
    write_nl(str(tmp_path), jphgr=0)
    r = run(driver, str(tmp_path))
    assert r.returncode != 0 and "It is not ready to Read in grid from a file" in r.stdout
    write_nl(str(tmp_path), jphgr=7)
    r = run(driver, str(tmp_path))
    assert r.returncode != 0 and "Wrong grid defination type" in r.stdout


def test_fortran_e_helper():
    assert fortran_e(0.0300871504, 16, 8) == "  0.30087150E-01"
    assert fortran_e(1234.5, 12, 5) == " 0.12345E+04"


@pytest.mark.gpu
@pytest.mark.parametrize("fused", [False, True])
def test_driver_run_matches_oracle(driver, tmp_path, oracle_mod, fused):
    d = str(tmp_path)
    write_nl(d, jpiglo=34, jpjglo=30, nitend=100, irecord=25,
             extra="   fused = %s\n" % (".true." if fused else ".false."))
    r = run(driver, d)
    assert r.returncode == 0, r.stdout + r.stderr
    o = oracle_mod.Model(jpi=32, jpj=28, rdt=20.0, cbfr=0.00015, visc=0.1)
    o.run(1, 100)
    ua, va = o.checksum(oracle_mod.UA), o.checksum(oracle_mod.VA)
    assert "ua checksum = %s" % fortran_e(ua, 16, 8) in r.stdout
    assert "va checksum = %s" % fortran_e(va, 16, 8) in r.stdout
    p = extractor_parse(r.stdout)
    assert p["jpiglo"] == 34 and p["jpjglo"] == 30
    assert p["Time-stepping"][0] == 1
    if not fused:
        for lab in ("Continuity", "Momentum", "BCs", "Next"):
            assert p[lab][0] == 100
    # per-record checksums
    rows = np.loadtxt(os.path.join(d, "checksums.csv"), delimiter=",", skiprows=1)
    assert list(rows[:, 0]) == [25, 50, 75, 100]
    np.testing.assert_allclose(rows[-1, 1:], [o.checksum(oracle_mod.SSHN), ua, va], rtol=1e-11)
    # gnuplot output at the last record: x, y, depth, ssh, u, v at T points
    dat = np.loadtxt(os.path.join(d, "go2d_00100.dat"))
    assert dat.shape == (32 * 28, 6)
    ssh = o.field(oracle_mod.SSHN).ravel()
    u = o.field(oracle_mod.UN)
    uc = (0.5 * (u[:, :-1] + u[:, 1:])).ravel()
    np.testing.assert_allclose(dat[:, 3], ssh, rtol=1e-6, atol=1e-12)
    np.testing.assert_allclose(dat[:, 4], uc, rtol=1e-6, atol=1e-12)
    assert os.path.exists(os.path.join(d, "go2d_00000.dat"))
