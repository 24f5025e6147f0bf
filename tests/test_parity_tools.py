"""Checksum-table and .dat comparison tools (CPU): the defects of the
reference's tools/csv-checksum.py (left compared with itself, v never
tested) and tools/diff.py (absolute differences only) are absent here."""
import numpy as np
import pytest

from nemo_b200 import parity


def write_csv(path, header, rows):
    with open(path, "w") as fh:
        fh.write(",".join(header) + "\n")
        for r in rows:
            fh.write(",".join(str(x) for x in r) + "\n")


def test_checksums_compare_left_against_right_for_both_fields(tmp_path):
    hdr = ["build", "scale", "repeat", "jpiglo", "jpjglo", "ua_checksum", "va_checksum"]
    left = tmp_path / "left.csv"
    right = tmp_path / "right.csv"
    write_csv(left, hdr, [["original", 128, 0, 130, 130, 1.25, 3.5], ["original", 256, 0, 258, 258, 2.0, 4.0]])
    # only a va checksum differs: the reference's tool reports "Correct!" here
    write_csv(right, hdr, [["cuda", 128, 0, 130, 130, 1.25, 3.5], ["cuda", 256, 0, 258, 258, 2.0, 4.0 + 1e-9]])
    rows, missing = parity.compare_checksums(parity.read_checksums(left), parity.read_checksums(right))
    assert not missing and len(rows) == 4
    bad = [r for r in rows if not r["ok"]]
    assert len(bad) == 1 and bad[0]["field"] == "va_checksum" and bad[0]["key"] == (256, 0)
    assert bad[0]["abs_diff"] == pytest.approx(1e-9, rel=1e-6)
    rows, _ = parity.compare_checksums(parity.read_checksums(left), parity.read_checksums(right), rtol=1e-9)
    assert all(r["ok"] for r in rows)
    assert parity.main(["checksums", str(left), str(right)]) == 1
    assert parity.main(["checksums", str(left), str(right), "--rtol", "1e-9"]) == 0


def test_driver_checksum_files_and_missing_records(tmp_path):
    hdr = ["istp", "ssh_checksum", "ua_checksum", "va_checksum"]
    a = tmp_path / "a.csv"
    b = tmp_path / "b.csv"
    write_csv(a, hdr, [[100, "1.00000000000000000e+00", 2.0, 3.0], [200, 1.5, 2.5, 3.5]])
    write_csv(b, hdr, [[100, 1.0, 2.0, 3.0]])
    rows, missing = parity.compare_checksums(parity.read_checksums(a), parity.read_checksums(b))
    assert all(r["ok"] for r in rows) and len(rows) == 3 and missing == [200]
    assert parity.main(["checksums", str(a), str(b)]) == 1  # a record is missing


def write_dat(path, a, ny, nx):
    """The model's go2d layout: 6e20.7e4 per point, a blank line after each row."""
    with open(path, "w") as fh:
        for j in range(ny):
            for i in range(nx):
                fh.write("".join("%20.7E" % v for v in a[j * nx + i]).replace("E+", "E+00").replace("E-", "E-00") + "\n")
            fh.write("\n")


def test_dat_relative_max_norm_per_column(tmp_path):
    rng = np.random.default_rng(1)
    ny, nx = 3, 4
    ref = rng.normal(size=(ny * nx, 6))
    ref[:, 5] *= 1e-3  # a small-magnitude column: only a relative norm judges it fairly
    smp = ref.copy()
    smp[5, 5] += 1e-6
    p, q = tmp_path / "ref.dat", tmp_path / "smp.dat"
    write_dat(p, ref, ny, nx)
    write_dat(q, smp, ny, nx)
    a, b = parity.read_dat(p), parity.read_dat(q)
    assert a.shape == (12, 6)
    np.testing.assert_allclose(a, ref, rtol=1e-7)
    res = parity.compare_dat(a, b)
    assert [k for k, r in res.items() if not r["ok"]] == ["v"]
    assert res["v"]["rel_max_norm"] == pytest.approx(1e-6 / np.abs(ref[:, 5]).max(), rel=1e-3)
    res = parity.compare_dat(a, b, rtol=2e-3)
    assert all(r["ok"] for r in res.values())
    assert parity.main(["dat", str(p), str(q)]) == 1
    assert parity.main(["dat", str(p), str(p)]) == 0
