"""Parity checks between two runs: checksum tables and .dat field files.

Does what the reference's tools/csv-checksum.py and tools/diff.py set out to
do, with their defects fixed: tools/csv-checksum.py:82-89 subtracts each left
checksum from itself (so every row compares equal), turns the u delta into a
boolean before thresholding it and selects incorrect rows with a query that
tests the u flag twice and never the v flag; tools/diff.py reports absolute
differences only.  Here both checksums (and the ssh checksum when present)
are compared left against right with absolute and relative tolerances, and
.dat files get, per column, the maximum absolute difference and the relative
max-norm max|a - b| / max|reference|.

Checksum tables are CSV files with a key column -- `scale` (and `repeat`, if
present) as written by tools/benchmark-extractor.py, or `istp` as written by
the host driver's checksums.csv -- and `ua_checksum`, `va_checksum` (and
optionally `ssh_checksum`) columns.  .dat files are the model's
`go2d_%05d.dat` output (original/nemolite2d.f90:773-799): six numbers per
line (x, y, depth, ssh, u, v), blank lines between grid rows.

Command line:
    python -m nemo_b200.parity checksums LEFT.csv RIGHT.csv [--rtol R] [--atol A]
    python -m nemo_b200.parity dat REFERENCE.dat SAMPLE.dat [--rtol R] [--atol A]
The exit status is 0 when everything agrees within the tolerances, 1 otherwise.
"""
import argparse
import csv
import sys

import numpy as np

CHECKSUM_FIELDS = ("ssh_checksum", "ua_checksum", "va_checksum")
DAT_COLUMNS = ("x", "y", "depth", "ssh", "u", "v")


def read_checksums(path):
    """{key: {field: value}} from a checksum CSV (key: `istp`, or `scale`
    with `repeat` when present; values averaged over rows sharing a key)."""
    with open(path, newline="") as fh:
        rows = list(csv.DictReader(fh))
    if not rows:
        return {}
    cols = rows[0].keys()
    if "istp" in cols:
        keycols = ("istp",)
    elif "scale" in cols:
        keycols = ("scale", "repeat") if "repeat" in cols else ("scale",)
    else:
        raise ValueError("%s: no istp or scale column" % path)
    fields = [f for f in CHECKSUM_FIELDS if f in cols]
    if not fields:
        raise ValueError("%s: no checksum columns" % path)
    acc = {}
    for r in rows:
        key = tuple(int(float(r[k])) for k in keycols)
        key = key[0] if len(key) == 1 else key
        d = acc.setdefault(key, {f: [] for f in fields})
        for f in fields:
            if r[f] not in ("", None):
                d[f].append(float(r[f].replace(",", "")))
    return {k: {f: float(np.mean(v)) for f, v in d.items() if v} for k, d in acc.items()}


def compare_checksums(left, right, rtol=0.0, atol=0.0):
    """Rows (key, field, left, right, abs_diff, rel_diff, ok) for every key and
    field present on both sides, and the keys present on one side only.  ok:
    |left - right| <= atol + rtol * |left|."""
    out = []
    for key in sorted(set(left) & set(right), key=lambda k: (str(type(k)), k)):
        for f in CHECKSUM_FIELDS:
            if f in left[key] and f in right[key]:
                a, b = left[key][f], right[key][f]
                d = abs(a - b)
                rel = d / abs(a) if a != 0 else (0.0 if d == 0 else float("inf"))
                ok = bool(d <= atol + rtol * abs(a))
                out.append(dict(key=key, field=f, left=a, right=b, abs_diff=d, rel_diff=rel, ok=ok))
    missing = sorted(set(left) ^ set(right), key=str)
    return out, missing


def read_dat(path):
    """(n, 6) float64 array of a .dat file (Fortran E format with wide
    exponents is read as is)."""
    vals = []
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            if not parts:
                continue
            if len(parts) != 6:
                raise ValueError("%s: expected 6 numbers per line, got %d" % (path, len(parts)))
            vals.append([float(p.replace("D", "E").replace("d", "e")) for p in parts])
    return np.asarray(vals, dtype=np.float64).reshape(-1, 6)


def compare_dat(ref, sample, rtol=0.0, atol=0.0):
    """Per column: max_abs, rel_max_norm (max|a-b| / max|ref|, 0 when both
    are 0), bad (rows with |a-b| > atol + rtol * max|ref|) and ok."""
    if ref.shape != sample.shape:
        raise ValueError("shapes differ: %s vs %s" % (ref.shape, sample.shape))
    out = {}
    for k, name in enumerate(DAT_COLUMNS):
        d = np.abs(ref[:, k] - sample[:, k])
        scale = np.abs(ref[:, k]).max() if ref.shape[0] else 0.0
        mx = float(d.max()) if d.size else 0.0
        rel = mx / scale if scale > 0 else (0.0 if mx == 0 else float("inf"))
        bad = int((d > atol + rtol * scale).sum())
        out[name] = dict(max_abs=mx, rel_max_norm=rel, bad=bad, ok=bad == 0)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m nemo_b200.parity")
    ap.add_argument("kind", choices=["checksums", "dat"])
    ap.add_argument("left")
    ap.add_argument("right")
    ap.add_argument("--rtol", type=float, default=0.0)
    ap.add_argument("--atol", type=float, default=0.0)
    a = ap.parse_args(argv)
    if a.kind == "checksums":
        rows, missing = compare_checksums(read_checksums(a.left), read_checksums(a.right), a.rtol, a.atol)
        bad = [r for r in rows if not r["ok"]]
        for r in bad:
            print("%-12s %-13s left %.16e right %.16e abs %.3e rel %.3e"
                  % (r["key"], r["field"], r["left"], r["right"], r["abs_diff"], r["rel_diff"]))
        if missing:
            print("keys on one side only:", ", ".join(str(m) for m in missing))
        print("%d of %d checksums agree (rtol %g, atol %g)" % (len(rows) - len(bad), len(rows), a.rtol, a.atol))
        return 0 if not bad and not missing and rows else 1
    res = compare_dat(read_dat(a.left), read_dat(a.right), a.rtol, a.atol)
    for name, r in res.items():
        print("%-6s max_abs %.3e rel_max_norm %.3e rows_over_tol %d" % (name, r["max_abs"], r["rel_max_norm"], r["bad"]))
    ok = all(r["ok"] for r in res.values())
    print("agree" if ok else "differ")
    return 0 if ok else 1


if __name__ == "__main__":
    sys.exit(main())
