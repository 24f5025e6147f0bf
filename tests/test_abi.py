"""The C-ABI libraries load and export every symbol include/nemo_b200.h declares.

CPU only: no call here touches a GPU.
"""
import os
import re
import subprocess

import pytest

from conftest import PKG, ROOT

HEADER = os.path.join(ROOT, "include", "nemo_b200.h")


def header_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|void|nemo_ctx\*|const char\*|long long)\s+\*?(\w+)\s*\(",
                                 text, flags=re.M)))


@pytest.fixture(scope="module")
def built():
    subprocess.run(["make", "-s", "-C", PKG], check=True)
    import nemo_b200
    return nemo_b200


@pytest.mark.parametrize("strict", [False, True])
def test_library_exports_every_declared_symbol(built, strict):
    lib = built.load(strict)
    syms = header_symbols()
    assert len(syms) >= 35
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(built.EXPORTED) == syms


def test_dynamic_symbol_table_has_cabi_names(built):
    out = subprocess.run(["nm", "-D", "--defined-only", built.lib_path(False)],
                         capture_output=True, text=True, check=True).stdout
    names = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for s in header_symbols():
        assert s in names, s


def test_strict_flag_distinguishes_builds(built):
    assert built.is_strict_build(True) is True
    assert built.is_strict_build(False) is False


def test_default_params_match_reference_defaults(built):
    p = built.default_params()
    # original/nemolite2d.f90:107-118 (jpiglo = 258 -> jpi = 256)
    assert (p.jpi, p.jpj, p.nit000, p.nitend, p.irecord) == (256, 256, 1, 1000, 1)
    assert (p.dx, p.dy, p.dep_const, p.rdt, p.cbfr, p.visc) == (1000.0, 1000.0, 100.0, 10.0, 0.001, 100.0)
    assert (p.amp_tide, p.tide_phase, p.lat, p.nbump) == (0.2, 0.0, 50.0, 0)


def test_status_strings(built):
    lib = built.load(False)
    assert lib.nemo_status_string(0) == b"ok"
    assert lib.nemo_status_string(1) == b"invalid argument"
    assert lib.nemo_status_string(99) == b"unknown status"


def test_null_handles_are_rejected_without_a_gpu(built):
    lib = built.load(False)
    assert lib.nemo_step_n(None, 1, 1) == 4
    assert lib.nemo_continuity(None) == 4
    assert lib.nemo_create(None, None) == 1
    assert lib.nemo_destroy(None) == 1
    assert lib.nemo_set_grid(None, None) == 1
    assert lib.nemo_record(None, None) == 1
    assert lib.nemo_record_wait(None) == 1


def test_field_shapes_follow_fortran_bounds(built):
    assert built.field_shape(built.SSHN, 7, 5) == (5, 7)
    assert built.field_shape(built.UN, 7, 5) == (5, 8)
    assert built.field_shape(built.VN, 7, 5) == (6, 7)


def test_missing_library_fails_loudly(built, monkeypatch, tmp_path):
    monkeypatch.setattr(built, "LIB_DIR", str(tmp_path))
    monkeypatch.setattr(built, "_libs", {})
    with pytest.raises(ImportError):
        built.load(False)


def test_member_recipe_is_seeded_and_bounded(built):
    """nemo_ens_generate is host-only: sides log-uniform in [64, 1024], aspect
    in [0.5, 2], tidal amplitude amp_scale*[0.5, 1.5], phase in [0, 2*pi)."""
    a = built.generate_members(42, 256)
    b = built.generate_members(42, 256)
    c = built.generate_members(43, 256)
    key = lambda ms: [(m.jpi, m.jpj, m.amp_tide, m.seed) for m in ms]
    assert key(a) == key(b) and key(a) != key(c)
    import math
    for m in a:
        assert 64 <= m.jpi <= 1024
        assert 0.5 - 1e-2 <= m.jpj / m.jpi <= 2.0 + 1e-2
        assert 0.5 <= m.amp_tide <= 1.5 and 0.0 <= m.tide_phase < 2 * math.pi
        assert (m.dep_const, m.nbump, m.hmin, m.hmax) == (100.0, 8, 50.0, 150.0)
    cells = sum(m.jpi * m.jpj for m in a)
    assert 2e7 < cells < 1.2e8
    s = built.generate_members(42, 8, amp_scale=0.2)
    assert all(0.1 <= m.amp_tide <= 0.3 for m in s)
