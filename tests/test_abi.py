"""The C-ABI library: builds, loads, exports every declared symbol; host-only calls."""
import ctypes
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "libcc_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", text)
    skip = {"if", "for", "while", "sizeof", "return"}
    return sorted({n for n in names if n not in skip and not n.isupper()})


def test_library_exports_every_declared_symbol():
    from libcc_b200 import _native as N
    lib = N.load()
    decl = declared_symbols()
    assert set(decl) == set(N.EXPORTS), (set(decl) ^ set(N.EXPORTS))
    for name in decl:
        assert hasattr(lib, name), name


def test_library_is_sm100a_only():
    so = (ROOT / "libcc_b200" / "_lib" / "libcc_b200.so").read_bytes()
    assert b"sm_100a" in so


def test_host_only_entry_points():
    from libcc_b200 import _native as N
    lib = N.load()
    assert lib.ccT_num_tuples(4) == 4 + 12
    assert lib.ccT_num_tuples(24) == 2024 + 552
    assert lib.ccT_status_string(0) == b"ok"
    assert lib.ccT_status_string(5).startswith(b"non-negative")
    opt = N.Options()
    lib.ccT_options_default(ctypes.byref(opt))
    assert opt.precision == 0 and opt.check_inputs == 1


def test_plan_rejects_bad_shapes_without_touching_a_gpu():
    from libcc_b200 import _native as N
    lib = N.load()
    h = ctypes.c_void_p()
    assert lib.ccT_plan_create(ctypes.byref(h), 1, 10, None) == 1
    assert lib.ccT_plan_create(ctypes.byref(h), 4, 0, None) == 1
    assert b"no" in lib.ccT_last_error()


def test_tuple_count_matches_reference_formula():
    from libcc_b200 import synthetic as S
    from libcc_b200 import _native as N
    lib = N.load()
    for no in (2, 3, 4, 12, 16, 24):
        ijk, iij, ijj = S.tuple_counts(no)
        assert lib.ccT_num_tuples(no) == ijk + iij + ijj
