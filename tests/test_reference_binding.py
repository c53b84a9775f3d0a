"""The reference's own Python binding loads this library unchanged (no device needed).

ArrowMetal's binding (python/arrowmetal/__init__.py:23-78 finds the library through
$ARROWMETAL_LIB; :80-1230 binds every entry point at import) is imported from a checkout of the
reference with $ARROWMETAL_LIB set to this library, in a child process so its module state stays out of
this one. Entry points outside the sort path are exported and answer "not served" with status 1.
Skipped where no checkout of the reference is present (set ARROWMETAL_REFERENCE to one).
"""
import ctypes
import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "arrowmetal_b200", "lib", "libArrowMetalC.so")
CHECKOUT = os.environ.get("ARROWMETAL_REFERENCE", os.path.join(os.sep, "root", "reference"))
BINDING = os.path.join(CHECKOUT, "python", "arrowmetal", "__init__.py")
HEADER = os.path.join(CHECKOUT, "include", "arrowmetal.h")

needs_checkout = pytest.mark.skipif(not os.path.exists(BINDING), reason="no checkout of the reference binding here")


def header_entry_points():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    return sorted(set(re.findall(r"\b(am_[a-z0-9_]+)\s*\(", text)))


@needs_checkout
def test_every_reference_entry_point_is_exported():
    lib = ctypes.CDLL(LIB)
    names = header_entry_points()
    assert len(names) > 250
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@needs_checkout
def test_reference_binding_imports_unchanged():
    code = ("import sys; sys.path.insert(0, sys.argv[1]); import arrowmetal as am; "
            "print(am.__file__); print(am._lib._name)")
    env = dict(os.environ, ARROWMETAL_LIB=LIB)
    r = subprocess.run([sys.executable, "-c", code, os.path.join(CHECKOUT, "python")], env=env,
                       capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    where, loaded = r.stdout.split()[-2:]
    assert where.startswith(CHECKOUT) and loaded == LIB


def test_unserved_entry_points_answer_not_served():
    lib = ctypes.CDLL(LIB)
    lib.am_last_error.restype = ctypes.c_char_p
    lib.am_filter.restype = ctypes.c_int
    assert lib.am_filter(None, None, None) == 1
    assert b"am_filter: not served" in lib.am_last_error()
    lib.am_parquet_num_rows.restype = ctypes.c_int64
    assert lib.am_parquet_num_rows(None) == -1
    lib.am_csv_batch_column_name.restype = ctypes.c_char_p
    assert lib.am_csv_batch_column_name(None, 0) is None
    assert b"am_csv_batch_column_name: not served" in lib.am_last_error()
