"""The C-ABI library without a GPU: it loads, exports every symbol include/*.h declares, and keeps the
reference's return-code and error conventions for calls that fail before touching the device."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

LIB = os.path.join(ROOT, "arrowmetal_b200", "lib", "libArrowMetalC.so")


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(am_[a-z0-9_]+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    assert os.path.exists(LIB), "build the library first (make -C arrowmetal_b200/csrc)"
    return ctypes.CDLL(LIB)


def test_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) >= 50
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def unserved_symbols():
    """The entry points outside the sort path that the library exports only so that the reference's
    callers load it (each answers "not served"), listed in csrc/unserved.cpp."""
    text = open(os.path.join(ROOT, "arrowmetal_b200", "csrc", "unserved.cpp")).read()
    return set(re.findall(r"\bX\((am_[a-z0-9_]+)\)", text))


def test_exports_nothing_else():
    out = os.popen(f"nm -D --defined-only {LIB}").read().split("\n")
    exported = {l.split()[-1] for l in out if l.strip()}
    extra = {e for e in exported if not e.startswith("am_")}
    assert not extra, sorted(extra)[:20]
    unserved = unserved_symbols()
    assert len(unserved) > 200 and not unserved & declared_symbols()
    assert exported == declared_symbols() | unserved


def test_reference_binding_sort_symbols_present(lib):
    # The sort-path symbols ArrowMetal's Python binding binds at import
    # (python/arrowmetal/__init__.py:80-118, :1219-1226, :3793-3794, :5684-5685).
    for n in ["am_version", "am_device_name", "am_last_error", "am_format", "am_compute_format", "am_length",
              "am_null_count", "am_release", "am_import", "am_import_chunks", "am_import_chunks_supported",
              "am_set_import_threads", "am_get_import_threads", "am_export", "am_take", "am_slice", "am_argsort",
              "am_sort", "am_top_k", "am_lexsort", "am_lexsort_ex", "am_lexsort_ex2", "am_argsort_ex",
              "am_argsort_ex2", "am_sort_ex", "am_sort_ex2", "am_top_k_ex", "am_batch_begin", "am_batch_end",
              "am_plan_source_create", "am_plan_run", "am_plan_column", "am_plan_result_release",
              "am_router_set_mode", "am_router_get_mode"]:
        assert hasattr(lib, n), n


def test_version_and_router(lib):
    lib.am_version.restype = ctypes.c_char_p
    assert lib.am_version() == b"0.6.1"
    assert lib.am_router_set_mode(1) == 0
    assert lib.am_router_get_mode() == 1
    assert lib.am_router_set_mode(7) == 2          # unknown mode (include/arrowmetal.h:1799)
    assert lib.am_router_set_mode(0) == 0


def test_null_handles_are_invalid_arguments(lib):
    P = ctypes.c_void_p
    out = P()
    lib.am_length.restype = ctypes.c_int64
    lib.am_length.argtypes = [P]
    assert lib.am_length(None) == -1
    lib.am_argsort.argtypes = [P, ctypes.c_int, ctypes.POINTER(P)]
    assert lib.am_argsort(None, 0, ctypes.byref(out)) == 2
    lib.am_take.argtypes = [P, P, ctypes.POINTER(P)]
    assert lib.am_take(None, None, ctypes.byref(out)) == 2
    lib.am_import.argtypes = [P, P, ctypes.POINTER(P)]
    assert lib.am_import(None, None, ctypes.byref(out)) == 2
    lib.am_lexsort.argtypes = [P, P, ctypes.c_int64, ctypes.POINTER(P)]
    assert lib.am_lexsort(None, None, 0, ctypes.byref(out)) == 2
    lib.am_plan_run.argtypes = [ctypes.c_char_p, P, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(P)]
    assert lib.am_plan_run(None, None, 0, 0, ctypes.byref(out)) == 2
    lib.am_release.argtypes = [P]
    lib.am_release(None)   # a no-op, as in the reference


def test_plan_errors_without_a_device(lib):
    lib.am_plan_explain.restype = ctypes.c_char_p
    lib.am_plan_explain.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int]
    lib.am_last_error.restype = ctypes.c_char_p
    assert lib.am_plan_explain(b'{"op": "scan", ', None, 0, 0) is None
    assert b"JSON" in lib.am_last_error()
    assert lib.am_plan_explain(b'{"op": "join", "input": {"op": "scan", "source": "t"}}', None, 0, 0) is None
    assert b"not supported" in lib.am_last_error()
    assert lib.am_plan_explain(b'{"op": "scan", "source": "t"}', None, 0, 0) is None
    assert b"unknown source" in lib.am_last_error()


def test_plan_json_nesting_and_mutations_fail_cleanly(lib):
    # Deep nesting is refused before it can overflow the caller's stack, and mangled plans (truncated,
    # bytes replaced or inserted) return an error instead of crashing.
    import random
    lib.am_plan_explain.restype = ctypes.c_char_p
    lib.am_plan_explain.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int]
    lib.am_last_error.restype = ctypes.c_char_p
    for depth in (513, 100_000, 1_000_000):
        assert lib.am_plan_explain(b"[" * depth + b"]" * depth, None, 0, 0) is None
        assert b"nested more than 512 levels" in lib.am_last_error()
    plan = (b'{"op": "limit", "count": 50, "offset": 3, "input": {"op": "sort", "by": [["k", true, '
            b'{"nulls": "first", "float_order": "total"}], ["v", false]], "input": {"op": "select", '
            b'"columns": ["k", "v"], "input": {"op": "scan", "source": "t"}}}}')
    rng = random.Random(7)
    alphabet = b'{}[]":,0123456789.eE+-\\u tnrfalsenull '
    for _ in range(3000):
        s = bytearray(plan)
        kind = rng.randrange(3)
        if kind == 0:
            s = s[:rng.randrange(len(s) + 1)]
        elif kind == 1:
            for _ in range(rng.randrange(1, 6)):
                s[rng.randrange(len(s))] = rng.choice(alphabet)
        else:
            at = rng.randrange(len(s))
            s = s[:at] + bytes(rng.choice(alphabet) for _ in range(rng.randrange(1, 20))) + s[at:]
        if lib.am_plan_explain(bytes(s), None, 0, 0) is None:
            assert lib.am_last_error()


def test_import_chunks_refuses_unsupported_types(lib):
    import pyarrow as pa
    from arrowmetal_b200 import _ArrowSchema
    s = _ArrowSchema()
    pa.array(["a"]).type._export_to_c(ctypes.addressof(s))
    lib.am_import_chunks_supported.argtypes = [ctypes.c_void_p]
    assert lib.am_import_chunks_supported(ctypes.addressof(s)) == 0
    out = ctypes.c_void_p()
    lib.am_import_chunks.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_void_p)]
    assert lib.am_import_chunks(ctypes.addressof(s), None, 0, ctypes.byref(out)) == 3
    ctypes.CFUNCTYPE(None, ctypes.c_void_p)(s.release)(ctypes.addressof(s))


def test_binding_validates_options_before_the_device():
    import arrowmetal_b200 as am
    with pytest.raises(am.ArrowMetalError, match="null_placement"):
        am._index_of(am.NULL_PLACEMENT, "middle", "null_placement")
    with pytest.raises(am.ArrowMetalError, match="float_order"):
        am._index_of(am.FLOAT_ORDERS, "lexicographic", "float_order")
    with pytest.raises(am.ArrowMetalError, match="lexsort needs"):
        am.lexsort_indices([])


def test_no_device_fails_loudly():
    import arrowmetal_b200 as am
    if os.environ.get("CUDA_VISIBLE_DEVICES", None) == "" or not _has_gpu():
        name = am.device_name()
        assert name.startswith("unavailable")
        with pytest.raises(am.ArrowMetalError, match="CUDA"):
            am.MetalArray.from_arrow([1, 2, 3])
        with pytest.raises(am.ArrowMetalError, match="CUDA"):
            am.Server(workers=2)
    else:
        pytest.skip("a GPU is present")


def test_import_checks_string_offsets_before_the_device():
    # Offsets that decrease or go negative are refused by am_import before any device work (the string
    # kernels read each row's bytes between its offsets); a well-formed array gets past the check.
    import numpy as np
    import pyarrow as pa
    import arrowmetal_b200 as am
    data = pa.py_buffer(b"abcdefghij")
    for offs, typ, dt in (([0, 3, 2, 6], pa.utf8(), np.int32), ([0, 2, -1, 4], pa.binary(), np.int32),
                          ([0, 5, 4, 9], pa.large_utf8(), np.int64)):
        bad = pa.Array.from_buffers(typ, 3, [None, pa.py_buffer(np.array(offs, dtype=dt).tobytes()), data])
        with pytest.raises(am.ArrowMetalError, match="negative or decrease"):
            am.MetalArray.from_arrow(bad)
        # The same array in a dictionary's values.
        dict_arr = pa.DictionaryArray.from_arrays(pa.array([0, 1, 2], type=pa.int32()), bad)
        with pytest.raises(am.ArrowMetalError, match="negative or decrease"):
            am.MetalArray.from_arrow(dict_arr)
    if not _has_gpu():
        good = pa.array(["ab", None, "cde"])
        with pytest.raises(am.ArrowMetalError, match="CUDA"):
            am.MetalArray.from_arrow(good)
        with pytest.raises(am.ArrowMetalError, match="CUDA"):
            am.MetalArray.from_arrow(pa.array([], type=pa.utf8()))


def test_server_rejects_bad_arguments(lib):
    import ctypes
    out = ctypes.c_void_p()
    i64 = ctypes.c_int64
    assert lib.am_server_create(0, i64(1 << 30), i64(0), ctypes.byref(out)) == 2
    assert lib.am_server_create(2, i64(0), i64(0), ctypes.byref(out)) == 2
    assert lib.am_server_wait(None, i64(1), ctypes.byref(out), None) == 2
    assert lib.am_server_release(None) == 2


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_stream_handles_without_a_device():
    """A record-batch stream is taken and its columns selected on the host; the sort itself needs the
    device and fails loudly without one; a missing IPC file is an error with its path."""
    import pyarrow as pa
    import arrowmetal_b200 as am
    s = am.scan_arrow(pa.table({"a": [3, 1, 2], "s": ["x", "y", "z"]}))
    s.select(["s", "a"])
    with pytest.raises(am.ArrowMetalError, match="no column named"):
        s.select(["nope"])
    with pytest.raises(am.ArrowMetalError, match="CUDA|device"):
        s.sort("a")
    with pytest.raises(am.ArrowMetalError, match="consumed"):
        s.sort("a")
    assert am._lib.am_stream_open_ipc(b"/nonexistent.arrow", 3, 1) is None
    assert b"cannot open /nonexistent.arrow" in am._lib.am_stream_last_error()


def _release(struct):
    if struct.release:
        ctypes.CFUNCTYPE(None, ctypes.c_void_p)(struct.release)(ctypes.addressof(struct))


def test_import_refuses_malformed_structs_and_keeps_them(lib):
    # A refused import leaves the array with its producer (release still set), as the reference's does
    # (CInterop.swift:119-131): the caller releases it. The checks run before any device work.
    import pyarrow as pa
    from arrowmetal_b200 import _ArrowArray as _Array, _ArrowSchema as _Schema
    lib.am_import.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    lib.am_last_error.restype = ctypes.c_char_p
    cases = [
        ("n_buffers", 1, "buffers"),
        ("length", -5, "negative length or offset"),
        ("offset", -1, "negative length or offset"),
        ("n_children", 1, "nested"),
    ]
    for field, value, message in cases:
        schema, array = _Schema(), _Array()
        pa.array([1, 2, None], type=pa.int64())._export_to_c(ctypes.addressof(array), ctypes.addressof(schema))
        saved = getattr(array, field)
        setattr(array, field, value)
        out = ctypes.c_void_p()
        rc = lib.am_import(ctypes.addressof(schema), ctypes.addressof(array), ctypes.byref(out))
        assert rc == 1 and message in lib.am_last_error().decode(), (field, rc, lib.am_last_error())
        assert array.release and not out.value
        setattr(array, field, saved)
        _release(array)
        _release(schema)
    # An unsupported type is refused by its format.
    schema, array = _Schema(), _Array()
    pa.array([[1], [2, 3]])._export_to_c(ctypes.addressof(array), ctypes.addressof(schema))
    out = ctypes.c_void_p()
    assert lib.am_import(ctypes.addressof(schema), ctypes.addressof(array), ctypes.byref(out)) != 0
    assert array.release
    _release(array)
    _release(schema)


def test_import_refuses_malformed_dictionary_structs(lib):
    # The dictionary of a dictionary array gets the same struct checks as the array itself, before
    # anything reads its buffers (its string offsets included).
    import pyarrow as pa
    from arrowmetal_b200 import _ArrowArray as _Array, _ArrowSchema as _Schema
    lib.am_import.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]
    lib.am_last_error.restype = ctypes.c_char_p
    cases = [("n_buffers", 1, "buffers"), ("n_buffers", 0, "buffers"), ("length", -3, "negative length or offset"),
             ("offset", -2, "negative length or offset"), ("n_children", 2, "nested")]
    for field, value, message in cases:
        schema, array = _Schema(), _Array()
        pa.array(["b", "a", None, "b"]).dictionary_encode()._export_to_c(ctypes.addressof(array),
                                                                        ctypes.addressof(schema))
        dictionary = ctypes.cast(array.dictionary, ctypes.POINTER(_Array)).contents
        saved = getattr(dictionary, field)
        setattr(dictionary, field, value)
        out = ctypes.c_void_p()
        rc = lib.am_import(ctypes.addressof(schema), ctypes.addressof(array), ctypes.byref(out))
        err = lib.am_last_error().decode()
        assert rc == 1 and message in err and "dictionary" in err, (field, rc, err)
        assert array.release and not out.value
        setattr(dictionary, field, saved)
        _release(array)
        _release(schema)
