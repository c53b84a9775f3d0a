"""am_argsort_device_noalloc, the argsort that allocates no device memory, against the ordinary
argsort (am_argsort_ex2) on the same columns, through the C ABI.

It is there for callers that cannot allocate on the device when they sort: a process whose device
memory belongs to its own pool allocator (a framework's caching allocator, an RMM pool), or a serving
loop that cannot afford cudaFree's wait for the whole device. Its scratch is one fixed block inside the
library that every call shares and that keeps what the last call left, so each check makes calls in a
row and compares every one of them. Row numbers are integers: the outputs must match exactly.

The file name makes pytest collect it last; it needs nothing that the other tests set up.
"""
import ctypes

import numpy as np
import pyarrow as pa
import pytest

from conftest import build_array

pytestmark = pytest.mark.gpu

MAX_ROWS = 1 << 18      # the entry point's stated limit
PLACEMENTS = ("at_end", "at_start")
FLOAT_ORDERS = ("ieee", "total", "nan_largest")


@pytest.fixture(scope="module")
def noalloc(am):
    import torch
    assert torch.cuda.is_available()
    f = am._lib.am_argsort_device_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                  ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]

    def run(arr, descending=False, null_placement="at_end", float_order="ieee"):
        """Copies the column's Arrow buffers to the device (the caller's memory, here torch's), sorts
        them with the entry point, returns the uint32 row numbers."""
        bufs = arr.buffers()
        dev = torch.device("cuda", am._lib.am_cuda_device())
        raw = bufs[1] if bufs[1] is not None else b""
        values = torch.from_numpy(np.frombuffer(raw, dtype=np.uint8).copy()).to(dev)
        validity = None
        if bufs[0] is not None and arr.null_count > 0:
            validity = torch.from_numpy(np.frombuffer(bufs[0], dtype=np.uint8).copy()).to(dev)
        out = torch.full((max(len(arr), 1),), -1, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev)
        rc = f(_format(arr.type).encode(), values.data_ptr(), validity.data_ptr() if validity is not None else None,
               arr.offset, len(arr), 1 if descending else 0, PLACEMENTS.index(null_placement),
               FLOAT_ORDERS.index(float_order), out.data_ptr(), stream.cuda_stream)
        if rc != 0:
            raise am.ArrowMetalError(am._lib.am_last_error().decode())
        return out[: len(arr)].cpu().numpy().view(np.uint32)

    run.entry = f
    return run


def _format(t):
    return {pa.bool_(): "b", pa.int8(): "c", pa.uint8(): "C", pa.int16(): "s", pa.uint16(): "S",
            pa.int32(): "i", pa.uint32(): "I", pa.int64(): "l", pa.uint64(): "L", pa.float16(): "e",
            pa.float32(): "f", pa.float64(): "g", pa.date32(): "tdD"}[t]


def existing(am, arr, descending=False, null_placement="at_end", float_order="ieee"):
    m = am.MetalArray.from_arrow(arr)
    return m.argsort(descending, null_placement, float_order).to_arrow().to_numpy(zero_copy_only=False)


def columns(seed):
    rng = np.random.default_rng(seed)

    def nulls(n, p):
        return rng.random(n) >= p

    n = 200_003
    i64 = build_array("int64", rng.integers(0, 1 << 40, n, dtype=np.int64) - (1 << 39), nulls(n, 0.1))
    f64v = rng.standard_normal(MAX_ROWS)
    f64v[rng.integers(0, MAX_ROWS, 2000)] = np.nan
    f64v[rng.integers(0, MAX_ROWS, 2000)] = -0.0
    f64v[rng.integers(0, MAX_ROWS, 2000)] = 0.0
    f64 = build_array("double", f64v, nulls(MAX_ROWS, 0.05))
    f32v = rng.standard_normal(70_001).astype(np.float32)
    f32v[::97] = np.float32("nan")
    f32v[1::89] = -np.float32("nan")
    f32 = build_array("float", f32v, nulls(70_001, 0.02))
    i32 = build_array("int32", rng.integers(-50, 50, 123_457).astype(np.int32))
    u8 = build_array("uint8", rng.integers(0, 256, 9_999).astype(np.uint8), nulls(9_999, 0.3))
    f16 = build_array("halffloat", rng.standard_normal(4097).astype(np.float16), nulls(4097, 0.1))
    b = pa.array(rng.random(33_333) < 0.5)
    return [
        ("int64 with nulls", i64, dict()),
        ("int64 sliced, descending", i64.slice(13, 150_000), dict(descending=True, null_placement="at_start")),
        ("float64 at the limit", f64, dict(null_placement="at_start")),
        ("float64 totalOrder descending", f64, dict(descending=True, float_order="total")),
        ("float32 nan_largest", f32, dict(float_order="nan_largest")),
        ("float32 ieee sliced", f32.slice(5, 60_000), dict(descending=True)),
        ("int32 no nulls", i32, dict()),
        ("uint8", u8, dict(descending=True)),
        ("float16", f16, dict(float_order="total")),
        ("bool", b, dict()),
        ("bool sliced", b.slice(3, 30_000), dict(descending=True)),
    ]


def test_matches_existing_argsort_call_after_call(am, noalloc):
    cases = columns(7)
    for name, arr, opts in cases:
        want = existing(am, arr, **opts)
        first = noalloc(arr, **opts)
        second = noalloc(arr, **opts)
        assert np.array_equal(first, want), name
        assert np.array_equal(second, want), name


def test_two_calls_in_a_row_on_different_columns(am, noalloc):
    # A long column, then a short one: the second call must not see the first call's rows.
    rng = np.random.default_rng(11)
    long_col = build_array("int64", rng.integers(0, 1 << 62, MAX_ROWS, dtype=np.int64), rng.random(MAX_ROWS) > 0.2)
    short_col = build_array("int64", rng.integers(0, 1000, 5000, dtype=np.int64), rng.random(5000) > 0.2)
    for arr in (long_col, short_col, long_col):
        assert np.array_equal(noalloc(arr), existing(am, arr))


def test_rejects_more_rows_than_the_limit(am, noalloc):
    arr = pa.array(np.zeros(MAX_ROWS + 1, dtype=np.int32))
    with pytest.raises(am.ArrowMetalError, match=str(MAX_ROWS)):
        noalloc(arr)
    # The refusal leaves the entry point usable.
    ok = pa.array(np.arange(100, 0, -1, dtype=np.int32))
    assert noalloc(ok).tolist() == list(range(99, -1, -1))


def test_empty_column(am, noalloc):
    assert len(noalloc(pa.array([], type=pa.int64()))) == 0


def test_calls_after_the_first_leave_device_memory_untouched(am, noalloc):
    # After a first call (which sets the entry point up on this device), further calls change neither
    # the library's memory pool (the device's default pool: in use and reserved) nor the device's free
    # memory. The column and the output are allocated once, before the figures are taken.
    import torch
    from cuda.bindings import runtime as cudart
    ordinal = am._lib.am_cuda_device()
    dev = torch.device("cuda", ordinal)
    rng = np.random.default_rng(5)
    n = 100_000
    values = torch.from_numpy(rng.integers(0, 1 << 40, n, dtype=np.int64)).to(dev)
    out = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream

    def call():
        assert noalloc.entry(b"l", values.data_ptr(), None, 0, n, 0, 0, 0, out.data_ptr(), stream) == 0
        torch.cuda.synchronize(dev)

    def figures():
        err, pool = cudart.cudaDeviceGetDefaultMemPool(ordinal)
        assert err == cudart.cudaError_t.cudaSuccess
        used = cudart.cudaMemPoolGetAttribute(pool, cudart.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
        reserved = cudart.cudaMemPoolGetAttribute(pool, cudart.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent)
        assert used[0] == reserved[0] == cudart.cudaError_t.cudaSuccess
        return int(used[1]), int(reserved[1]), torch.cuda.mem_get_info(dev)[0]

    call()
    before = figures()
    for _ in range(5):
        call()
    assert figures() == before
    want = np.argsort(values.cpu().numpy(), kind="stable").astype(np.uint32)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), want)
