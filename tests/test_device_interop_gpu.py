"""CUDA zero-copy interop: am_export_device hands out an ArrowDeviceArray (ARROW_DEVICE_CUDA) whose
buffers are the array's own HBM, and am_import_device takes one without a copy (the reference's
interface, include/arrowmetal.h:49-50, Sources/ArrowMetal/CInterop.swift:406-425, with CUDA in place of
Metal). Round trips through both, read back on the host and sorted, against pyarrow."""
import ctypes

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

pytestmark = pytest.mark.gpu

ARROW_DEVICE_CUDA = 2


def device_bytes(ptr, size):
    from cuda.bindings import runtime as cudart
    out = np.empty(size, dtype=np.uint8)
    if size:
        err, = cudart.cudaMemcpy(out.ctypes.data, ptr, size, cudart.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert err == cudart.cudaError_t.cudaSuccess
    return out


def export_device(am, arr):
    schema, darr = am._ArrowSchema(), am._ArrowDeviceArray()
    am._ok(am._lib.am_export_device(arr._h, ctypes.addressof(schema), ctypes.addressof(darr)))
    return schema, darr


def release(struct):
    if struct.release:
        ctypes.CFUNCTYPE(None, ctypes.c_void_p)(struct.release)(ctypes.addressof(struct))


def test_export_device_points_at_the_arrays_hbm(am):
    rng = np.random.default_rng(3)
    n = 1_000_003
    src = pa.array(rng.integers(-2**40, 2**40, n), mask=rng.random(n) < 0.1)
    m = am.MetalArray.from_arrow(src)
    idx = m.argsort()
    schema, darr = export_device(am, idx)
    try:
        assert darr.device_type == ARROW_DEVICE_CUDA and darr.device_id == am._lib.am_cuda_device()
        assert schema.format == b"I" and darr.array.length == n and darr.array.null_count == 0
        bufs = ctypes.cast(darr.array.buffers, ctypes.POINTER(ctypes.c_void_p * 2)).contents
        got = device_bytes(bufs[1], 4 * n).view(np.uint32)
        want = pc.array_sort_indices(src).to_numpy().astype(np.uint32)
        assert np.array_equal(got, want)
        # The key column, with its bitmap, exported the same way.
        ks, kd = export_device(am, m)
        try:
            kb = ctypes.cast(kd.array.buffers, ctypes.POINTER(ctypes.c_void_p * 2)).contents
            assert kd.array.null_count == src.null_count and kb[0]
            vals = device_bytes(kb[1], 8 * n).view(np.int64)
            bits = np.unpackbits(device_bytes(kb[0], (n + 7) // 8), bitorder="little")[:n].astype(bool)
            assert np.array_equal(bits, np.asarray(src.is_valid()))
            assert np.array_equal(vals[bits], src.to_numpy(zero_copy_only=False)[bits].astype(np.int64))
        finally:
            release(kd.array)
            release(ks)
    finally:
        release(darr.array)
        release(schema)
    # The handle outlives its export and stays usable.
    assert np.array_equal(idx.to_arrow().to_numpy(), want)


def test_import_device_round_trip_without_a_copy(am):
    rng = np.random.default_rng(4)
    n = 500_001
    src = pa.array(rng.standard_normal(n), mask=rng.random(n) < 0.05).slice(7, n - 20)
    m = am.MetalArray.from_arrow(src)
    schema, darr = export_device(am, m)
    bufs = ctypes.cast(darr.array.buffers, ctypes.POINTER(ctypes.c_void_p * 2)).contents
    values_ptr = bufs[1]
    out = ctypes.c_void_p()
    am._ok(am._lib.am_import_device(ctypes.addressof(schema), ctypes.addressof(darr), ctypes.byref(out)))
    assert not darr.array.release                      # moved into the library
    back = am.MetalArray(out)
    release(schema)
    assert back.to_arrow().equals(src)
    for d, p in ((False, "at_end"), (True, "at_start")):
        want = pc.array_sort_indices(src, order="descending" if d else "ascending", null_placement=p).to_numpy()
        assert np.array_equal(back.argsort(d, p).to_arrow().to_numpy(), want)
    # Zero copy: the re-imported array reads the exporter's buffer.
    s2, d2 = export_device(am, back)
    try:
        b2 = ctypes.cast(d2.array.buffers, ctypes.POINTER(ctypes.c_void_p * 2)).contents
        assert b2[1] == values_ptr
    finally:
        release(d2.array)
        release(s2)
    del m
    assert back.to_arrow().equals(src)                  # the exporter's memory lives on with the import


def test_import_device_from_framework_tensors(am):
    import torch
    dev = torch.device("cuda", am._lib.am_cuda_device())
    rng = np.random.default_rng(5)
    n = 300_000
    vals = rng.integers(0, 1000, n).astype(np.int32)
    valid = rng.random(n) >= 0.2
    tv = torch.from_numpy(vals).to(dev)
    tb = torch.from_numpy(np.packbits(valid, bitorder="little")).to(dev)
    arr = am.MetalArray.from_device(tv.data_ptr(), n, "i", tb.data_ptr(), int((~valid).sum()), keep=(tv, tb))
    want_arr = pa.array(vals, mask=~valid)
    assert arr.to_arrow().equals(want_arr)
    want = pc.array_sort_indices(want_arr, order="descending", null_placement="at_start").to_numpy()
    assert np.array_equal(arr.argsort(True, "at_start").to_arrow().to_numpy(), want)
