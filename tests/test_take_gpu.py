"""Take on the GPU: the golden fixtures (pyarrow's take), every index type, null indices, boolean and
narrow columns, slices, the multi-column form, and the out-of-range error."""
import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_golden_take(am):
    g = golden()
    n = 0
    for c in g.cases:
        if c["kind"] != "take":
            continue
        src = am.MetalArray.from_arrow(g.array(c["array"], c["type"]))
        idx = am.MetalArray.from_arrow(g.array(c["index"], c["index_type"]))
        got = src.take(idx).to_arrow()
        valid = np.asarray(got.is_valid().to_numpy(zero_copy_only=False))
        assert np.array_equal(valid, g[c["index"] + "_expect_valid"]), c
        vals = got.fill_null(0).to_numpy(zero_copy_only=False)
        want = g[c["index"] + "_expect_values"]
        assert np.array_equal(vals.view(want.dtype)[valid], want[valid]), c
        assert got.null_count == int((~valid).sum())
        n += 1
    assert n > 30


@pytest.mark.parametrize("t", [pa.int8(), pa.uint16(), pa.int32(), pa.float32(), pa.int64(), pa.float64(),
                               pa.bool_(), pa.timestamp("us"), pa.date32()])
def test_take_types_match_pyarrow(am, t):
    rng = np.random.default_rng(1)
    n = 100_003
    if t == pa.bool_():
        src = pa.array(rng.random(n) < 0.5, mask=rng.random(n) < 0.1)
    elif pa.types.is_floating(t):
        src = pa.array(rng.normal(size=n), mask=rng.random(n) < 0.1).cast(t)
    elif pa.types.is_temporal(t):
        storage = pa.int32() if t.bit_width == 32 else pa.int64()
        src = pa.array(rng.integers(0, 10**6, n), mask=rng.random(n) < 0.1).cast(storage).view(t)
    else:
        info = np.iinfo(t.to_pandas_dtype())
        src = pa.array(rng.integers(info.min, info.max, n, dtype=t.to_pandas_dtype()), mask=rng.random(n) < 0.1)
    m = am.MetalArray.from_arrow(src)
    for it in (pa.uint32(), pa.int32(), pa.int64()):
        for k in (0, 1, 127, 128, 129, 100_003):
            idx = pa.array(rng.integers(0, n, k), mask=rng.random(k) < 0.05).cast(it)
            got = m.take(idx).to_arrow()
            want = pc.take(src, idx)
            assert got.type == src.type
            assert got.equals(want), (t, it, k)


def test_take_through_argsort_is_sorted_copy(am):
    rng = np.random.default_rng(2)
    src = pa.array(rng.integers(-10**9, 10**9, 500_000), mask=rng.random(500_000) < 0.1)
    m = am.MetalArray.from_arrow(src)
    got = m.take(m.argsort()).to_arrow()
    assert got.equals(pc.take(src, pc.array_sort_indices(src)))


def test_take_columns_one_index_read(am):
    rng = np.random.default_rng(3)
    n = 300_001
    cols = [pa.array(rng.integers(0, 2**40, n), mask=rng.random(n) < 0.1), pa.array(rng.normal(size=n)),
            pa.array(rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32)), pa.array(rng.random(n) < 0.5)]
    idx = pa.array(rng.permutation(n).astype(np.uint32))
    outs = am.take_columns([am.MetalArray.from_arrow(c) for c in cols], idx)
    for c, o in zip(cols, outs):
        assert o.to_arrow().equals(pc.take(c, idx))


def test_take_from_slices(am):
    rng = np.random.default_rng(4)
    src = pa.array(rng.integers(0, 100, 10_000), mask=rng.random(10_000) < 0.3)
    m = am.MetalArray.from_arrow(src).slice(13, 5000)
    idx = pa.array(rng.integers(0, 5000, 777), type=pa.int64())
    assert m.take(idx).to_arrow().equals(pc.take(src.slice(13, 5000), idx))
    bsrc = pa.array(rng.random(10_000) < 0.5)
    bm = am.MetalArray.from_arrow(bsrc).slice(3, 9000)
    assert bm.take(idx).to_arrow().equals(pc.take(bsrc.slice(3, 9000), idx))


def test_take_out_of_range_raises(am):
    # IndexTypeTests.swift:109 and Take.swift:70-72: the error surfaces from the call.
    m = am.MetalArray.from_arrow(pa.array([1, 2, 3]))
    with pytest.raises(am.ArrowMetalError, match="out of range"):
        m.take(pa.array([0, 3], type=pa.int64()))
    with pytest.raises(am.ArrowMetalError, match="out of range"):
        m.take(pa.array([-1], type=pa.int32()))
    # The library stays usable afterwards.
    assert m.take(pa.array([2, 0], type=pa.uint32())).to_arrow().to_pylist() == [3, 1]


def test_take_error_deferred_to_batch_end(am):
    # BatchTests.swift:61: inside a batch the range error surfaces at the batch's end.
    m = am.MetalArray.from_arrow(pa.array([1, 2, 3]))
    with pytest.raises(am.ArrowMetalError, match="out of range"):
        with am.batch():
            m.take(pa.array([5], type=pa.int64()))
    assert m.take(pa.array([1], type=pa.int64())).to_arrow().to_pylist() == [2]


@pytest.mark.parametrize("idx_type", [pa.uint32(), pa.int64()])
def test_take_large(am, idx_type):
    # 6M output rows over 5M-row sources of every width, boolean and nullable ones included.
    rng = np.random.default_rng(12)
    n_src, n = 5_000_000, 6_000_000
    cols = [pa.array(rng.integers(-2**62, 2**62, n_src), mask=rng.random(n_src) < 0.1),
            pa.array(rng.standard_normal(n_src)),
            pa.array(rng.integers(-2**31, 2**31 - 1, n_src, dtype=np.int32)),
            pa.array(rng.random(n_src) < 0.5),
            pa.array(rng.integers(0, 255, n_src, dtype=np.uint8), mask=rng.random(n_src) < 0.3)]
    idx = pa.array(rng.integers(0, n_src, n), mask=rng.random(n) < 0.02).cast(idx_type)
    outs = am.take_columns([am.MetalArray.from_arrow(c) for c in cols], idx)
    for c, o in zip(cols, outs):
        got = o.to_arrow()
        want = pc.take(c, idx)
        assert got.null_count == want.null_count
        assert got.equals(want)


def test_take_through_sort_large(am):
    # The sorted-table gather of the ORDER BY workload shape, checked against numpy indexing.
    rng = np.random.default_rng(13)
    n = 8_000_000
    key = pa.array(rng.integers(0, 2**40, n), mask=rng.random(n) < 0.1)
    p1 = pa.array(rng.standard_normal(n))
    k, p = am.MetalArray.from_arrow(key), am.MetalArray.from_arrow(p1)
    idx = k.argsort()
    ko, po = am.take_columns([k, p], idx)
    ii = idx.to_arrow().to_numpy()
    assert np.array_equal(po.to_arrow().to_numpy(), p1.to_numpy()[ii])
    kv = ko.to_arrow()
    assert kv.equals(pc.take(key, pa.array(ii)))


def test_take_large_out_of_range(am):
    rng = np.random.default_rng(14)
    src = am.MetalArray.from_arrow(pa.array(rng.integers(0, 100, 5_000_000)))
    idx = rng.integers(0, 5_000_000, 5_000_000)
    idx[4_999_999] = 5_000_000
    with pytest.raises(am.ArrowMetalError, match="out of range"):
        am.take_columns([src, src], pa.array(idx))


def test_take_columns_through_row_records(am):
    # Several large columns through a permutation this library produced: the gather packs them into
    # 32-byte row records (7 columns of 27 bytes + a validity byte) and reads one record per row.
    rng = np.random.default_rng(15)
    n = 10_000_000
    cols = [pa.array(rng.integers(-2**62, 2**62, n), mask=rng.random(n) < 0.1),
            pa.array(rng.standard_normal(n)),
            pa.array(rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32)),
            pa.array(rng.standard_normal(n).astype(np.float32), mask=rng.random(n) < 0.5),
            pa.array(rng.integers(0, 2**16, n).astype(np.uint16)),
            pa.array(rng.integers(0, 255, n, dtype=np.uint8), mask=rng.random(n) < 0.3),
            pa.array(rng.random(n) < 0.5, mask=rng.random(n) < 0.05)]
    handles = [am.MetalArray.from_arrow(c) for c in cols]
    idx = am.MetalArray.from_arrow(pa.array(rng.integers(0, 2**40, n))).argsort()
    ii = pa.array(idx.to_arrow().to_numpy())
    for c, o in zip(cols, am.take_columns(handles, idx)):
        got = o.to_arrow()
        want = pc.take(c, ii)
        assert got.null_count == want.null_count
        assert got.equals(want)


def test_take_two_columns_through_16_byte_records(am):
    # The ORDER BY payload shape (float64 + int32, no nulls): 16-byte records, bit-exact values.
    rng = np.random.default_rng(16)
    n = 25_000_000
    p1 = rng.standard_normal(n)
    p2 = rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32)
    handles = [am.MetalArray.from_arrow(pa.array(p1)), am.MetalArray.from_arrow(pa.array(p2))]
    idx = am.MetalArray.from_arrow(pa.array(rng.integers(0, 2**40, n))).argsort()
    ii = idx.to_arrow().to_numpy()
    o1, o2 = am.take_columns(handles, idx)
    assert np.array_equal(o1.to_arrow().to_numpy().view(np.uint64), p1.view(np.uint64)[ii])
    assert np.array_equal(o2.to_arrow().to_numpy(), p2[ii])


def test_take_columns_through_8_byte_records(am):
    # int32 (nulls) + uint16 + boolean (nulls): 7 bytes and a validity byte, 8-byte row records. The
    # row count is not a multiple of the pack's row groups, so the last group is partial.
    rng = np.random.default_rng(17)
    n = 40_000_003
    cols = [pa.array(rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32), mask=rng.random(n) < 0.2),
            pa.array(rng.integers(0, 2**16, n).astype(np.uint16)),
            pa.array(rng.random(n) < 0.5, mask=rng.random(n) < 0.05)]
    handles = [am.MetalArray.from_arrow(c) for c in cols]
    idx = am.MetalArray.from_arrow(pa.array(rng.integers(0, 2**40, n))).argsort()
    ii = pa.array(idx.to_arrow().to_numpy())
    am.profile(True)
    am.profile_reset()
    try:
        outs = am.take_columns(handles, idx)
        assert am.profile_entries()["take_pack_records"][0] == 1      # the row-record form ran
    finally:
        am.profile(False)
    for c, o in zip(cols, outs):
        got = o.to_arrow()
        want = pc.take(c, ii)
        assert got.null_count == want.null_count
        assert got.equals(want)
