"""The out-of-core sort of a record-batch stream (am_stream_from_c_stream + am_stream_sort_ex) through
the C ABI: one run held in HBM, many runs spilled and merged on the GPU (a small run budget forces it),
LIMIT, the Arrow IPC stream output, and the edge cases. Every answer must equal pyarrow's stable
multi-key sort of the whole table (the reference's own test compares with pyarrow:
python/tests/test_stream.py:148-168)."""
import os

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

pytestmark = pytest.mark.gpu


def table_of(rng, n):
    words = ["", "a", "ab", "b", "ba", "zz", "héllo", "日本"]
    return pa.table({
        "k1": pa.array(rng.integers(0, 7, n), mask=rng.random(n) < 0.1),
        "k2": pa.array(np.where(rng.random(n) < 0.05, np.nan, np.round(rng.standard_normal(n), 1)),
                       mask=rng.random(n) < 0.05),
        "name": pa.array([words[int(i)] if rng.random() > 0.05 else None for i in rng.integers(0, len(words), n)]),
        "id": pa.array(np.arange(n, dtype=np.int64)),
        "flag": pa.array(rng.random(n) < 0.5),
    })


def reader(t, batch_rows):
    return pa.Table.from_batches(t.to_batches(max_chunksize=batch_rows)).to_reader()


def expected(t, keys, null_placement="at_end", limit=0):
    idx = pc.sort_indices(t, keys, null_placement=null_placement)
    out = t.take(idx)
    return out.slice(0, limit) if limit else out


@pytest.fixture
def small_runs():
    os.environ["ARROWMETAL_STREAM_RUN_BYTES"] = str(1 << 20)      # ~1 MiB of batches per run
    yield
    del os.environ["ARROWMETAL_STREAM_RUN_BYTES"]


def same(a, b):
    assert a.column_names == b.column_names
    for c in a.column_names:
        x, y = a[c].combine_chunks(), b[c].combine_chunks()
        if pa.types.is_floating(x.type):
            vx = x.is_valid().to_numpy(zero_copy_only=False)
            vy = y.is_valid().to_numpy(zero_copy_only=False)
            assert np.array_equal(vx, vy), c
            xv, yv = x.to_numpy(zero_copy_only=False)[vx], y.to_numpy(zero_copy_only=False)[vy]
            assert np.array_equal(xv.view(np.uint8), yv.view(np.uint8)), c
        else:
            assert x.equals(y), c


KEYS = [
    [("k1", "ascending")],
    [("k1", "descending"), ("name", "ascending")],
    [("name", "descending"), ("k2", "ascending"), ("k1", "descending")],
]


@pytest.mark.parametrize("keys", KEYS)
@pytest.mark.parametrize("placement", ["at_end", "at_start"])
def test_one_run_in_hbm(am, keys, placement):
    rng = np.random.default_rng(1)
    t = table_of(rng, 200_000)
    got = am.scan_arrow(reader(t, 30_000)).sort([(k, o == "descending") for k, o in keys], null_placement=placement)
    same(got, expected(t, keys, placement))


@pytest.mark.parametrize("keys", KEYS)
@pytest.mark.parametrize("placement", ["at_end", "at_start"])
def test_spilled_runs_merged_on_the_gpu(am, small_runs, keys, placement, tmp_path):
    rng = np.random.default_rng(2)
    t = table_of(rng, 300_000)
    s = am.scan_arrow(reader(t, 20_000), prefetch=2)
    got = s.sort([(k, o == "descending") for k, o in keys], scratch=tmp_path, null_placement=placement)
    same(got, expected(t, keys, placement))
    assert s.stats["batches"] == 15 and s.stats["rows"] == 300_000 and s.rows_out == 300_000
    assert s.stats["merge_s"] > 0
    assert not list(tmp_path.iterdir()), "the spilled runs are removed"


def test_limit_and_selected_columns(am, small_runs):
    rng = np.random.default_rng(3)
    t = table_of(rng, 250_000)
    keys = [("k2", "descending"), ("id", "ascending")]
    got = am.scan_arrow(reader(t, 10_000)).select(["id", "name"]).sort([("k2", True), ("id", False)], limit=1234)
    want = expected(t, keys, limit=1234).select(["id", "name"])
    same(got, want)
    one = am.scan_arrow(reader(t, 10_000), prefetch=0).sort("k1", limit=7)
    same(one, expected(t, [("k1", "ascending")], limit=7))


def test_float_orders(am, small_runs, oracle):
    rng = np.random.default_rng(4)
    n = 120_000
    v = rng.standard_normal(n)
    v[rng.random(n) < 0.1] = np.nan
    v[rng.random(n) < 0.1] = -0.0
    t = pa.table({"x": pa.array(v), "id": pa.array(np.arange(n))})
    for fo in ("total", "nan_largest"):
        got = am.scan_arrow(reader(t, 8_000)).sort(("x", True), float_order=fo)
        order = oracle.np_argsort(t["x"].combine_chunks(), True, "at_end", fo)
        assert np.array_equal(got["id"].to_numpy(), order), fo


@pytest.mark.parametrize("spill", [False, True])
def test_ipc_stream_output(am, tmp_path, spill):
    rng = np.random.default_rng(5)
    t = table_of(rng, 100_000)
    t = t.append_column("ts", pa.array(rng.integers(0, 10**12, len(t)), type=pa.timestamp("us", tz="UTC")))
    t = t.append_column("f32", pa.array(rng.standard_normal(len(t)).astype(np.float32)))
    if spill:
        os.environ["ARROWMETAL_STREAM_RUN_BYTES"] = str(1 << 20)
    try:
        path = tmp_path / "sorted.arrows"
        stats = am.scan_arrow(reader(t, 9_000)).sort_to_ipc([("name", False), ("k1", True)], path)
    finally:
        os.environ.pop("ARROWMETAL_STREAM_RUN_BYTES", None)
    got = pa.ipc.open_stream(str(path)).read_all()
    assert got.schema.names == t.schema.names and got.schema.types == t.schema.types
    same(got, expected(t, [("name", "ascending"), ("k1", "descending")]))
    assert stats["rows_out"] == len(t)


def test_empty_and_one_row_streams(am):
    schema = pa.schema([("a", pa.int64()), ("s", pa.utf8())])
    empty = am.scan_arrow(pa.RecordBatchReader.from_batches(schema, [])).sort("a")
    assert empty.num_rows == 0 and empty.schema.types == schema.types
    one = am.scan_arrow(pa.table({"a": [5], "s": ["x"]})).sort("a")
    assert one.to_pydict() == {"a": [5], "s": ["x"]}


def test_errors(am):
    t = pa.table({"a": [1, 2], "b": [3, 4]})
    s = am.scan_arrow(t)
    with pytest.raises(am.ArrowMetalError, match="no column named"):
        s.sort("zz")
    with pytest.raises(am.ArrowMetalError, match="consumed"):
        s.sort("a")


def test_sort_ipc_files_and_read_our_own_output(am, small_runs, tmp_path):
    rng = np.random.default_rng(6)
    t = table_of(rng, 150_000)
    data = tmp_path / "in"
    data.mkdir()
    for i, b in enumerate(t.to_batches(max_chunksize=40_000)):
        with pa.ipc.new_file(str(data / f"part-{i:03d}.arrow"), t.schema) as w:
            w.write_batch(b)
    keys = [("k2", "descending"), ("name", "ascending")]
    got = am.scan_ipc(data).sort([("k2", True), ("name", False)])
    same(got, expected(t, keys))
    out = tmp_path / "sorted.arrows"
    am.scan_ipc(data).sort_to_ipc([("k2", True), ("name", False)], out)
    same(am.scan_ipc(out).to_reader().read_all(), expected(t, keys))
