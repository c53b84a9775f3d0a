"""Arrow IPC input of the streaming sort, on the host (no device needed): am_stream_open_ipc reads
pyarrow-written IPC files (file and stream formats, a directory of them, slices, nulls, strings,
temporal types) and am_stream_export_c hands the batches, projected, back to pyarrow unchanged.
The reference reads the same inputs with am_stream_open_ipc (python/tests/test_stream.py)."""
import numpy as np
import pyarrow as pa
import pytest

import arrowmetal_b200 as am


def table_of(n, seed=0):
    rng = np.random.default_rng(seed)
    return pa.table({
        "i8": pa.array(rng.integers(-100, 100, n).astype(np.int8), mask=rng.random(n) < 0.1),
        "u32": pa.array(rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)),
        "f64": pa.array(rng.standard_normal(n), mask=rng.random(n) < 0.05),
        "f16": pa.array(rng.standard_normal(n).astype(np.float16)),
        "b": pa.array(rng.random(n) < 0.3, mask=rng.random(n) < 0.05),
        "s": pa.array([None if i % 17 == 0 else "x" * (i % 7) for i in range(n)]),
        "lb": pa.array([bytes([i % 251]) * (i % 5) for i in range(n)], type=pa.large_binary()),
        "ts": pa.array(rng.integers(0, 10**15, n), type=pa.timestamp("ns", tz="Europe/Paris")),
        "d": pa.array(rng.integers(0, 20000, n).astype(np.int32), type=pa.date32()),
        "t": pa.array(rng.integers(0, 86400, n).astype(np.int32), type=pa.time32("s")),
        "dur": pa.array(rng.integers(0, 10**9, n), type=pa.duration("ms")),
    })


def write_file(path, t, batch_rows):
    with pa.ipc.new_file(str(path), t.schema) as w:
        for b in t.to_batches(max_chunksize=batch_rows):
            w.write_batch(b)


def write_stream(path, t, batch_rows):
    with pa.ipc.new_stream(str(path), t.schema) as w:
        for b in t.to_batches(max_chunksize=batch_rows):
            w.write_batch(b)


@pytest.mark.parametrize("writer", [write_file, write_stream])
def test_ipc_round_trip(tmp_path, writer):
    t = table_of(10_000)
    path = tmp_path / "data.arrow"
    writer(path, t, 3_000)
    got = am.scan_ipc(path).to_reader().read_all()
    assert got.equals(t)


def test_directory_in_name_order_and_projection(tmp_path):
    parts = [table_of(2_000, seed=i) for i in range(3)]
    for i, p in enumerate(parts):
        write_file(tmp_path / f"part-{i}.arrow", p, 700)
    (tmp_path / "notes.txt").write_text("not arrow")
    got = am.scan_ipc(tmp_path, prefetch=0).select(["s", "f64"]).to_reader().read_all()
    want = pa.concat_tables(parts).select(["s", "f64"])
    assert got.equals(want)


def test_sliced_batches_and_projection_of_a_c_stream():
    t = table_of(5_000)
    batches = [b.slice(13, 900) for b in t.to_batches(max_chunksize=1_000)]
    src = pa.RecordBatchReader.from_batches(t.schema, batches)
    got = am.scan_arrow(src).select(["lb", "i8"]).to_reader().read_all()
    assert got.equals(pa.Table.from_batches(batches).select(["lb", "i8"]))


def test_ipc_errors(tmp_path):
    with pytest.raises(am.ArrowMetalError, match="cannot open"):
        am.scan_ipc(tmp_path / "missing.arrow")
    with pytest.raises(am.ArrowMetalError, match="no Arrow IPC files"):
        am.scan_ipc(tmp_path)
    t = pa.table({"d": pa.array(["a", "b", "a"]).dictionary_encode()})
    write_file(tmp_path / "dict.arrow", t, 10)
    with pytest.raises(am.ArrowMetalError, match="dictionary"):
        am.scan_ipc(tmp_path / "dict.arrow")
    c = tmp_path / "z.arrow"
    with pa.ipc.new_file(str(c), pa.schema([("x", pa.int64())]),
                         options=pa.ipc.IpcWriteOptions(compression="zstd")) as w:
        w.write_table(pa.table({"x": np.arange(1000)}))
    with pytest.raises(Exception, match="compressed"):
        am.scan_ipc(c).to_reader().read_all()
