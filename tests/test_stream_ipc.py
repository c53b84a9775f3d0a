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


# ---- malformed files: every column must fit its buffers before anything reads it

# A malformed batch surfaces as the stream's error: an ArrowMetalError, or pyarrow's OSError when
# pyarrow reads the exported C stream.

def messages_of(path):
    """(metadata bytes, body bytes) of each message of an IPC stream file."""
    reader = pa.ipc.MessageReader.open_stream(pa.OSFile(str(path)))
    out = []
    for m in reader:
        out.append((bytearray(m.metadata.to_pybytes()), bytearray(m.body.to_pybytes() if m.body else b"")))
    return out


def write_messages(path, msgs):
    import struct
    with open(path, "wb") as f:
        for meta, body in msgs:
            f.write(b"\xff\xff\xff\xff" + struct.pack("<i", len(meta)) + bytes(meta) + bytes(body))
        f.write(b"\xff\xff\xff\xff\x00\x00\x00\x00")


def patch_int64(buf, old, new, count=None):
    import struct
    pat, rep = struct.pack("<q", old), struct.pack("<q", new)
    hits = [i for i in range(len(buf) - 7) if buf[i:i + 8] == pat]
    if count is not None:
        assert len(hits) == count, hits
    for i in hits:
        buf[i:i + 8] = rep
    return len(hits)


def test_ipc_rows_past_their_buffers(tmp_path):
    src = tmp_path / "ok.arrows"
    write_stream(src, pa.table({"x": np.arange(1000, dtype=np.int64) * 7}), 1000)
    msgs = messages_of(src)
    assert patch_int64(msgs[1][0], 1000, 10**9) >= 2          # the batch's length and its column's
    bad = tmp_path / "rows.arrows"
    write_messages(bad, msgs)
    with pytest.raises((am.ArrowMetalError, OSError), match="values buffer shorter"):
        am.scan_ipc(bad).to_reader().read_all()


@pytest.mark.parametrize("column,rows", [(np.arange(1000, dtype=np.int64), 2**61),
                                         (pa.array(["ab"] * 1000), 2**62)])
def test_ipc_row_counts_that_would_wrap_a_size(tmp_path, column, rows):
    # 2^61 rows of 8 bytes (or 2^62 + 1 offsets of 4 bytes) is 2^64 bytes and more: a size formed by
    # multiplying would wrap to a few bytes and pass; the reader must still refuse it.
    src = tmp_path / "ok.arrows"
    write_stream(src, pa.table({"x": column}), 1000)
    msgs = messages_of(src)
    assert patch_int64(msgs[1][0], 1000, rows) >= 2
    bad = tmp_path / "wrap.arrows"
    write_messages(bad, msgs)
    with pytest.raises((am.ArrowMetalError, OSError), match="shorter than its column"):
        am.scan_ipc(bad).to_reader().read_all()


def test_ipc_nulls_without_a_bitmap(tmp_path):
    src = tmp_path / "ok.arrows"
    write_stream(src, pa.table({"x": np.arange(1000, dtype=np.int64)}), 1000)
    msgs = messages_of(src)
    import struct
    meta = msgs[1][0]
    node = struct.pack("<qq", 1000, 0)
    at = bytes(meta).find(node)
    assert at >= 0
    meta[at + 8:at + 16] = struct.pack("<q", 5)
    bad = tmp_path / "nulls.arrows"
    write_messages(bad, msgs)
    with pytest.raises((am.ArrowMetalError, OSError), match="nulls and no validity bitmap"):
        am.scan_ipc(bad).to_reader().read_all()


@pytest.mark.parametrize("corrupt,message", [("past_end", "past the end"), ("decreasing", "negative or decreasing")])
def test_ipc_string_offsets_checked(tmp_path, corrupt, message):
    n = 100
    vals = ["v%03d" % i for i in range(n)]                     # 4 bytes each, no nulls
    src = tmp_path / "ok.arrows"
    write_stream(src, pa.table({"s": pa.array(vals)}), n)
    msgs = messages_of(src)
    body = msgs[1][1]
    offs = np.frombuffer(bytes(body[:4 * (n + 1)]), dtype=np.int32).copy()
    assert offs[0] == 0 and offs[-1] == 4 * n                  # the offsets lead the body (no bitmap)
    if corrupt == "past_end":
        offs[-1] = 4 * n + 10_000
    else:
        offs[50] = offs[49] - 1
    body[:4 * (n + 1)] = offs.tobytes()
    bad = tmp_path / "offsets.arrows"
    write_messages(bad, msgs)
    with pytest.raises((am.ArrowMetalError, OSError), match=message):
        am.scan_ipc(bad).to_reader().read_all()
    # The same file unpatched still reads back.
    write_messages(tmp_path / "again.arrows", messages_of(src))
    assert am.scan_ipc(tmp_path / "again.arrows").to_reader().read_all().equals(pa.table({"s": pa.array(vals)}))


def test_ipc_mutated_files_fail_cleanly(tmp_path):
    # Truncated files, flipped bytes and overwritten 8-byte words (lengths and offsets among them):
    # each read either succeeds or raises, and the process survives.
    import random
    rng = random.Random(11)
    t = table_of(300, seed=11)
    sources = []
    for writer, name in ((write_file, "f.arrow"), (write_stream, "s.arrows")):
        writer(tmp_path / name, t, 100)
        sources.append((tmp_path / name).read_bytes())
    bad = tmp_path / "bad.arrow"
    failed = 0
    for _ in range(400):
        b = bytearray(rng.choice(sources))
        kind = rng.randrange(3)
        if kind == 0:
            b = b[:rng.randrange(len(b) + 1)]
        elif kind == 1:
            for _ in range(rng.randrange(1, 8)):
                b[rng.randrange(len(b))] = rng.randrange(256)
        else:
            for _ in range(rng.randrange(1, 4)):
                i = rng.randrange(len(b) - 8) & ~7
                b[i:i + 8] = rng.choice([0, 1, -1, 2**31, 2**40, -2**40, 10**12]).to_bytes(8, "little", signed=True)
        bad.write_bytes(bytes(b))
        try:
            am.scan_ipc(bad, prefetch=0).to_reader().read_all()
        except Exception:
            failed += 1
    assert 0 < failed < 400
