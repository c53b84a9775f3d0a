"""ORDER BY with the payload columns carried through the sort in row records: a one-key sort of a
frame whose other columns are fixed-width, complete on the device, without nulls and at most twelve
bytes a row moves each row's record (its id and payload) through the passes and unpacks it where the
row reaches its final place, so no gather follows. The result must equal pyarrow's sort_indices + take
(or the oracle's order at the large sizes), on every path the device can pick: one pass, several
passes, the two-level sort's local sorts and its fallback passes; for 8- and 4-byte keys, floats in
totalOrder, both directions and null placements, every payload layout, sliced columns. Frames that do
not qualify take the gather and must give the same answer."""
import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

pytestmark = pytest.mark.gpu


def sort_plan(key, desc, nulls_first, float_order="ieee"):
    return {"op": "sort", "by": [[key, desc, {"nulls": "first" if nulls_first else "last", "float_order": float_order}]],
            "input": {"op": "scan", "source": "t"}}


def run(am, cols, key, desc=False, nulls_first=False, float_order="ieee"):
    src = am.PlanSource("t", cols)
    out = am.run_plan(sort_plan(key, desc, nulls_first, float_order), [src])
    return {k: v.to_arrow() for k, v in out.items()}, am.last_sort_stats()


def bits(arr):
    """Validity and value bits of a fixed-width array (floats compared by their bits)."""
    valid = np.asarray(arr.is_valid())
    if pa.types.is_boolean(arr.type):
        return valid, np.where(valid, arr.fill_null(False).to_numpy(zero_copy_only=False), False)
    width = arr.type.bit_width // 8
    view = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[width]
    vals = np.frombuffer(arr.buffers()[1], dtype=view)[arr.offset:arr.offset + len(arr)]
    return valid, np.where(valid, vals, 0)


def check(out, table, order):
    for name in table.column_names:
        want = table[name].combine_chunks().take(pa.array(order))
        gv, gb = bits(out[name])
        wv, wb = bits(want)
        assert np.array_equal(gv, wv) and np.array_equal(gb, wb), name


def payload(rng, n, layout):
    cols = {}
    for i, t in enumerate(layout):
        if t == "f64":
            cols[f"p{i}"] = pa.array(rng.standard_normal(n))
        elif t == "i32":
            cols[f"p{i}"] = pa.array(rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32, endpoint=True))
        elif t == "u16":
            cols[f"p{i}"] = pa.array(rng.integers(0, 2**16, n).astype(np.uint16))
        elif t == "i8":
            cols[f"p{i}"] = pa.array(rng.integers(-128, 128, n).astype(np.int8))
        elif t == "f32":
            cols[f"p{i}"] = pa.array(rng.standard_normal(n).astype(np.float32))
        elif t == "i64":
            cols[f"p{i}"] = pa.array(rng.integers(-2**62, 2**62, n, dtype=np.int64))
    return cols


LAYOUTS = [["f64", "i32"], ["i32", "f32", "i32"], ["u16", "i8", "f64"], ["i8"], ["f64"], ["f32", "u16", "u16", "i32"]]


@pytest.mark.parametrize("layout", LAYOUTS, ids=["-".join(x) for x in LAYOUTS])
@pytest.mark.parametrize("n", [1, 1000, 5377, 250_003])
def test_payload_layouts_match_pyarrow(am, layout, n):
    rng = np.random.default_rng(n + len(layout))
    cols = {"k": pa.array(rng.integers(0, 2**40, n), mask=rng.random(n) < 0.1), **payload(rng, n, layout)}
    table = pa.table(cols)
    for desc, nf in ((False, False), (True, True), (True, False)):
        out, st = run(am, cols, "k", desc, nf)
        assert st["payload_in_records"], (layout, n)
        order = pc.sort_indices(table, [("k", "descending" if desc else "ascending")],
                                null_placement="at_start" if nf else "at_end")
        check(out, table, order.to_numpy())


@pytest.mark.parametrize("kind", ["int32", "int64_one_digit", "uint64_full", "f64_total", "f32_total", "int16"])
def test_key_types_and_pass_counts(am, oracle, kind):
    rng = np.random.default_rng(7)
    n = 300_001
    mask = rng.random(n) < 0.07
    if kind == "int32":
        key = pa.array(rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32), mask=mask)
    elif kind == "int64_one_digit":
        key = pa.array(rng.integers(0, 200, n, dtype=np.int64), mask=mask)      # one active digit
    elif kind == "uint64_full":
        key = pa.array(rng.integers(0, 2**64 - 1, n, dtype=np.uint64, endpoint=True))
    elif kind == "int16":
        key = pa.array(rng.integers(-2**15, 2**15, n).astype(np.int16), mask=mask)
    else:
        v = rng.standard_normal(n)
        v[rng.random(n) < 0.02] = np.nan
        v[rng.random(n) < 0.02] = -0.0
        key = pa.array(v.astype(np.float32) if kind == "f32_total" else v, mask=mask)
    fo = "total" if kind.endswith("total") else "ieee"
    cols = {"k": key, **payload(rng, n, ["f64", "i32"])}
    table = pa.table(cols)
    for desc, nf in ((False, False), (True, True)):
        out, st = run(am, cols, "k", desc, nf, fo)
        assert st["payload_in_records"], kind
        order = oracle.np_argsort(key, desc, "at_start" if nf else "at_end", fo)
        check(out, table, order)


def test_sliced_payload_and_key(am):
    rng = np.random.default_rng(8)
    n = 100_000
    full = {"k": pa.array(rng.integers(0, 2**30, n), mask=rng.random(n) < 0.1), **payload(rng, n, ["f64", "i32"])}
    cols = {k: v.slice(13, 70_000) for k, v in full.items()}
    out, st = run(am, cols, "k")
    assert st["payload_in_records"]
    table = pa.table(cols)
    check(out, table, pc.sort_indices(table, [("k", "ascending")]).to_numpy())


@pytest.mark.parametrize("why", ["nullable", "too_wide", "bool"])
def test_frames_that_take_the_gather(am, why):
    rng = np.random.default_rng(9)
    n = 60_000
    cols = {"k": pa.array(rng.integers(0, 2**40, n), mask=rng.random(n) < 0.1)}
    if why == "nullable":
        cols["p"] = pa.array(rng.standard_normal(n), mask=rng.random(n) < 0.1)
    elif why == "too_wide":
        cols.update(payload(rng, n, ["f64", "i64"]))
    else:
        cols["p"] = pa.array(rng.random(n) < 0.5)
    table = pa.table(cols)
    out, st = run(am, cols, "k")
    assert not st["payload_in_records"]
    check(out, table, pc.sort_indices(table, [("k", "ascending")]).to_numpy())


N_LARGE = 36_000_000        # 5% nulls leave more than 2^25 value rows: the two-level sort


@pytest.mark.parametrize("case", ["local_sorts", "fallback_passes"])
def test_two_level_sort_with_records(am, oracle, case):
    rng = np.random.default_rng(10)
    key = rng.integers(0, 2**40, N_LARGE, dtype=np.int64)
    if case == "fallback_passes":
        key[rng.random(N_LARGE) < 0.3] = 987_654_321_098       # one bucket of ~11M rows
    k = pa.array(key, mask=rng.random(N_LARGE) < 0.05)
    cols = {"k": k, **payload(rng, N_LARGE, ["f64", "i32"])}
    for desc, nf in ((False, False), (True, True)):
        out, st = run(am, cols, "k", desc, nf)
        assert st["payload_in_records"] and st["passes_run"] == (2 if case == "local_sorts" else 2 + 5)
        order = oracle.argsort(k, desc, "at_start" if nf else "at_end", threads=8)
        for name in ("p0", "p1"):
            want = cols[name].to_numpy()[order]
            assert np.array_equal(out[name].to_numpy(), want), (case, desc, name)
        kv, kb = bits(out["k"])
        wv, wb = bits(k.take(pa.array(order)))
        assert np.array_equal(kv, wv) and np.array_equal(kb, wb)
