"""The plan entry points with the plans the sort's callers send (the DataFusion rule's
select_all(sort(scan)) with limit, the Polars engine's per-key options), against pyarrow."""
import json

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

pytestmark = pytest.mark.gpu


def _table(rng, n):
    return pa.table({"c0": pa.array(rng.integers(0, 2**40, n), mask=rng.random(n) < 0.1),
                     "c1": pa.array(rng.normal(size=n)),
                     "c2": pa.array(rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32))})


def datafusion_plan(keys, fetch=None):
    # datafusion/src/gpu.rs:45-66 and :232-238, verbatim shape.
    by = ",".join(f'["c{c}",{"true" if d else "false"},{{"nulls":"{"first" if nf else "last"}","float_order":"total"}}]'
                  for c, d, nf in keys)
    node = f'{{"op":"sort","by":[{by}],"input":{{"op":"scan","source":"t"}}}}'
    if fetch is not None:
        node = f'{{"op":"limit","count":{fetch},"input":{node}}}'
    exprs = ",".join(f'["c{i}","(col \\"c{i}\\")"]' for i in range(3))
    return f'{{"op":"select","exprs":[{exprs}],"input":{node}}}'


@pytest.mark.parametrize("keys,fetch", [([(0, False, False)], None), ([(0, True, True)], None),
                                        ([(2, False, False), (1, True, False)], None),
                                        ([(0, False, False)], 1000)])
def test_datafusion_shaped_plans(am, keys, fetch):
    rng = np.random.default_rng(len(keys) + (fetch or 0))
    t = _table(rng, 200_001)
    src = am.PlanSource("t", {k: t[k].combine_chunks() for k in t.column_names})
    out = am.run_plan(datafusion_plan(keys, fetch), [src])
    assert list(out) == ["c0", "c1", "c2"]
    place = "at_start" if keys[0][2] else "at_end"
    idx = pc.sort_indices(t, [(f"c{c}", "descending" if d else "ascending") for c, d, _ in keys], null_placement=place)
    if fetch is not None:
        idx = idx[:fetch]
    want = t.take(idx)
    for k in out:
        assert out[k].to_arrow().equals(want[k].combine_chunks()), k


def test_polars_shaped_plan(am, oracle):
    # python/arrowmetal/polars_engine.py:944-998: nulls first unless nulls_last, nan_largest floats.
    rng = np.random.default_rng(5)
    n = 50_000
    v = rng.normal(size=n)
    v[rng.random(n) < 0.05] = np.nan
    a = pa.array(v, mask=rng.random(n) < 0.1)
    b = pa.array(rng.integers(0, 5, n))
    src = am.PlanSource("df", {"a": a, "b": b})
    plan = {"op": "limit", "count": 100, "offset": 10,
            "input": {"op": "sort", "input": {"op": "scan", "source": "df"},
                      "by": [["b", True], ["a", False, {"nulls": "first", "float_order": "nan_largest"}]]}}
    out = am.run_plan(json.dumps(plan), [src])
    idx = oracle.lexsort([b, a], [True, False], ["at_end", "at_start"], ["ieee", "nan_largest"])[10:110]
    assert out["a"].to_arrow().equals(a.take(pa.array(idx)))
    assert out["b"].to_arrow().equals(b.take(pa.array(idx)))
    assert "sort" in am.explain_plan(plan, [src])


def test_plan_errors(am):
    src = am.PlanSource("t", {"x": pa.array([1, 2, 3])})
    with pytest.raises(am.ArrowMetalError, match="unknown sort column"):
        am.run_plan({"op": "sort", "by": [["y", False]], "input": {"op": "scan", "source": "t"}}, [src])
    with pytest.raises(am.ArrowMetalError, match="float_order"):
        am.run_plan({"op": "sort", "by": [["x", False, {"float_order": "x"}]], "input": {"op": "scan", "source": "t"}}, [src])


@pytest.mark.parametrize("key_kind", ["int64", "uint32", "int8", "float64_ieee", "float64_total", "float32_nan_largest", "bool"])
@pytest.mark.parametrize("desc,nulls", [(False, "last"), (True, "first")])
def test_single_key_sort_all_columns(am, key_kind, desc, nulls):
    # One key: integer and totalOrder keys are rebuilt from the sorted keys, the other columns gathered;
    # other keys go through the permutation like every column.
    rng = np.random.default_rng(len(key_kind) * 7 + desc)
    n = 300_001
    fo = "ieee"
    if key_kind == "int64":
        key = pa.array(rng.integers(-2**62, 2**62, n), mask=rng.random(n) < 0.1)
    elif key_kind == "uint32":
        key = pa.array(rng.integers(0, 2**32, n, dtype=np.uint32), mask=rng.random(n) < 0.1)
    elif key_kind == "int8":
        key = pa.array(rng.integers(-128, 127, n, dtype=np.int8), mask=rng.random(n) < 0.1)
    elif key_kind == "bool":
        key = pa.array(rng.random(n) < 0.5, mask=rng.random(n) < 0.1)
    else:
        v = rng.normal(0, 100, n).astype(np.float64)
        v[rng.random(n) < 0.03] = np.nan
        v[rng.random(n) < 0.03] = -0.0
        key = pa.array(v, mask=rng.random(n) < 0.1)
        if key_kind.startswith("float32"):
            key = key.cast(pa.float32())
        fo = key_kind.split("_", 1)[1]
    cols = {"k": key, "f": pa.array(rng.standard_normal(n)), "i": pa.array(rng.integers(0, 9, n, dtype=np.int16)),
            "b": pa.array(rng.random(n) < 0.5, mask=rng.random(n) < 0.2),
            "u": pa.array(rng.integers(0, 200, n, dtype=np.uint8), mask=rng.random(n) < 0.3)}
    src = am.PlanSource("t", cols)
    plan = {"op": "sort", "input": {"op": "scan", "source": "t"},
            "by": [["k", desc, {"nulls": nulls, "float_order": fo}]]}
    out = am.run_plan(plan, [src])
    from oracle import oracle
    idx = oracle.argsort(key, desc, "at_start" if nulls == "first" else "at_end", fo)
    for name, col in cols.items():
        got = out[name].to_arrow()
        want = col.take(pa.array(idx))
        assert got.null_count == want.null_count, name
        assert same_bits(got, want), name


def same_bits(a, b):
    """Equal validity and equal value bits at every valid row (NaN payloads and -0.0 included;
    Array.equals treats NaN as unequal to itself)."""
    if len(a) != len(b) or a.type != b.type:
        return False
    va = np.asarray(a.is_valid().to_numpy(zero_copy_only=False))
    vb = np.asarray(b.is_valid().to_numpy(zero_copy_only=False))
    if not np.array_equal(va, vb):
        return False
    if pa.types.is_boolean(a.type):
        return np.array_equal(np.asarray(a.fill_null(False))[va], np.asarray(b.fill_null(False))[vb])
    width = a.type.bit_width // 8
    view = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[width]
    xa = np.frombuffer(a.buffers()[1], dtype=view)[a.offset:a.offset + len(a)]
    xb = np.frombuffer(b.buffers()[1], dtype=view)[b.offset:b.offset + len(b)]
    return np.array_equal(xa[va], xb[vb])


@pytest.mark.parametrize("t", [pa.int64(), pa.uint64(), pa.int32(), pa.int16(), pa.uint8()])
def test_sorted_copy_rebuilt_from_keys(am, t):
    rng = np.random.default_rng(3)
    n = 500_003
    info = np.iinfo(t.to_pandas_dtype())
    col = pa.array(rng.integers(info.min, info.max, n, dtype=t.to_pandas_dtype(), endpoint=True), mask=rng.random(n) < 0.05)
    m = am.MetalArray.from_arrow(col)
    for desc in (False, True):
        for place in ("at_end", "at_start"):
            got = m.sort(desc, place).to_arrow()
            want = pc.take(col, pc.array_sort_indices(col, order="descending" if desc else "ascending", null_placement=place))
            assert got.equals(want), (desc, place)


def test_sorted_copy_total_order_floats(am):
    rng = np.random.default_rng(4)
    bits = rng.integers(0, 2**64, 200_000, dtype=np.uint64)
    col = pa.Array.from_buffers(pa.float64(), len(bits), [None, pa.py_buffer(bits.tobytes())])
    m = am.MetalArray.from_arrow(col)
    got = m.sort(float_order="total").to_arrow()
    key = np.where(bits >> np.uint64(63), ~bits, bits | np.uint64(1 << 63))
    want = bits[np.argsort(key, kind="stable")]
    assert np.array_equal(got.to_numpy(zero_copy_only=False).view(np.uint64), want)


@pytest.mark.parametrize("key_kind", ["int64", "float64_ieee", "float64_total", "float32_nan_largest", "int32"])
@pytest.mark.parametrize("desc,nulls", [(False, "last"), (True, "first")])
def test_order_by_limit_is_the_sorted_prefix(am, key_kind, desc, nulls):
    # LIMIT over a one-key sort goes through radix selection: the rows must be those of the full sort.
    rng = np.random.default_rng(len(key_kind) * 3 + desc)
    n = 400_003
    fo = "ieee"
    if key_kind == "int64":
        key = pa.array(rng.integers(-2**50, 2**50, n), mask=rng.random(n) < 0.1)
    elif key_kind == "int32":
        key = pa.array(rng.integers(0, 1000, n).astype(np.int32), mask=rng.random(n) < 0.1)
    else:
        v = rng.standard_normal(n).astype(np.float32 if key_kind.startswith("float32") else np.float64)
        v[rng.random(n) < 0.05] = np.nan
        key = pa.array(v, mask=rng.random(n) < 0.1)
        fo = key_kind.split("_", 1)[1]
    t = {"k": key, "p": pa.array(rng.standard_normal(n)), "q": pa.array(rng.integers(0, 9, n).astype(np.int16))}
    src = am.PlanSource("t", t)
    sort = {"op": "sort", "by": [["k", desc, {"nulls": nulls, "float_order": fo}]], "input": {"op": "scan", "source": "t"}}
    full = am.run_plan(sort, [src])
    for off, count in [(0, 1), (0, 100), (17, 5000), (0, 20_000), (3, n), (n - 2, 10)]:
        out = am.run_plan({"op": "limit", "count": count, "offset": off, "input": sort}, [src])
        for name in t:
            want = full[name].to_arrow().slice(off, count)
            assert same_bits(out[name].to_arrow(), want), (name, off, count)
