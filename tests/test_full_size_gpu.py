"""The benchmark's workloads at their full sizes on the GPU, through the C ABI: bit-exact against pyarrow
where pyarrow finishes in seconds (1M full-range int64 keys), and through size-independent properties
at 50M rows (the result is a permutation; rows come out in key order; equal keys keep row order; the
taken columns are the inputs read through that permutation)."""
import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

import bench

pytestmark = pytest.mark.gpu


def is_permutation(idx, n):
    if len(idx) != n:
        return False
    seen = np.zeros(n, dtype=bool)
    seen[idx] = True
    return bool(seen.all())


def values_of(arr, dtype):
    """The value buffer of a primitive array, as `dtype` (null slots included, offset applied)."""
    return np.frombuffer(arr.buffers()[1], dtype=dtype)[arr.offset:arr.offset + len(arr)]


def test_full_range_int64_1M_matches_pyarrow(am):
    key = bench.make_full_range_keys(1_000_000)
    arr = pa.array(key)
    got = am.MetalArray.from_arrow(arr).argsort64().to_arrow().to_numpy()
    assert got.dtype == np.uint64
    assert np.array_equal(got, pc.array_sort_indices(arr).to_numpy())


def test_order_by_int64_50M(am):
    n = bench.N_ROWS
    key, valid, p1, p2 = bench.make_table(n)
    cols = bench.arrow_columns(key, valid, p1, p2)
    dcols = {k: am.MetalArray.from_arrow(v) for k, v in cols.items()}
    idx = dcols["c0"].argsort().to_arrow().to_numpy()
    assert is_permutation(idx, n)
    m = int(valid.sum())
    vi, ni = idx[:m].astype(np.int64), idx[m:].astype(np.int64)
    assert valid[vi].all() and not valid[ni].any()            # values first, nulls last
    d = np.diff(key[vi])
    assert (d >= 0).all()                                      # ascending
    assert (np.diff(vi)[d == 0] > 0).all()                     # equal keys keep row order
    assert (np.diff(ni) > 0).all()                             # null rows in row order

    out = am.run_plan(bench.PLAN, [am.PlanSource("t", dcols)])
    k = out["c0"].to_arrow()
    assert k.null_count == n - m
    assert np.array_equal(values_of(k, np.int64)[:m], key[vi])
    assert not np.asarray(k.is_valid())[m:].any()
    assert np.array_equal(values_of(out["c1"].to_arrow(), np.uint64), p1.view(np.uint64)[idx])
    assert np.array_equal(values_of(out["c2"].to_arrow(), np.int32), p2[idx])


def test_multikey_50M(am):
    n = bench.N_ROWS
    key1, key2, valid2, payload = bench.make_multikey_table(n)
    a1 = pa.array(key1)
    a2 = pa.array(key2, mask=~valid2, from_pandas=False)
    idx = am.lexsort_indices([am.MetalArray.from_arrow(a1), am.MetalArray.from_arrow(a2)],
                             descending=[True, False], null_placement="at_end", float_order="ieee")
    taken = am.take_columns([am.MetalArray.from_arrow(pa.array(payload))], idx)[0].to_arrow()
    idx = idx.to_arrow().to_numpy().astype(np.int64)
    assert is_permutation(idx, n)
    # Sort tuple: key1 descending; then key2 in Arrow's ieee order with nulls at the end: values
    # (-0.0 equal to +0.0), then NaN, then nulls.
    k1 = -key1.astype(np.int64)
    nan2 = np.isnan(key2) & valid2
    cat = np.where(~valid2, 2, np.where(nan2, 1, 0))
    v2 = np.where(cat == 0, key2 + 0.0, 0.0)
    a, b = idx[:-1], idx[1:]
    lt = (k1[a] < k1[b]) | ((k1[a] == k1[b]) & ((cat[a] < cat[b]) | ((cat[a] == cat[b]) & (v2[a] < v2[b]))))
    eq = (k1[a] == k1[b]) & (cat[a] == cat[b]) & (v2[a] == v2[b])
    assert (lt | (eq & (a < b))).all()
    assert np.array_equal(values_of(taken, np.uint64), payload.view(np.uint64)[idx])
