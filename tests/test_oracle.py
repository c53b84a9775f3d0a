"""The CPU oracle, pinned before it is trusted: the reference's known-answer vectors, and every golden
fixture pyarrow produced (tests/golden/make_golden.py), through both restatements (C and numpy)."""
import math
import zlib

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

from conftest import build_array, golden

NAN = float("nan")


# Tests/ArrowMetalTests/SortTests.swift:70-92: NaN and -0.0 placement, both widths, both directions.
KAT_FLOATS = [1.0, NAN, math.inf, -math.inf, -0.0, 0.0, None, NAN]
KAT_ASC = [3, 4, 5, 0, 2, 1, 7, 6]
KAT_DESC = [2, 0, 4, 5, 3, 1, 7, 6]

# Tests/ArrowMetalTests/SortNanLargestTests.swift:125-136: Polars' order (nan_largest).
POLARS_VALUES = [1, NAN, None, -0.0, 0.0, -1, math.inf, -math.inf, -NAN, None, 2, -0.0]
POLARS_ROWS = {(False, "at_start"): [2, 9, 7, 5, 3, 4, 11, 0, 10, 6, 1, 8],
               (False, "at_end"): [7, 5, 3, 4, 11, 0, 10, 6, 1, 8, 2, 9],
               (True, "at_start"): [2, 9, 1, 8, 6, 10, 0, 3, 4, 11, 5, 7],
               (True, "at_end"): [1, 8, 6, 10, 0, 3, 4, 11, 5, 7, 2, 9]}

# Tests/ArrowMetalTests/SortTests.swift:49-58: [5, nil, 3, 9, 1, 9].
INT_VALUES = [5, None, 3, 9, 1, 9]


@pytest.mark.parametrize("t", [pa.float32(), pa.float64()])
def test_kat_nan_and_negative_zero(oracle, t):
    a = pa.array(KAT_FLOATS, type=t, from_pandas=False)
    assert oracle.argsort(a).tolist() == KAT_ASC
    assert oracle.argsort(a, descending=True).tolist() == KAT_DESC
    assert oracle.np_argsort(a).tolist() == KAT_ASC
    assert oracle.np_argsort(a, descending=True).tolist() == KAT_DESC
    # pyarrow agrees with the reference's vector (the reference's own claim).
    assert pc.array_sort_indices(a).to_pylist() == KAT_ASC
    assert pc.array_sort_indices(a, order="descending").to_pylist() == KAT_DESC


@pytest.mark.parametrize("desc,place", list(POLARS_ROWS))
def test_kat_polars_nan_largest(oracle, desc, place):
    a = pa.array(POLARS_VALUES, type=pa.float64(), from_pandas=False)
    want = POLARS_ROWS[(desc, place)]
    assert oracle.argsort(a, desc, place, "nan_largest").tolist() == want
    assert oracle.np_argsort(a, desc, place, "nan_largest").tolist() == want


def test_kat_sorted_values(oracle):
    a = pa.array(INT_VALUES, type=pa.int32())
    idx = oracle.argsort(a)
    vals, valid = oracle.take(a, pa.array(idx, type=pa.uint32()))
    got = [int(np.int32(v)) if ok else None for v, ok in zip(vals.view(np.int32), valid)]
    assert got == [1, 3, 5, 9, 9, None]
    idx = oracle.argsort(a, descending=True)
    vals, valid = oracle.take(a, pa.array(idx, type=pa.uint32()))
    assert [int(v) if ok else None for v, ok in zip(vals.view(np.int32), valid)] == [9, 9, 5, 3, 1, None]
    # top_k = the first k of the argsort
    assert oracle.argsort(a, descending=True)[:2].tolist() == [3, 5]
    assert oracle.argsort(a)[:2].tolist() == [4, 2]


def test_stability_many_duplicates(oracle):
    # SortTests.swift:46: 50k rows of 3 distinct values keep input order within each value.
    a = pa.array(np.arange(50_000, dtype=np.int32) % 3)
    got = oracle.argsort(a)
    want = np.concatenate([np.arange(k, 50_000, 3) for k in range(3)])
    assert (got == want).all()


def _golden_cases(kind):
    return [c for c in golden().cases if c["kind"] == kind]


def test_golden_argsort_c_and_numpy(oracle):
    g = golden()
    checked = 0
    for c in _golden_cases("argsort"):
        a = g.array(c["array"], c["type"])
        want = g[c["expect"]]
        got = oracle.argsort(a, c["descending"], c["null_placement"], c["float_order"], threads=4)
        assert np.array_equal(got, want), c
        if c["n"] <= 4097:
            got2 = oracle.np_argsort(a, c["descending"], c["null_placement"], c["float_order"])
            assert np.array_equal(got2, want), c
        checked += 1
    assert checked > 500


def test_golden_lexsort(oracle):
    g = golden()
    for c in _golden_cases("lexsort"):
        arrays = [g.array(n, t) for n, t in zip(c["arrays"], c["types"])]
        want = g[c["expect"]]
        got = oracle.lexsort(arrays, c["descending"], c["null_placement"])
        assert np.array_equal(got, want), c
        got2 = oracle.np_lexsort(arrays, c["descending"], c["null_placement"])
        assert np.array_equal(got2, want), c


def test_golden_take(oracle):
    g = golden()
    for c in _golden_cases("take"):
        src = g.array(c["array"], c["type"])
        idx = g.array(c["index"], c["index_type"])
        vals, valid = oracle.take(src, idx)
        assert np.array_equal(valid, g[c["index"] + "_expect_valid"]), c
        want = g[c["index"] + "_expect_values"]
        assert np.array_equal(vals[valid], want.view(vals.dtype)[valid]), c


def test_take_out_of_range_is_an_error(oracle):
    # IndexTypeTests.swift:109: an out-of-range index is refused.
    with pytest.raises(IndexError):
        oracle.take(pa.array([1, 2, 3]), pa.array([0, 3], type=pa.int64()))
    with pytest.raises(IndexError):
        oracle.take(pa.array([1, 2, 3]), pa.array([-1], type=pa.int32()))


def test_oracle_threads_agree(oracle):
    rng = np.random.default_rng(5)
    a = pa.array(rng.integers(-2**63, 2**63 - 1, 300_000, dtype=np.int64), mask=rng.random(300_000) < 0.1)
    one = oracle.argsort(a, threads=1)
    many = oracle.argsort(a, threads=8)
    assert np.array_equal(one, many)
    want = pc.array_sort_indices(a).to_numpy()
    assert np.array_equal(one, want)


@pytest.mark.parametrize("t", ["int64", "double", "float", "uint8"])
def test_consumer_oracles_pinned_to_pyarrow(oracle, t):
    """The consumers' restatements agree with pyarrow's rank, rank_quantile, unique and value_counts on
    the same inputs (pyarrow is the reference's oracle for them: python/tests/test_options.py:125-405);
    the partition has the reference's block arrangement and its row at the pivot ties the sorted one."""
    import pyarrow.compute as pc
    rng = np.random.default_rng(zlib.crc32(t.encode()))
    n = 20_000
    valid = rng.random(n) > 0.1
    if t in ("double", "float"):
        v = np.round(rng.standard_normal(n), 1).astype(np.float64 if t == "double" else np.float32)
        v[rng.random(n) < 0.05] = np.nan
        v[rng.random(n) < 0.05] = 0.0
        v[rng.random(n) < 0.05] = -0.0
    elif t == "uint8":
        v = rng.integers(0, 256, n).astype(np.uint8)
    else:
        v = rng.integers(-40, 40, n).astype(np.int64)
    arr = build_array(t, v, valid)
    for desc in (False, True):
        sk = "descending" if desc else "ascending"
        for place in ("at_end", "at_start"):
            for tb in ("min", "max", "first", "dense"):
                want = pc.rank(arr, sort_keys=sk, null_placement=place, tiebreaker=tb).to_numpy()
                assert np.array_equal(oracle.rank(arr, tb, desc, place), want), (desc, place, tb)
            want_q = pc.rank_quantile(arr, sort_keys=sk, null_placement=place).to_numpy()
            assert np.allclose(oracle.rank_quantile(arr, desc, place), want_q, rtol=0, atol=1e-15)
    rows, counts = oracle.unique_rows(arr, "first_appearance")
    if t not in ("double", "float"):   # pyarrow keeps -0.0 and 0.0 apart; the sort's equality ties them
        assert arr.take(pa.array(rows, type=pa.int64())).equals(pc.unique(arr))
        assert np.array_equal(counts, pc.value_counts(arr).field("counts").to_numpy())
    full = oracle.np_argsort(arr)
    key, cat = oracle._keys_and_categories(arr, False, "ieee")
    for pivot in (0, n // 2, n - 1):
        got = oracle.partition_nth(arr, pivot)
        assert sorted(got) == list(range(n))
        a, b = got[pivot], full[pivot]
        assert cat[a] == cat[b] and (cat[a] != 0 or key[a] == key[b])
