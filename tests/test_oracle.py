"""The CPU oracle, pinned before it is trusted: the reference's known-answer vectors, and every golden
fixture pyarrow produced (tests/golden/make_golden.py), through both restatements (C and numpy)."""
import math

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
