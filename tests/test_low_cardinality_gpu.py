"""Low-cardinality integer keys: a key of at least 4M rows with at most 256 distinct values sorts by its
dense rank (one digit pass). Every order must equal the oracle's stable sort of the original values:
argsort and lexsort, both directions and null placements, 1, 200 and 256 distinct values, 257 (the
ordinary passes), keys that include the largest and smallest values of their type."""
import numpy as np
import pyarrow as pa
import pytest

pytestmark = pytest.mark.gpu

N = 5_000_000


def ids(m):
    return m.to_arrow().to_numpy(zero_copy_only=False)


def column(rng, distinct, dtype, null_fraction, extremes=False):
    info = np.iinfo(dtype)
    vals = rng.integers(info.min, info.max, distinct, dtype=dtype, endpoint=True)
    if extremes:
        vals[0], vals[-1] = info.max, info.min
    v = vals[rng.integers(0, distinct, N)]
    mask = rng.random(N) < null_fraction if null_fraction else None
    return pa.array(v, mask=mask)


@pytest.mark.parametrize("distinct", [1, 200, 256, 257])
@pytest.mark.parametrize("dtype", [np.int32, np.int64, np.uint64])
def test_argsort_of_few_distinct_values(am, oracle, distinct, dtype):
    rng = np.random.default_rng(distinct + np.dtype(dtype).itemsize)
    arr = column(rng, distinct, dtype, 0.05, extremes=distinct >= 2)
    h = am.MetalArray.from_arrow(arr)
    for desc, place in ((False, "at_end"), (True, "at_start"), (True, "at_end")):
        assert np.array_equal(ids(h.argsort(desc, place)), oracle.argsort(arr, desc, place, threads=8)), (desc, place)


def test_lexsort_with_a_low_cardinality_key(am, oracle):
    # The multi-key benchmark's shape: an int32 key of 200 values (descending) over a float64 key.
    rng = np.random.default_rng(31)
    k1 = column(rng, 200, np.int32, 0.0)
    v = rng.normal(0, 1e6, N)
    v[rng.random(N) < 0.01] = np.nan
    k2 = pa.array(v, mask=rng.random(N) < 0.05)
    h1, h2 = am.MetalArray.from_arrow(k1), am.MetalArray.from_arrow(k2)
    for d1, p in ((True, "at_end"), (False, "at_start")):
        got = ids(am.lexsort_indices([h1, h2], [d1, False], null_placement=p))
        want = oracle.lexsort([k1, k2], [d1, False], p, threads=8)
        assert np.array_equal(got, want), (d1, p)
    # Low-cardinality key as the less significant one.
    got = ids(am.lexsort_indices([h2, h1], [False, True]))
    assert np.array_equal(got, oracle.lexsort([k2, k1], [False, True], "at_end", threads=8))


def test_plan_sort_keeps_the_key_values(am):
    # An ORDER BY's sorted key column is rebuilt from its keys, so the ranks are not used there; the
    # rows and the key column must still be the values' order.
    rng = np.random.default_rng(32)
    k = column(rng, 50, np.int64, 0.1)
    p = pa.array(rng.standard_normal(N))
    src = am.PlanSource("t", {"k": k, "p": p})
    out = am.run_plan({"op": "sort", "by": [["k", True]], "input": {"op": "scan", "source": "t"}}, [src])
    import pyarrow.compute as pc
    order = pc.sort_indices(pa.table({"k": k}), [("k", "descending")], null_placement="at_end")
    assert out["k"].to_arrow().equals(k.take(order))
    assert out["p"].to_arrow().equals(p.take(order))
