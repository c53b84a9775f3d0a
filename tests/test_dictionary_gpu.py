"""Dictionary-encoded columns through the C ABI: import / export, slices and takes (the codes move, the
dictionary is shared), and every sort entry point ordering them by their values -- argsort, sorted
copies, lexsort keys, top-k, partition_nth, rank, plans and batches. The answers must equal the same
calls on the decoded column (the reference orders a dictionary column by its decoded values,
Sources/ArrowMetal/Kernels/MultiSort.swift:124-133), checked against the oracle and pyarrow."""
import zlib

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

pytestmark = pytest.mark.gpu

PLACEMENTS = ("at_end", "at_start")
INDEX_TYPES = (pa.int8(), pa.int16(), pa.int32(), pa.int64(), pa.uint8(), pa.uint32())


FORMATS = {pa.int8(): "c", pa.int16(): "s", pa.int32(): "i", pa.int64(): "l", pa.uint8(): "C", pa.uint32(): "I"}


def same_values(a, b):
    """Equal validity and values; float values compared by their bits (NaN payloads, -0.0)."""
    if a.type != b.type or len(a) != len(b):
        return False
    va, vb = a.is_valid().to_numpy(zero_copy_only=False), b.is_valid().to_numpy(zero_copy_only=False)
    if not np.array_equal(va, vb):
        return False
    if pa.types.is_floating(a.type):
        x, y = a.to_numpy(zero_copy_only=False)[va], b.to_numpy(zero_copy_only=False)[vb]
        return np.array_equal(x.view(np.uint8), y.view(np.uint8))
    return a.equals(b)


def ids(m):
    return m.to_arrow().to_numpy(zero_copy_only=False)


def rng_for(*parts):
    return np.random.default_rng(zlib.crc32("/".join(map(str, parts)).encode()))


def dictionary_values(rng, kind, d):
    """d dictionary entries with duplicates and a null among them."""
    if kind == "utf8":
        words = ["", "a", "ab", "abc", "b", "ba", "zz", "héllo", "hello", "日本", "Z"]
        vals = [words[int(i)] if rng.random() > 0.03 else None for i in rng.integers(0, len(words), d)]
        return pa.array(vals, type=pa.utf8())
    if kind == "large_binary":
        return pa.array([bytes(rng.integers(0, 3, int(k)).astype(np.uint8)) for k in rng.integers(0, 5, d)],
                        type=pa.large_binary())
    if kind == "int64":
        return pa.array(rng.integers(-20, 20, d), mask=rng.random(d) < 0.03)
    if kind == "float64":
        v = np.round(rng.standard_normal(d), 1)
        v[rng.random(d) < 0.1] = np.nan
        v[rng.random(d) < 0.1] = -0.0
        v[rng.random(d) < 0.1] = 0.0
        return pa.array(v, mask=rng.random(d) < 0.03)
    if kind == "float32":
        v = np.round(rng.standard_normal(d), 1).astype(np.float32)
        v[rng.random(d) < 0.1] = np.float32("nan")
        v[rng.random(d) < 0.05] = -np.float32("nan")
        return pa.array(v)
    raise AssertionError(kind)


def dictionary_column(rng, kind, n, d=100, index_type=pa.int32(), null_frac=0.08):
    values = dictionary_values(rng, kind, d)
    codes = rng.integers(0, d, n)
    valid = rng.random(n) >= null_frac
    idx = pa.array(codes, mask=~valid).cast(index_type)
    return pa.DictionaryArray.from_arrays(idx, values)


KINDS = ["utf8", "large_binary", "int64", "float64", "float32"]


def test_round_trip_slices_and_take(am):
    rng = rng_for("roundtrip")
    for kind in KINDS:
        for it in INDEX_TYPES:
            arr = dictionary_column(rng, kind, 5000, index_type=it)
            m = am.MetalArray.from_arrow(arr)
            assert m.format == FORMATS[it]          # am_format reports the codes' format
            back = m.to_arrow()
            assert back.type == arr.type and back.indices.equals(arr.indices), (kind, it)
            assert same_values(back.dictionary, arr.dictionary), (kind, it)
            for off, ln in [(0, 0), (7, 100), (4999, 1), (123, 3000)]:
                s = m.slice(off, ln).to_arrow()
                assert s.type == arr.type and s.indices.equals(arr.indices.slice(off, ln))
            idx = pa.array(rng.integers(0, 5000, 7000), type=pa.int64())
            t = m.take(idx).to_arrow()
            assert t.type == arr.type and t.indices.equals(arr.indices.take(idx))


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("placement", PLACEMENTS)
@pytest.mark.parametrize("desc", [False, True])
def test_argsort_orders_by_the_values(am, oracle, kind, placement, desc):
    rng = rng_for("argsort", kind, placement, desc)
    arr = dictionary_column(rng, kind, 200_003, d=int(rng.integers(1, 3000)))
    m = am.MetalArray.from_arrow(arr)
    decoded = arr.dictionary_decode()
    want = pc.array_sort_indices(decoded, order="descending" if desc else "ascending",
                                 null_placement=placement).to_numpy()
    got = ids(m.argsort(desc, placement))
    assert np.array_equal(got, want)
    assert np.array_equal(ids(am.MetalArray.from_arrow(decoded).argsort(desc, placement)), want)
    if kind.startswith("float"):
        for fo in ("total", "nan_largest"):
            got = ids(m.argsort(desc, placement, fo))
            assert np.array_equal(got, oracle.np_argsort(arr, desc, placement, fo)), fo


def test_sorted_copy_stays_a_dictionary(am):
    rng = rng_for("sorted")
    arr = dictionary_column(rng, "utf8", 50_000, d=40)
    m = am.MetalArray.from_arrow(arr)
    for desc in (False, True):
        s = m.sort(desc).to_arrow()
        order = pc.array_sort_indices(arr.dictionary_decode(), order="descending" if desc else "ascending")
        assert s.type == arr.type
        assert s.indices.equals(arr.indices.take(order))


def test_top_k_partition_and_rank(am, oracle):
    rng = rng_for("topk")
    for kind in ("utf8", "float64", "int64"):
        arr = dictionary_column(rng, kind, 300_000, d=500)
        decoded = arr.dictionary_decode()
        m = am.MetalArray.from_arrow(arr)
        for largest in (False, True):
            for placement in PLACEMENTS:
                full = ids(m.argsort(largest, placement))
                for k in (1, 100, 5000, 299_999):
                    assert np.array_equal(ids(m.top_k(k, largest, placement)), full[:k]), (kind, largest, k)
        for tb in ("min", "max", "first", "dense"):
            for placement in PLACEMENTS:
                want = pc.rank(decoded, null_placement=placement, tiebreaker=tb).to_numpy()
                assert np.array_equal(ids(m.rank(null_placement=placement, tiebreaker=tb)), want), (kind, tb)
        if kind != "utf8":
            for pivot in (0, 150_000, 299_999):
                got = ids(m.partition_nth_indices(pivot))
                assert np.array_equal(got, oracle.partition_nth(arr, pivot)), (kind, pivot)
        else:
            got = ids(m.partition_nth_indices(150_000))
            order = pc.array_sort_indices(decoded).to_numpy()
            vals = decoded.to_pylist()
            assert sorted(got) == list(range(len(vals)))
            assert vals[got[150_000]] == vals[order[150_000]]


def test_lexsort_plan_and_batch(am):
    rng = rng_for("lexsort")
    n = 120_000
    d = dictionary_column(rng, "utf8", n, d=30)
    k = pa.array(rng.integers(0, 7, n), mask=rng.random(n) < 0.1)
    v = pa.array(rng.standard_normal(n))
    decoded = pa.table({"d": d.dictionary_decode(), "k": k})
    for keys in ([("d", "ascending"), ("k", "descending")], [("k", "ascending"), ("d", "descending")]):
        for placement in PLACEMENTS:
            cols = {"d": d, "k": k}
            got = ids(am.lexsort_indices([am.MetalArray.from_arrow(cols[c]) for c, _ in keys],
                                         descending=[o == "descending" for _, o in keys], null_placement=placement))
            want = pc.sort_indices(decoded, keys, null_placement=placement).to_numpy()
            assert np.array_equal(got, want), (keys, placement)
    # A plan ORDER BY the dictionary column, with payload columns and a LIMIT.
    src = am.PlanSource("t", {"d": d, "k": k, "v": v})
    plan = {"op": "sort", "by": [["d", True, {"nulls": "last"}]], "input": {"op": "scan", "source": "t"}}
    out = am.run_plan(plan, [src])
    order = pc.array_sort_indices(d.dictionary_decode(), order="descending").to_numpy()
    assert out["d"].to_arrow().indices.equals(d.indices.take(pa.array(order)))
    assert out["v"].to_arrow().equals(v.take(pa.array(order)))
    lim = am.run_plan({"op": "limit", "count": 50, "offset": 3, "input": plan}, [src])
    assert lim["k"].to_arrow().equals(k.take(pa.array(order[3:53])))
    # Batches: dictionary arrays beside plain ones.
    arrays = [d, k, dictionary_column(rng, "float64", 3000, d=20), v]
    outs = am.argsort_batch([am.MetalArray.from_arrow(a) for a in arrays])
    for a, o in zip(arrays, outs):
        plain = a.dictionary_decode() if pa.types.is_dictionary(a.type) else a
        assert np.array_equal(ids(o), pc.array_sort_indices(plain).to_numpy())


def test_large_dictionary_column(am):
    rng = rng_for("large")
    n = 5_000_000
    arr = dictionary_column(rng, "int64", n, d=70_000, index_type=pa.int32())
    m = am.MetalArray.from_arrow(arr)
    want = pc.array_sort_indices(arr.dictionary_decode()).to_numpy()
    assert np.array_equal(ids(m.argsort()), want)


def test_bad_codes_and_unsupported_calls(am):
    bad = pa.DictionaryArray.from_arrays(pa.array([0, 5, 1], type=pa.int32()), pa.array(["a", "b"]), safe=False)
    m = am.MetalArray.from_arrow(bad)
    with pytest.raises(am.ArrowMetalError, match="out of range"):
        m.argsort()
    good = am.MetalArray.from_arrow(pa.DictionaryArray.from_arrays(pa.array([1, 0, 1], type=pa.int32()),
                                                                   pa.array(["b", "a"])))
    assert ids(good.argsort()).tolist() == pc.array_sort_indices(pa.array(["a", "b", "a"])).to_pylist()
    with pytest.raises(am.ArrowMetalError, match="dictionary"):
        good.unique()
