"""Single-key argsort on the GPU, bit-exact against the golden fixtures (pyarrow), the C oracle and
pyarrow itself; the shapes of the reference's own sort tests."""
import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

from conftest import build_array, golden

pytestmark = pytest.mark.gpu

OPTIONS = [(d, p) for d in (False, True) for p in ("at_end", "at_start")]


def ids(m):
    return m.to_arrow().to_numpy(zero_copy_only=False)


def test_golden_argsort(am):
    g = golden()
    n_checked = 0
    for c in g.cases:
        if c["kind"] != "argsort":
            continue
        a = am.MetalArray.from_arrow(g.array(c["array"], c["type"]))
        got = ids(a.argsort(c["descending"], c["null_placement"], c["float_order"]))
        assert got.dtype == np.uint32
        assert np.array_equal(got, g[c["expect"]]), c
        n_checked += 1
    assert n_checked > 500


def test_kat_nan_negative_zero(am):
    # Tests/ArrowMetalTests/SortTests.swift:70-92
    v = [1.0, float("nan"), float("inf"), float("-inf"), -0.0, 0.0, None, float("nan")]
    for t in (pa.float32(), pa.float64()):
        a = am.MetalArray.from_arrow(pa.array(v, type=t, from_pandas=False))
        assert ids(a.argsort()).tolist() == [3, 4, 5, 0, 2, 1, 7, 6]
        assert ids(a.argsort(True)).tolist() == [2, 0, 4, 5, 3, 1, 7, 6]
        assert ids(a.top_k(4)).tolist() == [2, 0, 4, 5]
        assert ids(a.top_k(4, largest=False)).tolist() == [3, 4, 5, 0]


def test_kat_sorted_and_topk(am):
    # Tests/ArrowMetalTests/SortTests.swift:49-58
    a = am.MetalArray.from_arrow(pa.array([5, None, 3, 9, 1, 9], type=pa.int32()))
    assert a.sort().to_arrow().to_pylist() == [1, 3, 5, 9, 9, None]
    assert a.sort(descending=True).to_arrow().to_pylist() == [9, 9, 5, 3, 1, None]
    assert ids(a.top_k(2)).tolist() == [3, 5]
    assert ids(a.top_k(2, largest=False)).tolist() == [4, 2]


# Sizes of Tests/ArrowMetalTests/RadixSortScaleTests.swift:28-29 (chunk, block and tile edges).
SCALE_SIZES = [0, 1, 2, 31, 32, 33, 63, 64, 65, 255, 256, 257, 511, 512, 513, 4095, 4096, 4097, 65536,
               2**18 - 1, 2**18, 2**18 + 1]


def shapes(n, rng):
    """RadixSortScaleTests.swift:59-125: random, all equal, narrow, low digits constant, sorted,
    reverse, runs."""
    full = rng.integers(-2**63, 2**63 - 1, n, dtype=np.int64, endpoint=True)
    yield "random", full
    yield "equal", np.full(n, 42, dtype=np.int64)
    yield "narrow", rng.integers(0, 1000, n).astype(np.int64)
    yield "low_constant", (rng.integers(-2**40, 2**40, n) << 16).astype(np.int64)
    yield "sorted", np.sort(full)
    yield "reverse", np.sort(full)[::-1].copy()
    yield "runs", np.repeat(rng.integers(-100, 100, max(n // 50 + 1, 1)), 50)[:n].astype(np.int64)


@pytest.mark.parametrize("n", SCALE_SIZES)
def test_scale_shapes_int64(am, oracle, n):
    rng = np.random.default_rng(n + 7)
    for name, v in shapes(n, rng):
        for nf in (0.0, 0.001, 0.25, 0.5, 1.0):
            mask = rng.random(n) < nf if nf else None
            arr = pa.array(v, type=pa.int64(), mask=mask)
            m = am.MetalArray.from_arrow(arr)
            for d, p in OPTIONS:
                want = oracle.argsort(arr, d, p, threads=8)
                got = ids(m.argsort(d, p))
                assert np.array_equal(got, want), (name, nf, d, p)


@pytest.mark.parametrize("t", [pa.int32(), pa.float32(), pa.uint32(), pa.int16(), pa.uint8(), pa.bool_(),
                               pa.float16(), pa.uint64()])
def test_scale_other_types(am, oracle, t):
    rng = np.random.default_rng(11)
    for n in (4097, 65536, 2**18 + 1):
        if t == pa.bool_():
            arr = pa.array(rng.random(n) < 0.5, mask=rng.random(n) < 0.1)
        elif pa.types.is_floating(t):
            v = rng.normal(0, 100, n).astype(np.float64)
            v[rng.random(n) < 0.02] = np.nan
            v[rng.random(n) < 0.02] = -0.0
            v[rng.random(n) < 0.01] = np.inf
            arr = pa.array(v, mask=rng.random(n) < 0.1).cast(t)
        else:
            info = np.iinfo(t.to_pandas_dtype())
            arr = pa.array(rng.integers(info.min, info.max, n, dtype=t.to_pandas_dtype(), endpoint=True),
                           mask=rng.random(n) < 0.1)
        m = am.MetalArray.from_arrow(arr)
        orders = ("ieee", "total", "nan_largest") if pa.types.is_floating(t) else ("ieee",)
        for fo in orders:
            for d, p in OPTIONS:
                want = oracle.argsort(arr, d, p, fo, threads=8)
                assert np.array_equal(ids(m.argsort(d, p, fo)), want), (t, n, fo, d, p)


def test_float_specials_at_scale(am):
    # RadixSortScaleTests.swift:132-160 and SortOptionsTests.swift:66-78 specials, checked against pyarrow.
    rng = np.random.default_rng(3)
    n = 1_000_003
    bits = rng.normal(0, 1e6, n).view(np.uint64).copy()
    specials = np.array([0x7FF8000000000000, 0xFFF8000000000000, 0x7FF0000000000001, 0xFFF8000000000042,
                         0x0000000000000000, 0x8000000000000000, 0x7FF0000000000000, 0xFFF0000000000000,
                         0x0000000000000001, 0x8000000000000001, 0x7FEFFFFFFFFFFFFF, 0xFFEFFFFFFFFFFFFF],
                        dtype=np.uint64)
    sp = rng.random(n) < 0.1
    bits[sp] = specials[rng.integers(0, len(specials), int(sp.sum()))]
    arr = build_array(pa.float64(), bits, rng.random(n) >= 0.05)
    m = am.MetalArray.from_arrow(arr)
    for d, p in OPTIONS:
        want = pc.array_sort_indices(arr, order="descending" if d else "ascending", null_placement=p).to_numpy()
        assert np.array_equal(ids(m.argsort(d, p)), want), (d, p)


def test_uint64_index_width(am):
    rng = np.random.default_rng(9)
    arr = pa.array(rng.integers(-2**63, 2**63 - 1, 1_000_000, dtype=np.int64))
    m = am.MetalArray.from_arrow(arr)
    got = m.argsort64().to_arrow()
    assert got.type == pa.uint64()
    want = pc.sort_indices(arr)       # pyarrow's own uint64 answer
    assert got.equals(want)


def test_sliced_input(am, oracle):
    # SortValuesTests.swift:141: a sliced array sorts as its slice.
    rng = np.random.default_rng(4)
    base = pa.array(rng.integers(-1000, 1000, 100_000), mask=rng.random(100_000) < 0.1)
    for off, ln in ((3, 50_001), (8, 4096), (1, 1)):
        s = base.slice(off, ln)
        m = am.MetalArray.from_arrow(s)
        assert np.array_equal(ids(m.argsort()), oracle.argsort(s))
        m2 = am.MetalArray.from_arrow(base).slice(off, ln)
        assert np.array_equal(ids(m2.argsort(True, "at_start")), oracle.argsort(s, True, "at_start"))


def test_stats_report_skipped_passes(am):
    # Keys in [0, 2^40): bytes 5..7 are constant, so 3 of 8 passes are skipped.
    rng = np.random.default_rng(2)
    m = am.MetalArray.from_arrow(pa.array(rng.integers(0, 2**40, 1_000_000), mask=rng.random(1_000_000) < 0.1))
    m.argsort()
    st = am.last_sort_stats()
    assert st["rows"] == 1_000_000
    assert st["passes_run"] == 5 and st["passes_skipped"] == 3
    assert 880_000 < st["value_rows"] < 920_000


def test_chunked_import(am, oracle):
    rng = np.random.default_rng(6)
    chunks = [pa.array(rng.integers(-50, 50, k), mask=rng.random(k) < 0.2) for k in (1, 7, 4096, 33, 10_001)]
    ca = pa.chunked_array(chunks)
    m = am.MetalArray.from_arrow(ca)
    assert len(m) == len(ca)
    assert m.to_arrow().equals(ca.combine_chunks())
    assert np.array_equal(ids(m.argsort()), oracle.argsort(ca.combine_chunks()))


def test_empty_and_all_null(am):
    e = am.MetalArray.from_arrow(pa.array([], type=pa.int64()))
    assert len(e.argsort().to_arrow()) == 0
    z = am.MetalArray.from_arrow(pa.array([None] * 5000, type=pa.float64()))
    assert ids(z.argsort()).tolist() == list(range(5000))
    assert ids(z.argsort(True, "at_start")).tolist() == list(range(5000))
