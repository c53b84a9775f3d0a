"""The cases of the reference's own sort-option tests, through this library's C ABI.

The reference checks its float orders in python/tests/test_sort_options.py and
python/tests/test_sort_nan_largest.py: sizes around its tile edges, columns with no, some and only
nulls, both directions and placements, float64 and float32 columns salted with special bit patterns
(NaN payloads of both signs, signalling NaNs, both zeros, both infinities, denormals), and top-k
prefixes. The same shapes run here against the same answers: pyarrow for the ieee order (the
reference's oracle for it), and the orders' definitions for totalOrder and nan_largest (the oracle's
numpy restatement, pinned in tests/test_oracle.py; the reference uses Polars for nan_largest, which is
not installed here). The reference's checkout is not on the GPU machine, so its test files cannot run
there; this file restates their cases.
"""
import struct

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

pytestmark = pytest.mark.gpu

# python/tests/test_sort_options.py:24-31
SIZES = [0, 1, 2, 33, 8191, 8192, 8193, 70_001]
OPTIONS = [(d, p) for d in (False, True) for p in ("at_end", "at_start")]
SPECIAL64 = np.array([0x7FF8000000000000, 0xFFF8000000000000, 0x7FF0000000000001, 0xFFF8000000000042,
                      0x7FF8000000000007, 0x0000000000000000, 0x8000000000000000, 0x7FF0000000000000,
                      0xFFF0000000000000, 0x0000000000000001, 0x8000000000000003, 0x000FFFFFFFFFFFFF],
                     dtype=np.uint64).view(np.float64)
SPECIAL32 = np.array([0x7FC00000, 0xFFC00000, 0x7F800001, 0xFFC00042, 0x80000000, 0],
                     dtype=np.uint32).view(np.float32)


def salted64(n, null_fraction, seed):
    """Uniform values in +-1e6, a quarter replaced by small repeated quarters and a quarter by the
    special bit patterns (python/tests/test_sort_options.py:34-42)."""
    rng = np.random.default_rng(seed)
    v = rng.uniform(-1e6, 1e6, n)
    rep = rng.random(n) < 0.25
    v[rep] = rng.integers(-20, 21, int(rep.sum())) / 4.0
    sp = rng.random(n) < 0.25
    v[sp] = SPECIAL64[rng.integers(0, len(SPECIAL64), int(sp.sum()))]
    return v, (rng.random(n) < null_fraction if null_fraction else None)


def salted32(n, null_fraction, seed):
    """The float64 column narrowed, then a tenth replaced by float32 specials (test_sort_options.py:45-54)."""
    v, _ = salted64(n, 0, seed)
    with np.errstate(invalid="ignore", over="ignore"):
        a = v.astype(np.float32)
    rng = np.random.default_rng(seed + 1)
    sp = rng.random(n) < 0.1
    a[sp] = SPECIAL32[rng.integers(0, len(SPECIAL32), int(sp.sum()))]
    return a, (rng.random(n) < null_fraction if null_fraction else None)


def column(make, n, null_fraction, seed):
    v, mask = make(n, null_fraction, seed)
    return pa.array(v, mask=mask, from_pandas=False)


def ids(m):
    return m.to_arrow().to_numpy(zero_copy_only=False).astype(np.int64)


def bits_of(arr):
    width = np.uint64 if arr.type == pa.float64() else np.uint32
    valid = np.asarray(arr.is_valid())
    return valid, np.where(valid, arr.fill_null(0).to_numpy(zero_copy_only=False).view(width), 0)


@pytest.mark.parametrize("make", [salted64, salted32], ids=["f64", "f32"])
@pytest.mark.parametrize("float_order", ["ieee", "total", "nan_largest"])
def test_float_orders_on_salted_columns(am, oracle, make, float_order):
    for n in SIZES:
        for null_fraction in (0.0, 0.1, 1.0):
            v = column(make, n, null_fraction, 7 * n + 3)
            x = am.MetalArray.from_arrow(v)
            for descending, placement in OPTIONS:
                if float_order == "ieee":
                    want = pc.array_sort_indices(v, order="descending" if descending else "ascending",
                                                 null_placement=placement).to_numpy().astype(np.int64)
                else:
                    want = oracle.np_argsort(v, descending, placement, float_order).astype(np.int64)
                case = (n, null_fraction, descending, placement)
                assert np.array_equal(ids(x.argsort(descending, placement, float_order)), want), case
                for k in (1, 17, 1500):
                    got = ids(x.top_k(k, largest=descending, null_placement=placement, float_order=float_order))
                    assert np.array_equal(got, want[:k]), case + (k,)
                if float_order == "total":
                    # The sorted copy is exact to the bit: NaN payloads and zero signs included.
                    s = x.sort(descending, placement, "total").to_arrow()
                    e = v.take(pa.array(want))
                    sv, sb = bits_of(s)
                    ev, eb = bits_of(e)
                    assert np.array_equal(sv, ev) and np.array_equal(sb, eb), case


def test_total_order_known_answer(am):
    # python/tests/test_sort_options.py:144-153
    nan, inf = float("nan"), float("inf")
    neg_nan = struct.unpack("<d", struct.pack("<Q", 0xFFF8000000000000))[0]
    v = pa.array([1.0, nan, -0.0, None, neg_nan, 0.0, -inf, inf, -0.0, -1.0, None], from_pandas=False)
    x = am.MetalArray.from_arrow(v)
    assert ids(x.argsort(float_order="total")).tolist() == [4, 6, 9, 2, 8, 5, 0, 7, 1, 3, 10]
    assert ids(x.argsort(True, "at_start", "total")).tolist() == [3, 10, 1, 7, 0, 5, 2, 8, 9, 6, 4]
    assert ids(x.argsort(True)).tolist() == pc.array_sort_indices(v, order="descending").to_pylist()


@pytest.mark.parametrize("descending,placement", OPTIONS)
def test_total_order_agrees_with_pyarrow_without_nan_or_negative_zero(am, descending, placement):
    # python/tests/test_sort_options.py:128-141
    rng = np.random.default_rng(5)
    v = rng.integers(-50, 50, 100_003) / 4.0
    v[v == 0] = 0.0
    v[::97] = np.inf
    v[1::89] = -np.inf
    arr = pa.array(v, mask=rng.random(len(v)) < 0.05)
    want = pc.array_sort_indices(arr, order="descending" if descending else "ascending",
                                 null_placement=placement).to_numpy().astype(np.int64)
    assert np.array_equal(ids(am.MetalArray.from_arrow(arr).argsort(descending, placement, "total")), want)


def test_integer_keys_ignore_the_float_order(am):
    # python/tests/test_sort_options.py:156-163
    v = pa.array([3, None, 1, 3, None, 2], pa.int64())
    x = am.MetalArray.from_arrow(v)
    for d, p in OPTIONS:
        want = pc.array_sort_indices(v, order="descending" if d else "ascending", null_placement=p).to_pylist()
        for order in ("total", "nan_largest"):
            assert ids(x.argsort(d, p, order)).tolist() == want
            assert ids(x.top_k(3, largest=d, null_placement=p, float_order=order)).tolist() == want[:3]


@pytest.mark.parametrize("n", [8193, 70_001])
def test_lexsort_per_key_float_orders(am, oracle, n):
    # python/tests/test_sort_options.py:174-198 and test_sort_nan_largest.py:100-113: an integer key with
    # nulls over a salted float key, every direction and placement of each, the float key in each order.
    rng = np.random.default_rng(n)
    k1 = pa.array(rng.integers(0, 4, n), mask=rng.random(n) < 0.1)
    k2 = column(salted64, n, 0.1, n)
    h1, h2 = am.MetalArray.from_arrow(k1), am.MetalArray.from_arrow(k2)
    for order in ("ieee", "total", "nan_largest"):
        for d1, p1 in OPTIONS:
            for d2, p2 in OPTIONS:
                got = ids(am.lexsort_indices([h1, h2], [d1, d2], null_placement=[p1, p2],
                                             float_order=["ieee", order]))
                want = oracle.np_lexsort([k1, k2], [d1, d2], [p1, p2], ["ieee", order]).astype(np.int64)
                assert np.array_equal(got, want), (order, d1, p1, d2, p2)


def test_bad_option_values_raise(am):
    # python/tests/test_sort_options.py:166-171
    x = am.MetalArray.from_arrow(pa.array([1.0, 2.0]))
    with pytest.raises(am.ArrowMetalError):
        x.argsort(float_order="bogus")
    with pytest.raises(am.ArrowMetalError):
        x.top_k(1, null_placement="middle")
