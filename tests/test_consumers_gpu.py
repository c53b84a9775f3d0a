"""Sort consumers through the C ABI: partition_nth_indices, rank (four tiebreakers), rank_quantile /
rank_normal, the window rankings, unique and value_counts. Each result is compared bit for bit with the
oracle's restatement on the same input, and with pyarrow wherever pyarrow defines the same answer (the
reference's own tests compare with pyarrow: python/tests/test_options.py:125-245, :332-405)."""
import zlib

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

from conftest import build_array

pytestmark = pytest.mark.gpu

PLACEMENTS = ("at_end", "at_start")
TIEBREAKERS = ("min", "max", "first", "dense")


def np_of(m):
    return m.to_arrow().to_numpy(zero_copy_only=False)


def column(rng, kind, n, null_frac=0.1):
    valid = rng.random(n) >= null_frac
    if kind == "int64":
        return build_array("int64", rng.integers(-2**62, 2**62, n, dtype=np.int64), valid)
    if kind == "int64_dups":
        return build_array("int64", rng.integers(0, 300, n, dtype=np.int64), valid)
    if kind == "int32_dups":
        return build_array("int32", rng.integers(-50, 50, n).astype(np.int32), valid)
    if kind == "uint8":
        return build_array("uint8", rng.integers(0, 256, n).astype(np.uint8), valid)
    if kind == "bool":
        return pa.array(rng.random(n) < 0.3, mask=~valid)
    if kind == "float64":
        v = np.round(rng.standard_normal(n), 2)
        v[rng.random(n) < 0.05] = np.nan
        v[rng.random(n) < 0.05] = -0.0
        v[rng.random(n) < 0.05] = 0.0
        v[rng.random(n) < 0.01] = -np.inf
        return build_array("double", v, valid)
    if kind == "float32":
        v = np.round(rng.standard_normal(n), 1).astype(np.float32)
        v[rng.random(n) < 0.05] = np.float32("nan")
        v[rng.random(n) < 0.02] = -np.float32("nan")
        return build_array("float", v, valid)
    raise AssertionError(kind)


KINDS = ["int64", "int64_dups", "int32_dups", "uint8", "bool", "float64", "float32"]


def same_bits(a, b):
    """Equal type, validity and value bits on the valid rows (NaN payloads and -0.0 compared exactly)."""
    if a.type != b.type or len(a) != len(b) or a.null_count != b.null_count:
        return False
    va, vb = a.is_valid().to_numpy(zero_copy_only=False), b.is_valid().to_numpy(zero_copy_only=False)
    if not np.array_equal(va, vb):
        return False
    if pa.types.is_floating(a.type):
        x = a.to_numpy(zero_copy_only=False)[va]
        y = b.to_numpy(zero_copy_only=False)[vb]
        return np.array_equal(x.view(np.uint8), y.view(np.uint8))
    return a.equals(b)


def rng_for(*parts):
    return np.random.default_rng(zlib.crc32("/".join(map(str, parts)).encode()))


# ---- partition_nth_indices

@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("placement", PLACEMENTS)
def test_partition_matches_the_oracle(am, oracle, kind, placement):
    rng = rng_for("partition", kind, placement)
    n = 300_001
    arr = column(rng, kind, n)
    m = am.MetalArray.from_arrow(arr)
    full = oracle.np_argsort(arr, False, placement)
    nulls = arr.null_count
    for pivot in sorted({0, 1, n // 3, n // 2, n - nulls - 1, n - nulls, n - 1, n}):
        got = np_of(m.partition_nth_indices(pivot, null_placement=placement))
        assert np.array_equal(got, oracle.partition_nth(arr, pivot, placement)), (kind, placement, pivot)
        if pivot < n:
            # The row at `pivot` ties with the one the full sort puts there.
            key, cat = oracle._keys_and_categories(arr, False, "ieee")
            a, b = got[pivot], full[pivot]
            assert cat[a] == cat[b] and (cat[a] != 0 or key[a] == key[b])


def test_partition_small_cases_and_errors(am, oracle):
    for vals in ([], [5], [None], [3, 1, 2], [2, 2, 2, None, 2], [None, None, 1]):
        arr = pa.array(vals, type=pa.int64())
        m = am.MetalArray.from_arrow(arr)
        for pivot in range(len(vals) + 1):
            for placement in PLACEMENTS:
                got = np_of(m.partition_nth_indices(pivot, null_placement=placement))
                assert np.array_equal(got, oracle.partition_nth(arr, pivot, placement)), (vals, pivot, placement)
    m = am.MetalArray.from_arrow(pa.array([1, 2, 3], type=pa.int64()))
    for bad in (-1, 4):
        with pytest.raises(am.ArrowMetalError, match="outside"):
            m.partition_nth_indices(bad)


def test_partition_of_strings_is_a_partition(am):
    rng = rng_for("partition-str")
    vals = ["".join(chr(97 + int(c)) for c in rng.integers(0, 3, int(rng.integers(0, 6)))) for _ in range(5000)]
    arr = pa.array(vals)
    order = pc.array_sort_indices(arr).to_numpy()
    got = np_of(am.MetalArray.from_arrow(arr).partition_nth_indices(2500))
    assert sorted(got) == list(range(5000))
    assert vals[got[2500]] == vals[order[2500]]
    assert all(vals[i] <= vals[got[2500]] for i in got[:2500])
    assert all(vals[i] >= vals[got[2500]] for i in got[2501:])


def test_partition_at_the_order_by_scale(am, oracle):
    rng = np.random.default_rng(20260906 + 2)
    n = 50_000_000
    arr = pa.array(rng.integers(0, 2**40, n, dtype=np.int64), mask=rng.random(n) < 0.10)
    m = am.MetalArray.from_arrow(arr)
    for pivot in (0, n // 2, n - 1):
        got = np_of(m.partition_nth_indices(pivot))
        assert np.array_equal(got, oracle.partition_nth(arr, pivot)), pivot


# ---- rank

@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("placement", PLACEMENTS)
@pytest.mark.parametrize("desc", [False, True])
def test_rank_every_option(am, oracle, kind, placement, desc):
    rng = rng_for("rank", kind, placement, desc)
    arr = column(rng, kind, 200_003)
    m = am.MetalArray.from_arrow(arr)
    sk = "descending" if desc else "ascending"
    for tb in TIEBREAKERS:
        got = np_of(m.rank(sort_keys=sk, null_placement=placement, tiebreaker=tb))
        assert got.dtype == np.uint32
        assert np.array_equal(got, oracle.rank(arr, tb, desc, placement)), tb
        want = pc.rank(arr, sort_keys=sk, null_placement=placement, tiebreaker=tb).to_numpy()
        assert np.array_equal(got, want), tb


def test_rank_floats_with_nan_small(am):
    v = pa.array([1.0, float("nan"), None, -0.0, 0.0, 2.5, float("nan")], type=pa.float64())
    m = am.MetalArray.from_arrow(v)
    for sk in ("ascending", "descending"):
        for placement in PLACEMENTS:
            for tb in TIEBREAKERS:
                got = np_of(m.rank(sort_keys=sk, null_placement=placement, tiebreaker=tb)).tolist()
                assert got == pc.rank(v, sort_keys=sk, null_placement=placement, tiebreaker=tb).to_pylist()


def test_rank_strings_and_edges(am):
    rng = rng_for("rank-str")
    words = ["", "a", "ab", "abc", "b", None, "zz", "héllo", "日本"]
    arr = pa.array([words[int(i)] for i in rng.integers(0, len(words), 20_000)])
    m = am.MetalArray.from_arrow(arr)
    for tb in TIEBREAKERS:
        for placement in PLACEMENTS:
            got = np_of(m.rank(null_placement=placement, tiebreaker=tb))
            assert np.array_equal(got, pc.rank(arr, null_placement=placement, tiebreaker=tb).to_numpy())
    assert len(am.MetalArray.from_arrow(pa.array([], type=pa.int32())).rank().to_arrow()) == 0
    with pytest.raises(am.ArrowMetalError):
        m.rank(tiebreaker="coin_toss")
    with pytest.raises(am.ArrowMetalError):
        m.rank(sort_keys="sideways")


@pytest.mark.parametrize("kind", ["int64_dups", "float64"])
@pytest.mark.parametrize("placement", PLACEMENTS)
@pytest.mark.parametrize("desc", [False, True])
def test_rank_quantile_and_normal(am, oracle, kind, placement, desc):
    rng = rng_for("quantile", kind, placement, desc)
    arr = column(rng, kind, 100_000)
    m = am.MetalArray.from_arrow(arr)
    sk = "descending" if desc else "ascending"
    q = np_of(m.rank_quantile(sort_keys=sk, null_placement=placement))
    assert np.array_equal(q, oracle.rank_quantile(arr, desc, placement))      # (s + e) / 2n, correctly rounded
    want = pc.rank_quantile(arr, sort_keys=sk, null_placement=placement).to_numpy()
    assert np.allclose(q, want, rtol=0, atol=1e-15)
    want_n = pc.rank_normal(arr, sort_keys=sk, null_placement=placement).to_numpy()
    got_n = np_of(m.rank_normal(sort_keys=sk, null_placement=placement))
    assert got_n.dtype == np.float64 and np.allclose(got_n, want_n, rtol=0, atol=1e-12)
    got_f = np_of(m.rank_normal(sort_keys=sk, null_placement=placement, float32=True))
    assert got_f.dtype == np.float32 and np.allclose(got_f, want_n, rtol=0, atol=2e-5)


@pytest.mark.parametrize("kind", ["int64_dups", "float64", "bool"])
def test_window_rankings(am, oracle, kind):
    rng = rng_for("window", kind)
    arr = column(rng, kind, 150_000)
    m = am.MetalArray.from_arrow(arr)
    for op in ("row_number", "rank", "dense_rank", "percent_rank", "cume_dist"):
        got = np_of(m.window(op))
        assert np.array_equal(got, oracle.window(arr, op)), op
    # row_number and rank are Arrow's rank with ties "first" / "min" when NaN sits apart from the nulls.
    if kind != "float64":
        assert np.array_equal(np_of(m.row_number()), pc.rank(arr, tiebreaker="first").to_numpy())
        assert np.array_equal(np_of(m.window("rank")), pc.rank(arr, tiebreaker="min").to_numpy())
    with pytest.raises(am.ArrowMetalError):
        m.window("lag")


# ---- unique / value_counts

@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("order", ["first_appearance", "sorted"])
def test_unique_and_value_counts(am, oracle, kind, order):
    rng = rng_for("unique", kind, order)
    arr = column(rng, kind, 250_000)
    m = am.MetalArray.from_arrow(arr)
    rows, counts = oracle.unique_rows(arr, order)
    want_values = arr.take(pa.array(rows, type=pa.int64()))
    got = m.unique(order).to_arrow()
    assert same_bits(got, want_values)
    vc = m.value_counts(order).to_arrow()
    assert vc.type == pa.struct([("values", arr.type), ("counts", pa.int64())])
    assert same_bits(vc.field("values"), want_values)
    assert np.array_equal(vc.field("counts").to_numpy(), counts)
    if order == "first_appearance" and not kind.startswith("float"):
        # Arrow's own answer (pyarrow keeps -0.0 apart from 0.0; the sort's equality does not).
        assert got.equals(pc.unique(arr))
        assert vc.equals(pc.value_counts(arr))


def test_unique_strings_and_edges(am):
    arr = pa.array(["pear", "apple", None, "pear", "fig", None, "apple", ""])
    m = am.MetalArray.from_arrow(arr)
    assert m.unique().to_arrow().to_pylist() == ["pear", "apple", "fig", ""]
    assert m.unique("sorted").to_arrow().to_pylist() == ["", "apple", "fig", "pear"]
    assert m.value_counts().to_arrow().to_pylist() == [
        {"values": "pear", "counts": 2}, {"values": "apple", "counts": 2}, {"values": "fig", "counts": 1},
        {"values": "", "counts": 1}]
    allnull = am.MetalArray.from_arrow(pa.array([None, None], type=pa.int64()))
    assert allnull.unique().to_arrow().to_pylist() == [None]
    assert allnull.unique("sorted").to_arrow().to_pylist() == []
    assert allnull.value_counts().to_arrow().to_pylist() == [{"values": None, "counts": 2}]
    empty = am.MetalArray.from_arrow(pa.array([], type=pa.float64()))
    assert len(empty.unique().to_arrow()) == 0 and len(empty.value_counts("sorted").to_arrow()) == 0
    f = am.MetalArray.from_arrow(pa.array([-0.0, float("nan"), 0.0, 1.0, float("nan"), None]))
    assert f.unique("sorted").to_arrow().to_pylist()[:2] == [-0.0, 1.0]
    assert np.signbit(f.unique("sorted").to_arrow().to_numpy()[0])
    assert f.value_counts().to_arrow().field("counts").to_pylist() == [2, 2, 1, 1]
    with pytest.raises(am.ArrowMetalError):
        m.unique("random")
    with pytest.raises(am.ArrowMetalError, match="struct"):
        m.value_counts().argsort()


def test_unique_large_strings(am):
    rng = rng_for("unique-lstr")
    words = [bytes(rng.integers(0, 4, int(k)).astype(np.uint8)) for k in rng.integers(0, 12, 300)]
    arr = pa.array([words[int(i)] if rng.random() > 0.05 else None for i in rng.integers(0, 300, 100_000)],
                   type=pa.large_binary())
    m = am.MetalArray.from_arrow(arr)
    vals = arr.to_pylist()
    seen = {}
    for v in vals:
        if v is not None:
            seen[v] = seen.get(v, 0) + 1
    assert m.unique().to_arrow().to_pylist() == list(seen)
    assert m.unique("sorted").to_arrow().to_pylist() == sorted(seen)
    vc = m.value_counts("sorted").to_arrow()
    assert vc.field("counts").to_pylist() == [seen[k] for k in sorted(seen)]
