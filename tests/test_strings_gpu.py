"""String and binary columns (utf8 / binary, large_utf8 / large_binary): import and export, argsort in
Arrow's byte order (a prefix before its extensions, ties in row order) at any key length, take, lexsort
with mixed keys, plan sorts, batches, top-k -- all against pyarrow on the same inputs."""
import numpy as np
import pyarrow as pa
import pyarrow.compute as pc
import pytest

pytestmark = pytest.mark.gpu

PLACEMENTS = ("at_end", "at_start")


def ids(m):
    return m.to_arrow().to_numpy(zero_copy_only=False)


def random_bytes(rng, n, max_len=40, alphabet=b"ab\x00\xff", null_frac=0.1):
    """Short strings over a tiny alphabet: many shared prefixes, ties, embedded zero bytes."""
    out = []
    for i in range(n):
        if rng.random() < null_frac:
            out.append(None)
            continue
        k = int(rng.integers(0, max_len + 1))
        out.append(bytes(alphabet[j] for j in rng.integers(0, len(alphabet), k)))
    return out


def random_text(rng, n, max_len=30, null_frac=0.1):
    words = ["", "a", "ab", "abc", "b", "ba", "zz", "héllo", "hello", "hello world", "日本", "日本語", "Z", "aa"]
    out = []
    for i in range(n):
        if rng.random() < null_frac:
            out.append(None)
        elif rng.random() < 0.5:
            out.append(words[int(rng.integers(len(words)))])
        else:
            k = int(rng.integers(0, max_len))
            out.append("".join(chr(int(c)) for c in rng.integers(32, 127, k)))
    return out


@pytest.mark.parametrize("typ", [pa.binary(), pa.large_binary(), pa.utf8(), pa.large_utf8()])
def test_round_trip_and_slices(am, typ):
    rng = np.random.default_rng(1)
    vals = random_bytes(rng, 5000) if typ in (pa.binary(), pa.large_binary()) else random_text(rng, 5000)
    arr = pa.array(vals, type=typ)
    m = am.MetalArray.from_arrow(arr)
    assert m.to_arrow().equals(arr)
    for off, ln in [(0, 0), (7, 100), (4999, 1), (123, 3000)]:
        assert am.MetalArray.from_arrow(arr.slice(off, ln)).to_arrow().equals(arr.slice(off, ln))
        assert m.slice(off, ln).to_arrow().equals(arr.slice(off, ln))


@pytest.mark.parametrize("typ", [pa.binary(), pa.large_utf8()])
@pytest.mark.parametrize("desc", [False, True])
@pytest.mark.parametrize("placement", PLACEMENTS)
def test_argsort_matches_pyarrow(am, typ, desc, placement):
    rng = np.random.default_rng(2 + desc)
    n = 200_003
    vals = random_bytes(rng, n) if typ == pa.binary() else random_text(rng, n)
    arr = pa.array(vals, type=typ)
    got = ids(am.MetalArray.from_arrow(arr).argsort(desc, placement))
    want = pc.array_sort_indices(arr, order="descending" if desc else "ascending", null_placement=placement).to_numpy()
    assert np.array_equal(got, want)


def test_prefixes_and_zero_bytes(am):
    vals = [b"ab", b"ab\x00", b"a", b"", b"ab\x00\x00", b"ab\x01", None, b"b", b"ab", b"\x00", b"\x00\x00",
            b"abcdefgh", b"abcdefgh\x00", b"abcdefg", b"abcdefghi", b"abcdefgh"]
    arr = pa.array(vals, type=pa.binary())
    for desc in (False, True):
        for placement in PLACEMENTS:
            got = ids(am.MetalArray.from_arrow(arr).argsort(desc, placement))
            want = pc.array_sort_indices(arr, order="descending" if desc else "ascending",
                                         null_placement=placement).to_numpy()
            assert np.array_equal(got, want), (desc, placement)


def test_take_strings(am):
    rng = np.random.default_rng(3)
    arr = pa.array(random_text(rng, 100_000), type=pa.utf8())
    idx = pa.array(rng.integers(0, len(arr), 150_000), mask=rng.random(150_000) < 0.05)
    got = am.MetalArray.from_arrow(arr).take(idx).to_arrow()
    assert got.equals(pc.take(arr, idx))
    with pytest.raises(am.ArrowMetalError, match="out of range"):
        am.MetalArray.from_arrow(arr).take(pa.array([0, len(arr)], type=pa.int64())).to_arrow()


def test_lexsort_with_string_keys(am):
    rng = np.random.default_rng(4)
    n = 100_000
    s = pa.array(random_bytes(rng, n, max_len=6, alphabet=b"ab"), type=pa.binary())
    k = pa.array(rng.integers(0, 5, n), mask=rng.random(n) < 0.1)
    t = pa.table({"s": s, "k": k})
    for keys in ([("s", "ascending"), ("k", "descending")], [("k", "ascending"), ("s", "descending")]):
        for placement in PLACEMENTS:
            cols = [t[c].combine_chunks() for c, _ in keys]
            got = ids(am.lexsort_indices(cols, descending=[o == "descending" for _, o in keys],
                                         null_placement=placement))
            want = pc.sort_indices(t, keys, null_placement=placement).to_numpy()
            assert np.array_equal(got, want), (keys, placement)


def test_plan_order_by_string_key_and_payload(am):
    rng = np.random.default_rng(5)
    n = 120_000
    t = pa.table({"name": pa.array(random_text(rng, n), type=pa.utf8()),
                  "v": pa.array(rng.standard_normal(n)),
                  "tag": pa.array(random_bytes(rng, n, max_len=4), type=pa.large_binary())})
    src = am.PlanSource("t", {c: t[c].combine_chunks() for c in t.column_names})
    for by, order in [("name", "ascending"), ("tag", "descending")]:
        plan = {"op": "sort", "by": [[by, order == "descending", {"nulls": "last"}]],
                "input": {"op": "scan", "source": "t"}}
        out = am.run_plan(plan, [src])
        want = t.take(pc.sort_indices(t, [(by, order)], null_placement="at_end"))
        for c in t.column_names:
            assert out[c].to_arrow().equals(want[c].combine_chunks()), (by, c)
        lim = am.run_plan({"op": "limit", "count": 100, "offset": 5, "input": plan}, [src])
        for c in t.column_names:
            assert lim[c].to_arrow().equals(want[c].combine_chunks().slice(5, 100)), (by, c)


def test_batch_top_k_and_sorted_copy(am):
    rng = np.random.default_rng(6)
    arrays = [pa.array(random_text(rng, 30_000), type=pa.utf8()), pa.array(rng.integers(0, 9, 5000)),
              pa.array(random_bytes(rng, 7), type=pa.binary())]
    outs = am.argsort_batch([am.MetalArray.from_arrow(a) for a in arrays])
    for a, o in zip(arrays, outs):
        assert np.array_equal(ids(o), pc.array_sort_indices(a).to_numpy())
    arr = arrays[0]
    m = am.MetalArray.from_arrow(arr)
    full = pc.array_sort_indices(arr, order="descending").to_numpy()
    assert np.array_equal(ids(m.top_k(50, True)), full[:50])
    assert m.sort(True).to_arrow().equals(arr.take(pa.array(full)))


def long_strings(rng, n, max_len=600, null_frac=0.05):
    """Strings past 120 bytes that share long prefixes: a few long stems, then short random tails."""
    stems = [bytes(rng.integers(97, 100, int(k)).astype(np.uint8)) for k in (0, 100, 119, 120, 121, 250, 500)]
    out = []
    for _ in range(n):
        if rng.random() < null_frac:
            out.append(None)
            continue
        stem = stems[int(rng.integers(len(stems)))]
        tail = bytes(rng.integers(0, 3, int(rng.integers(0, 12))).astype(np.uint8))
        out.append((stem + tail)[:max_len])
    return out


@pytest.mark.parametrize("typ", [pa.binary(), pa.large_utf8()])
@pytest.mark.parametrize("desc", [False, True])
@pytest.mark.parametrize("placement", PLACEMENTS)
def test_keys_longer_than_sixteen_chunks(am, typ, desc, placement):
    # More than 15 chunks: the key sorts in chained groups of 16 derived keys.
    rng = np.random.default_rng(7 + desc)
    vals = long_strings(rng, 60_000)
    if typ == pa.large_utf8():
        vals = [None if v is None else v.decode("latin-1") for v in vals]
    arr = pa.array(vals, type=typ)
    got = ids(am.MetalArray.from_arrow(arr).argsort(desc, placement))
    want = pc.array_sort_indices(arr, order="descending" if desc else "ascending", null_placement=placement).to_numpy()
    assert np.array_equal(got, want)


def test_long_keys_in_lexsort_plans_and_batches(am):
    rng = np.random.default_rng(8)
    n = 40_000
    s = pa.array(long_strings(rng, n, max_len=300), type=pa.binary())
    k = pa.array(rng.integers(0, 4, n), mask=rng.random(n) < 0.1)
    t = pa.table({"s": s, "k": k})
    for keys in ([("s", "ascending"), ("k", "descending")], [("k", "ascending"), ("s", "descending")]):
        cols = [t[c].combine_chunks() for c, _ in keys]
        got = ids(am.lexsort_indices(cols, descending=[o == "descending" for _, o in keys], null_placement="at_start"))
        want = pc.sort_indices(t, keys, null_placement="at_start").to_numpy()
        assert np.array_equal(got, want), keys
    outs = am.argsort_batch([am.MetalArray.from_arrow(s), am.MetalArray.from_arrow(k)])
    assert np.array_equal(ids(outs[0]), pc.array_sort_indices(s).to_numpy())
    src = am.PlanSource("t", {"s": s, "k": k})
    out = am.run_plan({"op": "sort", "by": [["s", False, {"nulls": "last"}]], "input": {"op": "scan", "source": "t"}},
                      [src])
    assert out["s"].to_arrow().equals(s.take(pc.array_sort_indices(s)))
    m = am.MetalArray.from_arrow(s)
    assert np.array_equal(ids(m.top_k(100, False)), pc.array_sort_indices(s).to_numpy()[:100])
    assert np.array_equal(ids(m.rank(tiebreaker="dense")), pc.rank(s, tiebreaker="dense").to_numpy())


def test_null_slots_that_span_bytes_keep_row_order(am):
    # Arrow lets a null row's slot cover bytes; the sort must still tie the null rows.
    vals = [b"zz", b"b", b"a", b"q", b"c", b"aa"]
    offsets = np.array([0, 2, 3, 4, 5, 6, 8], dtype=np.int32)
    data = b"".join(vals)
    valid = np.array([1, 0, 1, 0, 0, 1], dtype=np.uint8)
    arr = pa.Array.from_buffers(pa.binary(), 6, [pa.py_buffer(np.packbits(valid, bitorder="little").tobytes()),
                                                 pa.py_buffer(offsets.tobytes()), pa.py_buffer(data)], null_count=3)
    for desc in (False, True):
        for placement in PLACEMENTS:
            got = ids(am.MetalArray.from_arrow(arr).argsort(desc, placement))
            want = pc.array_sort_indices(arr, order="descending" if desc else "ascending",
                                         null_placement=placement).to_numpy()
            assert np.array_equal(got, want), (desc, placement)
