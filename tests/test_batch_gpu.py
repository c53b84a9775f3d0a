"""Segmented (batched) argsort, am_argsort_batch: every array's permutation must be identical to the
C oracle's argsort of that array with its options, and to am_argsort_ex2 on that array alone
(bit-exact), for mixed key types and widths, per-array options, empty, one-row, all-null and
tile-edge lengths, and the batch shape of the segmented benchmark (log-uniform lengths, int64 and
float32 alternating)."""
import numpy as np
import pyarrow as pa
import pytest

from conftest import build_array

pytestmark = pytest.mark.gpu

PLACEMENTS = ("at_end", "at_start")
ORDERS = ("ieee", "total", "nan_largest")


def ids(m):
    return m.to_arrow().to_numpy(zero_copy_only=False)


def random_array(rng, kind, n):
    nulls = rng.random(n) < rng.choice([0.0, 0.02, 0.3, 1.0], p=[0.4, 0.3, 0.25, 0.05])
    valid = ~nulls if nulls.any() else None
    if kind == "int64":
        v = rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n, dtype=np.int64, endpoint=True)
    elif kind == "int64_small":
        v = rng.integers(0, 50, n, dtype=np.int64)
    elif kind == "uint64":
        v = rng.integers(0, 2**64 - 1, n, dtype=np.uint64, endpoint=True)
    elif kind == "float64":
        v = rng.standard_normal(n)
        v[rng.random(n) < 0.03] = np.nan
        v[rng.random(n) < 0.03] = -0.0
    elif kind == "float32":
        v = rng.standard_normal(n).astype(np.float32)
        v[rng.random(n) < 0.03] = np.float32("nan")
    elif kind == "int32":
        v = rng.integers(-2**31, 2**31 - 1, n, dtype=np.int32, endpoint=True)
    elif kind == "uint16":
        v = rng.integers(0, 2**16, n).astype(np.uint16)
    elif kind == "int8":
        v = rng.integers(-128, 128, n).astype(np.int8)
    elif kind == "float16":
        v = rng.standard_normal(n).astype(np.float16)
    elif kind == "bool":
        return pa.array(rng.random(n) < 0.5, mask=None if valid is None else ~valid)
    else:
        raise AssertionError(kind)
    t = {"int64": "int64", "int64_small": "int64", "uint64": "uint64", "float64": "double", "float32": "float",
         "int32": "int32", "uint16": "uint16", "int8": "int8", "float16": "halffloat"}[kind]
    return build_array(t, v, valid)


def check_batch(am, oracle, arrays, opts):
    handles = [am.MetalArray.from_arrow(a) for a in arrays]
    desc = [o[0] for o in opts]
    place = [o[1] for o in opts]
    order = [o[2] for o in opts]
    outs = am.argsort_batch(handles, desc, place, order)
    assert len(outs) == len(arrays)
    for i, (h, o) in enumerate(zip(handles, outs)):
        got = ids(o)
        assert got.dtype == np.uint32
        case = (i, arrays[i].type, len(arrays[i]), opts[i])
        assert np.array_equal(got, oracle.argsort(arrays[i], desc[i], place[i], order[i])), case
        assert np.array_equal(got, ids(h.argsort(desc[i], place[i], order[i]))), case


KINDS = ["int64", "int64_small", "uint64", "float64", "float32", "int32", "uint16", "int8", "float16", "bool"]


def test_mixed_batch(am, oracle):
    rng = np.random.default_rng(101)
    lengths = [0, 1, 2, 31, 4095, 4096, 4097, 8191, 12_289, 100_003, 1, 0, 777, 65_536, 250_000]
    arrays, opts = [], []
    for i, n in enumerate(lengths):
        kind = KINDS[i % len(KINDS)]
        arrays.append(random_array(rng, kind, n))
        opts.append((bool(rng.integers(2)), PLACEMENTS[rng.integers(2)], ORDERS[rng.integers(3)]))
    check_batch(am, oracle, arrays, opts)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_many_small_and_large(am, oracle, seed):
    rng = np.random.default_rng(seed)
    arrays, opts = [], []
    for i in range(300):
        n = int(round(10 ** rng.uniform(0, 5.3)))
        kind = KINDS[int(rng.integers(len(KINDS)))]
        arrays.append(random_array(rng, kind, n))
        opts.append((bool(rng.integers(2)), PLACEMENTS[rng.integers(2)], ORDERS[rng.integers(3)]))
    check_batch(am, oracle, arrays, opts)


def test_segmented_benchmark_shape(am, oracle):
    # The segmented benchmark's arrays, fewer of them: int64 full range and float32 N(0,1) with 2% nulls
    # alternating, lengths log-uniform in [1e3, 1e6], with every combination of the options.
    rng = np.random.default_rng(20260906 + 4)
    arrays = []
    for i in range(64):
        n = int(round(10 ** rng.uniform(3, 6)))
        if i % 2 == 0:
            arrays.append(pa.array(rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n, dtype=np.int64,
                                                endpoint=True)))
        else:
            arrays.append(pa.array(rng.standard_normal(n).astype(np.float32), mask=rng.random(n) < 0.02))
    opts = [(bool(i % 3 == 1), PLACEMENTS[i % 2], ORDERS[(i // 2) % 3]) for i in range(len(arrays))]
    check_batch(am, oracle, arrays, opts)


def test_all_null_and_constant_arrays(am, oracle):
    arrays = [pa.array([None] * 5000, type=pa.int64()), pa.array(np.full(9000, 7, dtype=np.int32)),
              pa.array([None] * 3, type=pa.float32()), pa.array(np.full(5000, np.nan))]
    opts = [(False, "at_start", "ieee"), (True, "at_end", "ieee"), (False, "at_end", "total"),
            (True, "at_start", "nan_largest")]
    check_batch(am, oracle, arrays, opts)


def test_empty_batch(am):
    assert am.argsort_batch([]) == []


def test_repeated_shapes_replay_a_graph(am, oracle):
    # The second batch of a shape (same key widths and lengths) is captured into a CUDA graph and
    # later ones replay it with their own columns, options and outputs: every call must still match
    # am_argsort_ex2. Two shapes alternate, so both graphs stay in use.
    # Each position keeps its key width (8 or 4 bytes) from call to call; its type within that width,
    # its values and its options change.
    rng = np.random.default_rng(77)
    wide, narrow = ["int64", "uint64", "float64"], ["int32", "float32", "uint16", "int8", "bool", "float16"]
    shape_a = [(5000, wide), (1, narrow), (70_000, narrow), (4096, wide), (300_001, narrow)]
    shape_b = [(123, narrow), (45_678, wide)]
    for call in range(4):
        for shape in (shape_a, shape_b):
            arrays, opts = [], []
            for n, kinds in shape:
                arrays.append(random_array(rng, kinds[int(rng.integers(len(kinds)))], n))
                opts.append((bool(rng.integers(2)), PLACEMENTS[rng.integers(2)], ORDERS[rng.integers(3)]))
            check_batch(am, oracle, arrays, opts)
    am.profile(True)
    am.profile_reset()
    check_batch(am, oracle, [random_array(rng, "int64", n) if k is wide else random_array(rng, "int32", n)
                     for n, k in shape_a], [(False, "at_end", "ieee")] * len(shape_a))
    assert "batch_graph" in am.profile_entries()
    am.profile(False)


@pytest.mark.parametrize("shape", range(7))
def test_every_candidate_shape_against_the_oracle(am, oracle, shape):
    # Each shape the autotuner may pick, forced for every size class it serves: digit passes over three
    # tile shapes, and one CTA per array with two block shapes and 8- or 4-bit digits.
    rng = np.random.default_rng(200 + shape)
    lengths = [0, 1, 2, 31, 32, 33, 255, 256, 1000, 2047, 2048, 4095, 4096, 4097, 9000, 16384, 16385, 70_001]
    arrays, opts = [], []
    for i, n in enumerate(lengths * 2):
        arrays.append(random_array(rng, KINDS[(i * 7 + shape) % len(KINDS)], n))
        opts.append((bool(rng.integers(2)), PLACEMENTS[rng.integers(2)], ORDERS[rng.integers(3)]))
    am._ok(am._lib.am_debug_force_batch_shape(shape))
    try:
        check_batch(am, oracle, arrays, opts)
        check_batch(am, oracle, arrays, opts)            # the second batch of a shape replays a graph
    finally:
        am._ok(am._lib.am_debug_force_batch_shape(-1))


def test_autotuner_records_its_choice_per_size_class(am, oracle):
    # Enough rows in every size class to tune it: the chosen shape is recorded per key width and class,
    # and the batch that tuned it (every candidate run on it) is still exact.
    rng = np.random.default_rng(300)
    arrays = [random_array(rng, "int64", n) for n in [3000] * 100 + [12_000] * 200 + [150_000] * 16]
    opts = [(False, "at_end", "ieee")] * len(arrays)
    check_batch(am, oracle, arrays, opts)
    shapes = {(s["key_bytes"], s["size_class"]): s for s in am.batch_tuning()}
    for c in range(3):
        s = shapes[(8, c)]
        assert s["method"] in (0, 1) and s["threads"] > 0 and s["items"] > 0 and s["digit_bits"] in (4, 8), s
        if s["method"] == 1:
            assert c == 0 and s["threads"] * s["items"] >= 4096
    assert shapes[(8, 0)]["max_rows"] == 4096 and shapes[(8, 2)]["max_rows"] == -1
    check_batch(am, oracle, arrays, opts)
