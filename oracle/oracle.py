"""CPU oracle of the full-sort path -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this module; the
product (``arrowmetal_b200`` and ``libArrowMetalC.so``) never does.

Two independent restatements of ArrowMetal 0.6.1's sort semantics:

* ``argsort`` / ``lexsort`` / ``take`` call ``liboracle.so`` (``sort_oracle.c``), a C restatement of the
  reference's Metal algorithm: key maps (Sources/ArrowMetal/Kernels/SortSource.swift:131-190), stable
  three-way partition (SortSource.swift:226-330), 8-bit LSD passes with constant-digit skipping
  (Sort.swift:404-494), lexsort by take + argsort + compose (Kernels/MultiSort.swift:56-64), take with
  null indices and range errors (Kernels/Take.swift:41-79).
* ``np_argsort`` / ``np_lexsort`` restate the same orders from their definitions with numpy's stable
  sort (the reference's CPU reference of SortOptionsTests.swift:15-62 and the ``total_order_indices``
  oracle of python/tests/test_sort_options.py:58-76).

Both are pinned by the reference's known-answer vectors (tests/test_oracle.py) and by pyarrow's own
``sort_indices`` / ``take`` (the reference's oracle for the ieee order) through the fixtures in
tests/golden/.
"""
import ctypes
import os
import subprocess

import numpy as np
import pyarrow as pa

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

PT = {"bool": 0, "int8": 1, "uint8": 2, "int16": 3, "uint16": 4, "int32": 5, "uint32": 6,
      "int64": 7, "uint64": 8, "halffloat": 9, "float": 10, "double": 11}
FLOAT_ORDERS = {"ieee": 0, "total": 1, "nan_largest": 2}

_lib = None


def build():
    """Compiles liboracle.so with gcc (the oracle's own Makefile)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P, I64, I = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
        L.oracle_argsort.argtypes = [P, P, I64, I64, I64, I, I, I, I, P, I]
        L.oracle_take.argtypes = [P, P, I64, I64, I64, I, P, I, P, I64, I64, P, P]
        L.oracle_lexsort.argtypes = [I, P, P, P, P, P, P, P, P, I64, P, I]
        _lib = L
    return _lib


def _physical(arr):
    """(pt code, values address, validity address or 0, offset, byte width, keep-alive) of a pyarrow
    primitive array, read straight from its buffers (temporal types by their integer storage)."""
    t = arr.type
    if pa.types.is_timestamp(t) or pa.types.is_date64(t) or pa.types.is_time64(t) or pa.types.is_duration(t):
        storage = "int64"
    elif pa.types.is_date32(t) or pa.types.is_time32(t):
        storage = "int32"
    elif pa.types.is_boolean(t):
        storage = "bool"
    else:
        storage = str(t)   # 'int8' ... 'uint64', 'halffloat', 'float', 'double'
    if storage not in PT:
        raise TypeError(f"oracle: type {t} is not on the sort path")
    bufs = arr.buffers()
    vb = bufs[0] if arr.null_count > 0 else None
    width = {0: 0, 1: 1, 2: 1, 3: 2, 4: 2, 5: 4, 6: 4, 7: 8, 8: 8, 9: 2, 10: 4, 11: 8}[PT[storage]]
    return PT[storage], bufs[1].address, (vb.address if vb is not None else 0), arr.offset, width, bufs


def _as_array(a):
    """A plain array: chunks combined, and a dictionary array decoded -- the reference orders a dictionary
    column by its decoded values (Sources/ArrowMetal/Kernels/MultiSort.swift:124-133)."""
    if isinstance(a, pa.ChunkedArray):
        a = a.combine_chunks()
    if pa.types.is_dictionary(a.type):
        a = a.dictionary_decode()
    return a


def argsort(arr, descending=False, null_placement="at_end", float_order="ieee", threads=1):
    """uint32 indices of Arrow's stable array_sort_indices, by the C restatement."""
    arr = _as_array(arr)
    n = len(arr)
    out = np.empty(max(n, 1), dtype=np.uint32)
    pt, va, vb, off, width, keep = _physical(arr)
    # Values are addressed from element 0 of the buffer: fold the array offset into the address.
    vaddr = va + off * width if width else va
    boff = off if width == 0 else 0
    lib().oracle_argsort(vaddr, vb or None, off, boff, n, pt, int(bool(descending)),
                         1 if null_placement == "at_start" else 0, FLOAT_ORDERS[float_order],
                         out.ctypes.data, int(threads))
    del keep
    return out[:n]


def lexsort(arrays, descending=None, null_placement="at_end", float_order="ieee", threads=1):
    """uint32 indices of Arrow's multi-key sort_indices, by the C restatement (first key most
    significant); options are one value or one per key."""
    arrays = [_as_array(a) for a in arrays]
    K = len(arrays)
    n = len(arrays[0])
    desc = list(descending) if descending is not None else [False] * K
    place = [null_placement] * K if isinstance(null_placement, str) else list(null_placement)
    order = [float_order] * K if isinstance(float_order, str) else list(float_order)
    parts = [_physical(a) for a in arrays]
    P = ctypes.c_void_p * K
    I64 = ctypes.c_int64 * K
    Ia = ctypes.c_int * K
    vals = P(*[p[1] + (a.offset * p[4] if p[4] else 0) for p, a in zip(parts, arrays)])
    valid = P(*[p[2] or None for p in parts])
    voff = I64(*[a.offset for a in arrays])
    boff = I64(*[(a.offset if p[4] == 0 else 0) for p, a in zip(parts, arrays)])
    pts = Ia(*[p[0] for p in parts])
    out = np.empty(max(n, 1), dtype=np.uint32)
    lib().oracle_lexsort(K, vals, valid, voff, boff, pts, Ia(*[int(bool(d)) for d in desc]),
                         Ia(*[1 if p == "at_start" else 0 for p in place]),
                         Ia(*[FLOAT_ORDERS[f] for f in order]), n, out.ctypes.data, 1 if threads is None else int(threads))
    return out[:n]


def take(arr, indices):
    """(values as a numpy array of the storage type / packed bits for bool, validity bool array) of
    Arrow's take, by the C restatement; raises IndexError for an index out of range."""
    arr = _as_array(arr)
    indices = _as_array(indices)
    pt, va, vb, off, width, keep = _physical(arr)
    it = indices.type
    kind = 0 if it == pa.uint32() else 1 if it == pa.int32() else 2
    if it not in (pa.uint32(), pa.int32(), pa.int64()):
        raise TypeError("take indices must be int32, int64 or uint32")
    ib = indices.buffers()
    iwidth = 4 if kind < 2 else 8
    n = len(indices)
    if width:
        out = np.zeros(max(n, 1), dtype={1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[width])
    else:
        out = np.zeros(max((n + 7) // 8, 1), dtype=np.uint8)
    outv = np.zeros(max(n, 1), dtype=np.uint8)
    ivb = ib[0].address if indices.null_count > 0 else None
    vaddr = va + off * width if width else va
    bad = lib().oracle_take(vaddr, vb or None, off, off if width == 0 else 0, len(arr), width,
                            ib[1].address + indices.offset * iwidth, kind, ivb, indices.offset, n,
                            out.ctypes.data, outv.ctypes.data)
    del keep
    if bad:
        raise IndexError("take: index out of range")
    return (out[:n] if width else out), outv[:n].astype(bool)


# ---- numpy restatement (independent of the C one) --------------------------------------------------

def _keys_and_categories(arr, descending, float_order):
    """Order-preserving keys (uint64) and categories (0 value, 1 NaN block, 2 null) of every row."""
    arr = _as_array(arr)
    n = len(arr)
    valid = np.ones(n, bool) if arr.null_count == 0 else np.asarray(arr.is_valid().to_numpy(zero_copy_only=False))
    t = arr.type
    cat = np.where(valid, 0, 2).astype(np.int8)
    if pa.types.is_floating(t):
        if t == pa.float16():
            raw = np.asarray(arr.cast(pa.float32()).fill_null(0).to_numpy(zero_copy_only=False), dtype=np.float32)
            t32 = True
        else:
            raw = np.asarray(arr.fill_null(0).to_numpy(zero_copy_only=False))
            t32 = t == pa.float32()
        bits = raw.view(np.uint32).astype(np.uint64) if t32 else raw.view(np.uint64).copy()
        width = 32 if t32 else 64
        S = np.uint64(1 << (width - 1))
        full = np.uint64((1 << width) - 1)
        expmask = np.uint64(0x7F800000 if t32 else 0x7FF0000000000000)
        mag = bits & ~S & full
        nan = mag > expmask
        if float_order != "total":
            bits = np.where(mag == 0, np.uint64(0), bits)
            bits = np.where(nan, np.uint64(0x7F800001 if t32 else 0x7FF0000000000001), bits)
            if float_order == "ieee":
                cat = np.where(valid & nan, 1, cat).astype(np.int8)
        key = np.where(bits & S, ~bits & full, bits | S)
        if descending:
            key = ~key & full
        return key.astype(np.uint64), cat
    if pa.types.is_boolean(t):
        v = np.asarray(arr.fill_null(False).to_numpy(zero_copy_only=False)).astype(np.int64)
        key = (v.astype(np.int64) + (1 << 31)).astype(np.uint64)
        full = np.uint64(0xFFFFFFFF)
    else:
        storage = arr
        if pa.types.is_temporal(t):
            storage = arr.view(pa.int64() if t.bit_width == 64 else pa.int32())
        v = np.asarray(storage.fill_null(0).to_numpy(zero_copy_only=False))
        if v.dtype == np.uint64:
            key, full = v.astype(np.uint64), np.uint64(0xFFFFFFFFFFFFFFFF)
        elif v.dtype == np.int64:
            key, full = v.view(np.uint64) ^ np.uint64(1 << 63), np.uint64(0xFFFFFFFFFFFFFFFF)
        elif v.dtype == np.uint32:
            key, full = v.astype(np.uint64), np.uint64(0xFFFFFFFF)
        else:  # narrow integers widen to int32
            key = (v.astype(np.int64) + (1 << 31)).astype(np.uint64)
            full = np.uint64(0xFFFFFFFF)
    if descending:
        key = ~key & full
    return key, cat


def np_argsort(arr, descending=False, null_placement="at_end", float_order="ieee"):
    arr = _as_array(arr)
    key, cat = _keys_and_categories(arr, descending, float_order)
    order = np.argsort(key, kind="stable")
    vals = order[cat[order] == 0]
    nans = np.nonzero(cat == 1)[0]
    nulls = np.nonzero(cat == 2)[0]
    parts = [nulls, nans, vals] if null_placement == "at_start" else [vals, nans, nulls]
    return np.concatenate(parts).astype(np.uint32)


def np_lexsort(arrays, descending=None, null_placement="at_end", float_order="ieee"):
    """Multi-key order from the definition: per key a (category, key) pair, compared lexicographically
    over the keys, ties broken by row number."""
    K = len(arrays)
    desc = list(descending) if descending is not None else [False] * K
    place = [null_placement] * K if isinstance(null_placement, str) else list(null_placement)
    order = [float_order] * K if isinstance(float_order, str) else list(float_order)
    cols = []
    for a, d, p, f in zip(arrays, desc, place, order):
        key, cat = _keys_and_categories(_as_array(a), d, f)
        rank = np.where(cat == 0, 2, np.where(cat == 1, 1, 0)) if p == "at_start" else cat
        key = np.where(cat == 0, key, np.uint64(0))
        cols.append((rank.astype(np.int64), key))
    # np.lexsort sorts by the last key first; give it (least significant ... most significant).
    seq = []
    for rank, key in reversed(cols):
        seq.extend([key, rank])
    n = len(arrays[0])
    if n == 0:
        return np.empty(0, np.uint32)
    return np.lexsort(seq).astype(np.uint32)


# ---- sort consumers (numpy, on the orders above) ----------------------------------------------------
#
# Rank, the window rankings, unique / value_counts and partition_nth_indices restated from their
# definitions over np_argsort's order: a run is a maximal block of sorted positions whose rows are equal
# under the sort's value equality (same category; same key for a value row -- so -0.0 ties +0.0 and
# every NaN is one value). The reference builds these on its argsort the same way
# (Sources/ArrowMetal/Kernels/Window.swift:65-200, Kernels/Unique.swift:46-65,
# Kernels/UniqueOrder.swift:88-140, Kernels/PartitionNth.swift:215-235).

def _run_starts(arr, order, merge_nan):
    """True at each sorted position that starts a run. merge_nan: NaN rows and nulls are one run."""
    key, cat = _keys_and_categories(arr, False, "ieee")
    k = key[order]
    c = cat[order].copy()
    if merge_nan:
        c[c == 1] = 2
    start = np.ones(len(order), bool)
    start[1:] = (c[1:] != c[:-1]) | ((c[1:] == 0) & (k[1:] != k[:-1]))
    return start


def _rank_positions(arr, descending, null_placement, merge_nan):
    """(sorted order, run number per sorted position (1-based), first and one-past-last position of
    each position's run)."""
    order = np_argsort(arr, descending, null_placement).astype(np.int64)
    n = len(order)
    start = _run_starts(arr, order, merge_nan)
    run = np.cumsum(start)
    starts = np.nonzero(start)[0]
    ends = np.append(starts[1:], n)
    return order, run, starts[run - 1], ends[run - 1]


def rank(arr, tiebreaker="min", descending=False, null_placement="at_end"):
    """Arrow rank (pyarrow.compute.rank; the reference's am_rank_ex): 1-based ranks at the original rows,
    the nulls and NaN rows one tie group at the null_placement end; uint32."""
    arr = _as_array(arr)
    n = len(arr)
    if n == 0:
        return np.empty(0, np.uint32)
    order, run, s, e = _rank_positions(arr, descending, null_placement, True)
    val = {"min": s + 1, "max": e, "first": np.arange(1, n + 1), "dense": run}[tiebreaker]
    out = np.empty(n, np.uint32)
    out[order] = val
    return out


def rank_quantile(arr, descending=False, null_placement="at_end"):
    """Arrow rank_quantile: (s + e) / 2n over the row's run [s, e) of sorted positions, float64 (the
    run's average 1-based rank minus one half, over n)."""
    arr = _as_array(arr)
    n = len(arr)
    if n == 0:
        return np.empty(0, np.float64)
    order, run, s, e = _rank_positions(arr, descending, null_placement, True)
    out = np.empty(n, np.float64)
    out[order] = (s + e).astype(np.float64) / np.float64(2 * n)
    return out


def window(arr, op):
    """The SQL ranking window functions of am_window (ops 0-4): ascending, nulls last and one tie group,
    every NaN one value after +inf (include/arrowmetal.h:415-434 of the reference)."""
    arr = _as_array(arr)
    n = len(arr)
    if n == 0:
        return np.empty(0, np.float64 if op in ("percent_rank", "cume_dist") else np.uint32)
    order, run, s, e = _rank_positions(arr, False, "at_end", False)
    if op == "row_number":
        val, dt = np.arange(1, n + 1), np.uint32
    elif op == "rank":
        val, dt = s + 1, np.uint32
    elif op == "dense_rank":
        val, dt = run, np.uint32
    elif op == "percent_rank":
        val, dt = (s.astype(np.float64) / np.float64(n - 1)) if n > 1 else np.zeros(n), np.float64
    else:
        val, dt = e.astype(np.float64) / np.float64(n), np.float64
    out = np.empty(n, dt)
    out[order] = val
    return out


def unique_rows(arr, order="first_appearance"):
    """(representative rows, counts) of Arrow unique / value_counts: one row per distinct value, the
    earliest row carrying it. "sorted": ascending, nulls dropped; "first_appearance": in order of the
    representatives, with one null entry when there are nulls (not for string columns)."""
    arr = _as_array(arr)
    n = len(arr)
    is_str = pa.types.is_string(arr.type) or pa.types.is_binary(arr.type) or \
        pa.types.is_large_string(arr.type) or pa.types.is_large_binary(arr.type)
    if is_str:
        vals = arr.to_pylist()
        ordered = sorted((v, i) for i, v in enumerate(vals) if v is not None)
        heads, counts = [], []
        for v, i in ordered:
            if heads and vals[heads[-1]] == v:
                counts[-1] += 1
            else:
                heads.append(i)
                counts.append(1)
        heads, counts = np.array(heads, np.int64), np.array(counts, np.int64)
    else:
        srt = np_argsort(arr, False, "at_end").astype(np.int64)
        m = n if order == "first_appearance" else n - arr.null_count
        srt = srt[:m]
        if m == 0:
            return np.empty(0, np.int64), np.empty(0, np.int64)
        start = _run_starts(arr, srt, False)
        starts = np.nonzero(start)[0]
        heads = srt[starts]
        counts = np.diff(np.append(starts, m))
    if order == "first_appearance":
        o = np.argsort(heads, kind="stable")
        heads, counts = heads[o], counts[o]
    return heads, counts


def partition_nth(arr, pivot, null_placement="at_end"):
    """Arrow partition_nth_indices as the reference arranges it (Kernels/PartitionNth.swift:215-235):
    the rows ordered before the pivot row of the ascending stable argsort, then the rows equal to it,
    then the rest, each block in row order; uint32."""
    arr = _as_array(arr)
    n = len(arr)
    if n == 0:
        return np.empty(0, np.uint32)
    key, cat = _keys_and_categories(arr, False, "ieee")
    place = (2 - cat) if null_placement == "at_start" else cat.astype(np.int64)
    order = np_argsort(arr, False, null_placement)
    p = order[min(pivot, n - 1)]
    P, K = place[p], key[p]
    value = cat == 0
    before = (place < P) | ((place == P) & value & (key < K))
    equal = (place == P) & (~value | (key == K))
    rows = np.arange(n)
    return np.concatenate([rows[before], rows[equal], rows[~before & ~equal]]).astype(np.uint32)
