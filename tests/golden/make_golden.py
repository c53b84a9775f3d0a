"""Writes tests/golden/sort_golden.npz: seeded inputs and the answers the reference's oracle gives.

The reference checks its ieee-order sort against pyarrow (python/tests/test_sort_options.py:96-106,
python/tests/test_differential.py:962-1041 and :3167-3178), so pyarrow's ``array_sort_indices`` /
``sort_indices`` / ``take`` give the expected answers here. pyarrow has no totalOrder and no NaN-largest
float order; for those the expected answers come from the orders' definitions exactly as the reference
states them (``total_order_indices``, python/tests/test_sort_options.py:58-76; NaN one value above +inf in
both directions and -0.0 == +0.0, include/arrowmetal.h:1336-1347).

Generators follow the reference's tests: sizes around the chunk and block edges
(Tests/ArrowMetalTests/RadixSortScaleTests.swift:28-29, python/tests/test_sort_options.py:24), special
bit patterns (python/tests/test_sort_options.py:27-55), null fractions 0 / 0.1 / 1.0.

Run with ``python tests/golden/make_golden.py`` (pyarrow and numpy; no GPU).
"""
import json
import os
import struct

import numpy as np
import pyarrow as pa
import pyarrow.compute as pc

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sort_golden.npz")
SEED = 20260906

SPECIAL64 = [0x7FF8000000000000, 0xFFF8000000000000, 0x7FF0000000000001, 0xFFF8000000000042,
             0x7FF8000000000007, 0x0000000000000000, 0x8000000000000000, 0x7FF0000000000000,
             0xFFF0000000000000, 0x0000000000000001, 0x8000000000000003, 0x000FFFFFFFFFFFFF]
SPECIAL32 = [0x7FC00000, 0xFFC00000, 0x7F800001, 0xFFC00042, 0x80000000, 0, 0x7F800000, 0xFF800000, 1]

SIZES_INT64 = [0, 1, 2, 31, 32, 33, 255, 256, 257, 4095, 4096, 4097, 8191, 8192, 8193, 20001]
SIZES_FLOAT64 = [0, 1, 2, 33, 255, 256, 257, 4095, 4096, 4097]
SIZES_SMALL = [0, 1, 33, 4097]
OPTIONS = [(d, p) for d in (False, True) for p in ("at_end", "at_start")]


def physical_dtype(t):
    return {pa.int8(): np.int8, pa.uint8(): np.uint8, pa.int16(): np.int16, pa.uint16(): np.uint16,
            pa.int32(): np.int32, pa.uint32(): np.uint32, pa.int64(): np.int64, pa.uint64(): np.uint64,
            pa.float16(): np.uint16, pa.float32(): np.uint32, pa.float64(): np.uint64}[t]


def make_values(rng, t, n):
    if t == pa.float64():
        v = rng.uniform(-1e6, 1e6, n)
        dup = rng.random(n) < 0.25
        v[dup] = rng.integers(-20, 21, int(dup.sum())) / 4.0
        bits = v.view(np.uint64).copy()
        sp = rng.random(n) < 0.25
        bits[sp] = np.array(SPECIAL64, dtype=np.uint64)[rng.integers(0, len(SPECIAL64), int(sp.sum()))]
        return bits
    if t == pa.float32():
        v = rng.uniform(-1e3, 1e3, n).astype(np.float32)
        dup = rng.random(n) < 0.25
        v[dup] = (rng.integers(-20, 21, int(dup.sum())) / 4.0).astype(np.float32)
        bits = v.view(np.uint32).copy()
        sp = rng.random(n) < 0.25
        bits[sp] = np.array(SPECIAL32, dtype=np.uint32)[rng.integers(0, len(SPECIAL32), int(sp.sum()))]
        return bits
    if t == pa.float16():
        v = rng.uniform(-100, 100, n).astype(np.float16)
        bits = v.view(np.uint16).copy()
        sp = rng.random(n) < 0.2
        bits[sp] = np.array([0x7E00, 0xFE00, 0x8000, 0, 0x7C00, 0xFC00, 0x7C01], dtype=np.uint16)[
            rng.integers(0, 7, int(sp.sum()))]
        return bits
    dt = physical_dtype(t)
    info = np.iinfo(dt)
    if rng.random() < 0.5:
        return rng.integers(info.min, info.max, n, dtype=dt, endpoint=True)
    # narrow range with duplicates: constant high digits, stability matters
    lo = max(int(info.min), -1000)
    return rng.integers(lo, lo + 2000, n, dtype=np.int64).astype(dt)


def build_array(t, values, valid):
    n = len(values)
    vbuf = None
    if valid is not None:
        vbuf = pa.py_buffer(np.packbits(valid.astype(np.uint8), bitorder="little").tobytes())
    return pa.Array.from_buffers(t, n, [vbuf, pa.py_buffer(np.ascontiguousarray(values).tobytes())],
                                 null_count=-1 if valid is not None else 0)


def definition_order(arr, descending, placement, float_order):
    """total / nan_largest from the definitions (python/tests/test_sort_options.py:58-76)."""
    n = len(arr)
    valid = np.ones(n, bool) if arr.null_count == 0 else np.asarray(arr.is_valid().to_numpy(zero_copy_only=False))
    t = arr.type
    width = {pa.float16(): 16, pa.float32(): 32, pa.float64(): 64}[t]
    if width == 16:
        bits = np.asarray(arr.cast(pa.float32()).fill_null(0).to_numpy(zero_copy_only=False),
                          dtype=np.float32).view(np.uint32).astype(np.uint64)
        width = 32
    else:
        raw = arr.fill_null(0).to_numpy(zero_copy_only=False)
        bits = raw.view(np.uint64 if width == 64 else np.uint32).astype(np.uint64)
    sign = np.uint64(1 << (width - 1))
    full = np.uint64((1 << width) - 1)
    if float_order == "nan_largest":
        expo = np.uint64(0x7FF0000000000000 if width == 64 else 0x7F800000)
        mag = bits & ~sign & full
        bits = np.where(mag == 0, np.uint64(0), bits)
        bits = np.where(mag > expo, np.uint64(0x7FF0000000000001 if width == 64 else 0x7F800001), bits)
    key = np.where(bits & sign, ~bits & full, bits | sign)
    if descending:
        key = ~key & full
    rows = np.nonzero(valid)[0]
    ordered = rows[np.argsort(key[rows], kind="stable")]
    nulls = np.nonzero(~valid)[0]
    return np.concatenate([nulls, ordered] if placement == "at_start" else [ordered, nulls]).astype(np.uint32)


def main():
    rng = np.random.default_rng(SEED)
    cases, blobs = [], {}

    def add_array(name, t, n, null_fraction):
        values = make_values(rng, t, n)
        valid = None
        if null_fraction:
            valid = rng.random(n) >= null_fraction
        blobs[name + "_values"] = values
        if valid is not None:
            blobs[name + "_valid"] = valid
        return build_array(t, values, valid)

    # ---- single-key argsort
    types_main = [pa.int64(), pa.float64()]
    types_small = [pa.int8(), pa.uint8(), pa.int16(), pa.uint16(), pa.int32(), pa.uint32(), pa.uint64(),
                   pa.float32(), pa.float16()]
    k = 0
    for t in types_main + types_small:
        sizes = SIZES_INT64 if t == pa.int64() else SIZES_FLOAT64 if t == pa.float64() else SIZES_SMALL
        for n in sizes:
            for nf in (0.0, 0.1, 1.0) if n in (0, 33, 4097) else (0.1,):
                name = f"a{k}"
                k += 1
                arr = add_array(name, t, n, nf)
                orders = ["ieee", "total", "nan_largest"] if pa.types.is_floating(t) else ["ieee"]
                for fo in orders:
                    for d, p in OPTIONS:
                        if fo == "ieee":
                            if t == pa.float16():
                                want = pc.array_sort_indices(arr.cast(pa.float32()), order="descending" if d else "ascending",
                                                             null_placement=p)
                            else:
                                want = pc.array_sort_indices(arr, order="descending" if d else "ascending", null_placement=p)
                            want = want.to_numpy().astype(np.uint32)
                        else:
                            want = definition_order(arr, d, p, fo)
                        key = f"{name}_{fo}_{int(d)}_{p}"
                        blobs[key] = want
                        cases.append({"kind": "argsort", "array": name, "type": str(t), "n": n, "null_fraction": nf,
                                      "descending": d, "null_placement": p, "float_order": fo, "expect": key})

    # ---- multi-key sort_indices (pyarrow, one null placement for all keys)
    lk = 0
    for n in (0, 1, 257, 4097, 8193):
        for combo in ([pa.int32(), pa.float64()], [pa.int64(), pa.int64()], [pa.uint8(), pa.float32(), pa.int64()],
                      [pa.float64(), pa.int16()]):
            names = []
            for j, t in enumerate(combo):
                name = f"l{lk}_{j}"
                add_array(name, t, n, 0.1 if j != 0 or n < 4097 else 0.0)
                names.append(name)
            arrays = [build_array(t, blobs[nm + "_values"], blobs.get(nm + "_valid")) for t, nm in zip(combo, names)]
            for p in ("at_end", "at_start"):
                desc = [bool(rng.random() < 0.5) for _ in combo]
                table = pa.table({f"c{j}": a for j, a in enumerate(arrays)})
                want = pc.sort_indices(table, sort_keys=[(f"c{j}", "descending" if dd else "ascending")
                                                         for j, dd in enumerate(desc)],
                                       null_placement=p).to_numpy().astype(np.uint32)
                key = f"l{lk}_{p}"
                blobs[key] = want
                cases.append({"kind": "lexsort", "arrays": names, "types": [str(t) for t in combo], "n": n,
                              "descending": desc, "null_placement": p, "expect": key})
            lk += 1

    # ---- take with every index type, null indices, through a nullable source
    tk = 0
    for t in (pa.int64(), pa.float64(), pa.int32(), pa.int8(), pa.uint16()):
        for n_src, n_idx in ((1, 1), (1000, 257), (20001, 8193)):
            name = f"t{tk}"
            src = add_array(name, t, n_src, 0.1)
            for it in (pa.uint32(), pa.int32(), pa.int64()):
                idx_vals = rng.integers(0, n_src, n_idx).astype(it.to_pandas_dtype())
                idx_valid = rng.random(n_idx) >= 0.05
                iname = f"{name}_idx_{it}"
                blobs[iname + "_values"] = idx_vals
                blobs[iname + "_valid"] = idx_valid
                idx = build_array(it, idx_vals, idx_valid)
                got = pc.take(src, idx)
                ev = np.asarray(got.is_valid().to_numpy(zero_copy_only=False))
                vals = got.fill_null(0).to_numpy(zero_copy_only=False)
                if pa.types.is_floating(t):
                    vals = vals.view(physical_dtype(t))
                blobs[iname + "_expect_values"] = np.asarray(vals)
                blobs[iname + "_expect_valid"] = ev
                cases.append({"kind": "take", "array": name, "type": str(t), "n": n_src, "index": iname,
                              "index_type": str(it), "n_index": n_idx})
            tk += 1

    blobs["cases_json"] = np.frombuffer(json.dumps(cases).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **blobs)
    print(f"wrote {OUT}: {len(cases)} cases, {os.path.getsize(OUT) / 1e6:.2f} MB")


if __name__ == "__main__":
    main()
