// Device helpers shared by the sort kernels (radix_sort.cu) and the selection kernels (topk.cu): the
// order-preserving key maps of Arrow's sort orders, column loads and warp reductions.
#pragma once

#include <stdint.h>

#include "am_internal.h"
#include "radix_sort.cuh"

namespace am {
namespace rs {

__device__ __forceinline__ bool bit_at(const uint8_t* p, int64_t i) {
  return (p[i >> 3] >> (i & 7)) & 1;
}

// The ieee / nan_largest / total float maps on a float32 bit pattern (SortSource.swift:131-190).
// `cat` becomes 1 for a NaN that is its own block (ieee order).
__device__ __forceinline__ uint32_t key_f32_bits(uint32_t b, const ColView& c, int& cat) {
  const uint32_t S = 0x80000000u;
  uint32_t k;
  if (c.float_order == FO_TOTAL) {
    k = (b & S) ? ~b : (b | S);
  } else {
    const uint32_t mag = b & ~S;
    const bool nan = mag > 0x7F800000u;
    if (nan && c.nan_cat) { cat = 1; return 0u; }
    if (mag == 0u) b = 0u;
    if (nan) b = 0x7F800001u;
    k = (b & S) ? ~b : (b | S);
  }
  return c.desc ? ~k : k;
}

__device__ __forceinline__ uint64_t key_f64_bits(uint64_t b, const ColView& c, int& cat) {
  const uint64_t S = 0x8000000000000000ull;
  uint64_t k;
  if (c.float_order == FO_TOTAL) {
    k = (b & S) ? ~b : (b | S);
  } else {
    const uint64_t mag = b & ~S;
    const bool nan = mag > 0x7FF0000000000000ull;
    if (nan && c.nan_cat) { cat = 1; return 0ull; }
    if (mag == 0ull) b = 0ull;
    if (nan) b = 0x7FF0000000000001ull;
    k = (b & S) ? ~b : (b | S);
  }
  return c.desc ? ~k : k;
}

// Binary16 to binary32 bits, exactly and bit for bit: sign kept, exponent rebiased, subnormals
// normalised, a NaN's payload shifted into the wider mantissa. (A hardware conversion returns one
// canonical NaN, which would lose the sign totalOrder sorts -NaN by.)
__device__ __forceinline__ uint32_t f16_to_f32_bits(uint32_t h) {
  const uint32_t sign = (h & 0x8000u) << 16, exp = (h >> 10) & 0x1Fu, man = h & 0x3FFu;
  if (exp == 0x1Fu) return sign | 0x7F800000u | (man << 13);
  if (exp == 0u) {
    if (man == 0u) return sign;
    const uint32_t shift = uint32_t(__clz(int(man))) - 21u;   // brings the leading 1 to bit 10
    return sign | ((113u - shift) << 23) | (((man << shift) & 0x3FFu) << 13);
  }
  return sign | ((exp + 112u) << 23) | (man << 13);
}

// Raw bits of row `row`, widened to the key width: narrow integers sign- or zero-extended to 32 bits
// (the reference widens them to int32, Sort.swift:220-221), float16 as its 16 bits, boolean as its bit.
template <typename KeyT> __device__ __forceinline__ KeyT load_raw(const ColView& c, uint64_t row);
template <> __device__ __forceinline__ uint32_t load_raw<uint32_t>(const ColView& c, uint64_t row) {
  switch (c.pt) {
    case PT_BOOL: return bit_at(static_cast<const uint8_t*>(c.values), c.bool_off + int64_t(row)) ? 1u : 0u;
    case PT_I8: return uint32_t(int32_t(static_cast<const int8_t*>(c.values)[row]));
    case PT_U8: return static_cast<const uint8_t*>(c.values)[row];
    case PT_I16: return uint32_t(int32_t(static_cast<const int16_t*>(c.values)[row]));
    case PT_U16: case PT_F16: return static_cast<const uint16_t*>(c.values)[row];
    default: return static_cast<const uint32_t*>(c.values)[row];
  }
}
template <> __device__ __forceinline__ uint64_t load_raw<uint64_t>(const ColView& c, uint64_t row) {
  return static_cast<const uint64_t*>(c.values)[row];
}

// Loads the raw bits of ITEMS rows with the type dispatch outside the loop, so the loads are issued
// back to back. ok bit i: row i exists.
template <typename KeyT, int ITEMS>
__device__ __forceinline__ void load_raw_rows(const ColView& c, const uint32_t (&row)[ITEMS], uint32_t ok, KeyT (&raw)[ITEMS]) {
  if constexpr (sizeof(KeyT) == 8) {
    const uint64_t* v = static_cast<const uint64_t*>(c.values);
#pragma unroll
    for (int i = 0; i < ITEMS; i++) raw[i] = ((ok >> i) & 1u) ? v[row[i]] : 0ull;
  } else {
    switch (c.pt) {
      case PT_I32: case PT_U32: case PT_F32: {
        const uint32_t* v = static_cast<const uint32_t*>(c.values);
#pragma unroll
        for (int i = 0; i < ITEMS; i++) raw[i] = ((ok >> i) & 1u) ? v[row[i]] : 0u;
        break;
      }
      default:
#pragma unroll
        for (int i = 0; i < ITEMS; i++) raw[i] = ((ok >> i) & 1u) ? load_raw<uint32_t>(c, row[i]) : 0u;
    }
  }
}

// Key of raw bits `raw` (valid or null); `cat` is 0 for a value, 1 for a NaN block row, 2 for a null.
template <typename KeyT> __device__ __forceinline__ KeyT key_from_raw(const ColView& c, KeyT raw, bool valid, int& cat);

template <> __device__ __forceinline__ uint32_t key_from_raw<uint32_t>(const ColView& c, uint32_t raw, bool valid, int& cat) {
  cat = 0;
  if (!valid) { cat = 2; return 0u; }
  uint32_t k;
  switch (c.pt) {
    case PT_U32: k = raw; break;
    case PT_F16: return key_f32_bits(f16_to_f32_bits(raw), c, cat);
    case PT_F32: return key_f32_bits(raw, c, cat);
    default: k = raw ^ 0x80000000u;   // int32 and the narrow types widened to it
  }
  return c.desc ? ~k : k;
}

template <> __device__ __forceinline__ uint64_t key_from_raw<uint64_t>(const ColView& c, uint64_t raw, bool valid, int& cat) {
  cat = 0;
  if (!valid) { cat = 2; return 0ull; }
  if (c.pt == PT_F64) return key_f64_bits(raw, c, cat);
  const uint64_t k = (c.pt == PT_I64) ? (raw ^ 0x8000000000000000ull) : raw;
  return c.desc ? ~k : k;
}

// Validity of ITEMS rows held warp-striped from `first`: item i of lane l is row first + 32 i + l;
// bit i of `ok` says the row exists (rows before `end` do). When the bitmap's offset and `first` are
// multiples of 32 and the bitmap is word-aligned, an item's 32 rows are one bitmap word (lane l's bit
// l), one load for the warp; an item whose word reaches past the rows (the bitmap may end inside it)
// reads each row's own byte, placed at that byte's position in the word. Bit i of the result: the row
// exists and is valid.
template <int ITEMS>
__device__ __forceinline__ uint32_t striped_validity(const ColView& c, uint64_t first, uint64_t end, uint32_t ok) {
  if (!c.valid) return ok;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t vb[ITEMS];
  uint32_t valid = ok;
  if ((c.valid_off & 31) == 0 && (first & 31u) == 0 && (reinterpret_cast<uintptr_t>(c.valid) & 3u) == 0) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(c.valid) + ((uint64_t(c.valid_off) + first) >> 5);
    const uint64_t full = end > first ? (end - first) >> 5 : 0;   // items whose 32 rows all exist
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      if (uint64_t(i) < full) vb[i] = w[i];
      else vb[i] = ((ok >> i) & 1u) ? uint32_t(c.valid[(c.valid_off + int64_t(first + 32u * i + lane)) >> 3]) << (8u * (lane >> 3)) : 0u;
    }
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
      if (!((vb[i] >> lane) & 1u)) valid &= ~(1u << i);
  } else {
#pragma unroll
    for (int i = 0; i < ITEMS; i++) vb[i] = ((ok >> i) & 1u) ? c.valid[(c.valid_off + int64_t(first + 32u * i + lane)) >> 3] : 0u;
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
      if (!((vb[i] >> ((c.valid_off + int64_t(first + 32u * i + lane)) & 7)) & 1u)) valid &= ~(1u << i);
  }
  return valid;
}

// Keys and categories of ITEMS rows from their raw bits and validity (bit i: row i is valid), with the
// type and direction decided once for all the rows (the integer maps are one XOR a row, no branches).
// The same keys and categories as key_from_raw row by row.
template <typename KeyT, int ITEMS>
__device__ __forceinline__ void encode_raw(const ColView& c, const KeyT (&raw)[ITEMS], uint32_t valid, KeyT (&key)[ITEMS],
                                           int (&cat)[ITEMS]) {
  constexpr bool WIDE = sizeof(KeyT) == 8;
  const bool fl = WIDE ? c.pt == PT_F64 : (c.pt == PT_F32 || c.pt == PT_F16);
  if (!fl) {
    const KeyT sign = KeyT(KeyT(1) << (8 * sizeof(KeyT) - 1));
    const KeyT flip = WIDE ? (c.pt == PT_I64 ? sign : KeyT(0)) : (c.pt == PT_U32 ? KeyT(0) : sign);
    const KeyT x = flip ^ (c.desc ? KeyT(~KeyT(0)) : KeyT(0));
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const bool v = (valid >> i) & 1u;
      key[i] = v ? KeyT(raw[i] ^ x) : KeyT(0);
      cat[i] = v ? 0 : 2;
    }
  } else {
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      cat[i] = 0;
      if (!((valid >> i) & 1u)) {
        cat[i] = 2;
        key[i] = KeyT(0);
      } else if constexpr (WIDE) {
        key[i] = key_f64_bits(raw[i], c, cat[i]);
      } else {
        key[i] = key_f32_bits(c.pt == PT_F16 ? f16_to_f32_bits(uint32_t(raw[i])) : uint32_t(raw[i]), c, cat[i]);
      }
    }
  }
}

// Keys of ITEMS rows at any positions: all loads first (values and validity bytes), then the arithmetic.
template <typename KeyT, int ITEMS>
__device__ __forceinline__ void encode_rows(const ColView& c, const uint32_t (&row)[ITEMS], uint32_t ok, KeyT (&key)[ITEMS],
                                            int (&cat)[ITEMS]) {
  KeyT raw[ITEMS];
  uint32_t vb[ITEMS];
  load_raw_rows<KeyT, ITEMS>(c, row, ok, raw);
  uint32_t valid = ok;                 // bit i: row i exists and is not null
  if (c.valid) {
#pragma unroll
    for (int i = 0; i < ITEMS; i++) vb[i] = ((ok >> i) & 1u) ? c.valid[(c.valid_off + int64_t(row[i])) >> 3] : 0u;
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
      if (!((vb[i] >> ((c.valid_off + int64_t(row[i])) & 7)) & 1u)) valid &= ~(1u << i);
  }
  encode_raw<KeyT, ITEMS>(c, raw, valid, key, cat);
}

template <typename T> __device__ __forceinline__ T warp_or(T v);
template <> __device__ __forceinline__ uint32_t warp_or(uint32_t v) { return __reduce_or_sync(0xffffffffu, v); }
template <> __device__ __forceinline__ uint64_t warp_or(uint64_t v) {
  uint32_t lo = __reduce_or_sync(0xffffffffu, uint32_t(v));
  uint32_t hi = __reduce_or_sync(0xffffffffu, uint32_t(v >> 32));
  return (uint64_t(hi) << 32) | lo;
}
template <typename T> __device__ __forceinline__ T warp_and(T v);
template <> __device__ __forceinline__ uint32_t warp_and(uint32_t v) { return __reduce_and_sync(0xffffffffu, v); }
template <> __device__ __forceinline__ uint64_t warp_and(uint64_t v) {
  uint32_t lo = __reduce_and_sync(0xffffffffu, uint32_t(v));
  uint32_t hi = __reduce_and_sync(0xffffffffu, uint32_t(v >> 32));
  return (uint64_t(hi) << 32) | lo;
}
__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

}  // namespace rs
}  // namespace am
