// Stable LSD radix argsort for sm_100a: one key-encode + all-digit histogram read per key column,
// a one-block planning kernel, then onesweep digit passes with warp match_any ranking and decoupled
// look-back, skipping every digit that is constant over the column.
//
// What it computes is the reference's `radixSortRun` (Sources/ArrowMetal/Kernels/Sort.swift:190-504)
// and `lexsortIndices` (Sources/ArrowMetal/Kernels/MultiSort.swift:28-65):
//   * the order-preserving key maps key_from_{i32,u32,f32,i64,u64,f64}[_total|_nanlargest]
//     (Sources/ArrowMetal/Kernels/SortSource.swift:131-190): signed integers flip the sign bit,
//     floats map -0.0 onto +0.0 and every NaN onto one value, sign-magnitude to two's order;
//     descending is the complement; narrow integers widen to int32 (Sort.swift:220-221);
//   * the stable three-way split into values / NaN / nulls (SortSource.swift:226-330), with the NaN
//     block only for the ieee order, arranged [values][NaN][nulls] at the end or
//     [nulls][NaN][values] at the start (Sort.swift:11-28);
//   * dropping every pass whose digit is the same in every row (Sort.swift:404-417);
//   * multi-key order by stable passes from the least significant key upwards (MultiSort.swift:56-64).
// How it computes it is B200's own: no per-pass histogram or scan launch (one histogram read per key
// gives every digit's counts), no host readback (the planning kernel writes each pass's descriptor
// and inactive passes return at once), and the ids of the rows are synthesised by the first pass
// instead of being written by an iota kernel. A lexsort carries the row ids through every pass, so
// the reference's "take the next key column, argsort, compose" becomes one gather of the next key
// inside its first pass.
#include <algorithm>
#include <cstring>

#include "am_internal.h"
#include "radix_sort.cuh"

namespace am {
namespace rs {

// ------------------------------------------------------------------------------------------------
// Device helpers.

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint64_t pack_status(uint32_t epoch, uint32_t flag, uint32_t count) {
  return (uint64_t(epoch) << 34) | (uint64_t(flag) << 32) | uint64_t(count);
}

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

// Key of row `row` of column `c`; `cat` is 0 for a value, 1 for a NaN block row, 2 for a null.
template <typename KeyT> __device__ __forceinline__ KeyT encode_key(const ColView& c, uint64_t row, int& cat);

template <> __device__ __forceinline__ uint32_t encode_key<uint32_t>(const ColView& c, uint64_t row, int& cat) {
  cat = 0;
  if (c.valid && !bit_at(c.valid, c.valid_off + int64_t(row))) { cat = 2; return 0u; }
  int32_t v;
  switch (c.pt) {
    case PT_BOOL: v = bit_at(static_cast<const uint8_t*>(c.values), c.bool_off + int64_t(row)) ? 1 : 0; break;
    case PT_I8: v = static_cast<const int8_t*>(c.values)[row]; break;
    case PT_U8: v = static_cast<const uint8_t*>(c.values)[row]; break;
    case PT_I16: v = static_cast<const int16_t*>(c.values)[row]; break;
    case PT_U16: v = static_cast<const uint16_t*>(c.values)[row]; break;
    case PT_I32: v = static_cast<const int32_t*>(c.values)[row]; break;
    case PT_U32: {
      uint32_t k = static_cast<const uint32_t*>(c.values)[row];
      return c.desc ? ~k : k;
    }
    case PT_F16:
      return key_f32_bits(f16_to_f32_bits(static_cast<const unsigned short*>(c.values)[row]), c, cat);
    default:  // PT_F32
      return key_f32_bits(static_cast<const uint32_t*>(c.values)[row], c, cat);
  }
  const uint32_t k = uint32_t(v) ^ 0x80000000u;
  return c.desc ? ~k : k;
}

template <> __device__ __forceinline__ uint64_t encode_key<uint64_t>(const ColView& c, uint64_t row, int& cat) {
  cat = 0;
  if (c.valid && !bit_at(c.valid, c.valid_off + int64_t(row))) { cat = 2; return 0ull; }
  const uint64_t b = static_cast<const uint64_t*>(c.values)[row];
  if (c.pt == PT_F64) return key_f64_bits(b, c, cat);
  const uint64_t k = (c.pt == PT_I64) ? (b ^ 0x8000000000000000ull) : b;
  return c.desc ? ~k : k;
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

// ------------------------------------------------------------------------------------------------
// Kernel 1: key encode + all-digit histogram of one key column.
//
// One read of the column gives every digit's 256 counts (the reference reads the keys once per pass,
// SortSource.swift:31-73), the null and NaN-block counts, and the largest and smallest value key
// (for folding a lower key's null / NaN rows into its key range). A warp whose keys agree on a digit
// adds its count with one atomic instead of 32, so a digit that is constant over the column (the
// high bytes of keys drawn from [0, 2^40)) costs almost nothing.

template <typename KeyT, int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) key_histogram_kernel(const __grid_constant__ ColView col, KeyStats* __restrict__ st, uint64_t n) {
  constexpr int D = int(sizeof(KeyT));
  constexpr int CHUNK = THREADS * ITEMS;
  __shared__ uint32_t sh[D * 256];
  __shared__ uint32_t s_null, s_nan, s_val;
  __shared__ unsigned long long s_max, s_min_inv;
  for (int i = threadIdx.x; i < D * 256; i += THREADS) sh[i] = 0;
  if (threadIdx.x == 0) { s_null = 0; s_nan = 0; s_val = 0; s_max = 0; s_min_inv = 0; }
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t n_null = 0, n_nan = 0, n_val = 0;
  KeyT vmax = 0, vmin_inv = 0;

  for (uint64_t base = uint64_t(blockIdx.x) * CHUNK; base < n; base += uint64_t(gridDim.x) * CHUNK) {
    KeyT k[ITEMS];
    uint32_t valid_mask = 0;
    KeyT o = 0, a = KeyT(~KeyT(0));
    uint32_t nv = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const uint64_t g = base + uint64_t(warp) * (ITEMS * 32) + uint64_t(i) * 32 + lane;
      k[i] = 0;
      if (g < n) {
        int cat;
        const KeyT kk = encode_key<KeyT>(col, g, cat);
        if (cat == 0) {
          k[i] = kk;
          valid_mask |= 1u << i;
          o |= kk;
          a &= kk;
          nv++;
          vmax = kk > vmax ? kk : vmax;
          vmin_inv = KeyT(~kk) > vmin_inv ? KeyT(~kk) : vmin_inv;
        } else if (cat == 1) {
          n_nan++;
        } else {
          n_null++;
        }
      }
    }
    n_val += nv;
    const KeyT wo = warp_or<KeyT>(o), wa = warp_and<KeyT>(a);
    const uint32_t wnv = __reduce_add_sync(0xffffffffu, nv);
#pragma unroll
    for (int p = 0; p < D; p++) {
      const uint32_t diff = uint32_t((wo ^ wa) >> (8 * p)) & 255u;
      if (diff == 0u) {
        if (lane == 0 && wnv) atomicAdd(&sh[p * 256 + (uint32_t(wa >> (8 * p)) & 255u)], wnv);
      } else {
#pragma unroll
        for (int i = 0; i < ITEMS; i++)
          if (valid_mask & (1u << i)) atomicAdd(&sh[p * 256 + (uint32_t(k[i] >> (8 * p)) & 255u)], 1u);
      }
    }
  }
  // Block totals.
  n_null = __reduce_add_sync(0xffffffffu, n_null);
  n_nan = __reduce_add_sync(0xffffffffu, n_nan);
  n_val = __reduce_add_sync(0xffffffffu, n_val);
  const uint64_t wmax = warp_max_u64(uint64_t(vmax));
  const uint64_t wmin = warp_max_u64(uint64_t(vmin_inv));
  if (lane == 0) {
    if (n_null) atomicAdd(&s_null, n_null);
    if (n_nan) atomicAdd(&s_nan, n_nan);
    if (n_val) atomicAdd(&s_val, n_val);
    atomicMax(&s_max, (unsigned long long)wmax);
    atomicMax(&s_min_inv, (unsigned long long)wmin);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < D * 256; i += THREADS)
    if (sh[i]) atomicAdd(&st->hist[i >> 8][i & 255], sh[i]);
  if (threadIdx.x == 0) {
    if (s_null) atomicAdd(&st->n_null, s_null);
    if (s_nan) atomicAdd(&st->n_nan, s_nan);
    if (s_val) {
      atomicAdd(&st->n_value, s_val);
      atomicMax(&st->vmax, s_max);
      atomicMax(&st->vmin_inv, s_min_inv);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Kernel 2: the plan. One block decides, from the histograms alone, which digit passes run, where
// each pass reads and writes, and every pass's per-digit global base; the passes read it from HBM.

__device__ void block_exclusive_scan_256(const uint32_t* in, uint32_t* out, uint32_t* total, uint32_t* s_warp) {
  // 256 threads, one value each.
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  uint32_t v = in[t];
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < 8 ? s_warp[lane] : 0u;
    uint32_t z = w;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, z, o);
      if (lane >= o) z += y;
    }
    if (lane < 8) s_warp[8 + lane] = z - w;
    if (lane == 7) *total = z;
  }
  __syncthreads();
  out[t] = x - v + s_warp[8 + warp];
  __syncthreads();
}

__device__ __forceinline__ uint64_t key_max(int bytes) { return bytes == 8 ? ~0ull : 0xFFFFFFFFull; }

__global__ void __launch_bounds__(256) plan_kernel(PlanArgs a, KeyStats* __restrict__ st, KeyPlan* __restrict__ kp,
                                                   PassDesc* __restrict__ pd, SortSummary* __restrict__ sum) {
  __shared__ uint32_t s_vals[256];
  __shared__ uint32_t s_out[256];
  __shared__ uint32_t s_warp[16];
  __shared__ uint32_t s_total;
  __shared__ uint32_t s_max;
  __shared__ uint8_t s_active[MAX_SLOTS];
  const int t = threadIdx.x;
  const uint32_t n = uint32_t(a.n);

  // 1. Per key: fold a lower key's null / NaN-block rows into its key range when there is room,
  //    else give them key 0 and a category pass; add the folded rows to the histogram.
  if (t == 0) {
    for (int k = 0; k < a.nkeys; k++) {
      KeyStats& s = st[k];
      KeyPlan& p = kp[k];
      p.fold_mode = 0;
      p.fold_nan = 0;
      p.fold_null = 0;
      if (k == 0) continue;                 // the most significant key routes its categories
      const uint32_t ncat = (s.n_null ? 1u : 0u) + (s.n_nan ? 1u : 0u);
      if (ncat == 0) continue;
      const uint64_t kmax = key_max(a.key_bytes[k]);
      const bool first = a.nulls_first[k];
      if (s.n_value == 0) {
        // Only categories: any keys in category order.
        p.fold_nan = first ? 1 : 0;
        p.fold_null = first ? 0 : 1;
      } else if (!first && s.vmax <= kmax - ncat) {
        p.fold_nan = s.vmax + 1;
        p.fold_null = s.vmax + ncat;
      } else if (first && (~s.vmin_inv & kmax) >= ncat) {
        const uint64_t vmin = ~s.vmin_inv & kmax;
        p.fold_nan = vmin - 1;
        p.fold_null = vmin - ncat;
      } else {
        p.fold_mode = 1;                    // no room: placeholder key 0, category pass after
      }
      const int D = a.key_bytes[k];
      for (int d = 0; d < D; d++) {
        if (p.fold_mode == 0) {
          if (s.n_null) s.hist[d][(p.fold_null >> (8 * d)) & 255] += s.n_null;
          if (s.n_nan) s.hist[d][(p.fold_nan >> (8 * d)) & 255] += s.n_nan;
        } else {
          s.hist[d][0] += s.n_null + s.n_nan;
        }
      }
    }
  }
  __syncthreads();

  // 2. Which digit passes are not constant.
  for (int sl = 0; sl < a.nslots; sl++) {
    const int k = a.slot_key[sl], d = a.slot_digit[sl];
    if (d < 0) {
      if (t == 0) s_active[sl] = (kp[k].fold_mode == 1) ? 1 : 0;
      continue;
    }
    const uint32_t total = (k == 0) ? st[0].n_value : n;
    if (t == 0) s_max = 0;
    __syncthreads();
    uint32_t c = st[k].hist[d][t];
    uint32_t m = __reduce_max_sync(0xffffffffu, c);
    if ((t & 31) == 0) atomicMax(&s_max, m);
    __syncthreads();
    if (t == 0) s_active[sl] = (total > 0 && s_max < total) ? 1 : 0;
    __syncthreads();
  }

  // 3. Buffers: walk the active passes in order, least significant key first.
  if (t == 0) {
    const bool key0_cats = (st[0].n_null + st[0].n_nan) > 0;
    bool any_key0 = false, any = false;
    for (int sl = 0; sl < a.nslots; sl++) {
      if (s_active[sl]) { any = true; if (a.slot_key[sl] == 0) any_key0 = true; }
    }
    if ((key0_cats && !any_key0) || !any) s_active[a.slot_key0_first] = 1;

    int ids_src = -1, keys_src = -1;        // -1: identity ids / keys not in a buffer
    uint32_t run = 0;
    int last_any = -1;
    for (int sl = 0; sl < a.nslots; sl++) if (s_active[sl]) last_any = sl;
    for (int sl = 0; sl < a.nslots; sl++) {
      PassDesc& p = pd[sl];
      p.active = s_active[sl];
      if (!p.active) continue;
      run++;
      const int k = a.slot_key[sl], d = a.slot_digit[sl];
      int last_of_key = sl;
      for (int j = sl + 1; j < a.nslots && a.slot_key[j] == k; j++) if (s_active[j]) { last_of_key = j; break; }
      const bool is_last_of_key = (last_of_key == sl);
      const bool is_last = (sl == last_any);
      uint32_t flags = 0;
      if (d < 0) flags |= PF_CATPASS;
      else if (keys_src < 0) flags |= PF_ENCODE;
      if (k == 0 && (flags & PF_ENCODE)) flags |= PF_ROUTE;
      if (a.index_wide) flags |= PF_WIDE_OUT;
      p.flags = flags;
      p.key = uint32_t(k);
      p.shift = d < 0 ? 0u : uint32_t(8 * d);
      // Rows flowing: the most significant key drops its null / NaN rows in its first pass.
      p.count = (k == 0 && !(flags & PF_ENCODE)) ? st[0].n_value : n;
      p.src_keys = (flags & (PF_ENCODE | PF_CATPASS)) ? -1 : keys_src;
      p.src_ids = ids_src;
      if (is_last) {
        p.dst_keys = -1;
        p.dst_ids = -1;                      // the output index array
      } else if (is_last_of_key) {
        p.dst_keys = -1;
        p.dst_ids = (ids_src == 0) ? 1 : 0;
      } else {
        p.dst_keys = (keys_src == 0) ? 1 : 0;
        p.dst_ids = (ids_src == 0) ? 1 : 0;
      }
      p.value_base = (k == 0 && a.nulls_first[0]) ? (st[0].n_null + st[0].n_nan) : 0u;
      ids_src = p.dst_ids;
      keys_src = is_last_of_key ? -1 : p.dst_keys;
    }
    sum->value_rows = st[0].n_value;
    sum->null_rows = st[0].n_null;
    sum->nan_rows = st[0].n_nan;
    sum->passes_run = run;
    sum->passes_total = uint32_t(a.nslots);
  }
  __syncthreads();

  // 4. Per active pass, every bin's global base.
  for (int sl = 0; sl < a.nslots; sl++) {
    if (!s_active[sl]) continue;
    const int k = a.slot_key[sl], d = a.slot_digit[sl];
    PassDesc& p = pd[sl];
    if (d < 0) {
      // Category pass: bin 0 / 1 in category order.
      if (t == 0) {
        const uint32_t nn = st[k].n_null, nv = n - nn;
        const bool first = a.nulls_first[k];
        p.bin_base[0] = 0;
        p.bin_base[1] = first ? nn : nv;
        for (int b = 2; b < NBINS; b++) p.bin_base[b] = 0;
      }
      __syncthreads();
      continue;
    }
    s_vals[t] = st[k].hist[d][t];
    __syncthreads();
    block_exclusive_scan_256(s_vals, s_out, &s_total, s_warp);
    p.bin_base[t] = s_out[t];
    if (t == 0) {
      const uint32_t m = st[0].n_value, nn = st[0].n_null, nnan = st[0].n_nan;
      if (k == 0 && a.nulls_first[0]) {
        p.bin_base[NULL_BIN] = 0;
        p.bin_base[NAN_BIN] = nn;
      } else {
        p.bin_base[NAN_BIN] = m;
        p.bin_base[NULL_BIN] = m + nnan;
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------
// Kernel 3: one onesweep digit pass.
//
// Tiles of THREADS x ITEMS rows are claimed with an atomic ticket, so a tile only ever waits on tiles
// that have already started. Rows are held warp-striped (row = tile + warp*ITEMS*32 + i*32 + lane),
// which makes every load a coalesced warp access and makes "item i before item i+1, lower lane first"
// the input order; each warp ranks its rows with one __match_any_sync per item against its own
// per-digit counters in shared memory (the reference's ballot ranking, SortSource.swift:334-386, in
// one instruction). The tile's per-digit counts go out as look-back aggregates right away, the rows
// are staged in shared memory at their tile-local sorted slot, the look-back (bounded in time) turns
// the counts into global offsets, and the rows leave shared memory in order, so consecutive threads
// write consecutive addresses within every digit run.

template <typename KeyT, int THREADS, int ITEMS>
struct PassShared {
  static constexpr int WARPS = THREADS / 32;
  static constexpr int TILE = THREADS * ITEMS;
  PassDesc desc;
  uint32_t whist[WARPS][NBINS];
  uint32_t cnt[NBINS];
  uint32_t local[NBINS];
  uint32_t gdelta[NBINS];
  uint32_t scan_warp[16];
  uint32_t scan_total;
  uint32_t tile;
  uint16_t dig[TILE];
  KeyT keys[TILE];
  uint32_t ids[TILE];
};

template <typename KeyT, int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS, 2)
onesweep_pass_kernel(const __grid_constant__ PassArgs pa, const __grid_constant__ ColView col) {
  static_assert(THREADS == 256, "the digit scan assumes one thread per value digit");
  static_assert(THREADS * ITEMS <= 65536, "tile-local ranks are 16-bit");
  using SM = PassShared<KeyT, THREADS, ITEMS>;
  constexpr int TILE = SM::TILE;
  constexpr int WARPS = SM::WARPS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SM& sm = *reinterpret_cast<SM*>(smem_raw);

  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(pa.desc);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&sm.desc);
    for (int i = threadIdx.x; i < int(sizeof(PassDesc) / 4); i += THREADS) dst[i] = src[i];
  }
  __syncthreads();
  if (!sm.desc.active) return;

  const uint32_t flags = sm.desc.flags;
  const uint64_t count = sm.desc.count;
  const uint32_t shift = sm.desc.shift;
  const uint32_t ntiles = uint32_t((count + TILE - 1) / TILE);
  const int sk = sm.desc.src_keys, si = sm.desc.src_ids, dk = sm.desc.dst_keys, di = sm.desc.dst_ids;
  const KeyT* __restrict__ keys_in = sk < 0 ? nullptr : static_cast<const KeyT*>(sk == 0 ? pa.keys[0] : pa.keys[1]);
  const uint32_t* __restrict__ ids_in = si < 0 ? nullptr : (si == 0 ? pa.ids[0] : pa.ids[1]);
  KeyT* __restrict__ keys_out = dk < 0 ? nullptr : static_cast<KeyT*>(dk == 0 ? pa.keys[0] : pa.keys[1]);
  uint32_t* __restrict__ ids_out = di < 0 ? nullptr : (di == 0 ? pa.ids[0] : pa.ids[1]);
  const KeyPlan kplan = *pa.kplan;
  const uint32_t epoch = pa.epoch;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t lt_mask = (1u << lane) - 1u;

  for (;;) {
    if (threadIdx.x == 0) sm.tile = atomicAdd(pa.tile_counter, 1u);
    for (int b = lane; b < NBINS; b += 32) sm.whist[warp][b] = 0;
    __syncthreads();
    const uint32_t tile = sm.tile;
    if (tile >= ntiles) break;
    const uint64_t tile_base = uint64_t(tile) * TILE;

    // ---- load and digit
    KeyT key[ITEMS];
    uint32_t id[ITEMS];
    uint32_t dg[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const uint64_t g = tile_base + uint64_t(warp) * (ITEMS * 32) + uint64_t(i) * 32 + lane;
      key[i] = 0;
      id[i] = 0;
      dg[i] = INVALID_DIGIT;
      if (g < count) {
        id[i] = ids_in ? ids_in[g] : uint32_t(g);
        if (flags & PF_CATPASS) {
          const bool is_null = col.valid && !bit_at(col.valid, col.valid_off + int64_t(id[i]));
          dg[i] = (is_null != bool(col.nulls_first)) ? 1u : 0u;
        } else if (flags & PF_ENCODE) {
          int cat;
          KeyT k = encode_key<KeyT>(col, id[i], cat);
          if (cat && (flags & PF_ROUTE)) {
            dg[i] = (cat == 1) ? uint32_t(NAN_BIN) : uint32_t(NULL_BIN);
          } else {
            if (cat) k = kplan.fold_mode ? KeyT(0) : KeyT(cat == 1 ? kplan.fold_nan : kplan.fold_null);
            key[i] = k;
            dg[i] = uint32_t(k >> shift) & 255u;
          }
        } else {
          key[i] = keys_in[g];
          dg[i] = uint32_t(key[i] >> shift) & 255u;
        }
      }
    }

    // ---- warp ranking: rank among this warp's rows of the same digit, in input order
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const uint32_t d = dg[i];
      const uint32_t peers = __match_any_sync(0xffffffffu, d);
      const int leader = __ffs(peers) - 1;
      uint32_t base = 0;
      if (lane == leader && d != INVALID_DIGIT) {
        base = sm.whist[warp][d];
        sm.whist[warp][d] = base + __popc(peers);
      }
      base = __shfl_sync(0xffffffffu, base, leader);
      __syncwarp();
      dg[i] = d | ((base + __popc(peers & lt_mask)) << 16);
    }
    __syncthreads();

    // ---- per digit: warps' exclusive offsets and the tile's count; publish the aggregate
    for (int b = threadIdx.x; b < NBINS; b += THREADS) {
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < WARPS; w++) {
        const uint32_t c = sm.whist[w][b];
        sm.whist[w][b] = run;
        run += c;
      }
      sm.cnt[b] = run;
      st_relaxed_u64(pa.status + uint64_t(tile) * NBINS + b, pack_status(epoch, tile == 0 ? ST_INCL : ST_AGG, run));
    }
    __syncthreads();
    // Tile-local digit starts: value digits in order, then the NaN and null routing bins.
    block_exclusive_scan_256(sm.cnt, sm.local, &sm.scan_total, sm.scan_warp);
    if (threadIdx.x == 0) {
      const uint32_t tot = sm.local[255] + sm.cnt[255];
      sm.local[NAN_BIN] = tot;
      sm.local[NULL_BIN] = tot + sm.cnt[NAN_BIN];
    }
    __syncthreads();

    // ---- stage keys, ids and digits at their tile-local sorted slot (frees the registers)
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const uint32_t d = dg[i] & 0xFFFFu;
      if (d != INVALID_DIGIT) {
        const uint32_t pos = sm.local[d] + sm.whist[warp][d] + (dg[i] >> 16);
        sm.keys[pos] = key[i];
        sm.ids[pos] = id[i];
        sm.dig[pos] = uint16_t(d);
      }
    }

    // ---- decoupled look-back, one thread per digit, LOOKBACK_WINDOW predecessors per round trip:
    // the window's loads are independent, so the inclusive-prefix frontier moves a whole window of
    // tiles per L2 round trip instead of one. Every wait is bounded in time.
    for (int b = threadIdx.x; b < NBINS; b += THREADS) {
      uint32_t excl = 0;
      if (tile > 0) {
        int64_t j = int64_t(tile) - 1;
        bool done = false;
        while (!done) {
          uint64_t st[LOOKBACK_WINDOW];
#pragma unroll
          for (int i = 0; i < LOOKBACK_WINDOW; i++)
            st[i] = (j - i >= 0) ? ld_relaxed_u64(pa.status + uint64_t(j - i) * NBINS + b) : pack_status(epoch, ST_INCL, 0);
#pragma unroll
          for (int i = 0; i < LOOKBACK_WINDOW; i++) {
            uint64_t s = st[i];
            if (uint32_t(s >> 34) != epoch || ((s >> 32) & 3u) == 0u) {
              const uint64_t* p = pa.status + uint64_t(j - i) * NBINS + b;
              const uint64_t t0 = globaltimer_ns();
              uint32_t polls = 0;
              for (;;) {
                s = ld_relaxed_u64(p);
                if (uint32_t(s >> 34) == epoch && ((s >> 32) & 3u) != 0u) break;
                if (++polls > 8) __nanosleep(32);
                if ((polls & 63u) == 0u && globaltimer_ns() - t0 > LOOKBACK_TIMEOUT_NS) {
                  atomicOr(pa.err, ERR_LOOKBACK_TIMEOUT);
                  s = pack_status(epoch, ST_INCL, 0);
                  break;
                }
              }
            }
            excl += uint32_t(s);
            if (((s >> 32) & 3u) == ST_INCL) { done = true; break; }
          }
          j -= LOOKBACK_WINDOW;
          if (j < 0) done = true;
        }
        st_relaxed_u64(pa.status + uint64_t(tile) * NBINS + b, pack_status(epoch, ST_INCL, excl + sm.cnt[b]));
      }
      sm.gdelta[b] = sm.desc.bin_base[b] + excl - sm.local[b];
    }
    __syncthreads();

    const uint32_t tile_n = uint32_t((count - tile_base) < uint64_t(TILE) ? (count - tile_base) : uint64_t(TILE));
    // ---- keys out, then ids out; consecutive threads write consecutive addresses of a digit run
    if (keys_out) {
      for (uint32_t j = threadIdx.x; j < tile_n; j += THREADS) {
        const uint32_t d = sm.dig[j];
        if (d < RADIX) keys_out[sm.gdelta[d] + j] = sm.keys[j];
      }
    }
    for (uint32_t j = threadIdx.x; j < tile_n; j += THREADS) {
      const uint32_t d = sm.dig[j];
      const uint32_t v = sm.ids[j];
      uint32_t dst = sm.gdelta[d] + j;
      if (d >= RADIX || !ids_out) {
        if (d < RADIX) dst += sm.desc.value_base;
        if (flags & PF_WIDE_OUT) static_cast<uint64_t*>(pa.final_out)[dst] = v;
        else static_cast<uint32_t*>(pa.final_out)[dst] = v;
      } else {
        ids_out[dst] = v;
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------
// Host side.

template <typename KeyT>
struct PassConfig;
template <> struct PassConfig<uint32_t> { static constexpr int THREADS = 256, ITEMS = 16; };
template <> struct PassConfig<uint64_t> { static constexpr int THREADS = 256, ITEMS = 16; };

constexpr int HIST_THREADS = 256, HIST_ITEMS = 8;

template <typename KeyT>
static size_t pass_smem() {
  using C = PassConfig<KeyT>;
  return sizeof(PassShared<KeyT, C::THREADS, C::ITEMS>);
}

template <typename KeyT>
static int pass_blocks_per_sm() {
  using C = PassConfig<KeyT>;
  static int cached = -1;
  static std::once_flag once;
  std::call_once(once, [] {
    auto fn = onesweep_pass_kernel<KeyT, C::THREADS, C::ITEMS>;
    AM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(pass_smem<KeyT>())));
    int b = 0;
    AM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, C::THREADS, pass_smem<KeyT>()));
    cached = std::max(1, b);
  });
  return cached;
}

template <typename KeyT>
static void launch_histogram(const ColView& cv, KeyStats* st, uint64_t n, cudaStream_t s) {
  constexpr int CHUNK = HIST_THREADS * HIST_ITEMS;
  const uint64_t chunks = (n + CHUNK - 1) / CHUNK;
  const int grid = int(std::min<uint64_t>(chunks, uint64_t(device().sm_count) * 8));
  KernelTimer kt("radix_histogram", s);
  key_histogram_kernel<KeyT, HIST_THREADS, HIST_ITEMS><<<grid, HIST_THREADS, 0, s>>>(cv, st, n);
  AM_CUDA(cudaGetLastError());
}

template <typename KeyT>
static void launch_pass(const PassArgs& pa, const ColView& cv, uint64_t n, cudaStream_t s) {
  using C = PassConfig<KeyT>;
  constexpr int TILE = C::THREADS * C::ITEMS;
  const uint64_t tiles = (n + TILE - 1) / TILE;
  const int grid = int(std::min<uint64_t>(tiles, uint64_t(device().sm_count) * pass_blocks_per_sm<KeyT>()));
  KernelTimer kt("radix_onesweep_pass", s);
  onesweep_pass_kernel<KeyT, C::THREADS, C::ITEMS><<<std::max(grid, 1), C::THREADS, pass_smem<KeyT>(), s>>>(pa, cv);
  AM_CUDA(cudaGetLastError());
}

static int min_tile() {
  return std::min(PassConfig<uint32_t>::THREADS * PassConfig<uint32_t>::ITEMS,
                  PassConfig<uint64_t>::THREADS * PassConfig<uint64_t>::ITEMS);
}

ColView make_view(const SortKey& k) {
  ColView v{};
  const am_array* a = k.col;
  v.values = a->data();
  v.valid = (a->null_count != 0) ? a->valid_bits() : nullptr;
  v.valid_off = a->validity_offset;
  v.bool_off = a->pt == PT_BOOL ? a->value_offset : 0;
  v.pt = a->pt;
  v.desc = k.descending ? 1 : 0;
  v.nulls_first = k.nulls_first ? 1 : 0;
  const bool fl = pt_float(a->pt);
  v.float_order = fl ? uint8_t(k.float_order) : uint8_t(FO_IEEE);
  v.nan_cat = (fl && k.float_order == FO_IEEE) ? 1 : 0;
  return v;
}

SortSummary* last_summary_host() {
  static thread_local SortSummary* host_sum = nullptr;
  if (!host_sum) host_sum = static_cast<SortSummary*>(pinned_alloc(sizeof(SortSummary)));
  return host_sum;
}

}  // namespace rs

void fill_last_sort_stats(am_sort_stats* out) {
  ThreadState& t = tls();
  *out = t.last_stats;
  if (!t.stats_stream) return;
  AM_CUDA(cudaStreamSynchronize(t.stats_stream));
  const rs::SortSummary* h = rs::last_summary_host();
  out->value_rows = h->value_rows;
  out->passes_run = int32_t(h->passes_run);
  out->passes_skipped = int32_t(h->passes_total - h->passes_run);
}

void radix_argsort(const std::vector<SortKey>& keys, int64_t n64, void* out, int index_width, cudaStream_t s,
                   am_sort_stats* stats) {
  using namespace rs;
  const int K = int(keys.size());
  if (K < 1 || K > MAX_KEYS) throw invalid("sort takes 1 to " + std::to_string(MAX_KEYS) + " key columns");
  if (n64 <= 0) return;
  const uint64_t n = uint64_t(n64);

  // Slots: least significant key first; its digits low to high, then (lower keys) a category slot.
  PlanArgs pa{};
  pa.nkeys = K;
  pa.n = n;
  pa.index_wide = index_width == 8 ? 1 : 0;
  std::vector<int> slot_bytes;
  int S = 0;
  for (int k = K - 1; k >= 0; k--) {
    const int kb = pt_key_bytes(keys[k].col->pt);
    pa.key_bytes[k] = uint8_t(kb);
    pa.nulls_first[k] = keys[k].nulls_first ? 1 : 0;
    for (int d = 0; d < kb; d++) {
      if (k == 0 && d == 0) pa.slot_key0_first = S;
      pa.slot_key[S] = int8_t(k);
      pa.slot_digit[S] = int8_t(d);
      slot_bytes.push_back(kb);
      S++;
    }
    if (k > 0) {
      pa.slot_key[S] = int8_t(k);
      pa.slot_digit[S] = -1;
      slot_bytes.push_back(4);
      S++;
    }
  }
  pa.nslots = S;

  int max_kb = 4;
  for (auto& k : keys) max_kb = std::max(max_kb, pt_key_bytes(k.col->pt));

  // Per-call scratch: stats, plans, pass descriptors, tickets, summary (one memset), then the
  // ping-pong key and id buffers.
  const size_t off_stats = 0;
  const size_t off_kplan = off_stats + sizeof(KeyStats) * K;
  const size_t off_desc = (off_kplan + sizeof(KeyPlan) * K + 255) & ~size_t(255);
  const size_t off_tick = off_desc + sizeof(PassDesc) * S;
  const size_t off_sum = (off_tick + sizeof(uint32_t) * S + 15) & ~size_t(15);
  const size_t header = (off_sum + sizeof(SortSummary) + 255) & ~size_t(255);
  const size_t kbuf = ((n * max_kb) + 255) & ~size_t(255);
  const size_t ibuf = ((n * 4) + 255) & ~size_t(255);
  char* base = static_cast<char*>(dmalloc(header + 2 * kbuf + 2 * ibuf, s));
  AM_CUDA(cudaMemsetAsync(base, 0, header, s));
  KeyStats* st = reinterpret_cast<KeyStats*>(base + off_stats);
  KeyPlan* kp = reinterpret_cast<KeyPlan*>(base + off_kplan);
  PassDesc* pd = reinterpret_cast<PassDesc*>(base + off_desc);
  uint32_t* tick = reinterpret_cast<uint32_t*>(base + off_tick);
  SortSummary* sum = reinterpret_cast<SortSummary*>(base + off_sum);
  void* kbufA = base + header;
  void* kbufB = base + header + kbuf;
  uint32_t* ibufA = reinterpret_cast<uint32_t*>(base + header + 2 * kbuf);
  uint32_t* ibufB = reinterpret_cast<uint32_t*>(base + header + 2 * kbuf + ibuf);
  if (debug_skip_first_tile()) {
    // Test hook: every pass's ticket starts at 1, so tile 0 is never processed and the look-back of
    // tile 1 runs into its time limit.
    const std::vector<uint32_t> ones(size_t(S), 1u);
    AM_CUDA(cudaMemcpyAsync(tick, ones.data(), sizeof(uint32_t) * S, cudaMemcpyHostToDevice, s));
    AM_CUDA(cudaStreamSynchronize(s));
  }

  std::vector<ColView> views(K);
  for (int k = 0; k < K; k++) {
    views[k] = make_view(keys[k]);
    if (pt_key_bytes(keys[k].col->pt) == 8) launch_histogram<uint64_t>(views[k], st + k, n, s);
    else launch_histogram<uint32_t>(views[k], st + k, n, s);
  }
  {
    KernelTimer kt("radix_plan", s);
    plan_kernel<<<1, 256, 0, s>>>(pa, st, kp, pd, sum);
    AM_CUDA(cudaGetLastError());
  }

  const uint64_t max_tiles = (n + min_tile() - 1) / min_tile();
  StreamScratch& sc = stream_scratch(s, size_t(max_tiles) * NBINS);
  for (int sl = 0; sl < S; sl++) {
    if (sc.epoch >= (1u << 30) - 1) {
      AM_CUDA(cudaMemsetAsync(sc.status, 0, sc.status_words * sizeof(uint64_t), s));
      sc.epoch = 0;
    }
    PassArgs a{};
    a.desc = pd + sl;
    a.kplan = kp + pa.slot_key[sl];
    a.keys[0] = kbufA;
    a.keys[1] = kbufB;
    a.ids[0] = ibufA;
    a.ids[1] = ibufB;
    a.final_out = out;
    a.status = sc.status;
    a.epoch = ++sc.epoch;
    a.tile_counter = tick + sl;
    a.err = sc.err;
    const ColView& cv = views[pa.slot_key[sl]];
    if (slot_bytes[sl] == 8) launch_pass<uint64_t>(a, cv, n, s);
    else launch_pass<uint32_t>(a, cv, n, s);
  }
  if (stats) {
    // Counters arrive asynchronously; am_last_sort_stats waits for them.
    stats->rows = int64_t(n);
    AM_CUDA(cudaMemcpyAsync(last_summary_host(), sum, sizeof(SortSummary), cudaMemcpyDeviceToHost, s));
    tls().stats_stream = s;
  }
  dfree(base, s);
}

}  // namespace am
