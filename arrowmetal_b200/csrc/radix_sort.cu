// Stable LSD radix argsort for sm_100a: one key-encode + all-digit histogram read per key column,
// a one-block planning kernel, then onesweep digit passes with warp-ballot multisplit ranking and
// decoupled look-back, skipping every digit that is constant over the column.
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
#include <atomic>
#include <cstdlib>
#include <list>
#include <memory>
#include <cstring>
#include <type_traits>

#include "am_internal.h"
#include "radix_sort.cuh"
#include "key_encode.cuh"


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
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Byte p of a key (digit p), zero-extended: one byte permute.
__device__ __forceinline__ uint32_t key_byte(uint32_t k, int p) { return __byte_perm(k, 0u, 0x4440u | uint32_t(p)); }
__device__ __forceinline__ uint32_t key_byte(uint64_t k, int p) {
  return p < 4 ? __byte_perm(uint32_t(k), 0u, 0x4440u | uint32_t(p)) : __byte_perm(uint32_t(k >> 32), 0u, 0x4440u | uint32_t(p - 4));
}

// Look-back status words. 32-bit: flag (2 bits) | count (30 bits), zeroed before every pass; used when a
// pass has fewer than 2^30 rows. 64-bit: the pass epoch (30 bits) | flag | count (32 bits), never
// cleared: a word of an older pass has another epoch.
template <typename S> struct Status;
template <> struct Status<uint32_t> {
  static constexpr int WINDOW = 8;        // measured passes: 8 a round trip 1.46 ms, 16 1.49, 32 1.55
  static __device__ __forceinline__ uint32_t make(uint32_t, uint32_t flag, uint32_t count) { return (flag << 30) | count; }
  static __device__ __forceinline__ bool ready(uint32_t s, uint32_t) { return (s >> 30) != 0u; }
  static __device__ __forceinline__ uint32_t flag(uint32_t s) { return s >> 30; }
  static __device__ __forceinline__ uint32_t count(uint32_t s) { return s & 0x3FFFFFFFu; }
  static __device__ __forceinline__ uint32_t load(const uint32_t* p) { return ld_relaxed_u32(p); }
  static __device__ __forceinline__ void store(uint32_t* p, uint32_t v) { st_relaxed_u32(p, v); }
};
template <> struct Status<uint64_t> {
  static constexpr int WINDOW = 16;
  static __device__ __forceinline__ uint64_t make(uint32_t e, uint32_t flag, uint32_t count) { return pack_status(e, flag, count); }
  static __device__ __forceinline__ bool ready(uint64_t s, uint32_t e) { return uint32_t(s >> 34) == e && ((s >> 32) & 3u) != 0u; }
  static __device__ __forceinline__ uint32_t flag(uint64_t s) { return uint32_t(s >> 32) & 3u; }
  static __device__ __forceinline__ uint32_t count(uint64_t s) { return uint32_t(s); }
  static __device__ __forceinline__ uint64_t load(const uint64_t* p) { return ld_relaxed_u64(p); }
  static __device__ __forceinline__ void store(uint64_t* p, uint64_t v) { st_relaxed_u64(p, v); }
};

// ------------------------------------------------------------------------------------------------
// Kernel 1: key encode + all-digit histogram of one key column.
//
// One read of the column gives every digit's 256 counts (the reference reads the keys once per pass,
// SortSource.swift:31-73), the null and NaN-block counts, and the largest and smallest value key
// (for folding a lower key's null / NaN rows into its key range). A warp whose keys agree on a digit
// adds its count with one atomic instead of 32, so a digit that is constant over the column (the
// high bytes of keys drawn from [0, 2^40)) costs almost nothing.

// The block's share of one column: rows [first, end) in chunks of THREADS x ITEMS rows, `stride` rows
// apart, added into `st`.
// RANGE: also the largest and smallest value key (only a lower key of a multi-key sort folds its null and
// NaN rows into its key range; for any other key the two 64-bit maxima per row are left out).
template <typename KeyT, int THREADS, int ITEMS, bool RANGE = true>
__device__ __forceinline__ void histogram_rows(const ColView& col, KeyStats* __restrict__ st, uint64_t first,
                                               uint64_t end, uint64_t stride) {
  constexpr int D = int(sizeof(KeyT));
  // Per digit 256 bins and one more, which takes the (discarded) counts of rows that are not values,
  // so every item adds to a bin without a branch.
  constexpr int STRIDE = 257;
  __shared__ uint32_t sh[D * STRIDE];
  __shared__ uint32_t s_null, s_nan, s_val;
  __shared__ unsigned long long s_max, s_min_inv;
  for (int i = threadIdx.x; i < D * STRIDE; i += THREADS) sh[i] = 0;
  if (threadIdx.x == 0) { s_null = 0; s_nan = 0; s_val = 0; s_max = 0; s_min_inv = 0; }
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t n_null = 0, n_nan = 0, n_val = 0;
  KeyT vmax = 0, vmin_inv = 0;

  for (uint64_t base = first; base < end; base += stride) {
    KeyT k[ITEMS];
    int cat[ITEMS];
    uint32_t row[ITEMS];
    uint32_t ok = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const uint64_t g = base + uint64_t(warp) * (ITEMS * 32) + uint64_t(i) * 32 + lane;
      row[i] = uint32_t(g);
      if (g < end) ok |= 1u << i;
    }
    {
      // The block's rows are warp-striped from a multiple of 32: validity a bitmap word an item.
      KeyT raw[ITEMS];
      load_raw_rows<KeyT, ITEMS>(col, row, ok, raw);
      const uint32_t vmask = striped_validity<ITEMS>(col, base + uint64_t(warp) * (ITEMS * 32), end, ok);
      encode_raw<KeyT, ITEMS>(col, raw, vmask, k, cat);
    }
    uint32_t valid_mask = 0;
    KeyT o = 0, a = KeyT(~KeyT(0));
    uint32_t nv = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      if (!((ok >> i) & 1u)) continue;
      if (cat[i] == 0) {
        const KeyT kk = k[i];
        valid_mask |= 1u << i;
        o |= kk;
        a &= kk;
        nv++;
        if constexpr (RANGE) {
          vmax = kk > vmax ? kk : vmax;
          vmin_inv = KeyT(~kk) > vmin_inv ? KeyT(~kk) : vmin_inv;
        }
      } else if (cat[i] == 1) {
        n_nan++;
      } else {
        n_null++;
      }
    }
    n_val += nv;
    const KeyT wo = warp_or<KeyT>(o), wa = warp_and<KeyT>(a);
    const KeyT wdiff = KeyT(wo ^ wa);
    const uint32_t wnv = __reduce_add_sync(0xffffffffu, nv);
    // Rows that are not values count in the extra bin: their key is taken as 0 and offset by 256.
    KeyT km[ITEMS];
    uint32_t pad[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const bool v = (valid_mask >> i) & 1u;
      km[i] = v ? k[i] : KeyT(0);
      pad[i] = v ? 0u : 256u;
    }
#pragma unroll
    for (int p = 0; p < D; p++) {
      if (key_byte(wdiff, p) == 0u) {
        if (lane == 0 && wnv) atomicAdd(&sh[p * STRIDE + key_byte(wa, p)], wnv);
      } else {
#pragma unroll
        for (int i = 0; i < ITEMS; i++) atomicAdd(&sh[p * STRIDE + key_byte(km[i], p) + pad[i]], 1u);
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
  for (int i = threadIdx.x; i < D * 256; i += THREADS) {
    const uint32_t c = sh[(i >> 8) * STRIDE + (i & 255)];
    if (c) atomicAdd(&st->hist[i >> 8][i & 255], c);
  }
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

template <typename KeyT, int THREADS, int ITEMS, bool RANGE = true>
__global__ void __launch_bounds__(THREADS) key_histogram_kernel(const __grid_constant__ ColView col, KeyStats* __restrict__ st, uint64_t n) {
  constexpr uint64_t CHUNK = uint64_t(THREADS) * ITEMS;
  histogram_rows<KeyT, THREADS, ITEMS, RANGE>(col, st, uint64_t(blockIdx.x) * CHUNK, n, uint64_t(gridDim.x) * CHUNK);
}

// ------------------------------------------------------------------------------------------------
// Kernel 2: the plan. One block decides, from the histograms alone, which digit passes run, where
// each pass reads and writes, and every pass's per-digit global base; the passes read it from HBM.

// Exclusive scan of 256 values held in shared memory; the first 256 threads of the block take part in
// the arithmetic and every thread in the barriers.
__device__ void block_exclusive_scan_256(const uint32_t* in, uint32_t* out, uint32_t* total, uint32_t* s_warp) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  uint32_t v = 0, x = 0;
  if (t < 256) {
    v = in[t];
    x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
  }
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
  if (t < 256) out[t] = x - v + s_warp[8 + warp];
  __syncthreads();
}

__device__ __forceinline__ uint64_t key_max(int bytes) { return bytes == 8 ? ~0ull : 0xFFFFFFFFull; }

__device__ void plan_body(const PlanArgs& a, KeyStats* __restrict__ st, KeyPlan* __restrict__ kp,
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
      if (is_last) flags |= PF_LAST;
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
      p.buf_rows = n;         // the ping-pong buffers and the output hold n rows
      p.out_rows = n;
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

__global__ void __launch_bounds__(256) plan_kernel(PlanArgs a, KeyStats* __restrict__ st, KeyPlan* __restrict__ kp,
                                                   PassDesc* __restrict__ pd, SortSummary* __restrict__ sum) {
  plan_body(a, st, kp, pd, sum);
}

// Segmented sorts: one histogram launch and one plan launch for all arrays of a key width.

// The last s in [0, count) with start[s] <= x (start ascending, start[0] = 0).
__device__ __forceinline__ uint32_t segment_of(const uint32_t* __restrict__ start, uint32_t count, uint32_t x) {
  uint32_t lo = 0, hi = count;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (start[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Block b histograms rows [r, r + rows_per_item) of the array whose items contain b.
template <typename KeyT, int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS) segmented_histogram_kernel(const SegDesc* __restrict__ segs,
                                                                      const uint32_t* __restrict__ item_start,
                                                                      uint32_t nsegs, uint32_t rows_per_item,
                                                                      KeyStats* __restrict__ st) {
  const uint32_t seg = segment_of(item_start, nsegs, blockIdx.x);
  const ColView col = segs[seg].col;
  const uint64_t n = segs[seg].n;
  const uint64_t lo = uint64_t(blockIdx.x - item_start[seg]) * rows_per_item;
  const uint64_t hi = lo + rows_per_item < n ? lo + rows_per_item : n;
  histogram_rows<KeyT, THREADS, ITEMS, false>(col, st + seg, lo, hi, uint64_t(THREADS) * ITEMS);
}

// Block s plans array s: one key of `key_bytes` bytes, uint32 indices.
__global__ void __launch_bounds__(256) segmented_plan_kernel(const SegDesc* __restrict__ segs, int key_bytes,
                                                             KeyStats* __restrict__ st, KeyPlan* __restrict__ kp,
                                                             PassDesc* __restrict__ pd, SortSummary* __restrict__ sum) {
  const uint32_t seg = blockIdx.x;
  PlanArgs a{};
  a.n = segs[seg].n;
  a.nkeys = 1;
  a.nslots = key_bytes;
  a.slot_key0_first = 0;
  a.index_wide = 0;
  a.key_bytes[0] = uint8_t(key_bytes);
  a.nulls_first[0] = segs[seg].col.nulls_first;
  for (int d = 0; d < key_bytes; d++) {
    a.slot_key[d] = 0;
    a.slot_digit[d] = int8_t(d);
  }
  plan_body(a, st + seg, kp + seg, pd + size_t(seg) * key_bytes, sum + seg);
}

// ------------------------------------------------------------------------------------------------
// Segmented sort of the arrays that fit one CTA: each such array of a batch is sorted by one CTA in
// shared memory, all of them in one persistent launch. A CTA encodes its array's rows (the key maps
// and categories of the digit passes), finds the digits that vary over its value rows, and ranks the
// rows by each varying digit, least significant first, then by their arrangement class (values, NaN
// block, nulls, in the order the null placement asks): DBITS-bit digits, one ballot per digit bit, so
// every pass is stable and so is the result. The same arrays through the digit passes give the same
// permutation; the autotuner picks DBITS and the block shape per size class by measurement.

// One stable ranking pass over a CTA's rows in shared memory by NB-bit digits `dg` (empty slots carry
// the largest digit and come last, never counted or stored): every row's place, rows then moved there.
template <int NBITS, int THREADS, int ITEMS, typename KeyT>
__device__ __forceinline__ void cta_rank_pass(KeyT (&key)[ITEMS], uint32_t (&id)[ITEMS], const uint32_t (&dg)[ITEMS],
                                              uint32_t ok, uint32_t size, int nit, KeyT* skeys, uint32_t* sids,
                                              uint32_t* whist, uint32_t* local, uint32_t* wsum) {
  constexpr int NB = 1 << NBITS, WARPS = THREADS / 32;
  constexpr int DPT = NB >= THREADS ? NB / THREADS : 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  for (int x = lane; x < NB; x += 32) whist[warp * NB + x] = 0;
  __syncwarp();
#pragma unroll
  for (int i = 0; i < ITEMS; i++)
    if ((ok >> i) & 1u) atomicAdd(&whist[warp * NB + dg[i]], 1u);
  __syncthreads();
  // Per digit: the warps' exclusive starts and the digit's total; then a scan over the digits.
  uint32_t tots[DPT];
  uint32_t tot = 0;
  const bool owner = int(threadIdx.x) * DPT < NB;
  if (owner) {
#pragma unroll
    for (int q = 0; q < DPT; q++) {
      const int d = int(threadIdx.x) * DPT + q;
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < WARPS; w++) {
        const uint32_t c = whist[w * NB + d];
        whist[w * NB + d] = run;
        run += c;
      }
      tots[q] = run;
      tot += run;
    }
  }
  uint32_t x = tot;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (owner) {
    uint32_t at = x - tot;
    for (int w = 0; w < warp; w++) at += wsum[w];
#pragma unroll
    for (int q = 0; q < DPT; q++) {
      local[int(threadIdx.x) * DPT + q] = at;
      at += tots[q];
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    if (i >= nit) break;
    const uint32_t d = dg[i];
    uint32_t peers = 0xffffffffu;
#pragma unroll
    for (int k = 0; k < NBITS; k++) {
      const uint32_t bit = (d >> k) & 1u;
      const uint32_t bl = __ballot_sync(0xffffffffu, bit);
      peers &= bit ? bl : ~bl;
    }
    const uint32_t b0 = whist[warp * NB + d];
    __syncwarp();
    if (lane == __ffs(peers) - 1) whist[warp * NB + d] = b0 + __popc(peers);
    const uint32_t p = local[d] + b0 + __popc(peers & lt);
    if (p < size) {
      skeys[p] = key[i];
      sids[p] = id[i];
    }
    __syncwarp();
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    const uint32_t r = uint32_t(warp) * (ITEMS * 32) + uint32_t(i) * 32 + lane;
    if ((ok >> i) & 1u) {
      key[i] = skeys[r];
      id[i] = sids[r];
    }
  }
  __syncthreads();
}

template <typename KeyT, int THREADS, int ITEMS, int DBITS>
__host__ __device__ constexpr size_t cta_sort_smem() {
  return size_t(THREADS) * ITEMS * (sizeof(KeyT) + 4) + size_t(THREADS / 32) * (size_t(1) << DBITS) * 4 +
         (size_t(1) << DBITS) * 4 + size_t(THREADS / 32) * 4 + 2 * sizeof(unsigned long long) + 16;
}

// Arrays list[0 .. count) of `segs`, each of at most THREADS x ITEMS rows, one CTA at a time.
template <typename KeyT, int THREADS, int ITEMS, int DBITS>
__global__ void __launch_bounds__(THREADS) segment_cta_sort_kernel(const SegDesc* __restrict__ segs, uint32_t count,
                                                                   uint32_t* __restrict__ err) {
  constexpr int CAP = THREADS * ITEMS, WARPS = THREADS / 32, NB = 1 << DBITS;
  constexpr int KBITS = int(sizeof(KeyT)) * 8;
  static_assert(DBITS >= 2, "the arrangement pass uses 2-bit digits within the same histogram space");
  extern __shared__ __align__(16) unsigned char cta_smem[];
  KeyT* skeys = reinterpret_cast<KeyT*>(cta_smem);
  uint32_t* sids = reinterpret_cast<uint32_t*>(skeys + CAP);
  uint32_t* whist = sids + CAP;                           // [WARPS][NB]
  uint32_t* local = whist + WARPS * NB;                   // [NB]
  uint32_t* wsum = local + NB;                            // [WARPS]
  unsigned long long* red = reinterpret_cast<unsigned long long*>(
      (reinterpret_cast<uintptr_t>(wsum + WARPS) + 15) & ~uintptr_t(15));   // OR and AND of the value keys
  uint32_t* any_cat = reinterpret_cast<uint32_t*>(red + 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t j = blockIdx.x; j < count; j += gridDim.x) {
    const SegDesc& sd = segs[j];
    const uint32_t size = sd.n;
    if (size > uint32_t(CAP)) {           // the host sends only arrays that fit; never read past the tile
      if (threadIdx.x == 0) atomicOr(err, ERR_BOUNDS);
      continue;
    }
    if (threadIdx.x == 0) {
      red[0] = 0ull;
      red[1] = ~0ull;
      *any_cat = 0;
    }
    __syncthreads();
    const ColView col = sd.col;
    uint32_t row[ITEMS];
    uint32_t ok = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      row[i] = uint32_t(warp) * (ITEMS * 32) + uint32_t(i) * 32 + lane;
      if (row[i] < size) ok |= 1u << i;
    }
    KeyT key[ITEMS];
    int cat[ITEMS];
    encode_rows<KeyT, ITEMS>(col, row, ok, key, cat);
    uint32_t id[ITEMS];
    KeyT kor = 0, kand = ~KeyT(0);
    uint32_t cats = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      id[i] = row[i];
      if (!((ok >> i) & 1u)) continue;
      if (cat[i] == 0) {
        kor |= key[i];
        kand &= key[i];
      } else {
        key[i] = 0;
        cats = 1;
      }
    }
    kor = warp_or(kor);
    kand = warp_and(kand);
    cats = __reduce_or_sync(0xffffffffu, cats);
    if (lane == 0) {
      atomicOr(&red[0], (unsigned long long)kor);
      atomicAnd(&red[1], (unsigned long long)kand);
      if (cats) atomicOr(any_cat, 1u);
    }
    __syncthreads();
    // A CTA with no value rows has OR 0 and AND all ones: no varying digit.
    const KeyT diff = red[0] <= red[1] ? KeyT(0) : KeyT(red[0] ^ red[1]);
    const bool arrange = *any_cat != 0;
    const uint32_t w_first = uint32_t(warp) * (ITEMS * 32);
    const int nit = size > w_first ? int(min(uint32_t(ITEMS), (size - w_first + 31) / 32)) : 0;
    // Every row's arrangement class before any pass moves it.
    uint32_t cls[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) cls[i] = col.nulls_first ? uint32_t(2 - cat[i]) : uint32_t(cat[i]);
    if (arrange) {
      // The class rides in the key's place for the value digits' passes: carried in the row id's top
      // bits (ids are below 2^16 here).
#pragma unroll
      for (int i = 0; i < ITEMS; i++) id[i] |= cls[i] << 30;
    }
    for (int shift = 0; shift < KBITS; shift += DBITS) {
      const KeyT mask = KeyT((uint64_t(1) << DBITS) - 1) << shift;
      if (!(diff & mask)) continue;
      uint32_t dg[ITEMS];
#pragma unroll
      for (int i = 0; i < ITEMS; i++) dg[i] = ((ok >> i) & 1u) ? uint32_t(key[i] >> shift) & uint32_t(NB - 1) : uint32_t(NB - 1);
      cta_rank_pass<DBITS, THREADS, ITEMS, KeyT>(key, id, dg, ok, size, nit, skeys, sids, whist, local, wsum);
    }
    if (arrange) {
      uint32_t dg[ITEMS];
#pragma unroll
      for (int i = 0; i < ITEMS; i++) dg[i] = ((ok >> i) & 1u) ? (id[i] >> 30) : 3u;
      cta_rank_pass<2, THREADS, ITEMS, KeyT>(key, id, dg, ok, size, nit, skeys, sids, whist, local, wsum);
    }
    uint32_t* out = static_cast<uint32_t*>(sd.out);
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const uint32_t r = uint32_t(warp) * (ITEMS * 32) + uint32_t(i) * 32 + lane;
      if ((ok >> i) & 1u) out[r] = id[i] & 0x3FFFFFFFu;
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
// the input order. The tile's digit counts go out as look-back aggregates before any ranking; each
// warp then ranks its rows (one ballot per digit bit, the reference's ballot multisplit of
// SortSource.swift:334-386) and stages them in shared memory at their tile-local sorted slot; the
// decoupled look-back (a window of predecessors per L2 round trip, bounded in time) turns the counts
// into global offsets; and the rows leave shared memory in order, so consecutive threads write
// consecutive addresses within every digit run.

template <typename KeyT, int THREADS, int ITEMS, typename IdT = uint32_t>
struct PassShared {
  static constexpr int WARPS = THREADS / 32;
  static constexpr int TILE = THREADS * ITEMS;
  SegDesc sdesc;                 // segmented passes: the tile's array
  PassDesc desc;
  uint32_t whist[WARPS][NBINS];
  uint32_t cnt[NBINS];
  uint32_t local[NBINS];
  uint32_t gdelta[NBINS];
  uint32_t scan_warp[16];
  uint32_t scan_total;
  uint32_t ticket;
  uint32_t seg;
  uint32_t lo_first, lo_last;    // PF_BUCKETS: the lower bucket digit of the tile's first and last rows
  // Each staged row's digit; in record passes (16-bit places) the digit << 16 | the row's place within
  // the tile, one word read for both.
  using DigT = std::conditional_t<sizeof(IdT) == 2, uint32_t, uint16_t>;
  DigT dig[TILE];
  KeyT keys[TILE];
  IdT ids[sizeof(IdT) == 2 ? 1 : TILE];   // row ids (passes that carry them)
};

// Inverse of the integer and totalOrder key maps (SortSource.swift:131-190 read backwards): the value
// bits of a key, at the key's width.
template <typename KeyT>
__device__ __forceinline__ uint64_t unkey_bits(KeyT k, int pt, int desc) {
  if (desc) k = KeyT(~k);
  if constexpr (sizeof(KeyT) == 8) {
    const uint64_t S = 0x8000000000000000ull;
    if (pt == PT_I64) return k ^ S;
    if (pt == PT_F64) return (k & S) ? (k ^ S) : ~k;
    return k;
  } else {
    const uint32_t S = 0x80000000u;
    if (pt == PT_U32) return k;
    if (pt == PT_F32) return (k & S) ? (k ^ S) : uint32_t(~k);
    return uint32_t(k ^ S);          // int32 and the narrow types widened to it (truncated on store)
  }
}

__device__ __forceinline__ void store_width(void* base, uint64_t i, int width, uint64_t v) {
  switch (width) {
    case 8: static_cast<uint64_t*>(base)[i] = v; break;
    case 4: static_cast<uint32_t*>(base)[i] = uint32_t(v); break;
    case 2: static_cast<uint16_t*>(base)[i] = uint16_t(v); break;
    default: static_cast<uint8_t*>(base)[i] = uint8_t(v); break;
  }
}
// ---- payload records (RecLayout)

__device__ __forceinline__ uint64_t load_width(const void* base, uint64_t i, int width) {
  switch (width) {
    case 8: return static_cast<const uint64_t*>(base)[i];
    case 4: return static_cast<const uint32_t*>(base)[i];
    case 2: return static_cast<const uint16_t*>(base)[i];
    default: return static_cast<const uint8_t*>(base)[i];
  }
}

// Row `row`'s record: its id and its payload fields read from the columns.
__device__ __forceinline__ uint4 build_record(const RecLayout& L, uint32_t row) {
  if (L.pair) {
    const uint64_t w = static_cast<const uint64_t*>(L.src[L.wide])[row];
    return make_uint4(row, uint32_t(w), uint32_t(w >> 32), static_cast<const uint32_t*>(L.src[L.narrow])[row]);
  }
  uint64_t lo = 0;           // payload bytes 0-7
  uint32_t hi = 0;           // payload bytes 8-11
  for (int c = 0; c < L.ncols; c++) {
    const uint64_t v = load_width(L.src[c], row, L.width[c]);
    const int o = L.off[c];
    if (o < 8) lo |= v << (8 * o);
    else hi |= uint32_t(v) << (8 * (o - 8));
  }
  return make_uint4(row, uint32_t(lo), uint32_t(lo >> 32), hi);
}

// A record's payload fields, written to row `dst` of the sorted payload columns.
__device__ __forceinline__ void unpack_record(const RecLayout& L, const uint4& r, uint64_t dst) {
  const uint64_t lo = uint64_t(r.y) | (uint64_t(r.z) << 32);
  if (L.pair) {
    static_cast<uint64_t*>(L.dst[L.wide])[dst] = lo;
    static_cast<uint32_t*>(L.dst[L.narrow])[dst] = r.w;
    return;
  }
  for (int c = 0; c < L.ncols; c++) {
    const int o = L.off[c];
    const uint64_t v = o < 8 ? (lo >> (8 * o)) : uint64_t(r.w >> (8 * (o - 8)));
    store_width(L.dst[c], dst, L.width[c], v);
  }
}

template <typename KeyT, typename StatusT, int THREADS, int ITEMS, bool SEG, bool REC = false>
__global__ void __launch_bounds__(THREADS, 2)
onesweep_pass_kernel(const __grid_constant__ PassArgs pa, const __grid_constant__ ColView col_arg) {
  static_assert(THREADS >= NBINS && THREADS % 32 == 0, "one thread per digit bin");
  static_assert(THREADS * ITEMS <= 65536, "tile-local ranks are 16-bit");
  static_assert(!(SEG && REC), "record passes sort one array");
  using ST = Status<StatusT>;
  using SM = PassShared<KeyT, THREADS, ITEMS, std::conditional_t<REC, uint16_t, uint32_t>>;
  constexpr int TILE = SM::TILE;
  constexpr int WARPS = SM::WARPS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SM& sm = *reinterpret_cast<SM*>(smem_raw);
  StatusT* __restrict__ status = static_cast<StatusT*>(pa.status);

  auto copy_words = [](void* dst, const void* src, int words) {
    for (int i = threadIdx.x; i < words; i += THREADS)
      static_cast<uint32_t*>(dst)[i] = static_cast<const uint32_t*>(src)[i];
  };
  // What the pass descriptor says, for the arrays at `row_off` of the buffers.
  uint32_t flags = 0, shift = 0, ntiles = 0;
  uint64_t count = 0;
  int si = -1, di = -1;
  const KeyT* __restrict__ keys_in = nullptr;
  const uint32_t* __restrict__ ids_in = nullptr;
  KeyT* __restrict__ keys_out = nullptr;
  uint32_t* __restrict__ ids_out = nullptr;
  auto bind = [&](uint64_t row_off) {
    flags = sm.desc.flags;
    count = sm.desc.count;
    shift = sm.desc.shift;
    ntiles = uint32_t((count + TILE - 1) / TILE);
    const int sk = sm.desc.src_keys, dk = sm.desc.dst_keys;
    si = sm.desc.src_ids;
    di = sm.desc.dst_ids;
    keys_in = sk < 0 ? nullptr : static_cast<const KeyT*>(sk == 0 ? pa.keys[0] : pa.keys[1]) + row_off;
    ids_in = si < 0 ? nullptr : (si == 0 ? pa.ids[0] : pa.ids[1]) + row_off;
    keys_out = dk < 0 ? nullptr : static_cast<KeyT*>(dk == 0 ? pa.keys[0] : pa.keys[1]) + row_off;
    ids_out = di < 0 ? nullptr : (di == 0 ? pa.ids[0] : pa.ids[1]) + row_off;
  };
  KeyPlan kplan{};
  void* final_out = pa.final_out;
  const ColView* colp = &col_arg;
  if constexpr (!SEG) {
    copy_words(&sm.desc, pa.desc, int(sizeof(PassDesc) / 4));
    __syncthreads();
    if (!sm.desc.active) return;
    bind(0);
    kplan = *pa.kplan;
  }
  const uint32_t epoch = pa.epoch;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t lt_mask = (1u << lane) - 1u;

  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t t = atomicAdd(pa.tile_counter, 1u);
      sm.ticket = t;
      if constexpr (SEG) {
        // The segment of tile t: the last s with tile_start[s] <= t.
        uint32_t lo = 0, hi = pa.nsegs;
        if (t < pa.total_tiles) {
          while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (pa.tile_start[mid] <= t) lo = mid;
            else hi = mid;
          }
        }
        sm.seg = lo;
      }
    }
    for (int b = lane; b < NBINS; b += 32) sm.whist[warp][b] = 0;
    __syncthreads();
    const uint32_t T = sm.ticket;   // the launch's tile number
    uint32_t tile;                   // the tile within its array
    if constexpr (SEG) {
      if (T >= pa.total_tiles) break;
      const uint32_t seg = sm.seg;
      copy_words(&sm.desc, pa.desc + size_t(seg) * pa.nslots + pa.slot, int(sizeof(PassDesc) / 4));
      copy_words(&sm.sdesc, pa.segs + seg, int(sizeof(SegDesc) / 4));
      __syncthreads();
      bind(sm.sdesc.row_off);
      kplan = pa.kplan[seg];
      colp = &sm.sdesc.col;
      final_out = sm.sdesc.out;
      tile = T - pa.tile_start[seg];
      // An array whose digit is constant, or a tile past its rows (its later passes see only its value
      // rows): nothing to do, and no tile of the array waits on it.
      if (!sm.desc.active || tile >= ntiles) continue;
    } else {
      tile = T;
      if (tile >= ntiles) break;
    }
    const ColView& col = *colp;
    const uint64_t first_tile = uint64_t(T) - tile;   // status index of the array's tile 0
    const uint64_t tile_base = uint64_t(tile) * TILE;

    // ---- load and digit: row ids first, then every item's key load back to back
    KeyT key[ITEMS];
    uint32_t id[ITEMS];
    uint32_t dg[ITEMS];
    const uint64_t wbase = tile_base + uint64_t(warp) * (ITEMS * 32) + lane;
    uint32_t ok = (1u << ITEMS) - 1u;      // a full tile: every item holds a row
    if (count - tile_base < uint64_t(TILE)) {
      ok = 0;
#pragma unroll
      for (int i = 0; i < ITEMS; i++)
        if (wbase + uint64_t(i) * 32 < count) ok |= 1u << i;
    }
    if (ids_in && pa.carry_ids && !REC) {
#pragma unroll
      for (int i = 0; i < ITEMS; i++) id[i] = ((ok >> i) & 1u) ? ids_in[wbase + uint64_t(i) * 32] : 0u;
    } else {
#pragma unroll
      for (int i = 0; i < ITEMS; i++) id[i] = uint32_t(wbase + uint64_t(i) * 32);
    }
    if (flags & PF_CATPASS) {
#pragma unroll
      for (int i = 0; i < ITEMS; i++) {
        key[i] = 0;
        const bool is_null = ((ok >> i) & 1u) && col.valid && !bit_at(col.valid, col.valid_off + int64_t(id[i]));
        dg[i] = ((ok >> i) & 1u) ? ((is_null != bool(col.nulls_first)) ? 1u : 0u) : INVALID_DIGIT;
      }
    } else if (flags & PF_ENCODE) {
      // Raw values and validity bytes loaded together; then each row's key, category and digit in one
      // step, so only one row's category is live at a time.
      KeyT raw[ITEMS];
      uint32_t vb[ITEMS];
      load_raw_rows<KeyT, ITEMS>(col, id, ok, raw);
      // Validity: rows in their own order are warp-striped from a multiple of 32 (a bitmap word an
      // item); rows reached through gathered ids read their bytes.
      uint32_t vmask = ok;
      if (col.valid) {
        if (!(ids_in && pa.carry_ids && !REC)) {
          vmask = striped_validity<ITEMS>(col, wbase - lane, count, ok);
        } else {
#pragma unroll
          for (int i = 0; i < ITEMS; i++) vb[i] = ((ok >> i) & 1u) ? col.valid[(col.valid_off + int64_t(id[i])) >> 3] : 0u;
#pragma unroll
          for (int i = 0; i < ITEMS; i++)
            if (!((vb[i] >> ((col.valid_off + int64_t(id[i])) & 7)) & 1u)) vmask &= ~(1u << i);
        }
      }
      // A row's key, digit and routing from its key and category.
      auto place = [&](int i, KeyT k, int cat) {
        if (cat && (flags & PF_ROUTE)) {
          dg[i] = (cat == 1) ? uint32_t(NAN_BIN) : uint32_t(NULL_BIN);
        } else {
          if (cat) k = kplan.fold_mode ? KeyT(0) : KeyT(cat == 1 ? kplan.fold_nan : kplan.fold_null);
          dg[i] = uint32_t(k >> shift) & 255u;
        }
        if (!((ok >> i) & 1u)) dg[i] = INVALID_DIGIT;
        key[i] = k;
      };
      constexpr bool WIDE = sizeof(KeyT) == 8;
      const bool fl = WIDE ? col.pt == PT_F64 : (col.pt == PT_F32 || col.pt == PT_F16);
      if (!fl) {
        // Integer keys: one XOR a row (sign flip and direction decided once), no branch on the type.
        const KeyT sign = KeyT(KeyT(1) << (8 * sizeof(KeyT) - 1));
        const KeyT flip = WIDE ? (col.pt == PT_I64 ? sign : KeyT(0)) : (col.pt == PT_U32 ? KeyT(0) : sign);
        const KeyT x = flip ^ (col.desc ? KeyT(~KeyT(0)) : KeyT(0));
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
          const bool valid = (vmask >> i) & 1u;
          place(i, valid ? KeyT(raw[i] ^ x) : KeyT(0), valid ? 0 : 2);
        }
      } else {
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
          const bool valid = (vmask >> i) & 1u;
          int cat;
          const KeyT k = key_from_raw<KeyT>(col, raw[i], valid, cat);
          place(i, k, cat);
        }
      }
    } else {
#pragma unroll
      for (int i = 0; i < ITEMS; i++) key[i] = ((ok >> i) & 1u) ? keys_in[wbase + uint64_t(i) * 32] : KeyT(0);
#pragma unroll
      for (int i = 0; i < ITEMS; i++) dg[i] = ((ok >> i) & 1u) ? (uint32_t(key[i] >> shift) & 255u) : INVALID_DIGIT;
    }

    // The two-level sort's second pass counts its buckets (this pass's digit, the lower digit). Its rows
    // arrive ordered by the lower digit (the first pass sorted by it), so the tile's first and last rows
    // tell whether one lower digit covers the whole tile.
    if ((flags & PF_BUCKETS) && threadIdx.x == 0) {
      // Thread 0's first item is the tile's first row; the last row's key is read again (L2).
      const uint32_t lsh = sm.desc.bucket_shift;
      const uint64_t last_row = (count - tile_base < uint64_t(TILE) ? count : tile_base + TILE) - 1;
      sm.lo_first = uint32_t(key[0] >> lsh) & 255u;
      sm.lo_last = uint32_t(keys_in[last_row] >> lsh) & 255u;
    }

    // ---- early counts: the tile's per-digit counts go out as look-back aggregates before any
    // ranking, so the tiles after this one can resolve their prefixes as early as possible.
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
      if (dg[i] != INVALID_DIGIT) atomicAdd(&sm.whist[warp][dg[i]], 1u);
    __syncthreads();
    const bool one_lower = (flags & PF_BUCKETS) && sm.lo_first == sm.lo_last;
    for (int b = threadIdx.x; b < NBINS; b += THREADS) {
      uint32_t run = 0;
#pragma unroll
      for (int w = 0; w < WARPS; w++) {
        const uint32_t c = sm.whist[w][b];
        sm.whist[w][b] = run;
        run += c;
      }
      sm.cnt[b] = run;
      ST::store(status + uint64_t(T) * NBINS + b, ST::make(epoch, tile == 0 ? ST_INCL : ST_AGG, run));
      // One lower digit in the tile: each digit's count is its bucket's share.
      if (one_lower && b < RADIX && run) atomicAdd(pa.bucket_count + ((uint32_t(b) << 8) | sm.lo_first), run);
    }
    if ((flags & PF_BUCKETS) && !one_lower) {
      // The tile holds a change of the lower digit (at most 255 tiles of the pass do): one count a row.
      const uint32_t lsh = sm.desc.bucket_shift;
#pragma unroll
      for (int i = 0; i < ITEMS; i++)
        if (dg[i] < uint32_t(RADIX)) atomicAdd(pa.bucket_count + ((dg[i] << 8) | (uint32_t(key[i] >> lsh) & 255u)), 1u);
    }
    // Tile-local digit starts: value digits in order, then the NaN and null routing bins.
    block_exclusive_scan_256(sm.cnt, sm.local, &sm.scan_total, sm.scan_warp);
    if (threadIdx.x == 0) {
      const uint32_t t = sm.local[255] + sm.cnt[255];
      sm.local[NAN_BIN] = t;
      sm.local[NULL_BIN] = t + sm.cnt[NAN_BIN];
    }
    __syncthreads();

    // Passes that neither route nor sort categories take each staged row's digit from its key again
    // instead of staging it.
    const bool dig_from_key = !REC && !(flags & (PF_ROUTE | PF_CATPASS));
    // ---- warp ranking and staging: each row goes to its tile-local sorted slot. The rows of a lane's
    // item that share its digit come from one ballot per digit bit, and the item is placed right after
    // its ballots: holding every item's peer mask first overlaps more ballots but pushes the 8-byte
    // key's pass past its 80 registers into spills, which measured slower.
    {
      const int nbits = (flags & PF_ROUTE) ? 9 : 8;
      // Rows past the end carry INVALID_DIGIT. Nine digit bits already tell it apart (its low nine bits
      // are 511, no bin's); with eight, only a tile that ends early has such rows and needs the ballot.
      const bool invalid_ballot = nbits == 8 && count - tile_base < uint64_t(TILE);
#pragma unroll
      for (int i = 0; i < ITEMS; i++) {
        const uint32_t d = dg[i];
        uint32_t peers = invalid_ballot ? __ballot_sync(0xffffffffu, d != INVALID_DIGIT) : 0xffffffffu;
#pragma unroll
        for (int k = 0; k < 9; k++) {
          if (k < nbits) {
            const uint32_t bit = (d >> k) & 1u;
            const uint32_t bl = __ballot_sync(0xffffffffu, bit);
            peers &= bit ? bl : ~bl;
          }
        }
        uint32_t base = 0;
        if (d != INVALID_DIGIT) base = sm.whist[warp][d];
        __syncwarp();
        if (d != INVALID_DIGIT) {
          if (lane == __ffs(peers) - 1) sm.whist[warp][d] = base + __popc(peers);
          const uint32_t pos = sm.local[d] + base + __popc(peers & lt_mask);
          sm.keys[pos] = key[i];
          if constexpr (REC) {
            sm.dig[pos] = (d << 16) | (id[i] - uint32_t(tile_base));
          } else {
            if (pa.carry_ids) sm.ids[pos] = id[i];
            if (!dig_from_key) sm.dig[pos] = uint16_t(d);
          }
        }
        __syncwarp();
      }
    }

    // ---- decoupled look-back, one thread per digit, a window of predecessors per round trip:
    // the window's loads are independent, so the inclusive-prefix frontier moves a whole window of
    // tiles per L2 round trip instead of one. Every wait is bounded in time.
    for (int b = threadIdx.x; b < NBINS; b += THREADS) {
      uint32_t excl = 0;
      if (tile > 0) {
        int64_t j = int64_t(tile) - 1;
        bool done = false;
        while (!done) {
          constexpr int W = ST::WINDOW;
          StatusT st[W];
#pragma unroll
          for (int i = 0; i < W; i++)
            st[i] = (j - i >= 0) ? ST::load(status + (first_tile + uint64_t(j - i)) * NBINS + b) : ST::make(epoch, ST_INCL, 0);
#pragma unroll
          for (int i = 0; i < W; i++) {
            StatusT s = st[i];
            if (!ST::ready(s, epoch)) {
              const StatusT* p = status + (first_tile + uint64_t(j - i)) * NBINS + b;
              const uint64_t t0 = globaltimer_ns();
              uint32_t polls = 0;
              for (;;) {
                s = ST::load(p);
                if (ST::ready(s, epoch)) break;
                if (++polls > 8) __nanosleep(32);
                if ((polls & 63u) == 0u && globaltimer_ns() - t0 > LOOKBACK_TIMEOUT_NS) {
                  atomicOr(pa.err, ERR_LOOKBACK_TIMEOUT);
                  s = ST::make(epoch, ST_INCL, 0);
                  break;
                }
              }
            }
            excl += ST::count(s);
            if (ST::flag(s) == ST_INCL) { done = true; break; }
          }
          j -= W;
          if (j < 0) done = true;
        }
        ST::store(status + uint64_t(T) * NBINS + b, ST::make(epoch, ST_INCL, excl + sm.cnt[b]));
      }
      sm.gdelta[b] = sm.desc.bin_base[b] + excl - sm.local[b];
    }
    __syncthreads();

    const uint32_t tile_n = uint32_t((count - tile_base) < uint64_t(TILE) ? (count - tile_base) : uint64_t(TILE));
    auto dig_at = [&](uint32_t j) -> uint32_t {
      if constexpr (REC) return sm.dig[j] >> 16;
      else return dig_from_key ? (uint32_t(sm.keys[j] >> shift) & 255u) : uint32_t(sm.dig[j]);
    };
    // ---- keys and ids out; consecutive threads write consecutive addresses of a digit run. A pass that
    // moves both writes them in one loop (one digit and base lookup per row). Every destination is
    // checked against its array: an offset error is reported, never written.
    const uint32_t buf_rows = sm.desc.buf_rows, out_rows = sm.desc.out_rows;
    const bool last = (flags & PF_LAST) != 0;
    const bool merged = keys_out && ids_out && pa.carry_ids;
    if constexpr (REC) {
      // Keys and records in one loop. A row's record comes from its place in the tile's input (the
      // tile's records, read in sorted order, stay within one L2-resident span), or is built from the
      // payload columns in the first pass; a row reaching its final place has its record unpacked.
      // Two rows a thread per round, their record loads in flight together (each is a random read
      // within the tile's span, an L2 round trip).
      const uint4* __restrict__ rin = reinterpret_cast<const uint4*>(ids_in);
      uint4* __restrict__ rout = reinterpret_cast<uint4*>(ids_out);
      constexpr int U = 2;
      const bool encode = (flags & PF_ENCODE) != 0;
      for (uint32_t j0 = threadIdx.x; j0 < tile_n; j0 += THREADS * U) {
        uint4 r[U];
        uint32_t dg[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const uint32_t j = j0 + uint32_t(u) * THREADS;
          dg[u] = INVALID_DIGIT;
          if (j >= tile_n) continue;
          const uint32_t w = sm.dig[j];
          dg[u] = w >> 16;
          const uint64_t src_row = tile_base + (w & 0xFFFFu);
          r[u] = encode ? build_record(pa.rec, uint32_t(src_row)) : rin[src_row];
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
          const uint32_t j = j0 + uint32_t(u) * THREADS;
          const uint32_t d = dg[u];
          if (d == INVALID_DIGIT) continue;
          uint32_t dst = sm.gdelta[d] + j;
          if (d < RADIX && rout) {
            if (dst < buf_rows) {
              if (keys_out) keys_out[dst] = sm.keys[j];
              rout[dst] = r[u];
            } else {
              atomicOr(pa.err, ERR_BOUNDS);
            }
            continue;
          }
          if (d < RADIX) dst += sm.desc.value_base;
          if (dst >= out_rows) {
            atomicOr(pa.err, ERR_BOUNDS);
            continue;
          }
          if (final_out) {
            if (flags & PF_WIDE_OUT) static_cast<uint64_t*>(final_out)[dst] = r[u].x;
            else static_cast<uint32_t*>(final_out)[dst] = r[u].x;
          }
          unpack_record(pa.rec, r[u], dst);
          // The sorted key column at the same row: null rows as zero, value rows (last pass) unkeyed.
          if (pa.key_out_mode == KEY_OUT_UNKEY)
            store_width(pa.key_out, dst, pt_bytes(pa.key_out_pt),
                        d < RADIX ? unkey_bits<KeyT>(sm.keys[j], pa.key_out_pt, pa.key_desc) : 0ull);
        }
      }
    } else if (merged) {
      for (uint32_t j = threadIdx.x; j < tile_n; j += THREADS) {
        const uint32_t d = dig_at(j);
        const uint32_t dst = sm.gdelta[d] + j;
        if (d < RADIX) {
          if (dst < buf_rows) {
            keys_out[dst] = sm.keys[j];
            ids_out[dst] = sm.ids[j];
          } else {
            atomicOr(pa.err, ERR_BOUNDS);
          }
        } else if (final_out) {
          if (dst >= out_rows) atomicOr(pa.err, ERR_BOUNDS);
          else if (flags & PF_WIDE_OUT) static_cast<uint64_t*>(final_out)[dst] = sm.ids[j];
          else static_cast<uint32_t*>(final_out)[dst] = sm.ids[j];
        }
      }
    } else if (keys_out) {
      for (uint32_t j = threadIdx.x; j < tile_n; j += THREADS) {
        const uint32_t d = dig_at(j);
        const uint32_t dst = sm.gdelta[d] + j;
        if (d < RADIX) {
          if (dst < buf_rows) keys_out[dst] = sm.keys[j];
          else atomicOr(pa.err, ERR_BOUNDS);
        }
      }
    }
    // The sorted key column: value rows from their keys in the last pass, null rows (first pass of the
    // most significant key) as zero. Record passes write it in their own loop, beside the payload.
    if (!REC && pa.key_out_mode == KEY_OUT_UNKEY && (last || (flags & PF_ROUTE))) {
      const int kw = pt_bytes(pa.key_out_pt);
      for (uint32_t j = threadIdx.x; j < tile_n; j += THREADS) {
        const uint32_t d = dig_at(j);
        if (d < RADIX && !last) continue;
        uint32_t dst = sm.gdelta[d] + j;
        if (d < RADIX) dst += sm.desc.value_base;
        if (dst >= out_rows) { atomicOr(pa.err, ERR_BOUNDS); continue; }
        const uint64_t v = d < RADIX ? unkey_bits<KeyT>(sm.keys[j], pa.key_out_pt, pa.key_desc) : 0ull;
        store_width(pa.key_out, dst, kw, v);
      }
    }
    if (pa.carry_ids && !merged && !REC) {
      for (uint32_t j = threadIdx.x; j < tile_n; j += THREADS) {
        const uint32_t d = dig_at(j);
        const uint32_t v = sm.ids[j];
        uint32_t dst = sm.gdelta[d] + j;
        if (d >= RADIX || !ids_out) {
          if (!final_out) continue;
          if (d < RADIX) dst += sm.desc.value_base;
          if (dst >= out_rows) { atomicOr(pa.err, ERR_BOUNDS); continue; }
          if (flags & PF_WIDE_OUT) static_cast<uint64_t*>(final_out)[dst] = v;
          else static_cast<uint32_t*>(final_out)[dst] = v;
        } else {
          if (dst < buf_rows) ids_out[dst] = v;
          else atomicOr(pa.err, ERR_BOUNDS);
        }
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------------
// Kernel 4: after the passes, the sorted key column's validity bitmap.

// The sorted key column's validity: the null block of the most significant key is
// [0, nulls) with nulls first, [n - nulls, n) with nulls last; its null count is that block's size.
__global__ void __launch_bounds__(256) key_validity_kernel(const SortSummary* __restrict__ sum, int nulls_first,
                                                           uint32_t* __restrict__ bits, uint64_t n,
                                                           unsigned long long* null_count) {
  const uint64_t nn = sum->null_rows;
  const uint64_t lo = nulls_first ? 0 : n - nn, hi = nulls_first ? nn : n;   // null rows [lo, hi)
  const uint64_t words = (n + 31) / 32;
  for (uint64_t w = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; w < words; w += uint64_t(gridDim.x) * blockDim.x) {
    // Bit b is row w * 32 + b: set unless the row is null (in [lo, hi)) or past the end.
    const uint64_t r0 = w * 32;
    uint32_t v = r0 + 32 <= n ? 0xFFFFFFFFu : ((1u << uint32_t(n - r0)) - 1u);   // n - r0 < 32 there
    const uint64_t a = lo > r0 ? lo : r0, b = hi < r0 + 32 ? hi : r0 + 32;
    if (a < b) {
      const uint32_t len = uint32_t(b - a);
      v &= len == 32 ? 0u : ~(((1u << len) - 1u) << uint32_t(a - r0));
    }
    bits[w] = v;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *null_count = nn;
}

// ------------------------------------------------------------------------------------------------
// The large single-key sort: two passes on the top digits, then local sorts in shared memory.
//
// One 8-byte key over at least 2^25 value rows with three or more active digits. Two onesweep passes
// on the two highest active digits (the lower of them first: LSD order) leave the value rows grouped
// by those digits -- at most 65,536 buckets, a few hundred rows each at the benchmark's size -- with
// every bucket in row order. Each bucket is then sorted by the remaining active digits inside one
// CTA's shared memory (the same warp-ballot ranking as the passes, no look-back), and written to its
// final place: one read and one write of the rows instead of a global pass per remaining digit.
// Buckets too large for every local shape make the sort run the remaining passes instead: the low
// digits, then the two top digits again (a complete LSD sequence after the first two passes, so the
// answer is the same). Every choice is made on the device, with no host round trip.

constexpr uint64_t HYB_MIN_ROWS = uint64_t(1) << 25;     // one pass saved; ARROWMETAL_HYBRID_MIN_ROWS overrides
constexpr uint64_t HYB_MIN_ANY = uint64_t(1) << 21;      // the smallest sort that may take it (6 passes saved)
constexpr int HYB_STEPS = 10;                 // two top-digit passes, then up to eight fallback passes
constexpr int HYB_BUCKETS = 65536;            // (higher digit, lower digit) buckets of the two passes
constexpr int LOC_ITEMS = 7;
constexpr int LOC_VARIANTS = 3;               // 128, 256 and 512 threads x 7 rows
__host__ __device__ constexpr int loc_threads(int v) { return v == 0 ? 128 : v == 1 ? 256 : 512; }
__host__ __device__ constexpr uint32_t loc_cap(int v) { return uint32_t(loc_threads(v) * LOC_ITEMS); }

struct HybridState {
  uint32_t mode;          // 1: the hybrid sort runs
  uint32_t fallback;      // 1: a bucket exceeds every local shape; the remaining passes run
  uint32_t variant;       // the local shape that runs
  uint32_t buckets;       // non-empty buckets
  uint32_t m;             // value rows
  uint32_t value_base;    // the value rows' first output row
  uint32_t nlocal;        // digits left to the local sorts, low to high
  uint32_t nfall;         // fallback passes prepared
  uint32_t hi_shift, lo_shift;   // the two bucket digits
  uint32_t max_bucket;
  uint32_t local_shift[8];
  uint32_t scan_done, count_error;   // bucket_scan_kernel: blocks finished, a digit's counts off
};

// One block: the hybrid's pass descriptors from the plan's (one descriptor per digit slot), or the
// plan's own passes unchanged when the hybrid does not apply.
__global__ void __launch_bounds__(256) hybrid_plan_kernel(PlanArgs a, const KeyStats* __restrict__ st,
                                                          const PassDesc* __restrict__ normal,
                                                          PassDesc* __restrict__ steps, HybridState* __restrict__ hs) {
  __shared__ int s_src[HYB_STEPS];      // the normal slot each step copies (-1: none)
  __shared__ int s_hyb, s_na, s_act[8];
  if (threadIdx.x == 0) {
    int na = 0;
    for (int d = 0; d < a.nslots && d < 8; d++)
      if (normal[d].active) s_act[na++] = d;
    // The two-level sort replaces na - 2 global passes by the bucket boundaries and the local sorts,
    // whose cost barely depends on the digits left: it pays from about 16M / (na - 2) value rows
    // (measured on B200: from 2-4M rows with 6 passes saved, 4-8M with 3), and from 2^25 rows when it
    // saves one pass. hyb_min_rows, when set, is one threshold for every digit count.
    const uint64_t saved = na >= 3 ? uint64_t(na - 2) : 0;
    const uint64_t thr = a.hyb_min_rows ? a.hyb_min_rows : saved >= 2 ? (uint64_t(16) << 20) / saved : HYB_MIN_ROWS;
    const bool hyb = a.nkeys == 1 && a.key_bytes[0] == 8 && uint64_t(st->n_value) >= thr && na >= 3;
    s_hyb = hyb ? 1 : 0;
    s_na = na;
    for (int i = 0; i < HYB_STEPS; i++) s_src[i] = -1;
    if (hyb) {
      s_src[0] = s_act[na - 2];
      s_src[1] = s_act[na - 1];
      for (int i = 0; i < na; i++) s_src[2 + i] = s_act[i];   // low digits, then the top two again
    } else {
      for (int i = 0; i < a.nslots && i < 8; i++) s_src[2 + i] = i;
    }
  }
  __syncthreads();
  // The descriptors' words, copied by the whole block.
  constexpr int W = int(sizeof(PassDesc) / 4);
  for (int i = 0; i < HYB_STEPS; i++) {
    uint32_t* dst = reinterpret_cast<uint32_t*>(steps + i);
    if (s_src[i] < 0) {
      for (int w = threadIdx.x; w < W; w += blockDim.x) dst[w] = 0;
    } else {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(normal + s_src[i]);
      for (int w = threadIdx.x; w < W; w += blockDim.x) dst[w] = src[w];
    }
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  const uint32_t m = st->n_value;
  hs->mode = uint32_t(s_hyb);
  hs->fallback = 0;
  hs->variant = 0;
  hs->buckets = 0;
  hs->m = m;
  hs->value_base = a.nulls_first[0] ? st->n_null + st->n_nan : 0u;
  hs->max_bucket = 0;
  hs->scan_done = 0;
  hs->count_error = 0;
  if (!s_hyb) {
    hs->nlocal = 0;
    hs->nfall = 0;
    return;                              // steps 2.. are the plan's passes, as planned
  }
  const int na = s_na;
  const uint32_t wide = a.index_wide ? PF_WIDE_OUT : 0u;
  PassDesc& h0 = steps[0];
  h0.active = 1;
  h0.flags = PF_ENCODE | PF_ROUTE | wide;
  h0.count = uint32_t(a.n);
  h0.src_keys = -1;
  h0.src_ids = -1;
  h0.dst_keys = 0;
  h0.dst_ids = 0;
  PassDesc& h1 = steps[1];
  h1.active = 1;
  h1.flags = wide | PF_BUCKETS;
  h1.bucket_shift = uint32_t(8 * s_act[na - 2]);
  h1.count = m;
  h1.src_keys = 0;
  h1.src_ids = 0;
  h1.dst_keys = 1;
  h1.dst_ids = 1;
  int cur = 1;
  for (int i = 0; i < na; i++) {
    PassDesc& f = steps[2 + i];
    const bool last = i == na - 1;
    f.active = 0;                        // activated by the decision when a bucket is too large
    f.flags = wide | (last ? PF_LAST : 0u);
    f.count = m;
    f.src_keys = cur;
    f.src_ids = cur;
    if (last) {
      f.dst_keys = -1;
      f.dst_ids = -1;
    } else {
      f.dst_keys = 1 - cur;
      f.dst_ids = 1 - cur;
      cur = 1 - cur;
    }
  }
  hs->nfall = uint32_t(na);
  hs->nlocal = uint32_t(na - 2);
  for (int i = 0; i < na - 2; i++) hs->local_shift[i] = uint32_t(8 * s_act[i]);
  hs->hi_shift = uint32_t(8 * s_act[na - 1]);
  hs->lo_shift = uint32_t(8 * s_act[na - 2]);
}

// After the second pass: the buckets' starts, the largest bucket, and the local shape or the
// fallback passes. The second pass counted every bucket (65,536: its digit, then the lower digit);
// the buckets of one digit d start where the second pass put digit d (its bin base), so block d scans
// its 256 lower-digit counts on its own: pos[d * 256 + l] = base[d] + the counts before l. The last
// block to finish decides from the largest bucket; pos[65,536] is the value rows.
__global__ void __launch_bounds__(256) bucket_scan_kernel(HybridState* __restrict__ hs, const uint32_t* __restrict__ counts,
                                                          uint32_t* __restrict__ pos, PassDesc* __restrict__ steps,
                                                          SortSummary* __restrict__ sum, uint32_t* __restrict__ err) {
  __shared__ uint32_t s_sum[8], s_max[8];
  __shared__ uint32_t s_last;
  if (!hs->mode) return;
  const uint32_t d = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint32_t c = counts[d * 256 + t];
  uint32_t x = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  const uint32_t mx = __reduce_max_sync(0xffffffffu, c);
  if (lane == 31) s_sum[warp] = x;
  if (lane == 0) s_max[warp] = mx;
  __syncthreads();
  uint32_t add = 0, tot = 0, bmax = 0;
#pragma unroll
  for (int w = 0; w < 8; w++) {
    if (w < int(warp)) add += s_sum[w];
    tot += s_sum[w];
    bmax = max(bmax, s_max[w]);
  }
  const uint32_t base = steps[1].bin_base[d];
  pos[d * 256 + t] = base + x - c + add;
  if (t == 0) {
    // The digit's buckets must hold exactly its rows; otherwise no local sort runs on them.
    const uint32_t end = d + 1 < 256 ? steps[1].bin_base[d + 1] : hs->m;
    if (base + tot != end) atomicOr(&hs->count_error, 1u);
    atomicMax(&hs->max_bucket, bmax);
    __threadfence();
    s_last = atomicAdd(&hs->scan_done, 1u) == gridDim.x - 1 ? 1u : 0u;
  }
  __syncthreads();
  if (!s_last || t != 0) return;
  __threadfence();
  const uint32_t big = atomicAdd(&hs->max_bucket, 0u);
  const bool bad = atomicAdd(&hs->count_error, 0u) != 0u;
  pos[HYB_BUCKETS] = hs->m;
  hs->buckets = HYB_BUCKETS;
  int v = -1;
  for (int i = LOC_VARIANTS - 1; i >= 0; i--)
    if (big <= loc_cap(i)) v = i;
  if (bad) {
    atomicOr(err, ERR_BOUNDS);
    v = -1;
  }
  if (v >= 0) {
    hs->variant = uint32_t(v);
    sum->passes_run = 2;                 // the local sorts stand in for the others
  } else {
    hs->fallback = 1;
    for (uint32_t i = 0; i < hs->nfall; i++) steps[2 + i].active = 1;
    sum->passes_run = 2 + hs->nfall;
  }
}

// The local sorts: each bucket of the value rows, sorted by the digits below the bucket digits in
// shared memory, then written to its final rows (ids, and the key column rebuilt when asked). A
// persistent grid of CTAs walks the buckets; a shape that is not the chosen one returns at once.
template <int THREADS, int VARIANT, bool REC = false>
__global__ void __launch_bounds__(THREADS, THREADS == 128 ? 8 : THREADS == 256 ? 4 : 2) local_sort_kernel(const uint64_t* __restrict__ keys,
                                                             const void* __restrict__ ids_or_recs,
                                                             const uint32_t* __restrict__ pos,
                                                             const HybridState* __restrict__ hs,
                                                             const __grid_constant__ PassArgs pa) {
  constexpr int ITEMS = LOC_ITEMS, WARPS = THREADS / 32, CAP = THREADS * ITEMS;
  extern __shared__ __align__(16) unsigned char loc_smem[];
  uint64_t* skeys = reinterpret_cast<uint64_t*>(loc_smem);
  uint32_t* sids = reinterpret_cast<uint32_t*>(skeys + CAP);
  uint32_t* whist = sids + CAP;                       // [WARPS][256]
  uint32_t* local = whist + WARPS * 256;              // [256]
  uint32_t* wsum = local + 256;                       // [WARPS]
  if (!hs->mode || hs->fallback || hs->variant != uint32_t(VARIANT)) return;
  // Row ids, or (record sorts) 16-byte records; a record sort ranks each row's place in its bucket.
  const uint32_t* __restrict__ ids = static_cast<const uint32_t*>(ids_or_recs);
  const uint4* __restrict__ recs = static_cast<const uint4*>(ids_or_recs);
  const uint32_t g = hs->buckets, nloc = hs->nlocal, vbase = hs->value_base;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  constexpr int DPT = THREADS >= 256 ? 1 : 256 / THREADS;
  // What the output loop needs, read once: the bounds, the index width, and how a key leaves.
  const uint64_t out_rows = pa.desc->out_rows;
  const bool wide_out = (pa.desc->flags & PF_WIDE_OUT) != 0;
  const bool unkey = pa.key_out_mode == KEY_OUT_UNKEY;
  // An 8-byte integer key (the two-level sort's keys are 8 bytes) inverts its key map with one XOR.
  const bool unkey_xor = unkey && (pa.key_out_pt == PT_I64 || pa.key_out_pt == PT_U64);
  const uint64_t key_xor = (pa.key_out_pt == PT_I64 ? 0x8000000000000000ull : 0ull) ^ (pa.key_desc ? ~0ull : 0ull);
  auto key_out = [&](uint64_t dst, uint64_t k) {
    if (unkey_xor) static_cast<uint64_t*>(pa.key_out)[dst] = k ^ key_xor;
    else if (unkey) store_width(pa.key_out, dst, pt_bytes(pa.key_out_pt), unkey_bits<uint64_t>(k, pa.key_out_pt, pa.key_desc));
  };
  // The counting step's bins: the top bits of the two highest local digits.
  const uint32_t sh_top = hs->local_shift[nloc - 1];
  const uint32_t sh_next = nloc >= 2 ? hs->local_shift[nloc - 2] : 0u;
  const bool two = nloc >= 2;
  const uint64_t lmask = (uint64_t(1) << hs->lo_shift) - 1u;     // lo_shift <= 48
  for (uint32_t j = blockIdx.x; j < g; j += gridDim.x) {
    const uint32_t start = pos[j], size = pos[j + 1] - start;
    if (size > uint32_t(CAP)) {            // the decision rules it out; never read past the tile
      if (threadIdx.x == 0) atomicOr(pa.err, ERR_BOUNDS);
      continue;
    }
    if (size == 0) continue;               // an empty bucket (the same for every thread)
    uint64_t key[ITEMS];
    uint32_t id[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
      const uint32_t r = uint32_t(warp) * (ITEMS * 32) + uint32_t(i) * 32 + lane;
      key[i] = r < size ? keys[start + r] : 0ull;
      if constexpr (REC) id[i] = r;
      else id[i] = r < size ? ids[start + r] : 0u;
    }
    // The tile's empty slots (r >= size) are the last rows in order. They take digit 255 in the ballots
    // but are neither counted nor stored: every row before them keeps its place in [0, size), and their
    // own places come out at size or later.
    uint32_t ok = 0;
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
      if (uint32_t(warp) * (ITEMS * 32) + uint32_t(i) * 32 + lane < size) ok |= 1u << i;
    // Items of this warp holding any row (the same for all its lanes): the ranking skips the others,
    // whose slots are all empty and all after every row.
    const uint32_t w_first = uint32_t(warp) * (ITEMS * 32);
    const int nit = size > w_first ? int(min(uint32_t(ITEMS), (size - w_first + 31) / 32)) : 0;

    // ---- Ranking by one counting step. Rows go to NB bins by the top bits of their two highest local
    // digits (shared-memory atomics: in no particular order within a bin); a row's place is its bin's
    // start plus the number of its bin's rows that order before it by (the key bits below the bucket
    // digits, the row's place in the bucket): a unique pair, so the order is total and ties keep bucket
    // order, which is row order. Taken when no bin holds more than HASH_MAX_BIN rows (uniform keys put
    // one to three rows in a bin); otherwise the ballot ranking below runs, one pass per local digit.
    bool hashed = false;
    {
      constexpr int NB = WARPS * 128;                     // cnt and bstart fill whist's WARPS x 256 words
      constexpr int NBB = NB == 512 ? 9 : NB == 1024 ? 10 : 11;
      constexpr int PER = NB / THREADS;
      constexpr uint32_t HASH_MAX_BIN = 32;
      static_assert(NB == 512 || NB == 1024 || NB == 2048, "bins per local-sort shape");
      uint32_t* cnt = whist;
      uint32_t* bstart = whist + NB;
      auto bin_of = [&](uint64_t k) {
        const uint32_t hi16 = ((uint32_t(k >> sh_top) & 255u) << 8) | (two ? (uint32_t(k >> sh_next) & 255u) : 0u);
        return hi16 >> (16 - NBB);
      };
      for (int x = threadIdx.x; x < NB; x += THREADS) cnt[x] = 0;
      if (threadIdx.x == 0) local[0] = 0;
      __syncthreads();
      // Each item's bin (high half) and its arrival within the bin (low half; fewer than 2^16 rows).
      uint32_t slot[ITEMS];
#pragma unroll
      for (int i = 0; i < ITEMS; i++) {
        slot[i] = 0u;
        if ((ok >> i) & 1u) {
          const uint32_t b = bin_of(key[i]);
          slot[i] = (b << 16) | atomicAdd(&cnt[b], 1u);
        }
      }
      __syncthreads();
      // Bin starts (exclusive scan over the bins, PER consecutive bins a thread) and the largest bin.
      uint32_t c[PER];
      uint32_t tot = 0, mx = 0;
#pragma unroll
      for (int q = 0; q < PER; q++) {
        c[q] = cnt[int(threadIdx.x) * PER + q];
        tot += c[q];
        mx = max(mx, c[q]);
      }
      uint32_t x = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      mx = __reduce_max_sync(0xffffffffu, mx);
      if (lane == 31) wsum[warp] = x;
      if (lane == 0) atomicMax(&local[0], mx);
      __syncthreads();
      uint32_t at = x - tot;
      for (int w = 0; w < warp; w++) at += wsum[w];
#pragma unroll
      for (int q = 0; q < PER; q++) {
        bstart[int(threadIdx.x) * PER + q] = at;
        at += c[q];
      }
      __syncthreads();
      if (local[0] <= HASH_MAX_BIN) {
        hashed = true;
        uint64_t* comp = skeys;                           // the tile holds the bins' pairs first
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
          if (!((ok >> i) & 1u)) continue;
          const uint32_t r = uint32_t(warp) * (ITEMS * 32) + uint32_t(i) * 32 + lane;
          comp[bstart[slot[i] >> 16] + (slot[i] & 0xFFFFu)] = ((key[i] & lmask) << 12) | r;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
          if (!((ok >> i) & 1u)) continue;
          const uint32_t r = uint32_t(warp) * (ITEMS * 32) + uint32_t(i) * 32 + lane;
          const uint32_t b = slot[i] >> 16;
          const uint32_t s0 = bstart[b], nb = cnt[b];
          const uint64_t me = ((key[i] & lmask) << 12) | r;
          uint32_t rank = 0;
          for (uint32_t q = 0; q < nb; q++) rank += comp[s0 + q] < me ? 1u : 0u;
          slot[i] = s0 + rank;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
          if (!((ok >> i) & 1u)) continue;
          skeys[slot[i]] = key[i];
          sids[slot[i]] = id[i];
        }
        __syncthreads();
      }
    }
    for (uint32_t dgi = 0; dgi < nloc && !hashed; dgi++) {
      const uint32_t shift = hs->local_shift[dgi];
      uint32_t dg[ITEMS];
#pragma unroll
      for (int i = 0; i < ITEMS; i++) dg[i] = ((ok >> i) & 1u) ? (uint32_t(key[i] >> shift) & 255u) : 255u;
      for (int x = lane; x < 256; x += 32) whist[warp * 256 + x] = 0;
      __syncwarp();
#pragma unroll
      for (int i = 0; i < ITEMS; i++)
        if ((ok >> i) & 1u) atomicAdd(&whist[warp * 256 + dg[i]], 1u);
      __syncthreads();
      // Per digit: the warps' exclusive starts, and the digit's total; then a scan over digits.
      uint32_t tots[DPT];
      uint32_t tot = 0;
      if (threadIdx.x * DPT < 256) {
#pragma unroll
        for (int q = 0; q < DPT; q++) {
          const int d = int(threadIdx.x) * DPT + q;
          uint32_t run = 0;
#pragma unroll
          for (int w = 0; w < WARPS; w++) {
            const uint32_t c = whist[w * 256 + d];
            whist[w * 256 + d] = run;
            run += c;
          }
          tots[q] = run;
          tot += run;
        }
      }
      uint32_t x = tot;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) wsum[warp] = x;
      __syncthreads();
      uint32_t add = 0;
      for (int w = 0; w < warp; w++) add += wsum[w];
      if (threadIdx.x * DPT < 256) {
        uint32_t at = x - tot + add;
#pragma unroll
        for (int q = 0; q < DPT; q++) {
          local[int(threadIdx.x) * DPT + q] = at;
          at += tots[q];
        }
      }
      __syncthreads();
      // Stable ranks: one ballot per digit bit; the warp's counters advance item by item.
#pragma unroll
      for (int i = 0; i < ITEMS; i++) {
        if (i >= nit) break;
        const uint32_t d = dg[i];
        uint32_t peers = 0xffffffffu;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const uint32_t bit = (d >> k) & 1u;
          const uint32_t bl = __ballot_sync(0xffffffffu, bit);
          peers &= bit ? bl : ~bl;
        }
        const uint32_t b0 = whist[warp * 256 + d];
        __syncwarp();
        if (lane == __ffs(peers) - 1) whist[warp * 256 + d] = b0 + __popc(peers);
        const uint32_t p = local[d] + b0 + __popc(peers & lt);
        if (p < size) {
          skeys[p] = key[i];
          sids[p] = id[i];
        }
        __syncwarp();
      }
      __syncthreads();
      // The next digit's rows, back from the tile. No barrier after: the tile is next written after
      // the next digit's histogram barrier, which every warp reaches only once it has read its rows.
      if (dgi + 1 < nloc) {
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
          const uint32_t r = uint32_t(warp) * (ITEMS * 32) + uint32_t(i) * 32 + lane;
          if ((ok >> i) & 1u) {
            key[i] = skeys[r];
            id[i] = sids[r];
          }
        }
      }
    }
    // The bucket's rows, in order, to their final places.
    const uint64_t out0 = uint64_t(vbase) + start;
    if constexpr (REC) {
      // Each row's record from its place in the bucket's input (one L2-resident span), four rows a
      // thread per round with their loads in flight together.
      constexpr int U = 4;
      for (uint32_t r0 = threadIdx.x; r0 < size; r0 += THREADS * U) {
        uint4 rr[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const uint32_t r = r0 + uint32_t(u) * THREADS;
          if (r < size) rr[u] = recs[start + sids[r]];
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
          const uint32_t r = r0 + uint32_t(u) * THREADS;
          if (r >= size) continue;
          const uint64_t dst = out0 + r;
          if (dst >= out_rows) {
            atomicOr(pa.err, ERR_BOUNDS);
            continue;
          }
          if (pa.final_out) {
            if (wide_out) static_cast<uint64_t*>(pa.final_out)[dst] = rr[u].x;
            else static_cast<uint32_t*>(pa.final_out)[dst] = rr[u].x;
          }
          unpack_record(pa.rec, rr[u], dst);
          key_out(dst, skeys[r]);
        }
      }
    } else {
      for (uint32_t r = threadIdx.x; r < size; r += THREADS) {
        const uint64_t dst = out0 + r;
        if (dst >= out_rows) {
          atomicOr(pa.err, ERR_BOUNDS);
          continue;
        }
        if (pa.final_out) {
          if (wide_out) static_cast<uint64_t*>(pa.final_out)[dst] = sids[r];
          else static_cast<uint32_t*>(pa.final_out)[dst] = sids[r];
        }
        key_out(dst, skeys[r]);
      }
    }
    // No barrier here either: the next bucket writes the tile only after its first histogram barrier.
  }
}

template <int THREADS>
constexpr size_t loc_smem_bytes() {
  return size_t(THREADS) * LOC_ITEMS * 12 + size_t(THREADS / 32) * 256 * 4 + 256 * 4 + size_t(THREADS / 32) * 4;
}

// ------------------------------------------------------------------------------------------------
// Host side.

template <typename KeyT>
struct PassConfig;
// Tile shape of a single sort's digit passes: 512 threads x 10 rows (5,120-row tiles, two blocks per SM,
// 64 registers a thread). Measured on B200 with the record passes: ORDER BY 2.558 ms against 2.575 for
// 384 x 14, 2.566 for 512 x 8 and 2.724 for 448 x 12.
template <> struct PassConfig<uint32_t> { static constexpr int THREADS = 512, ITEMS = 10; };
template <> struct PassConfig<uint64_t> { static constexpr int THREADS = 512, ITEMS = 10; };
constexpr int HIST_THREADS = 256, HIST_ITEMS = 8;

template <typename KeyT, int ITEMS = PassConfig<KeyT>::ITEMS, int THREADS = PassConfig<KeyT>::THREADS, bool REC = false>
static size_t pass_smem() {
  return sizeof(PassShared<KeyT, THREADS, ITEMS, std::conditional_t<REC, uint16_t, uint32_t>>);
}

template <typename KeyT, typename StatusT, bool SEG = false, int ITEMS = PassConfig<KeyT>::ITEMS,
          int THREADS = PassConfig<KeyT>::THREADS, bool REC = false>
static int pass_blocks_per_sm() {
  static int cached = -1;
  static std::once_flag once;
  std::call_once(once, [] {
    auto fn = onesweep_pass_kernel<KeyT, StatusT, THREADS, ITEMS, SEG, REC>;
    const size_t smem = pass_smem<KeyT, ITEMS, THREADS, REC>();
    AM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int b = 0;
    AM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, THREADS, smem));
    cached = std::max(1, b);
  });
  return cached;
}

// `range`: the key range too (a lower key of a multi-key sort).
template <typename KeyT>
static void launch_histogram(const ColView& cv, KeyStats* st, uint64_t n, cudaStream_t s, bool range = false) {
  constexpr int CHUNK = HIST_THREADS * HIST_ITEMS;
  const uint64_t chunks = (n + CHUNK - 1) / CHUNK;
  const int grid = int(std::min<uint64_t>(chunks, uint64_t(device().sm_count) * 8));
  KernelTimer kt("radix_histogram", s);
  if (range) key_histogram_kernel<KeyT, HIST_THREADS, HIST_ITEMS, true><<<grid, HIST_THREADS, 0, s>>>(cv, st, n);
  else key_histogram_kernel<KeyT, HIST_THREADS, HIST_ITEMS, false><<<grid, HIST_THREADS, 0, s>>>(cv, st, n);
  AM_CUDA(cudaGetLastError());
}

template <typename KeyT, typename StatusT>
static void launch_pass(const PassArgs& pa, const ColView& cv, uint64_t n, cudaStream_t s) {
  using C = PassConfig<KeyT>;
  constexpr int TILE = C::THREADS * C::ITEMS;
  const uint64_t tiles = (n + TILE - 1) / TILE;
  KernelTimer kt("radix_onesweep_pass", s);
  if (pa.rec_mode) {
    const int bps = pass_blocks_per_sm<KeyT, StatusT, false, C::ITEMS, C::THREADS, true>();
    const int grid = int(std::min<uint64_t>(tiles, uint64_t(device().sm_count) * bps));
    onesweep_pass_kernel<KeyT, StatusT, C::THREADS, C::ITEMS, false, true>
        <<<std::max(grid, 1), C::THREADS, pass_smem<KeyT, C::ITEMS, C::THREADS, true>(), s>>>(pa, cv);
  } else {
    const int grid = int(std::min<uint64_t>(tiles, uint64_t(device().sm_count) * pass_blocks_per_sm<KeyT, StatusT>()));
    onesweep_pass_kernel<KeyT, StatusT, C::THREADS, C::ITEMS, false><<<std::max(grid, 1), C::THREADS, pass_smem<KeyT>(), s>>>(pa, cv);
  }
  AM_CUDA(cudaGetLastError());
}

// Zeroes a pass's look-back words, unless the pass is inactive (the hybrid's passes are decided on the
// device, so a memset that always runs would clear the words for passes that never run).
__global__ void __launch_bounds__(256) zero_status_kernel(const PassDesc* __restrict__ desc, uint4* __restrict__ words,
                                                          uint64_t n16) {
  if (!desc->active) return;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n16; i += uint64_t(gridDim.x) * blockDim.x)
    words[i] = make_uint4(0, 0, 0, 0);
}

// One local-sort shape as a persistent grid (it returns at once unless the decision chose it).
template <int VARIANT, bool REC>
static void launch_local_as(const uint64_t* keys, const void* ids, const uint32_t* pos, const HybridState* hs,
                            const PassArgs& a, cudaStream_t s) {
  constexpr int THREADS = loc_threads(VARIANT);
  constexpr size_t SMEM = loc_smem_bytes<THREADS>();
  static int blocks = 0;
  static std::once_flag once;
  std::call_once(once, [] {
    auto fn = local_sort_kernel<THREADS, VARIANT, REC>;
    AM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM)));
    int b = 0;
    AM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, THREADS, SMEM));
    blocks = std::max(1, b);
  });
  local_sort_kernel<THREADS, VARIANT, REC><<<device().sm_count * blocks, THREADS, SMEM, s>>>(keys, ids, pos, hs, a);
  AM_CUDA(cudaGetLastError());
}

template <int VARIANT>
static void launch_local(const uint64_t* keys, const void* ids, const uint32_t* pos, const HybridState* hs,
                         const PassArgs& a, cudaStream_t s) {
  if (a.rec_mode) launch_local_as<VARIANT, true>(keys, ids, pos, hs, a, s);
  else launch_local_as<VARIANT, false>(keys, ids, pos, hs, a, s);
}

// ARROWMETAL_HYBRID_MIN_ROWS: one two-level threshold for every digit count (0: the per-count rule).
static uint64_t hybrid_min_rows() {
  static const uint64_t v = [] {
    const char* e = std::getenv("ARROWMETAL_HYBRID_MIN_ROWS");
    const long long x = e ? std::atoll(e) : 0;
    return x > 0 ? uint64_t(x) : uint64_t(0);
  }();
  return v;
}

// Rows per look-back entry (a tile), the smallest over the key widths.
static uint64_t min_super() {
  using A = PassConfig<uint32_t>;
  using B = PassConfig<uint64_t>;
  return std::min<uint64_t>(uint64_t(A::THREADS) * A::ITEMS, uint64_t(B::THREADS) * B::ITEMS);
}

ColView make_view(const SortKey& k) {
  ColView v{};
  const am_array* a = k.col;
  if (a->pt == PT_STRUCT) throw unsupported("+s: a struct result is exported, not computed on");
  if (a->dictionary) throw Error("radix sort: a dictionary column must be sorted through its key column");
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

void key_statistics(const SortKey& k, rs::KeyStats* st, cudaStream_t s) {
  const rs::ColView cv = rs::make_view(k);
  AM_CUDA(cudaMemsetAsync(st, 0, sizeof(rs::KeyStats), s));
  if (pt_key_bytes(k.col->pt) == 8) rs::launch_histogram<uint64_t>(cv, st, uint64_t(k.col->length), s);
  else rs::launch_histogram<uint32_t>(cv, st, uint64_t(k.col->length), s);
}

bool key_invertible(const SortKey& k) {
  if (k.col->dictionary) return false;   // the codes do not order the column
  switch (k.col->pt) {
    case PT_I8: case PT_U8: case PT_I16: case PT_U16: case PT_I32: case PT_U32: case PT_I64: case PT_U64:
      return true;
    case PT_F32: case PT_F64:
      return k.float_order == rs::FO_TOTAL;
    default:
      return false;
  }
}

bool payload_record_layout(const std::vector<am_array*>& cols, rs::RecLayout* L) {
  using namespace rs;
  if (cols.empty() || cols.size() > size_t(REC_MAX_COLS)) return false;
  int total = 0;
  for (am_array* c : cols) {
    const int w = pt_bytes(c->pt);
    if (c->pt == PT_STRUCT || c->dictionary || pt_var(c->pt) || c->pt == PT_BOOL || w <= 0 || c->null_count != 0)
      return false;
    total += w;
  }
  if (total > REC_PAYLOAD_BYTES) return false;
  // Widest first: each field then starts at a multiple of its width, and an 8-byte field at byte 0.
  std::vector<int> order(cols.size());
  for (size_t i = 0; i < order.size(); i++) order[i] = int(i);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return pt_bytes(cols[x]->pt) > pt_bytes(cols[y]->pt); });
  *L = RecLayout{};
  L->ncols = int32_t(cols.size());
  int off = 0;
  for (int i : order) {
    L->src[i] = cols[size_t(i)]->data();
    L->width[i] = pt_bytes(cols[size_t(i)]->pt);
    L->off[i] = off;
    off += L->width[i];
  }
  // The common payload (a float64 or int64 beside a 32-bit column) is read and written without the
  // per-field loop.
  if (cols.size() == 2 && L->width[order[0]] == 8 && L->width[order[1]] == 4) {
    L->pair = 1;
    L->wide = order[0];
    L->narrow = order[1];
  }
  return true;
}

void radix_argsort(const std::vector<SortKey>& keys, int64_t n, void* out, int index_width, cudaStream_t s,
                   am_sort_stats* stats) {
  radix_sort(keys, n, out, index_width, nullptr, s, stats);
}

void radix_sort(const std::vector<SortKey>& keys_in, int64_t n64, void* out, int index_width, am_array* key_dst,
                cudaStream_t s, am_sort_stats* stats, const rs::RecLayout* payload) {
  using namespace rs;
  // An integer key with at most 256 distinct values sorts by its dense rank (one digit), where its
  // values are not needed back (no sorted copy of the key is written).
  std::vector<SortKey> keys = keys_in;
  std::vector<am_array*> rank_cols;
  struct RankRelease {
    std::vector<am_array*>& cols;
    ~RankRelease() {
      for (am_array* r : cols) am::release(r);
    }
  } rank_release{rank_cols};
  if (!key_dst && !payload && n64 > 0) {
    for (auto& k : keys) {
      if (am_array* r = low_cardinality_ranks(k, s)) {
        rank_cols.push_back(r);
        k = SortKey{r, false, k.nulls_first, 0};
      }
    }
  }
  const int K = int(keys.size());
  if (K < 1 || K > MAX_KEYS) throw invalid("sort takes 1 to " + std::to_string(MAX_KEYS) + " key columns (a string key counts as its 8-byte chunks plus one)");
  for (auto& k : keys)
    if (pt_var(k.col->pt)) throw Error("radix_sort: string keys must be expanded to their chunk keys first");
  if (n64 <= 0) return;
  const uint64_t n = uint64_t(n64);
  if (key_dst && (K != 1 || !key_invertible(keys[0])))
    throw invalid("the sorted key column is rebuilt only for one integer or totalOrder float key");
  if (payload && K != 1) throw invalid("payload columns ride through a sort by one key only");
  // Row ids move through the passes when an index is wanted or a lower key's column is gathered;
  // with payload columns, 16-byte row records (id and payload) move instead.
  const bool carry_ids = out != nullptr || K > 1 || payload != nullptr;
  const size_t id_bytes = payload ? sizeof(uint4) : sizeof(uint32_t);

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
  // A single 8-byte key over at least 2^21 rows may take the two-level sort (the device decides).
  pa.hyb_min_rows = hybrid_min_rows();
  const bool hybrid = K == 1 && pt_key_bytes(keys[0].col->pt) == 8 && n < (uint64_t(1) << 32) &&
                      n >= (pa.hyb_min_rows ? pa.hyb_min_rows : HYB_MIN_ANY);
  const int NT = S + (hybrid ? HYB_STEPS : 0);          // tile counters: one per launched pass
  const size_t off_stats = 0;
  const size_t off_kplan = off_stats + sizeof(KeyStats) * K;
  const size_t off_desc = (off_kplan + sizeof(KeyPlan) * K + 255) & ~size_t(255);
  const size_t off_steps = off_desc + sizeof(PassDesc) * S;
  const size_t off_hs = (off_steps + (hybrid ? sizeof(PassDesc) * HYB_STEPS : 0) + 15) & ~size_t(15);
  const size_t off_bcount = (off_hs + (hybrid ? sizeof(HybridState) : 0) + 15) & ~size_t(15);
  const size_t off_bpos = off_bcount + (hybrid ? sizeof(uint32_t) * HYB_BUCKETS : 0);
  const size_t off_tick = (off_bpos + (hybrid ? sizeof(uint32_t) * (HYB_BUCKETS + 1) : 0) + 15) & ~size_t(15);
  const size_t off_sum = (off_tick + sizeof(uint32_t) * NT + 15) & ~size_t(15);
  const size_t header = (off_sum + sizeof(SortSummary) + 255) & ~size_t(255);
  const size_t kbuf = ((n * max_kb) + 255) & ~size_t(255);
  const size_t ibuf = carry_ids ? ((n * id_bytes) + 255) & ~size_t(255) : 0;
  ScratchBlock scratch(s, header + 2 * kbuf + 2 * ibuf);
  char* base = scratch.data();
  AM_CUDA(cudaMemsetAsync(base, 0, header, s));
  KeyStats* st = reinterpret_cast<KeyStats*>(base + off_stats);
  KeyPlan* kp = reinterpret_cast<KeyPlan*>(base + off_kplan);
  PassDesc* pd = reinterpret_cast<PassDesc*>(base + off_desc);
  uint32_t* tick = reinterpret_cast<uint32_t*>(base + off_tick);
  SortSummary* sum = reinterpret_cast<SortSummary*>(base + off_sum);
  PassDesc* steps = reinterpret_cast<PassDesc*>(base + off_steps);
  HybridState* hs = reinterpret_cast<HybridState*>(base + off_hs);
  uint32_t* bcount = reinterpret_cast<uint32_t*>(base + off_bcount);
  uint32_t* bpos = reinterpret_cast<uint32_t*>(base + off_bpos);
  void* kbufA = base + header;
  void* kbufB = base + header + kbuf;
  uint32_t* ibufA = carry_ids ? reinterpret_cast<uint32_t*>(base + header + 2 * kbuf) : nullptr;
  uint32_t* ibufB = carry_ids ? reinterpret_cast<uint32_t*>(base + header + 2 * kbuf + ibuf) : nullptr;
  if (key_dst) {
    const size_t words = size_t((n + 127) / 128) * 4;
    key_dst->values = DevBuffer::alloc(n * pt_bytes(keys[0].col->pt) + 16, s);
    key_dst->last_stream = s;
    if (keys[0].col->null_count != 0) {
      key_dst->validity = DevBuffer::alloc(words * 4, s);
      key_dst->null_count_dev = DevBuffer::alloc(sizeof(unsigned long long), s);
      // The sorted column has the input's null rows: a known count needs no device round trip.
      key_dst->null_count = keys[0].col->null_count > 0 ? keys[0].col->null_count : -1;
    } else {
      key_dst->null_count = 0;
    }
  }
  if (debug_skip_first_tile()) {
    // Test hook: every pass's ticket starts at 1, so tile 0 is never processed and the look-back of
    // tile 1 runs into its time limit.
    const std::vector<uint32_t> ones(size_t(NT), 1u);
    AM_CUDA(cudaMemcpyAsync(tick, ones.data(), sizeof(uint32_t) * NT, cudaMemcpyHostToDevice, s));
    AM_CUDA(cudaStreamSynchronize(s));
  }

  std::vector<ColView> views(K);
  for (int k = 0; k < K; k++) {
    views[k] = make_view(keys[k]);
    if (pt_key_bytes(keys[k].col->pt) == 8) launch_histogram<uint64_t>(views[k], st + k, n, s, k > 0);
    else launch_histogram<uint32_t>(views[k], st + k, n, s, k > 0);
  }
  {
    KernelTimer kt("radix_plan", s);
    plan_kernel<<<1, 256, 0, s>>>(pa, st, kp, pd, sum);
    AM_CUDA(cudaGetLastError());
  }

  const uint64_t max_tiles = (n + min_super() - 1) / min_super();
  // Passes of fewer than 2^30 rows use 32-bit look-back words, zeroed before each pass.
  const bool narrow_status = n < (uint64_t(1) << 30);
  StreamScratch& sc = stream_scratch(s, size_t(max_tiles) * NBINS);
  // The arguments every pass and the local sorts share.
  auto args_for = [&](const PassDesc* desc, uint32_t* counter, const KeyPlan* plan) {
    PassArgs a{};
    a.desc = desc;
    a.kplan = plan;
    a.keys[0] = kbufA;
    a.keys[1] = kbufB;
    a.ids[0] = ibufA;
    a.ids[1] = ibufB;
    a.final_out = out;
    a.status = sc.status;
    a.tile_counter = counter;
    a.err = sc.err;
    a.carry_ids = carry_ids ? 1 : 0;
    a.bucket_count = hybrid ? bcount : nullptr;
    if (key_dst) {
      a.key_out_mode = KEY_OUT_UNKEY;
      a.key_out_pt = keys[0].col->pt;
      a.key_desc = keys[0].descending ? 1 : 0;
      a.key_float_order = keys[0].float_order;
      a.key_out = key_dst->values->ptr;
    }
    if (payload) {
      a.rec_mode = 1;
      a.rec = *payload;
    }
    return a;
  };
  auto launch_one = [&](const PassDesc* desc, uint32_t* counter, const KeyPlan* plan, const ColView& cv, int kb) {
    if (narrow_status) {
      const uint64_t bytes = uint64_t(max_tiles) * NBINS * sizeof(uint32_t);
      const uint64_t n16 = (bytes + 15) / 16;
      const int grid = int(std::min<uint64_t>((n16 + 255) / 256, uint64_t(device().sm_count) * 4));
      zero_status_kernel<<<std::max(grid, 1), 256, 0, s>>>(desc, reinterpret_cast<uint4*>(sc.status), n16);
      AM_CUDA(cudaGetLastError());
    } else if (sc.epoch >= (1u << 30) - 1) {
      AM_CUDA(cudaMemsetAsync(sc.status, 0, sc.status_words * sizeof(uint64_t), s));
      sc.epoch = 0;
    }
    PassArgs a = args_for(desc, counter, plan);
    a.epoch = ++sc.epoch;
    if (kb == 8) {
      if (narrow_status) launch_pass<uint64_t, uint32_t>(a, cv, n, s);
      else launch_pass<uint64_t, uint64_t>(a, cv, n, s);
    } else {
      if (narrow_status) launch_pass<uint32_t, uint32_t>(a, cv, n, s);
      else launch_pass<uint32_t, uint64_t>(a, cv, n, s);
    }
  };
  if (hybrid) {
    {
      KernelTimer kt("radix_plan", s);
      hybrid_plan_kernel<<<1, 256, 0, s>>>(pa, st, pd, steps, hs);
      AM_CUDA(cudaGetLastError());
    }
    launch_one(steps + 0, tick + S + 0, kp, views[0], 8);
    launch_one(steps + 1, tick + S + 1, kp, views[0], 8);
    {
      KernelTimer kt("radix_buckets", s);
      bucket_scan_kernel<<<HYB_BUCKETS / 256, 256, 0, s>>>(hs, bcount, bpos, steps, sum, sc.err);
      AM_CUDA(cudaGetLastError());
    }
    for (int i = 2; i < HYB_STEPS; i++) launch_one(steps + i, tick + S + i, kp, views[0], 8);
    {
      KernelTimer kt("radix_local_sort", s);
      const PassArgs a = args_for(steps + 1, nullptr, kp);
      launch_local<0>(static_cast<const uint64_t*>(kbufB), ibufB, bpos, hs, a, s);
      launch_local<1>(static_cast<const uint64_t*>(kbufB), ibufB, bpos, hs, a, s);
      launch_local<2>(static_cast<const uint64_t*>(kbufB), ibufB, bpos, hs, a, s);
    }
  }
  for (int sl = 0; sl < S && !hybrid; sl++) {
    if (narrow_status) {
      AM_CUDA(cudaMemsetAsync(sc.status, 0, size_t(max_tiles) * NBINS * sizeof(uint32_t), s));
    } else if (sc.epoch >= (1u << 30) - 1) {
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
    a.carry_ids = carry_ids ? 1 : 0;
    if (key_dst) {
      a.key_out_mode = KEY_OUT_UNKEY;
      a.key_out_pt = keys[0].col->pt;
      a.key_desc = keys[0].descending ? 1 : 0;
      a.key_float_order = keys[0].float_order;
      a.key_out = key_dst->values->ptr;
    }
    if (payload) {
      a.rec_mode = 1;
      a.rec = *payload;
    }
    const ColView& cv = views[pa.slot_key[sl]];
    if (slot_bytes[sl] == 8) {
      if (narrow_status) launch_pass<uint64_t, uint32_t>(a, cv, n, s);
      else launch_pass<uint64_t, uint64_t>(a, cv, n, s);
    } else {
      if (narrow_status) launch_pass<uint32_t, uint32_t>(a, cv, n, s);
      else launch_pass<uint32_t, uint64_t>(a, cv, n, s);
    }
  }
  // The sorted key column's validity: one block of nulls at one end.
  const int fin_grid = int(std::min<uint64_t>((n + 8191) / 8192, uint64_t(device().sm_count) * 4));
  if (key_dst && key_dst->validity) {
    KernelTimer kt("sort_finish", s);
    key_validity_kernel<<<std::max(fin_grid, 1), 256, 0, s>>>(sum, keys[0].nulls_first ? 1 : 0,
                                                            static_cast<uint32_t*>(key_dst->validity->ptr), n,
                                                            static_cast<unsigned long long*>(key_dst->null_count_dev->ptr));
    AM_CUDA(cudaGetLastError());
  }
  if (key_dst) key_dst->ready = std::make_shared<ReadyEvent>(s);
  if (stats) {
    // Counters arrive asynchronously; am_last_sort_stats waits for them.
    stats->rows = int64_t(n);
    stats->payload_in_records = payload ? 1 : 0;
    AM_CUDA(cudaMemcpyAsync(last_summary_host(), sum, sizeof(SortSummary), cudaMemcpyDeviceToHost, s));
    tls().stats_stream = s;
  }
}


// ------------------------------------------------------------------------------------------------
// Segmented (batched) argsort: the arrays of one key width share every launch.

namespace rs {
namespace {

constexpr uint32_t SEG_HIST_ROWS = 32768;   // rows per histogram block

// One key width's arrays of a batch: the tables the kernels read and where everything sits in the
// group's scratch.
template <typename KeyT, int THREADS, int ITEMS>
struct GroupLayout {
  static constexpr uint64_t TILE = uint64_t(THREADS) * ITEMS;
  static constexpr int S = int(sizeof(KeyT));
  uint32_t G = 0;
  uint64_t rows = 0, tiles = 0, items = 0, max_n = 0;
  std::vector<uint32_t> lens;
  std::vector<char> host;              // segment table, tile starts, item starts
  size_t off_tiles = 0, off_items = 0, tables = 0;
  size_t off_stats = 0, off_kplan = 0, off_desc = 0, off_sum = 0, off_tick = 0, header = 0;
  size_t kbuf = 0, ibuf = 0;
  size_t bytes() const { return header + 2 * kbuf + 2 * ibuf; }
  bool narrow() const { return max_n < (uint64_t(1) << 30); }

  GroupLayout(const std::vector<SortKey>& keys, const std::vector<void*>& outs, const std::vector<size_t>& group) {
    G = uint32_t(group.size());
    std::vector<SegDesc> segs(G);
    std::vector<uint32_t> tile_start(G + 1), item_start(G + 1);
    lens.resize(G);
    for (uint32_t g = 0; g < G; g++) {
      const SortKey& k = keys[group[g]];
      const uint64_t n = uint64_t(k.col->length);
      segs[g].col = make_view(k);
      segs[g].row_off = rows;
      segs[g].out = outs[group[g]];
      segs[g].n = uint32_t(n);
      lens[g] = uint32_t(n);
      tile_start[g] = uint32_t(tiles);
      item_start[g] = uint32_t(items);
      rows += n;
      tiles += (n + TILE - 1) / TILE;
      items += (n + SEG_HIST_ROWS - 1) / SEG_HIST_ROWS;
      max_n = std::max(max_n, n);
    }
    tile_start[G] = uint32_t(tiles);
    item_start[G] = uint32_t(items);
    if (tiles >= (uint64_t(1) << 32) || items >= (uint64_t(1) << 31))
      throw invalid("a batch of " + std::to_string(rows) + " rows is too large for one segmented sort");
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    off_tiles = up(sizeof(SegDesc) * G);
    off_items = up(off_tiles + sizeof(uint32_t) * (G + 1));
    tables = up(off_items + sizeof(uint32_t) * (G + 1));
    off_stats = tables;
    off_kplan = up(off_stats + sizeof(KeyStats) * G);
    off_desc = up(off_kplan + sizeof(KeyPlan) * G);
    off_sum = up(off_desc + sizeof(PassDesc) * G * S);
    off_tick = up(off_sum + sizeof(SortSummary) * G);
    header = up(off_tick + sizeof(uint32_t) * S);
    kbuf = up(rows * sizeof(KeyT));
    ibuf = up(rows * 4);
    host.assign(tables, 0);
    std::memcpy(host.data(), segs.data(), sizeof(SegDesc) * G);
    std::memcpy(host.data() + off_tiles, tile_start.data(), sizeof(uint32_t) * (G + 1));
    std::memcpy(host.data() + off_items, item_start.data(), sizeof(uint32_t) * (G + 1));
  }
};

// The launches of one group, with its scratch at `base` and its tables already there or copied from
// `pinned_tables` (a graph's first node) when that is given. `timed`: a KernelTimer per launch (not
// inside a graph capture).
template <typename KeyT, int THREADS, int ITEMS>
void enqueue_group(const GroupLayout<KeyT, THREADS, ITEMS>& L, char* base, void* status, uint32_t* err,
                   const void* pinned_tables, bool timed, cudaStream_t s) {
  constexpr int S = GroupLayout<KeyT, THREADS, ITEMS>::S;
  if (pinned_tables) AM_CUDA(cudaMemcpyAsync(base, pinned_tables, L.tables, cudaMemcpyHostToDevice, s));
  AM_CUDA(cudaMemsetAsync(base + L.tables, 0, L.header - L.tables, s));
  const SegDesc* d_segs = reinterpret_cast<const SegDesc*>(base);
  const uint32_t* d_tiles = reinterpret_cast<const uint32_t*>(base + L.off_tiles);
  const uint32_t* d_items = reinterpret_cast<const uint32_t*>(base + L.off_items);
  KeyStats* st = reinterpret_cast<KeyStats*>(base + L.off_stats);
  KeyPlan* kp = reinterpret_cast<KeyPlan*>(base + L.off_kplan);
  PassDesc* pd = reinterpret_cast<PassDesc*>(base + L.off_desc);
  SortSummary* sum = reinterpret_cast<SortSummary*>(base + L.off_sum);
  uint32_t* tick = reinterpret_cast<uint32_t*>(base + L.off_tick);
  char* kbufA = base + L.header;
  char* kbufB = kbufA + L.kbuf;
  uint32_t* ibufA = reinterpret_cast<uint32_t*>(kbufB + L.kbuf);
  uint32_t* ibufB = reinterpret_cast<uint32_t*>(kbufB + L.kbuf + L.ibuf);
  {
    std::unique_ptr<KernelTimer> kt(timed ? new KernelTimer("batch_histogram", s) : nullptr);
    segmented_histogram_kernel<KeyT, HIST_THREADS, HIST_ITEMS><<<uint32_t(L.items), HIST_THREADS, 0, s>>>(
        d_segs, d_items, L.G, SEG_HIST_ROWS, st);
    AM_CUDA(cudaGetLastError());
  }
  {
    std::unique_ptr<KernelTimer> kt(timed ? new KernelTimer("batch_plan", s) : nullptr);
    segmented_plan_kernel<<<L.G, 256, 0, s>>>(d_segs, S, st, kp, pd, sum);
    AM_CUDA(cudaGetLastError());
  }
  // Every array's counts fit 30 bits below 2^30 rows: 32-bit look-back words, zeroed per pass. Above,
  // 64-bit words whose pass epochs (1..S) start over from a zeroed array in every call.
  const bool narrow = L.narrow();
  if (!narrow) AM_CUDA(cudaMemsetAsync(status, 0, size_t(L.tiles) * NBINS * sizeof(uint64_t), s));
  const int bps = narrow ? pass_blocks_per_sm<KeyT, uint32_t, true, ITEMS, THREADS>()
                         : pass_blocks_per_sm<KeyT, uint64_t, true, ITEMS, THREADS>();
  const int grid = int(std::min<uint64_t>(L.tiles, uint64_t(device().sm_count) * bps));
  for (int sl = 0; sl < S; sl++) {
    if (narrow) AM_CUDA(cudaMemsetAsync(status, 0, size_t(L.tiles) * NBINS * sizeof(uint32_t), s));
    PassArgs a{};
    a.desc = pd;
    a.kplan = kp;
    a.keys[0] = kbufA;
    a.keys[1] = kbufB;
    a.ids[0] = ibufA;
    a.ids[1] = ibufB;
    a.final_out = nullptr;
    a.status = status;
    a.epoch = uint32_t(sl + 1);
    a.tile_counter = tick + sl;
    a.err = err;
    a.carry_ids = 1;
    a.segs = d_segs;
    a.tile_start = d_tiles;
    a.nsegs = L.G;
    a.total_tiles = uint32_t(L.tiles);
    a.slot = uint32_t(sl);
    a.nslots = uint32_t(S);
    const ColView none{};
    std::unique_ptr<KernelTimer> kt(timed ? new KernelTimer("batch_pass", s) : nullptr);
    constexpr size_t smem = sizeof(PassShared<KeyT, THREADS, ITEMS>);
    if (narrow)
      onesweep_pass_kernel<KeyT, uint32_t, THREADS, ITEMS, true><<<std::max(grid, 1), THREADS, smem, s>>>(a, none);
    else
      onesweep_pass_kernel<KeyT, uint64_t, THREADS, ITEMS, true><<<std::max(grid, 1), THREADS, smem, s>>>(a, none);
    AM_CUDA(cudaGetLastError());
  }
}

// ---- CUDA graphs for repeated batch shapes.
//
// A batch's launches depend on its key width and its arrays' lengths only: the columns, options and
// output arrays reach the kernels through the segment table. The second time a thread sorts a batch of
// the same shape on the same stream, the launches are captured into a graph whose first node copies the
// table from a pinned host buffer; later batches of that shape write their table there and launch the
// graph: one launch instead of 2 + 2 x digits, and no scratch allocation. Two graph instances with
// their own pinned tables alternate, so a batch never waits for the one just before it.
struct BatchGraph {
  int width = 0;
  int items = 0;
  cudaStream_t stream = nullptr;
  std::vector<uint32_t> lens;
  char* base = nullptr;                 // scratch (device)
  void* status = nullptr;               // look-back words (device)
  size_t tables = 0;
  struct Slot {
    void* host = nullptr;               // pinned segment table
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done = nullptr;
    bool launched = false;
  } slot[2];
  int next = 0;
  ~BatchGraph() {
    for (auto& sl : slot) {
      if (sl.launched) (void)cudaEventSynchronize(sl.done);
      if (sl.exec) (void)cudaGraphExecDestroy(sl.exec);
      if (sl.done) (void)cudaEventDestroy(sl.done);
      pinned_free(sl.host);
    }
    if (base) (void)cudaFree(base);
    if (status) (void)cudaFree(status);
  }
};

constexpr size_t kGraphCacheEntries = 4;
constexpr size_t kGraphMaxScratch = size_t(16) << 30;    // larger batches run without a graph

struct GraphCache {
  std::list<std::unique_ptr<BatchGraph>> graphs;          // most recently used first
  std::list<std::pair<int, std::vector<uint32_t>>> seen;  // shapes seen once
};
GraphCache& graph_cache() {
  static thread_local GraphCache c;
  return c;
}

bool graphs_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("ARROWMETAL_BATCH_GRAPHS");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename KeyT, int THREADS, int ITEMS>
BatchGraph* find_or_capture(const GroupLayout<KeyT, THREADS, ITEMS>& L, uint32_t* err, cudaStream_t s) {
  GraphCache& c = graph_cache();
  const int width = int(sizeof(KeyT)) * 100000 + THREADS * 100 + ITEMS;    // key width and tile shape
  for (auto it = c.graphs.begin(); it != c.graphs.end(); ++it) {
    if ((*it)->width == width && (*it)->stream == s && (*it)->lens == L.lens) {
      c.graphs.splice(c.graphs.begin(), c.graphs, it);
      return c.graphs.front().get();
    }
  }
  bool seen = false;
  for (auto& sh : c.seen) if (sh.first == width && sh.second == L.lens) seen = true;
  if (!seen) {
    c.seen.emplace_front(width, L.lens);
    if (c.seen.size() > 16) c.seen.pop_back();
    return nullptr;
  }
  if (L.bytes() > kGraphMaxScratch) return nullptr;
  auto g = std::make_unique<BatchGraph>();
  g->width = width;
  g->stream = s;
  g->lens = L.lens;
  g->tables = L.tables;
  AM_CUDA(cudaMalloc(reinterpret_cast<void**>(&g->base), L.bytes()));
  const size_t status_bytes = size_t(L.tiles) * NBINS * (L.narrow() ? sizeof(uint32_t) : sizeof(uint64_t));
  AM_CUDA(cudaMalloc(&g->status, std::max<size_t>(status_bytes, 16)));
  // Launch attributes and occupancy are looked up before the capture.
  (void)pass_blocks_per_sm<KeyT, uint32_t, true, ITEMS, THREADS>();
  (void)pass_blocks_per_sm<KeyT, uint64_t, true, ITEMS, THREADS>();
  for (auto& sl : g->slot) {
    sl.host = pinned_alloc(L.tables);
    AM_CUDA(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
    cudaGraph_t graph = nullptr;
    AM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue_group<KeyT, THREADS, ITEMS>(L, g->base, g->status, err, sl.host, false, s);
    } catch (...) {
      cudaGraph_t discard = nullptr;
      (void)cudaStreamEndCapture(s, &discard);
      if (discard) (void)cudaGraphDestroy(discard);
      throw;
    }
    AM_CUDA(cudaStreamEndCapture(s, &graph));
    const cudaError_t e = cudaGraphInstantiate(&sl.exec, graph, 0);
    (void)cudaGraphDestroy(graph);
    AM_CUDA(e);
  }
  c.graphs.push_front(std::move(g));
  if (c.graphs.size() > kGraphCacheEntries) c.graphs.pop_back();
  return c.graphs.front().get();
}

template <typename KeyT, int THREADS, int ITEMS>
void sort_segment_class(const std::vector<SortKey>& keys, const std::vector<void*>& outs,
                        const std::vector<size_t>& group, bool allow_graph, cudaStream_t s) {
  GroupLayout<KeyT, THREADS, ITEMS> L(keys, outs, group);
  StreamScratch& sc = stream_scratch(s, L.narrow() ? (size_t(L.tiles) * NBINS + 1) / 2 : size_t(L.tiles) * NBINS);
  if (allow_graph && graphs_enabled()) {
    if (BatchGraph* g = find_or_capture<KeyT, THREADS, ITEMS>(L, sc.err, s)) {
      BatchGraph::Slot& sl = g->slot[g->next];
      g->next ^= 1;
      if (sl.launched) AM_CUDA(cudaEventSynchronize(sl.done));
      std::memcpy(sl.host, L.host.data(), L.tables);
      KernelTimer kt("batch_graph", s);
      AM_CUDA(cudaGraphLaunch(sl.exec, s));
      AM_CUDA(cudaEventRecord(sl.done, s));
      sl.launched = true;
      return;
    }
  }
  char* base = static_cast<char*>(dmalloc(L.bytes(), s));
  copy_h2d(base, L.host.data(), L.tables, s);
  enqueue_group<KeyT, THREADS, ITEMS>(L, base, sc.status, sc.err, nullptr, true, s);
  dfree(base, s);
}

// One launch sorts every array of a size class that fits a CTA (at most CTA_SORT_ROWS rows).
template <typename KeyT, int THREADS, int ITEMS, int DBITS>
void sort_segment_cta(const std::vector<SortKey>& keys, const std::vector<void*>& outs,
                      const std::vector<size_t>& group, cudaStream_t s) {
  static_assert(THREADS * ITEMS >= 4096, "the one-CTA class holds arrays of up to 4,096 rows");
  constexpr size_t SMEM = cta_sort_smem<KeyT, THREADS, ITEMS, DBITS>();
  static int blocks = 0;
  static std::once_flag once;
  std::call_once(once, [] {
    auto fn = segment_cta_sort_kernel<KeyT, THREADS, ITEMS, DBITS>;
    AM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(SMEM)));
    int b = 0;
    AM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, THREADS, SMEM));
    blocks = std::max(1, b);
  });
  std::vector<SegDesc> segs(group.size());
  for (size_t g = 0; g < group.size(); g++) {
    const SortKey& k = keys[group[g]];
    segs[g] = SegDesc{};
    segs[g].col = make_view(k);
    segs[g].out = outs[group[g]];
    segs[g].n = uint32_t(k.col->length);
  }
  const size_t bytes = sizeof(SegDesc) * segs.size();
  SegDesc* d = static_cast<SegDesc*>(dmalloc(bytes, s));
  copy_h2d(d, segs.data(), bytes, s);
  const int grid = int(std::min<uint64_t>(segs.size(), uint64_t(device().sm_count) * blocks));
  StreamScratch& sc = stream_scratch(s, 0);
  {
    KernelTimer kt("batch_cta_sort", s);
    segment_cta_sort_kernel<KeyT, THREADS, ITEMS, DBITS><<<std::max(grid, 1), THREADS, SMEM, s>>>(d, uint32_t(segs.size()), sc.err);
    AM_CUDA(cudaGetLastError());
  }
  dfree(d, s);
}

// ---- Shapes per size class, chosen by measurement.
//
// A batch's arrays of one key width fall into three size classes: up to CTA_SORT_ROWS rows, up to
// SMALL_ARRAY_ROWS, and larger. Each class has its candidate shapes: the digit passes with a tile of
// `threads` x `items` rows, or (the smallest class) one CTA per array with `threads` threads, `items`
// rows a thread and `digit_bits`-bit digits. The first batch whose class holds at least its class's
// tuning rows (2^18, 2^20 and 2^21 rows) runs the class with every candidate, timed by CUDA events (each run leaves the same,
// final output), and the fastest serves the class from then on. ARROWMETAL_SEG_ITEMS=4 or 8 fixes the
// passes' tile at 512 x 4 or 512 x 8 rows for every class instead.
constexpr uint32_t CTA_SORT_ROWS = 4096;
constexpr uint32_t SMALL_ARRAY_ROWS = 16384;
constexpr int SEG_CLASSES = 3;

struct SegShape {
  int method;          // 0: digit passes, 1: one CTA per array
  int threads, items, digit_bits;
};
constexpr SegShape kSegShapes[] = {
    {0, 512, 8, 8}, {0, 512, 4, 8}, {0, 384, 12, 8},
    {1, 256, 16, 8}, {1, 256, 16, 4}, {1, 512, 8, 8}, {1, 512, 8, 4},
};
constexpr int kNumSegShapes = int(sizeof(kSegShapes) / sizeof(kSegShapes[0]));
const std::vector<int>& class_candidates(int cls) {
  static const std::vector<int> c0 = {3, 4, 5, 6, 1}, c12 = {0, 1, 2};
  static_assert(kNumSegShapes == 7, "every shape is a candidate of some class");
  return cls == 0 ? c0 : c12;
}
uint64_t class_tune_rows(int cls) { return cls == 0 ? (uint64_t(1) << 18) : cls == 1 ? (uint64_t(1) << 20) : (uint64_t(2) << 20); }

std::mutex g_tune_mu;
int g_tuned_shape[2][SEG_CLASSES] = {{-1, -1, -1}, {-1, -1, -1}};   // [key width 4 / 8][class]

int forced_items() {
  static const int v = [] {
    const char* e = std::getenv("ARROWMETAL_SEG_ITEMS");
    const int x = e ? std::atoi(e) : 0;
    return (x == 4 || x == 8) ? x : 0;
  }();
  return v;
}

int tuned_shape(int width, int cls) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  return g_tuned_shape[width == 8][cls];
}

std::atomic<int> g_forced_shape{-1};     // test hook: one shape for every class it can serve

template <typename KeyT>
void run_segment_shape(int shape, const std::vector<SortKey>& keys, const std::vector<void*>& outs,
                       const std::vector<size_t>& group, bool allow_graph, cudaStream_t s) {
  switch (shape) {
    case 0: sort_segment_class<KeyT, 512, 8>(keys, outs, group, allow_graph, s); break;
    case 1: sort_segment_class<KeyT, 512, 4>(keys, outs, group, allow_graph, s); break;
    case 2: sort_segment_class<KeyT, 384, 12>(keys, outs, group, allow_graph, s); break;
    case 3: sort_segment_cta<KeyT, 256, 16, 8>(keys, outs, group, s); break;
    case 4: sort_segment_cta<KeyT, 256, 16, 4>(keys, outs, group, s); break;
    case 5: sort_segment_cta<KeyT, 512, 8, 8>(keys, outs, group, s); break;
    default: sort_segment_cta<KeyT, 512, 8, 4>(keys, outs, group, s); break;
  }
}

template <typename KeyT>
void sort_segment_group(const std::vector<SortKey>& keys, const std::vector<void*>& outs,
                        const std::vector<size_t>& group, cudaStream_t s) {
  std::vector<size_t> cls[SEG_CLASSES];
  uint64_t cls_rows[SEG_CLASSES] = {0, 0, 0};
  for (size_t i : group) {
    const uint64_t n = uint64_t(keys[i].col->length);
    const int c = n <= CTA_SORT_ROWS ? 0 : n <= SMALL_ARRAY_ROWS ? 1 : 2;
    cls[c].push_back(i);
    cls_rows[c] += n;
  }
  const int width = int(sizeof(KeyT));
  for (int c = 0; c < SEG_CLASSES; c++) {
    if (cls[c].empty()) continue;
    if (const int f = forced_items()) {
      run_segment_shape<KeyT>(f == 4 ? 1 : 0, keys, outs, cls[c], true, s);
      continue;
    }
    if (const int f = g_forced_shape.load(); f >= 0 && (kSegShapes[f].method == 0 || c == 0)) {
      run_segment_shape<KeyT>(f, keys, outs, cls[c], true, s);
      continue;
    }
    int shape = tuned_shape(width, c);
    if (shape < 0 && cls_rows[c] >= class_tune_rows(c)) {
      // Measure every candidate on this batch; each run leaves the same output.
      const std::vector<int>& cand = class_candidates(c);
      std::vector<float> ms(cand.size(), 0.0f);
      cudaEvent_t e0, e1;
      AM_CUDA(cudaEventCreate(&e0));
      AM_CUDA(cudaEventCreate(&e1));
      for (size_t k = 0; k < cand.size(); k++) {
        AM_CUDA(cudaEventRecord(e0, s));
        run_segment_shape<KeyT>(cand[k], keys, outs, cls[c], false, s);
        AM_CUDA(cudaEventRecord(e1, s));
        AM_CUDA(cudaEventSynchronize(e1));
        AM_CUDA(cudaEventElapsedTime(&ms[k], e0, e1));
      }
      (void)cudaEventDestroy(e0);
      (void)cudaEventDestroy(e1);
      const size_t best = size_t(std::min_element(ms.begin(), ms.end()) - ms.begin());
      std::lock_guard<std::mutex> g(g_tune_mu);
      g_tuned_shape[width == 8][c] = cand[best];
      continue;
    }
    if (shape < 0) shape = c == 0 ? 5 : 0;     // untuned: one CTA per array, or 512 x 8 tiles
    run_segment_shape<KeyT>(shape, keys, outs, cls[c], true, s);
  }
}

}  // namespace
}  // namespace rs

void debug_force_batch_shape(int shape) {
  if (shape >= rs::kNumSegShapes) throw invalid("no batch shape " + std::to_string(shape));
  rs::g_forced_shape.store(shape < 0 ? -1 : shape);
}

std::vector<std::array<int32_t, 7>> batch_tuning() {
  std::vector<std::array<int32_t, 7>> out;
  std::lock_guard<std::mutex> g(rs::g_tune_mu);
  const int32_t bound[rs::SEG_CLASSES] = {int32_t(rs::CTA_SORT_ROWS), int32_t(rs::SMALL_ARRAY_ROWS), -1};
  for (int w = 0; w < 2; w++)
    for (int c = 0; c < rs::SEG_CLASSES; c++) {
      const int sh = rs::g_tuned_shape[w][c];
      if (sh < 0) {
        out.push_back({w ? 8 : 4, c, bound[c], -1, 0, 0, 0});
        continue;
      }
      const rs::SegShape& x = rs::kSegShapes[sh];
      out.push_back({w ? 8 : 4, c, bound[c], x.method, x.threads, x.items, x.digit_bits});
    }
  return out;
}

void radix_argsort_batch(const std::vector<SortKey>& keys, const std::vector<void*>& outs, cudaStream_t s) {
  std::vector<size_t> g4, g8;
  for (size_t i = 0; i < keys.size(); i++) {
    if (keys[i].col->length <= 0) continue;
    if (pt_var(keys[i].col->pt) || keys[i].col->dictionary) {
      // A string or dictionary array: sorted on its own through its derived keys.
      argsort_any({keys[i]}, keys[i].col->length, outs[i], 4, s, nullptr);
      continue;
    }
    (pt_key_bytes(keys[i].col->pt) == 8 ? g8 : g4).push_back(i);
  }
  if (!g4.empty()) rs::sort_segment_group<uint32_t>(keys, outs, g4, s);
  if (!g8.empty()) rs::sort_segment_group<uint64_t>(keys, outs, g8, s);
}

// ------------------------------------------------------------------------------------------------
// Argsort that allocates nothing.
//
// Some callers cannot allocate device memory when they need a sort. A process whose device memory
// is owned by its own pool allocator (a framework's caching allocator, an RMM pool reserved at start)
// has no room outside that pool and must not have a library take memory behind it. A serving loop
// that must not stall cannot call cudaFree, which waits for the whole device. For them
// am_argsort_device_noalloc sorts one key column with all of its scratch in one fixed block of device
// memory that belongs to this library's image: every GPU the library is loaded on holds the block,
// about 6.1 MiB, until the process exits. The caller passes the input column and the output index
// array as device pointers. One call sorts at most NOALLOC_MAX_ROWS rows.

namespace rs {

constexpr uint64_t NOALLOC_MAX_ROWS = uint64_t(1) << 18;   // 262,144 rows per call
constexpr uint64_t NOALLOC_TILE_ROWS = uint64_t(PassConfig<uint64_t>::THREADS) * PassConfig<uint64_t>::ITEMS;
static_assert(NOALLOC_TILE_ROWS == uint64_t(PassConfig<uint32_t>::THREADS) * PassConfig<uint32_t>::ITEMS,
              "both key widths use the same tile");
constexpr int NOALLOC_MAX_PASSES = 8;                       // one key of at most 8 bytes

// What one call keeps besides the ping-pong buffers. All of it must be zero when a call starts (the
// histogram adds into `stats`, the passes take tiles from `tickets`, kernels OR into `err`), and so
// must the look-back status words before every pass.
struct NoAllocHeader {
  KeyStats stats;
  KeyPlan kplan;
  PassDesc desc[NOALLOC_MAX_PASSES];
  uint32_t tickets[NOALLOC_MAX_PASSES];
  SortSummary summary;
  uint32_t err;
};

constexpr size_t round256(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t NOALLOC_HEADER = round256(sizeof(NoAllocHeader));
constexpr size_t NOALLOC_KEYS = round256(NOALLOC_MAX_ROWS * 8);
constexpr size_t NOALLOC_IDS = round256(NOALLOC_MAX_ROWS * 4);
constexpr size_t NOALLOC_TILES = (NOALLOC_MAX_ROWS + NOALLOC_TILE_ROWS - 1) / NOALLOC_TILE_ROWS;
constexpr size_t NOALLOC_STATUS = round256(NOALLOC_TILES * NBINS * sizeof(uint32_t));
constexpr size_t NOALLOC_BYTES = NOALLOC_HEADER + 2 * NOALLOC_KEYS + 2 * NOALLOC_IDS + NOALLOC_STATUS;

// The block. In host code this name is only a stand-in for the device variable, never an address a
// kernel may be given: the host looks the address up per device (cudaGetSymbolAddress) and passes that.
static __device__ __align__(256) unsigned char noalloc_scratch[NOALLOC_BYTES];

namespace {

constexpr int NOALLOC_MAX_DEVICES = 64;

struct NoAllocDevice {
  bool ready = false;
  unsigned char* scratch = nullptr;   // device address of noalloc_scratch on this device
  int hist_grid_cap = 0;
  int pass_grid_cap[2] = {0, 0};      // 4-byte and 8-byte keys
};

// Calls share the block, so they take turns: the lock is held until the call's work has finished on
// its stream.
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc[NOALLOC_MAX_DEVICES];

template <typename KeyT>
int noalloc_pass_cap(int sm_count) {
  using C = PassConfig<KeyT>;
  auto fn = onesweep_pass_kernel<KeyT, uint32_t, C::THREADS, C::ITEMS, false>;
  AM_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(pass_smem<KeyT>())));
  int b = 0;
  AM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, C::THREADS, pass_smem<KeyT>()));
  return sm_count * std::max(1, b);
}

// Set-up of the calling thread's current device, once: the block's device address, the kernels'
// shared-memory limit and grid caps. It runs inside the first call on each device.
NoAllocDevice& noalloc_device() {
  int dev = 0;
  AM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    throw unsupported("argsort without allocation runs on devices 0 to " + std::to_string(NOALLOC_MAX_DEVICES - 1));
  NoAllocDevice& d = g_noalloc[dev];
  if (d.ready) return d;
  unsigned char* ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, noalloc_scratch);
  if (e != cudaSuccess || ptr == nullptr) {
    (void)cudaGetLastError();
    throw Error(std::string("argsort without allocation: no device address for its scratch block on device ") +
                std::to_string(dev) + ": " + (e != cudaSuccess ? cudaGetErrorString(e) : "null address"));
  }
  int sm = 0;
  AM_CUDA(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, dev));
  d.scratch = ptr;
  d.hist_grid_cap = std::max(1, sm) * 8;
  d.pass_grid_cap[0] = noalloc_pass_cap<uint32_t>(std::max(1, sm));
  d.pass_grid_cap[1] = noalloc_pass_cap<uint64_t>(std::max(1, sm));
  d.ready = true;
  return d;
}

template <typename KeyT>
void noalloc_launch_pass(const PassArgs& a, const ColView& cv, uint64_t n, int cap, cudaStream_t s) {
  using C = PassConfig<KeyT>;
  const uint64_t tiles = (n + NOALLOC_TILE_ROWS - 1) / NOALLOC_TILE_ROWS;
  const int grid = int(std::min<uint64_t>(tiles, uint64_t(cap)));
  onesweep_pass_kernel<KeyT, uint32_t, C::THREADS, C::ITEMS, false><<<std::max(grid, 1), C::THREADS, pass_smem<KeyT>(), s>>>(a, cv);
  AM_CUDA(cudaGetLastError());
}

template <typename KeyT>
void noalloc_launch_histogram(const ColView& cv, KeyStats* st, uint64_t n, int cap, cudaStream_t s) {
  constexpr int CHUNK = HIST_THREADS * HIST_ITEMS;
  const uint64_t chunks = (n + CHUNK - 1) / CHUNK;
  const int grid = int(std::min<uint64_t>(chunks, uint64_t(cap)));
  key_histogram_kernel<KeyT, HIST_THREADS, HIST_ITEMS, false><<<std::max(grid, 1), HIST_THREADS, 0, s>>>(cv, st, n);
  AM_CUDA(cudaGetLastError());
}

}  // namespace
}  // namespace rs

uint64_t noalloc_max_rows() { return rs::NOALLOC_MAX_ROWS; }

void argsort_noalloc(int pt, const void* values, const uint8_t* validity, int64_t offset, int64_t length,
                     bool descending, bool nulls_first, int float_order, uint32_t* indices, cudaStream_t s) {
  using namespace rs;
  if (pt_var(pt)) throw unsupported("argsort without allocation takes fixed-width columns");
  if (length < 0) throw invalid("negative length " + std::to_string(length));
  if (offset < 0) throw invalid("negative offset " + std::to_string(offset));
  if (uint64_t(length) > NOALLOC_MAX_ROWS)
    throw invalid("argsort without allocation takes at most " + std::to_string(NOALLOC_MAX_ROWS) + " rows (" +
                  std::to_string(length) + " given): its fixed scratch block holds no more");
  if (float_order < 0 || float_order > 2) throw invalid("unknown float_order " + std::to_string(float_order));
  if (length == 0) return;
  if (!values) throw invalid("no values buffer");
  if (!indices) throw invalid("no output index buffer");
  const uint64_t n = uint64_t(length);
  const int kb = pt_key_bytes(pt);

  ColView cv{};
  cv.values = pt == PT_BOOL ? values : static_cast<const void*>(static_cast<const char*>(values) + offset * pt_bytes(pt));
  cv.valid = validity;
  cv.valid_off = offset;
  cv.bool_off = pt == PT_BOOL ? offset : 0;
  cv.pt = pt;
  cv.desc = descending ? 1 : 0;
  cv.nulls_first = nulls_first ? 1 : 0;
  const bool fl = pt_float(pt);
  cv.float_order = fl ? uint8_t(float_order) : uint8_t(FO_IEEE);
  cv.nan_cat = (fl && float_order == FO_IEEE) ? 1 : 0;

  PlanArgs pa{};
  pa.n = n;
  pa.nkeys = 1;
  pa.nslots = kb;
  pa.slot_key0_first = 0;
  pa.index_wide = 0;
  pa.key_bytes[0] = uint8_t(kb);
  pa.nulls_first[0] = nulls_first ? 1 : 0;
  for (int d = 0; d < kb; d++) {
    pa.slot_key[d] = 0;
    pa.slot_digit[d] = int8_t(d);
  }

  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocDevice& dev = noalloc_device();
  unsigned char* base = dev.scratch;
  NoAllocHeader* h = reinterpret_cast<NoAllocHeader*>(base);
  unsigned char* keysA = base + NOALLOC_HEADER;
  unsigned char* keysB = keysA + NOALLOC_KEYS;
  uint32_t* idsA = reinterpret_cast<uint32_t*>(keysB + NOALLOC_KEYS);
  uint32_t* idsB = reinterpret_cast<uint32_t*>(keysB + NOALLOC_KEYS + NOALLOC_IDS);
  uint32_t* status = reinterpret_cast<uint32_t*>(keysB + NOALLOC_KEYS + 2 * NOALLOC_IDS);
  const size_t status_bytes = ((n + NOALLOC_TILE_ROWS - 1) / NOALLOC_TILE_ROWS) * NBINS * sizeof(uint32_t);

  try {
    // The block keeps whatever the previous call left in it.
    AM_CUDA(cudaMemsetAsync(h, 0, sizeof(NoAllocHeader), s));
    if (kb == 8) noalloc_launch_histogram<uint64_t>(cv, &h->stats, n, dev.hist_grid_cap, s);
    else noalloc_launch_histogram<uint32_t>(cv, &h->stats, n, dev.hist_grid_cap, s);
    plan_kernel<<<1, 256, 0, s>>>(pa, &h->stats, &h->kplan, h->desc, &h->summary);
    AM_CUDA(cudaGetLastError());
    for (int sl = 0; sl < kb; sl++) {
      AM_CUDA(cudaMemsetAsync(status, 0, status_bytes, s));
      PassArgs a{};
      a.desc = h->desc + sl;
      a.kplan = &h->kplan;
      a.keys[0] = keysA;
      a.keys[1] = keysB;
      a.ids[0] = idsA;
      a.ids[1] = idsB;
      a.final_out = indices;
      a.status = status;
      a.epoch = 1;
      a.tile_counter = h->tickets + sl;
      a.err = &h->err;
      a.carry_ids = 1;
      if (kb == 8) noalloc_launch_pass<uint64_t>(a, cv, n, dev.pass_grid_cap[1], s);
      else noalloc_launch_pass<uint32_t>(a, cv, n, dev.pass_grid_cap[0], s);
    }
    // Wait for the sort and read its error word into a host variable.
    uint32_t err = 0;
    AM_CUDA(cudaMemcpyAsync(&err, &h->err, sizeof(err), cudaMemcpyDeviceToHost, s));
    AM_CUDA(cudaStreamSynchronize(s));
    if (err & ERR_LOOKBACK_TIMEOUT) throw Error("radix sort: a look-back wait timed out on the device");
    if (err & ERR_BOUNDS) throw Error("radix sort: a destination fell outside its array (write skipped)");
    if (err) throw Error("device error word " + std::to_string(err));
  } catch (...) {
    // Leave no work in flight on the block for the next call.
    (void)cudaStreamSynchronize(s);
    (void)cudaGetLastError();
    throw;
  }
}

}  // namespace am
