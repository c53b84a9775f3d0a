// Sort consumers: Arrow's rank with its four tiebreakers, rank_quantile / rank_normal, the SQL window
// ranking functions (row_number, rank, dense_rank, percent_rank, cume_dist), unique and value_counts.
// Each is one stable argsort of the column and a few passes over its sorted order (the reference builds
// them the same way: Sources/ArrowMetal/Kernels/Window.swift:106-200 for the rankings,
// Kernels/Unique.swift:46-65 and Kernels/UniqueOrder.swift:88-140 for the distinct values):
//   1. run marks: sorted position i starts a run when its row is not equal to the row at i - 1, with
//      the sort's value equality (-0.0 ties +0.0, every NaN is one value, the nulls are one run; Arrow's
//      rank functions also put the NaN rows and the nulls in one run, as pyarrow ranks them). One byte
//      per position, and a count of marks per block;
//   2. an exclusive scan of the block counts (one block; the total run count lands after them);
//   3. every position's run number (its block's offset plus a block scan of the marks); a run's first
//      position is recorded as the run's start, and its row as the run's representative (the earliest
//      row of the run: the sort is stable);
//   4. one pass over the positions turns run numbers into the answer (the run's first or last
//      position, its quantile), or one over the runs gives their lengths;
//   5. the answers go to their original rows by a scatter in two steps that keeps every random store
//      inside L2: the (row, value) pairs are appended to the bucket of the row's high bits (a bucket's
//      size is known, the order being a permutation), then drained bucket after bucket.
#include <algorithm>
#include <vector>

#include "am_internal.h"
#include "key_encode.cuh"
#include "radix_sort.cuh"

namespace am {
namespace rs {
namespace {

constexpr int RUN_THREADS = 256, RUN_ITEMS = 16;
constexpr uint64_t RUN_CHUNK = uint64_t(RUN_THREADS) * RUN_ITEMS;

// A string column as the run marks read it.
struct StrView {
  const void* offsets;        // row 0's offset
  const uint8_t* bytes;
  const uint8_t* valid;       // NULL: no nulls
  int64_t valid_off;
};

// The equality class of a fixed-width row: its sort key and category (0 value, 1 NaN, 2 null).
template <typename KeyT>
__device__ __forceinline__ void run_key(const ColView& c, uint32_t row, bool merge_nan, KeyT& key, int& cat) {
  const KeyT raw = load_raw<KeyT>(c, row);
  const bool valid = !c.valid || bit_at(c.valid, c.valid_off + int64_t(row));
  key = key_from_raw<KeyT>(c, raw, valid, cat);
  if (merge_nan && cat == 1) cat = 2;
}

template <typename OffT>
__device__ __forceinline__ bool same_string(const StrView& v, uint32_t a, uint32_t b) {
  const bool va = !v.valid || bit_at(v.valid, v.valid_off + int64_t(a));
  const bool vb = !v.valid || bit_at(v.valid, v.valid_off + int64_t(b));
  if (va != vb) return false;
  if (!va) return true;
  const OffT* off = static_cast<const OffT*>(v.offsets);
  const uint64_t sa = uint64_t(off[a]), sb = uint64_t(off[b]);
  const uint64_t la = uint64_t(off[a + 1]) - sa, lb = uint64_t(off[b + 1]) - sb;
  if (la != lb) return false;
  for (uint64_t j = 0; j < la; j++)
    if (v.bytes[sa + j] != v.bytes[sb + j]) return false;
  return true;
}

__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* s_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = __reduce_add_sync(0xffffffffu, v);
  if (lane == 0) s_warp[warp] = v;
  __syncthreads();
  uint32_t all = 0;
#pragma unroll
  for (int w = 0; w < RUN_THREADS / 32; w++) all += s_warp[w];
  return all;
}

// Block-wide exclusive scan of one value per thread.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t* s_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  uint32_t add = 0;
#pragma unroll
  for (int w = 0; w < RUN_THREADS / 32; w++)
    if (w < warp) add += s_warp[w];
  return x - v + add;
}

// Writes one thread's RUN_ITEMS marks at position `base` (a multiple of RUN_ITEMS), 16 bytes at once
// when all of them exist.
__device__ __forceinline__ void store_marks(uint8_t* marks, uint64_t base, uint64_t m, const uint8_t (&mk)[RUN_ITEMS]) {
  if (base + RUN_ITEMS <= m) {
    uint32_t w[4];
#pragma unroll
    for (int q = 0; q < 4; q++)
      w[q] = uint32_t(mk[4 * q]) | (uint32_t(mk[4 * q + 1]) << 8) | (uint32_t(mk[4 * q + 2]) << 16) |
             (uint32_t(mk[4 * q + 3]) << 24);
    *reinterpret_cast<uint4*>(marks + base) = make_uint4(w[0], w[1], w[2], w[3]);
  } else {
    for (int i = 0; i < RUN_ITEMS && base + i < m; i++) marks[base + i] = mk[i];
  }
}

// 1. Run marks of sorted positions [0, m) of a fixed-width column, and their count per block.
template <typename KeyT>
__global__ void __launch_bounds__(RUN_THREADS) run_marks_kernel(const __grid_constant__ ColView c, int merge_nan,
                                                                const uint32_t* __restrict__ perm, uint64_t m,
                                                                uint8_t* __restrict__ marks,
                                                                uint32_t* __restrict__ block_counts) {
  __shared__ uint32_t s_warp[RUN_THREADS / 32];
  const uint64_t base = uint64_t(blockIdx.x) * RUN_CHUNK + uint64_t(threadIdx.x) * RUN_ITEMS;
  uint8_t mk[RUN_ITEMS];
  uint32_t cnt = 0;
  if (base < m) {
    // Rows of positions base - 1 .. base + RUN_ITEMS - 1: all the index loads, then the value loads.
    uint32_t row[RUN_ITEMS + 1];
#pragma unroll
    for (int i = 0; i <= RUN_ITEMS; i++) {
      const uint64_t pos = base + i - 1;
      row[i] = (i == 0 && base == 0) || pos >= m ? 0u : perm[pos];
    }
    KeyT key[RUN_ITEMS + 1];
    int cat[RUN_ITEMS + 1];
#pragma unroll
    for (int i = 0; i <= RUN_ITEMS; i++) run_key<KeyT>(c, row[i], merge_nan != 0, key[i], cat[i]);
#pragma unroll
    for (int i = 0; i < RUN_ITEMS; i++) {
      const uint64_t pos = base + i;
      const bool start = pos == 0 || cat[i] != cat[i + 1] || (cat[i + 1] == 0 && key[i] != key[i + 1]);
      mk[i] = (pos < m && start) ? 1 : 0;
      cnt += mk[i];
    }
    store_marks(marks, base, m, mk);
  }
  const uint32_t total = block_sum(cnt, s_warp);
  if (threadIdx.x == 0) block_counts[blockIdx.x] = total;
}

// 1'. The same for a string column (bytes compared, lengths first).
template <typename OffT>
__global__ void __launch_bounds__(RUN_THREADS) run_marks_str_kernel(const __grid_constant__ StrView v,
                                                                    const uint32_t* __restrict__ perm, uint64_t m,
                                                                    uint8_t* __restrict__ marks,
                                                                    uint32_t* __restrict__ block_counts) {
  __shared__ uint32_t s_warp[RUN_THREADS / 32];
  const uint64_t base = uint64_t(blockIdx.x) * RUN_CHUNK + uint64_t(threadIdx.x) * RUN_ITEMS;
  uint8_t mk[RUN_ITEMS];
  uint32_t cnt = 0;
  if (base < m) {
    uint32_t prev = base == 0 ? 0u : perm[base - 1];
    for (int i = 0; i < RUN_ITEMS; i++) {
      const uint64_t pos = base + i;
      mk[i] = 0;
      if (pos >= m) continue;
      const uint32_t r = perm[pos];
      mk[i] = (pos == 0 || !same_string<OffT>(v, prev, r)) ? 1 : 0;
      cnt += mk[i];
      prev = r;
    }
    store_marks(marks, base, m, mk);
  }
  const uint32_t total = block_sum(cnt, s_warp);
  if (threadIdx.x == 0) block_counts[blockIdx.x] = total;
}

// 2. One block: exclusive scan of the block counts in place; the total run count lands at [blocks].
__global__ void __launch_bounds__(1024) run_scan_kernel(uint32_t* __restrict__ counts, uint32_t blocks) {
  __shared__ uint32_t s[32];
  __shared__ uint32_t carry;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < blocks; base += 1024) {
    const uint32_t i = base + uint32_t(t);
    const uint32_t v = i < blocks ? counts[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s[warp] = x;
    __syncthreads();
    uint32_t add = carry, all = 0;
    for (int w = 0; w < 32; w++) {
      if (w < warp) add += s[w];
      all += s[w];
    }
    if (i < blocks) counts[i] = x - v + add;
    __syncthreads();
    if (t == 0) carry += all;
    __syncthreads();
  }
  if (t == 0) counts[blocks] = carry;
}

// 3. Run numbers (1-based) of positions [0, m): run_of_pos[i] (when wanted), and for each run's first
// position its start and its row.
__global__ void __launch_bounds__(RUN_THREADS) run_ids_kernel(const uint8_t* __restrict__ marks,
                                                              const uint32_t* __restrict__ block_off,
                                                              const uint32_t* __restrict__ perm, uint64_t m,
                                                              uint32_t* __restrict__ run_of_pos,
                                                              uint32_t* __restrict__ starts,
                                                              uint32_t* __restrict__ heads) {
  __shared__ uint32_t s_warp[RUN_THREADS / 32];
  const uint64_t base = uint64_t(blockIdx.x) * RUN_CHUNK + uint64_t(threadIdx.x) * RUN_ITEMS;
  uint8_t mk[RUN_ITEMS];
  if (base + RUN_ITEMS <= m) {
    const uint4 w = *reinterpret_cast<const uint4*>(marks + base);
    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int i = 0; i < RUN_ITEMS; i++) mk[i] = uint8_t(ws[i >> 2] >> (8 * (i & 3)));
  } else {
#pragma unroll
    for (int i = 0; i < RUN_ITEMS; i++) mk[i] = base + i < m ? marks[base + i] : 0;
  }
  uint32_t cnt = 0;
#pragma unroll
  for (int i = 0; i < RUN_ITEMS; i++) cnt += mk[i];
  uint32_t run = block_off[blockIdx.x] + block_exclusive(cnt, s_warp);
#pragma unroll
  for (int i = 0; i < RUN_ITEMS; i++) {
    const uint64_t pos = base + i;
    if (pos >= m) break;
    run += mk[i];
    if (run_of_pos) run_of_pos[pos] = run;
    if (mk[i]) {
      if (starts) starts[run - 1] = uint32_t(pos);
      if (heads) heads[run - 1] = perm[pos];
    }
  }
}

// 4. Run numbers into the answer, per sorted position. A run [s, e) of sorted positions:
//   FIN_MIN s + 1; FIN_MAX e; FIN_QUANTILE (s + e) / 2n, the run's average 1-based rank minus one
//   half over n; FIN_NORMAL64 / FIN_NORMAL32 the standard normal quantile of that; FIN_PERCENT
//   s / (n - 1) (0 for one row); FIN_CUME e / n.
enum Finish { FIN_MIN = 0, FIN_MAX, FIN_QUANTILE, FIN_NORMAL64, FIN_NORMAL32, FIN_PERCENT, FIN_CUME };

__global__ void __launch_bounds__(256) rank_finish_kernel(const uint32_t* run_of_pos,
                                                          const uint32_t* __restrict__ starts,
                                                          const uint32_t* __restrict__ total_runs, uint64_t n,
                                                          int mode, void* out) {
  const uint32_t runs = *total_runs;
  for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t g = run_of_pos[r];
    const uint64_t s = starts[g - 1];
    const uint64_t e = g < runs ? uint64_t(starts[g]) : n;
    switch (mode) {
      case FIN_MIN: static_cast<uint32_t*>(out)[r] = uint32_t(s + 1); break;
      case FIN_MAX: static_cast<uint32_t*>(out)[r] = uint32_t(e); break;
      case FIN_QUANTILE: static_cast<double*>(out)[r] = double(s + e) / double(2 * n); break;
      case FIN_NORMAL64: static_cast<double*>(out)[r] = normcdfinv(double(s + e) / double(2 * n)); break;
      case FIN_NORMAL32: static_cast<float*>(out)[r] = float(normcdfinv(double(s + e) / double(2 * n))); break;
      case FIN_PERCENT: static_cast<double*>(out)[r] = n > 1 ? double(s) / double(n - 1) : 0.0; break;
      default: static_cast<double*>(out)[r] = double(e) / double(n); break;
    }
  }
}

// 5. The scatter to the original rows: out[perm[i]] = val[i] (val NULL: i + 1). perm is a permutation of
// [0, n), so the pairs whose row lies in [b << shift, (b + 1) << shift) are exactly 2^shift (fewer in
// the last bucket) and bucket b's pairs go to [b << shift, ...) of the pair arrays, each block reserving
// its share of every bucket with one atomic. The drain then reads the pairs in order: the blocks in
// flight work on a few neighbouring buckets, whose rows span a region L2 holds.
constexpr int SC_THREADS = 512, SC_ITEMS = 8;
constexpr uint64_t SC_CHUNK = uint64_t(SC_THREADS) * SC_ITEMS;

// Each warp ranks its pairs within their buckets by ballots on the bucket's bits (no shared atomics:
// the warp's counters advance item by item, as in the sort's ranking); then one thread per bucket
// reserves the block's share with one atomic and hands each warp its offset.
constexpr int SC_WARPS = SC_THREADS / 32;
constexpr int SC_MAX_BUCKETS = 64, SC_BUCKET_BITS = 6;

template <typename V>
__global__ void __launch_bounds__(SC_THREADS) bucket_pairs_kernel(const uint32_t* __restrict__ perm,
                                                                  const V* __restrict__ val, uint64_t n, int shift,
                                                                  int nb, uint32_t* __restrict__ cursor,
                                                                  uint32_t* __restrict__ rows_out, V* __restrict__ vals_out,
                                                                  uint32_t* __restrict__ err) {
  __shared__ uint32_t wcnt[SC_WARPS][SC_MAX_BUCKETS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  for (int b = lane; b < SC_MAX_BUCKETS; b += 32) wcnt[warp][b] = 0;
  __syncwarp();
  // A warp's items: SC_ITEMS x 32 consecutive positions.
  const uint64_t start = uint64_t(blockIdx.x) * SC_CHUNK + uint64_t(warp) * (SC_ITEMS * 32);
  uint32_t row[SC_ITEMS], slot[SC_ITEMS];
  V v[SC_ITEMS];
#pragma unroll
  for (int i = 0; i < SC_ITEMS; i++) {
    const uint64_t pos = start + uint64_t(i) * 32 + lane;
    const bool live = pos < n;
    row[i] = live ? perm[pos] : 0u;
    v[i] = live ? (val ? val[pos] : V(pos + 1)) : V(0);
  }
#pragma unroll
  for (int i = 0; i < SC_ITEMS; i++) {
    const uint64_t pos = start + uint64_t(i) * 32 + lane;
    const bool live = pos < n;
    const uint32_t b = live ? (row[i] >> shift) : 0u;
    uint32_t peers = __ballot_sync(0xffffffffu, live);
#pragma unroll
    for (int k = 0; k < SC_BUCKET_BITS; k++) {
      const uint32_t bit = (b >> k) & 1u;
      const uint32_t bl = __ballot_sync(0xffffffffu, bit);
      peers &= bit ? bl : ~bl;
    }
    const uint32_t base = live ? wcnt[warp][b] : 0u;
    __syncwarp();
    if (live) {
      if (lane == __ffs(peers) - 1) wcnt[warp][b] = base + __popc(peers);
      slot[i] = base + __popc(peers & lt);
    }
    __syncwarp();
  }
  __syncthreads();
  // Per bucket: the block's total, one reservation, and each warp's offset within it.
  for (int b = threadIdx.x; b < nb; b += SC_THREADS) {
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < SC_WARPS; w++) total += wcnt[w][b];
    uint32_t at = total ? (uint32_t(b) << shift) + atomicAdd(&cursor[b], total) : 0u;
#pragma unroll
    for (int w = 0; w < SC_WARPS; w++) {
      const uint32_t c = wcnt[w][b];
      wcnt[w][b] = at;
      at += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < SC_ITEMS; i++) {
    const uint64_t pos = start + uint64_t(i) * 32 + lane;
    if (pos >= n) continue;
    const uint64_t dst = uint64_t(wcnt[warp][row[i] >> shift]) + slot[i];
    if (dst >= n) {
      atomicOr(err, ERR_BOUNDS);
      continue;
    }
    rows_out[dst] = row[i];
    vals_out[dst] = v[i];
  }
}

template <typename V>
__global__ void __launch_bounds__(256) drain_pairs_kernel(const uint32_t* __restrict__ rows, const V* __restrict__ vals,
                                                          uint64_t n, V* __restrict__ out, uint32_t* __restrict__ err) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t r = rows[i];
    if (r < n) out[r] = vals[i];
    else atomicOr(err, ERR_BOUNDS);
  }
}

// Run lengths: counts[g] = start of run g + 1 (or m) - start of run g.
__global__ void __launch_bounds__(256) run_lengths_kernel(const uint32_t* __restrict__ starts, const uint32_t* __restrict__ total_runs,
                                                          uint64_t m, int64_t* __restrict__ counts) {
  const uint32_t runs = *total_runs;
  for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < runs; g += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t e = g + 1 < runs ? uint64_t(starts[g + 1]) : m;
    counts[g] = int64_t(e - starts[g]);
  }
}

// rows_out[i] = heads[order[i]], counts_out[i] = counts[order[i]] (when counts are wanted).
__global__ void __launch_bounds__(256) runs_in_order_kernel(const uint32_t* __restrict__ order, const uint32_t* __restrict__ heads,
                                                            const int64_t* __restrict__ counts, uint64_t runs,
                                                            uint32_t* __restrict__ rows_out, int64_t* __restrict__ counts_out) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < runs; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t g = order[i];
    rows_out[i] = heads[g];
    if (counts) counts_out[i] = counts[g];
  }
}

// A dictionary column's values as the key builder reads them: validity, and (ieee float values) the
// bits that tell a NaN.
struct DictView {
  const void* values;
  const uint8_t* valid;       // NULL: no null entries
  int64_t valid_off;
  int32_t pt;
  int32_t nan_cat;            // a NaN value is its own block (ieee order)
};

__device__ __forceinline__ int64_t load_code(const void* codes, int pt, uint64_t r) {
  switch (pt) {
    case PT_I8: return static_cast<const int8_t*>(codes)[r];
    case PT_U8: return static_cast<const uint8_t*>(codes)[r];
    case PT_I16: return static_cast<const int16_t*>(codes)[r];
    case PT_U16: return static_cast<const uint16_t*>(codes)[r];
    case PT_I32: return static_cast<const int32_t*>(codes)[r];
    case PT_U32: return static_cast<const uint32_t*>(codes)[r];
    case PT_U64: {
      const uint64_t v = static_cast<const uint64_t*>(codes)[r];
      return v > uint64_t(INT64_MAX) ? -1 : int64_t(v);
    }
    default: return static_cast<const int64_t*>(codes)[r];
  }
}

__device__ __forceinline__ bool entry_is_nan(const DictView& d, uint64_t c) {
  switch (d.pt) {
    case PT_F16: return (static_cast<const uint16_t*>(d.values)[c] & 0x7FFFu) > 0x7C00u;
    case PT_F32: return (static_cast<const uint32_t*>(d.values)[c] & 0x7FFFFFFFu) > 0x7F800000u;
    case PT_F64: return (static_cast<const uint64_t*>(d.values)[c] & 0x7FFFFFFFFFFFFFFFull) > 0x7FF0000000000000ull;
    default: return false;
  }
}

// Row keys of a dictionary column: the dense rank (1-based) of the row's value among the dictionary's
// distinct values, minus one, as a float; NaN for a NaN value in the ieee order; null where the code or
// the value is null. A warp handles 32 consecutive rows and writes their validity word.
template <typename OutT>
__global__ void __launch_bounds__(256) dict_row_keys_kernel(const void* __restrict__ codes, int code_pt,
                                                            const uint8_t* __restrict__ code_valid, int64_t code_voff,
                                                            uint64_t n, const __grid_constant__ DictView dict,
                                                            const uint32_t* __restrict__ dense, uint64_t d,
                                                            OutT* __restrict__ key, uint32_t* __restrict__ valid_words,
                                                            unsigned long long* __restrict__ null_count,
                                                            uint32_t* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
  unsigned long long nulls = 0;
  for (uint64_t w = uint64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); w * 32 < n; w += warps) {
    const uint64_t r = w * 32 + lane;
    bool valid = false;
    OutT k = OutT(0);
    if (r < n && (!code_valid || bit_at(code_valid, code_voff + int64_t(r)))) {
      const int64_t c = load_code(codes, code_pt, r);
      if (c < 0 || uint64_t(c) >= d) {
        atomicOr(err, ERR_DICT_CODE);
      } else if (!dict.valid || bit_at(dict.valid, dict.valid_off + c)) {
        valid = true;
        k = (dict.nan_cat && entry_is_nan(dict, uint64_t(c))) ? OutT(NAN) : OutT(dense[c] - 1u);
      }
    }
    const uint32_t word = __ballot_sync(0xffffffffu, valid);
    if (r < n) key[r] = k;
    if (lane == 0) {
      valid_words[w] = word;
      const uint64_t live = n - w * 32 < 32 ? n - w * 32 : 32;
      nulls += live - uint64_t(__popc(word));
    }
  }
  if (lane == 0 && nulls) atomicAdd(null_count, nulls);
}

int grid_for(uint64_t n) {
  return int(std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, uint64_t(device().sm_count) * 8)));
}

}  // namespace
}  // namespace rs

namespace {

using namespace rs;

// The stable argsort (uint32) of one column.
BufPtr sorted_order(am_array* a, bool desc, bool nulls_first, int float_order, cudaStream_t s) {
  const int64_t n = a->length;
  BufPtr perm = DevBuffer::alloc(size_t(n) * 4 + 16, s);
  argsort_any({SortKey{a, desc, nulls_first, float_order}}, n, perm->ptr, 4, s, nullptr);
  return perm;
}

// Steps 1 and 2 over sorted positions [0, m): marks and scanned block counts (blocks + 1 words).
struct Runs {
  BufPtr marks, counts;
  uint32_t blocks = 0;
  const uint32_t* total() const { return static_cast<const uint32_t*>(counts->ptr) + blocks; }
};

Runs mark_runs(am_array* a, const uint32_t* perm, uint64_t m, bool merge_nan, int float_order, cudaStream_t s) {
  Runs r;
  r.blocks = uint32_t((m + RUN_CHUNK - 1) / RUN_CHUNK);
  r.marks = DevBuffer::alloc(size_t(m) + 16, s);
  r.counts = DevBuffer::alloc(size_t(r.blocks + 1) * 4, s);
  uint8_t* marks = static_cast<uint8_t*>(r.marks->ptr);
  uint32_t* counts = static_cast<uint32_t*>(r.counts->ptr);
  KernelTimer kt("run_marks", s);
  if (pt_var(a->pt)) {
    const StrView v{a->data(), static_cast<const uint8_t*>(a->bytes->ptr), a->null_count != 0 ? a->valid_bits() : nullptr,
                    a->validity_offset};
    if (a->pt == PT_LSTR) run_marks_str_kernel<int64_t><<<r.blocks, RUN_THREADS, 0, s>>>(v, perm, m, marks, counts);
    else run_marks_str_kernel<int32_t><<<r.blocks, RUN_THREADS, 0, s>>>(v, perm, m, marks, counts);
  } else {
    const ColView c = make_view(SortKey{a, false, false, float_order});
    if (pt_key_bytes(a->pt) == 8)
      run_marks_kernel<uint64_t><<<r.blocks, RUN_THREADS, 0, s>>>(c, merge_nan ? 1 : 0, perm, m, marks, counts);
    else run_marks_kernel<uint32_t><<<r.blocks, RUN_THREADS, 0, s>>>(c, merge_nan ? 1 : 0, perm, m, marks, counts);
  }
  AM_CUDA(cudaGetLastError());
  run_scan_kernel<<<1, 1024, 0, s>>>(counts, r.blocks);
  AM_CUDA(cudaGetLastError());
  return r;
}

void run_ids(const Runs& r, const uint32_t* perm, uint64_t m, uint32_t* run_of_row, uint32_t* starts, uint32_t* heads,
             cudaStream_t s) {
  KernelTimer kt("run_ids", s);
  run_ids_kernel<<<r.blocks, RUN_THREADS, 0, s>>>(static_cast<const uint8_t*>(r.marks->ptr),
                                                  static_cast<const uint32_t*>(r.counts->ptr), perm, m, run_of_row,
                                                  starts, heads);
  AM_CUDA(cudaGetLastError());
}

// out[perm[i]] = vals[i] for i < n (vals NULL: i + 1), perm a permutation of [0, n).
template <typename V>
void scatter_to_rows(const uint32_t* perm, const V* vals, uint64_t n, V* out, cudaStream_t s) {
  int bits = 0;
  while ((uint64_t(1) << bits) < n) bits++;
  // At most 64 buckets: a block's 4,096 pairs make runs of ~64 per bucket, and a bucket's rows (at
  // most 2^26 of the 2^32 rows, 4-8 MB at 50M rows) still sit well inside L2 while they drain.
  const int shift = std::max(12, bits - 6);
  const int nb = int((n + (uint64_t(1) << shift) - 1) >> shift);
  BufPtr cursor = DevBuffer::alloc(size_t(nb) * 4 + 16, s);
  BufPtr rows = DevBuffer::alloc(size_t(n) * 4 + 16, s);
  BufPtr pv = DevBuffer::alloc(size_t(n) * sizeof(V) + 16, s);
  AM_CUDA(cudaMemsetAsync(cursor->ptr, 0, size_t(nb) * 4, s));
  uint32_t* err = stream_scratch(s, 0).err;
  KernelTimer kt("rank_scatter", s);
  const uint32_t blocks = uint32_t((n + SC_CHUNK - 1) / SC_CHUNK);
  if (nb > SC_MAX_BUCKETS) throw Error("rank scatter: more buckets than the kernel ranks");
  bucket_pairs_kernel<V><<<blocks, SC_THREADS, 0, s>>>(perm, vals, n, shift, nb,
                                                                    static_cast<uint32_t*>(cursor->ptr),
                                                                    static_cast<uint32_t*>(rows->ptr),
                                                                    static_cast<V*>(pv->ptr), err);
  AM_CUDA(cudaGetLastError());
  drain_pairs_kernel<V><<<grid_for(n), 256, 0, s>>>(static_cast<const uint32_t*>(rows->ptr),
                                                    static_cast<const V*>(pv->ptr), n, out, err);
  AM_CUDA(cudaGetLastError());
}

am_array* new_filled(int pt, const char* format, int64_t n, cudaStream_t s) {
  am_array* o = new_array(pt, format, n);
  o->values = DevBuffer::alloc(size_t(std::max<int64_t>(n, 1)) * std::max(pt_bytes(pt), 1) + 16, s);
  o->null_count = 0;
  o->last_stream = s;
  return o;
}

}  // namespace

am_array* rank_of(am_array* a, int fn, bool desc, bool nulls_first, bool merge_nan, cudaStream_t s, int float_order) {
  const int64_t n = a->length;
  if (a->dictionary && n > 0) {
    // A dictionary column ranks as its sort key, which orders and ties exactly as its values.
    use_on(a, s);
    am_array* key = dictionary_key_column(SortKey{a, desc, nulls_first, float_order}, s);
    am_array* r = nullptr;
    try {
      r = rank_of(key, fn, desc, nulls_first, merge_nan, s, FO_IEEE);
    } catch (...) {
      release(key);
      throw;
    }
    release(key);
    return r;
  }
  const bool f32 = fn == RANK_NORMAL32;
  const bool f64 = fn == RANK_QUANTILE || fn == RANK_NORMAL64 || fn == RANK_PERCENT || fn == RANK_CUME;
  am_array* out = f32 ? new_filled(PT_F32, "f", n, s) : f64 ? new_filled(PT_F64, "g", n, s) : new_filled(PT_U32, "I", n, s);
  if (n == 0) return out;
  try {
    use_on(a, s);
    BufPtr perm = sorted_order(a, desc, nulls_first, float_order, s);
    const uint32_t* p = static_cast<const uint32_t*>(perm->ptr);
    if (fn == RANK_FIRST) {
      scatter_to_rows<uint32_t>(p, nullptr, uint64_t(n), static_cast<uint32_t*>(out->values->ptr), s);
      return out;
    }
    const Runs r = mark_runs(a, p, uint64_t(n), merge_nan, float_order, s);
    // Run numbers by position; the uint32 answers are computed in place, the float ones beside them.
    BufPtr run_of_pos = DevBuffer::alloc(size_t(n) * 4 + 16, s);
    uint32_t* rp = static_cast<uint32_t*>(run_of_pos->ptr);
    BufPtr starts = fn == RANK_DENSE ? nullptr : DevBuffer::alloc(size_t(n) * 4 + 16, s);
    run_ids(r, p, uint64_t(n), rp, starts ? static_cast<uint32_t*>(starts->ptr) : nullptr, nullptr, s);
    BufPtr val_pos = (f32 || f64) ? DevBuffer::alloc(size_t(n) * (f64 ? 8 : 4) + 16, s) : nullptr;
    if (fn != RANK_DENSE) {
      static const int finish[] = {FIN_MIN, FIN_MAX, -1, -1, FIN_QUANTILE, FIN_NORMAL64, FIN_NORMAL32, FIN_PERCENT, FIN_CUME};
      KernelTimer kt("rank_finish", s);
      rank_finish_kernel<<<grid_for(uint64_t(n)), 256, 0, s>>>(rp, static_cast<const uint32_t*>(starts->ptr),
                                                               r.total(), uint64_t(n), finish[fn],
                                                               val_pos ? val_pos->ptr : static_cast<void*>(rp));
      AM_CUDA(cudaGetLastError());
    }
    if (f64) scatter_to_rows<double>(p, static_cast<const double*>(val_pos->ptr), uint64_t(n),
                                     static_cast<double*>(out->values->ptr), s);
    else if (f32) scatter_to_rows<float>(p, static_cast<const float*>(val_pos->ptr), uint64_t(n),
                                         static_cast<float*>(out->values->ptr), s);
    else scatter_to_rows<uint32_t>(p, rp, uint64_t(n), static_cast<uint32_t*>(out->values->ptr), s);
    // The scratch buffers are freed in stream order after the kernels that read them.
  } catch (...) {
    release(out);
    throw;
  }
  return out;
}

am_array* unique_of(am_array* a, bool first_appearance, am_array** counts_out, cudaStream_t s) {
  if (a->dictionary) throw unsupported("unique / value_counts of a dictionary column (its dictionary holds the distinct values)");
  const int64_t n = a->length;
  const int64_t nulls = resolve_null_count(a);
  // The nulls sort last and are one run; a fixed-width column keeps it in first-appearance order, as
  // Arrow does, and a string column drops it in both orders (the reference's string dictionary has no
  // slot for it, Kernels/UniqueOrder.swift:165-200).
  const bool keep_null = first_appearance && !pt_var(a->pt);
  const uint64_t m = uint64_t(keep_null ? n : n - nulls);
  am_array* values = nullptr;
  am_array* counts = nullptr;
  auto empty = [&]() {
    values = new_array(a->pt, a->format, 0);
    values->null_count = 0;
    if (pt_var(a->pt)) {
      values->values = DevBuffer::alloc(16, s);
      AM_CUDA(cudaMemsetAsync(values->values->ptr, 0, 16, s));
      values->bytes = DevBuffer::alloc(16, s);
    } else {
      values->values = DevBuffer::alloc(16, s);
    }
    values->last_stream = s;
    if (counts_out) *counts_out = new_filled(PT_I64, "l", 0, s);
    return values;
  };
  if (m == 0) return empty();
  use_on(a, s);
  BufPtr perm = sorted_order(a, false, false, FO_IEEE, s);
  const uint32_t* p = static_cast<const uint32_t*>(perm->ptr);
  const Runs r = mark_runs(a, p, m, false, FO_IEEE, s);
  BufPtr starts = DevBuffer::alloc(size_t(m) * 4 + 16, s);
  BufPtr heads = DevBuffer::alloc(size_t(m) * 4 + 16, s);
  run_ids(r, p, m, nullptr, static_cast<uint32_t*>(starts->ptr), static_cast<uint32_t*>(heads->ptr), s);
  uint32_t runs = 0;
  AM_CUDA(cudaMemcpyAsync(&runs, r.total(), 4, cudaMemcpyDeviceToHost, s));
  AM_CUDA(cudaStreamSynchronize(s));
  if (runs == 0) return empty();

  BufPtr run_counts;
  if (counts_out) {
    run_counts = DevBuffer::alloc(size_t(runs) * 8 + 16, s);
    KernelTimer kt("run_lengths", s);
    run_lengths_kernel<<<grid_for(runs), 256, 0, s>>>(static_cast<const uint32_t*>(starts->ptr), r.total(), m,
                                                      static_cast<int64_t*>(run_counts->ptr));
    AM_CUDA(cudaGetLastError());
  }
  // The representatives' rows: ascending order as they are; first-appearance order by a sort of the
  // runs' earliest rows (distinct, so the order is total).
  am_array* rows = new_filled(PT_U32, "I", int64_t(runs), s);
  rows->perm_of = n;
  try {
    if (!first_appearance) {
      AM_CUDA(cudaMemcpyAsync(rows->values->ptr, heads->ptr, size_t(runs) * 4, cudaMemcpyDeviceToDevice, s));
      if (counts_out) {
        counts = new_filled(PT_I64, "l", int64_t(runs), s);
        AM_CUDA(cudaMemcpyAsync(counts->values->ptr, run_counts->ptr, size_t(runs) * 8, cudaMemcpyDeviceToDevice, s));
      }
    } else {
      am_array* head_col = new_array(PT_U32, "I", int64_t(runs));
      head_col->values = heads;
      head_col->null_count = 0;
      head_col->last_stream = s;
      BufPtr order = DevBuffer::alloc(size_t(runs) * 4 + 16, s);
      try {
        radix_argsort({SortKey{head_col, false, false, 0}}, int64_t(runs), order->ptr, 4, s, nullptr);
      } catch (...) {
        release(head_col);
        throw;
      }
      release(head_col);
      if (counts_out) counts = new_filled(PT_I64, "l", int64_t(runs), s);
      KernelTimer kt("runs_in_order", s);
      runs_in_order_kernel<<<grid_for(runs), 256, 0, s>>>(
          static_cast<const uint32_t*>(order->ptr), static_cast<const uint32_t*>(heads->ptr),
          counts_out ? static_cast<const int64_t*>(run_counts->ptr) : nullptr, runs,
          static_cast<uint32_t*>(rows->values->ptr), counts ? static_cast<int64_t*>(counts->values->ptr) : nullptr);
      AM_CUDA(cudaGetLastError());
    }
    values = new_array(a->pt, a->format, int64_t(runs));
    take_columns(&a, 1, rows, &values, false, s);
  } catch (...) {
    release(rows);
    if (values) release(values);
    if (counts) release(counts);
    throw;
  }
  release(rows);
  if (counts_out) *counts_out = counts;
  return values;
}

namespace {

// One derived key of argsort_any: a column as it is (chunk == -2), or a string column's chunk `chunk`
// or (chunk == -1) its length.
struct Piece {
  SortKey key;
  int chunk;
};

__global__ void __launch_bounds__(256) compose_kernel(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ order,
                                                      uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    out[i] = perm[order[i]];
}

__global__ void __launch_bounds__(256) widen_kernel(const uint32_t* __restrict__ in, uint64_t n, uint64_t* __restrict__ out) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    out[i] = in[i];
}

// The columns of pieces [lo, hi), in row order: consecutive chunks of one string column are derived
// in one pass over its bytes.
std::vector<am_array*> materialize(const std::vector<Piece>& p, size_t lo, size_t hi, cudaStream_t s) {
  std::vector<am_array*> cols;
  try {
    for (size_t i = lo; i < hi;) {
      if (p[i].chunk == -2) {
        retain(p[i].key.col);
        cols.push_back(p[i].key.col);
        i++;
        continue;
      }
      if (p[i].chunk == -1) {
        // A length piece on its own (its chunks sit in the group before).
        std::vector<am_array*> c = string_key_columns(p[i].key.col, 0, 0, true, s);
        cols.insert(cols.end(), c.begin(), c.end());
        i++;
        continue;
      }
      size_t j = i;
      while (j + 1 < hi && p[j + 1].key.col == p[i].key.col && p[j + 1].chunk == p[j].chunk + 1) j++;
      const bool with_length = j + 1 < hi && p[j + 1].key.col == p[i].key.col && p[j + 1].chunk == -1;
      std::vector<am_array*> c = string_key_columns(p[i].key.col, p[i].chunk, int(j - i + 1), with_length, s);
      cols.insert(cols.end(), c.begin(), c.end());
      i = j + 1 + (with_length ? 1 : 0);
    }
  } catch (...) {
    for (am_array* c : cols) release(c);
    throw;
  }
  return cols;
}

}  // namespace

void argsort_any(const std::vector<SortKey>& keys, int64_t n, void* out, int width, cudaStream_t s,
                 am_sort_stats* stats) {
  if (n <= 0) return;
  std::vector<am_array*> owned;
  std::vector<Piece> pieces;
  auto release_all = [&](std::vector<am_array*>& v) {
    for (am_array* c : v) release(c);
    v.clear();
  };
  try {
    for (const SortKey& k : keys) {
      if (k.col->dictionary) {
        am_array* c = dictionary_key_column(k, s);
        owned.push_back(c);
        pieces.push_back(Piece{SortKey{c, k.descending, k.nulls_first, FO_IEEE}, -2});
      } else if (pt_var(k.col->pt)) {
        const int m = string_chunk_count(k.col, s);
        for (int j = 0; j < m; j++) pieces.push_back(Piece{SortKey{k.col, k.descending, k.nulls_first, 0}, j});
        pieces.push_back(Piece{SortKey{k.col, k.descending, k.nulls_first, 0}, -1});
      } else {
        pieces.push_back(Piece{k, -2});
      }
    }
    auto sort_keys_of = [&](const std::vector<am_array*>& cols, size_t lo) {
      std::vector<SortKey> ks;
      for (size_t c = 0; c < cols.size(); c++) {
        const SortKey& pk = pieces[lo + c].key;
        ks.push_back(SortKey{cols[c], pk.descending, pk.nulls_first, pieces[lo + c].chunk == -2 ? pk.float_order : 0});
      }
      return ks;
    };
    const size_t P = pieces.size(), G = size_t(MAX_KEYS);
    if (P <= G) {
      std::vector<am_array*> cols = materialize(pieces, 0, P, s);
      try {
        radix_sort(sort_keys_of(cols, 0), n, out, width, nullptr, s, stats);
      } catch (...) {
        release_all(cols);
        throw;
      }
      release_all(cols);
      release_all(owned);
      return;
    }
    // Groups of MAX_KEYS derived keys, least significant first: each sorted stably in the order the
    // groups after it left, so the composed order sorts by every key.
    am_array* perm = nullptr;      // the order so far (uint32 row numbers), NULL: the identity
    try {
      for (size_t hi = P; hi > 0;) {
        const size_t lo = hi > G ? hi - G : 0;
        std::vector<am_array*> cols = materialize(pieces, lo, hi, s);
        std::vector<am_array*> moved;
        BufPtr order = DevBuffer::alloc(size_t(n) * 4 + 16, s);
        try {
          if (perm) {
            // This group's keys in the current order.
            moved.assign(cols.size(), nullptr);
            for (size_t c = 0; c < cols.size(); c++) moved[c] = new_array(cols[c]->pt, cols[c]->format, n);
            take_columns(cols.data(), int(cols.size()), perm, moved.data(), false, s);
          }
          radix_sort(sort_keys_of(perm ? moved : cols, lo), n, order->ptr, 4, nullptr, s, stats);
        } catch (...) {
          release_all(cols);
          release_all(moved);
          throw;
        }
        release_all(cols);
        release_all(moved);
        am_array* next = new_array(PT_U32, "I", n);
        next->null_count = 0;
        next->perm_of = n;
        next->last_stream = s;
        if (perm) {
          next->values = DevBuffer::alloc(size_t(n) * 4 + 16, s);
          compose_kernel<<<grid_for(uint64_t(n)), 256, 0, s>>>(static_cast<const uint32_t*>(perm->values->ptr),
                                                               static_cast<const uint32_t*>(order->ptr), uint64_t(n),
                                                               static_cast<uint32_t*>(next->values->ptr));
          AM_CUDA(cudaGetLastError());
          release(perm);
        } else {
          next->values = order;
        }
        perm = next;
        hi = lo;
      }
      if (width == 8) {
        widen_kernel<<<grid_for(uint64_t(n)), 256, 0, s>>>(static_cast<const uint32_t*>(perm->values->ptr), uint64_t(n),
                                                          static_cast<uint64_t*>(out));
        AM_CUDA(cudaGetLastError());
      } else {
        AM_CUDA(cudaMemcpyAsync(out, perm->values->ptr, size_t(n) * 4, cudaMemcpyDeviceToDevice, s));
      }
    } catch (...) {
      if (perm) release(perm);
      throw;
    }
    release(perm);
  } catch (...) {
    release_all(owned);
    throw;
  }
  release_all(owned);
}

am_array* dictionary_key_column(const SortKey& k, cudaStream_t s) {
  am_array* a = k.col;
  am_array* dict = a->dictionary;
  const int64_t n = a->length, d = dict->length;
  if (dict->dictionary) throw unsupported("a dictionary whose values are themselves dictionary-encoded");
  use_on(dict, s);
  // Dense ranks of the dictionary's values (ascending, in the key's float order): equal values share one.
  am_array* dense = d > 0 ? rank_of(dict, RANK_DENSE, false, false, false, s, k.float_order) : nullptr;
  // A float32 key holds every rank exactly below 2^24 distinct values; a float64 one beyond.
  const bool wide = d > (int64_t(1) << 24);
  am_array* key = new_array(wide ? PT_F64 : PT_F32, wide ? "g" : "f", n);
  try {
    const uint64_t words = uint64_t(n + 31) / 32;
    key->values = DevBuffer::alloc(size_t(std::max<int64_t>(n, 1)) * (wide ? 8 : 4) + 16, s);
    key->validity = DevBuffer::alloc(size_t(words) * 4 + 16, s);
    key->null_count_dev = DevBuffer::alloc(16, s);
    key->null_count = -1;
    key->last_stream = s;
    AM_CUDA(cudaMemsetAsync(key->null_count_dev->ptr, 0, sizeof(unsigned long long), s));
    const bool fl = pt_float(dict->pt);
    const DictView dv{pt_var(dict->pt) ? nullptr : dict->data(), dict->null_count != 0 ? dict->valid_bits() : nullptr,
                      dict->validity_offset, dict->pt, (fl && k.float_order == FO_IEEE) ? 1 : 0};
    const uint32_t* dn = dense ? static_cast<const uint32_t*>(dense->values->ptr) : nullptr;
    const int grid = int(std::max<uint64_t>(1, std::min<uint64_t>(words / 8 + 1, uint64_t(device().sm_count) * 8)));
    uint32_t* err = stream_scratch(s, 0).err;
    auto* nc = static_cast<unsigned long long*>(key->null_count_dev->ptr);
    const uint8_t* cv = a->null_count != 0 ? a->valid_bits() : nullptr;
    KernelTimer kt("dictionary_keys", s);
    if (wide)
      dict_row_keys_kernel<double><<<grid, 256, 0, s>>>(a->data(), a->pt, cv, a->validity_offset, uint64_t(n), dv, dn,
                                                        uint64_t(d), static_cast<double*>(key->values->ptr),
                                                        static_cast<uint32_t*>(key->validity->ptr), nc, err);
    else
      dict_row_keys_kernel<float><<<grid, 256, 0, s>>>(a->data(), a->pt, cv, a->validity_offset, uint64_t(n), dv, dn,
                                                       uint64_t(d), static_cast<float*>(key->values->ptr),
                                                       static_cast<uint32_t*>(key->validity->ptr), nc, err);
    AM_CUDA(cudaGetLastError());
    // A code outside the dictionary is an invalid array: report it here, not in a later call.
    check_device_errors(s);
  } catch (...) {
    release(key);
    if (dense) release(dense);
    throw;
  }
  if (dense) release(dense);
  return key;
}

}  // namespace am
