// Top-k by radix selection: the first k indices of the stable argsort without sorting every row.
//
// am_top_k_ex answers with the first k indices am_argsort_ex2 gives with the same options
// (include/arrowmetal.h:1345-1350; the reference selects on the same key maps in TopK.swift and
// RadixSelect.swift). In the argsort's arrangement the value rows come in key order and the NaN-block
// and null rows in row order ([values][NaN][nulls] with nulls at the end, [nulls][NaN][values] at the
// start), so the answer is some category rows in row order plus the kv smallest value keys, ties in
// row order. On the order-preserving unsigned keys of the sort, reading the column twice:
//   1. the key statistics give the category counts and every digit's histogram; on the host, the
//      digits that are constant over the value keys and the first one that is not (digit dv, whose
//      histogram is then exact for the rows that share the constant ones) fix the threshold's leading
//      digits and the rank k_rem of the wanted key within its bucket;
//   2. one ordered compaction of the column extracts every value row whose leading digits (down to dv)
//      are at most the threshold's -- all rows below the bucket and the bucket itself -- as
//      (key, row) pairs in row order;
//   3. on that buffer, a histogram per lower digit over the pairs that share the digits chosen so far
//      narrows the threshold key T to its last digit;
//   4. an ordered compaction of the buffer takes every pair with key < T and the first `need` pairs
//      with key == T: exactly kv candidates, in row order;
//   5. the candidates are argsorted by the radix sort (stable, so equal keys stay in row order) and
//      their rows written out, beside the category rows, compacted in row order the same way.
// The output is bit-identical to the prefix of the full argsort.
#include <algorithm>
#include <vector>

#include "am_internal.h"
#include "key_encode.cuh"
#include "radix_sort.cuh"

namespace am {
namespace rs {
namespace {

constexpr int SEL_THREADS = 256, SEL_ITEMS = 8;
constexpr uint64_t SEL_CHUNK = uint64_t(SEL_THREADS) * SEL_ITEMS;   // rows per block in a compaction

struct SelState {
  unsigned long long prefix;    // the threshold key's digits chosen so far
  unsigned long long k_rem;     // rank of the wanted key among the keys that share them (1-based)
};

// Where a selection step reads: the key column itself (each key encoded on the fly), or a buffer of
// encoded value keys with their row numbers.
template <typename KeyT>
struct Source {
  ColView col;
  const KeyT* keys;       // NULL: the column
  const uint32_t* rows;
  uint64_t n;
};

// Positions pos[i] of the source: keys, categories (0 value, 1 NaN block, 2 null) and row numbers.
template <typename KeyT>
__device__ __forceinline__ void load_source(const Source<KeyT>& s, const uint32_t (&pos)[SEL_ITEMS], uint32_t ok,
                                            KeyT (&key)[SEL_ITEMS], int (&cat)[SEL_ITEMS],
                                            uint32_t (&row)[SEL_ITEMS]) {
  if (s.keys) {
#pragma unroll
    for (int i = 0; i < SEL_ITEMS; i++) {
      const bool live = (ok >> i) & 1u;
      key[i] = live ? s.keys[pos[i]] : KeyT(0);
      row[i] = live ? s.rows[pos[i]] : 0u;
      cat[i] = 0;
    }
  } else {
    encode_rows<KeyT, SEL_ITEMS>(s.col, pos, ok, key, cat);
#pragma unroll
    for (int i = 0; i < SEL_ITEMS; i++) row[i] = pos[i];
  }
}

// Digit `shift` of the value keys whose digits above it equal the state's prefix.
template <typename KeyT>
__global__ void __launch_bounds__(SEL_THREADS) select_histogram_kernel(const __grid_constant__ Source<KeyT> src,
                                                                       int shift, const SelState* __restrict__ st,
                                                                       uint32_t* __restrict__ hist) {
  __shared__ uint32_t sh[256];
  for (int i = threadIdx.x; i < 256; i += SEL_THREADS) sh[i] = 0;
  __syncthreads();
  const KeyT want = KeyT(st->prefix >> (shift + 8));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint64_t base = uint64_t(blockIdx.x) * SEL_CHUNK; base < src.n; base += uint64_t(gridDim.x) * SEL_CHUNK) {
    uint32_t pos[SEL_ITEMS];
    uint32_t ok = 0;
#pragma unroll
    for (int i = 0; i < SEL_ITEMS; i++) {
      const uint64_t g = base + uint64_t(warp) * (SEL_ITEMS * 32) + uint64_t(i) * 32 + lane;
      pos[i] = uint32_t(g);
      if (g < src.n) ok |= 1u << i;
    }
    KeyT key[SEL_ITEMS];
    int cat[SEL_ITEMS];
    uint32_t row[SEL_ITEMS];
    load_source<KeyT>(src, pos, ok, key, cat, row);
#pragma unroll
    for (int i = 0; i < SEL_ITEMS; i++) {
      if (!((ok >> i) & 1u) || cat[i] != 0) continue;
      if (KeyT(key[i] >> (shift + 8)) == want) atomicAdd(&sh[uint32_t(key[i] >> shift) & 255u], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += SEL_THREADS)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// One block: the digit at which the k_rem-th key sits; it joins the prefix and k_rem becomes the rank
// among the keys with that digit.
__global__ void __launch_bounds__(256) select_step_kernel(const uint32_t* __restrict__ hist, int shift,
                                                          SelState* __restrict__ st) {
  __shared__ uint32_t wsum[8];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const unsigned long long k = st->k_rem;     // read by every thread before the one writer below
  const uint32_t v = hist[t];
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  uint32_t add = 0;
  for (int w = 0; w < warp; w++) add += wsum[w];
  const uint32_t incl = x + add, before = incl - v;
  if (v > 0 && before < k && k <= incl) {
    st->prefix |= (unsigned long long)t << shift;
    st->k_rem = k - before;
  }
}

// Block-wide exclusive scan of one value per thread (SEL_THREADS threads); *total gets the sum.
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  __syncthreads();
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  uint32_t add = 0, all = 0;
#pragma unroll
  for (int w = 0; w < SEL_THREADS / 32; w++) {
    const uint32_t c = s_warp[w];
    if (w < warp) add += c;
    all += c;
  }
  if (total) *total = all;
  return x - v + add;
}

// The entries a compaction takes, in source order: every entry of class A, and class-B entries up to
// `limit`.
//   PRED_PREFIX: A = value keys with (key >> shift) < p, B = those with (key >> shift) == p, no limit;
//   PRED_THRESHOLD: A = keys < T, B = keys == T, limit k_rem (T, k_rem: the selection state);
//   PRED_CATEGORY: B = rows of category `cat` (1 NaN block, 2 null), up to `limit`;
//   PRED_PARTITION: against the pivot (category place `cat` in the sorted arrangement, key T when that
//     is the value block): A = rows before it, B = rows equal to it; every row is written.
constexpr int PRED_PREFIX = 0, PRED_THRESHOLD = 1, PRED_CATEGORY = 2, PRED_PARTITION = 3;
struct Compact {
  int mode;
  int cat;
  int shift;
  unsigned long long p;
  unsigned long long limit;
  const SelState* st;
  int nulls_first;            // PRED_PARTITION: the arrangement is [nulls][NaN][values]
};

template <typename KeyT>
__device__ __forceinline__ void classify(const Source<KeyT>& src, const Compact& c, uint64_t base,
                                         uint32_t (&a)[SEL_ITEMS], uint32_t (&b)[SEL_ITEMS], KeyT (&key)[SEL_ITEMS],
                                         uint32_t (&row)[SEL_ITEMS]) {
  uint32_t pos[SEL_ITEMS];
  uint32_t ok = 0;
#pragma unroll
  for (int i = 0; i < SEL_ITEMS; i++) {
    const uint64_t g = base + uint64_t(threadIdx.x) * SEL_ITEMS + i;   // consecutive entries per thread
    pos[i] = uint32_t(g);
    if (g < src.n) ok |= 1u << i;
  }
  int cat[SEL_ITEMS];
  load_source<KeyT>(src, pos, ok, key, cat, row);
  const KeyT T = KeyT((c.mode == PRED_THRESHOLD || c.mode == PRED_PARTITION) ? c.st->prefix : 0);
#pragma unroll
  for (int i = 0; i < SEL_ITEMS; i++) {
    const bool live = (ok >> i) & 1u;
    if (c.mode == PRED_PREFIX) {
      const KeyT hi = KeyT(key[i] >> c.shift);
      a[i] = live && cat[i] == 0 && hi < KeyT(c.p);
      b[i] = live && cat[i] == 0 && hi == KeyT(c.p);
    } else if (c.mode == PRED_THRESHOLD) {
      a[i] = live && cat[i] == 0 && key[i] < T;
      b[i] = live && cat[i] == 0 && key[i] == T;
    } else if (c.mode == PRED_PARTITION) {
      const int place = c.nulls_first ? 2 - cat[i] : cat[i];   // the category's block in the arrangement
      const bool same = place == c.cat;
      a[i] = live && (place < c.cat || (same && cat[i] == 0 && key[i] < T));
      b[i] = live && same && (cat[i] != 0 || key[i] == T);
    } else {
      a[i] = 0;
      b[i] = live && cat[i] == c.cat;
    }
  }
}

template <typename KeyT>
__global__ void __launch_bounds__(SEL_THREADS) compact_count_kernel(const __grid_constant__ Source<KeyT> src,
                                                                    const __grid_constant__ Compact c,
                                                                    uint32_t* __restrict__ count_a,
                                                                    uint32_t* __restrict__ count_b) {
  __shared__ uint32_t s_warp[SEL_THREADS / 32];
  uint32_t a[SEL_ITEMS], b[SEL_ITEMS], row[SEL_ITEMS];
  KeyT key[SEL_ITEMS];
  classify<KeyT>(src, c, uint64_t(blockIdx.x) * SEL_CHUNK, a, b, key, row);
  uint32_t ca = 0, cb = 0;
#pragma unroll
  for (int i = 0; i < SEL_ITEMS; i++) {
    ca += a[i];
    cb += b[i];
  }
  uint32_t ta = 0, tb = 0;
  block_scan(ca, s_warp, &ta);
  block_scan(cb, s_warp, &tb);
  if (threadIdx.x == 0) {
    count_a[blockIdx.x] = ta;
    count_b[blockIdx.x] = tb;
  }
}

// One block: exclusive scans of the per-block counts, in place; the totals land at [blocks].
__global__ void __launch_bounds__(1024) compact_scan_kernel(uint32_t* __restrict__ count_a, uint32_t* __restrict__ count_b,
                                                            uint32_t blocks) {
  __shared__ unsigned long long s[2][32];
  __shared__ unsigned long long carry[2];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) carry[0] = carry[1] = 0;
  __syncthreads();
  for (uint32_t base = 0; base < blocks; base += 1024) {
    const uint32_t i = base + uint32_t(t);
    unsigned long long v[2] = {i < blocks ? count_a[i] : 0u, i < blocks ? count_b[i] : 0u};
    unsigned long long x[2] = {v[0], v[1]};
#pragma unroll
    for (int q = 0; q < 2; q++) {
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x[q], o);
        if (lane >= o) x[q] += y;
      }
      if (lane == 31) s[q][warp] = x[q];
    }
    __syncthreads();
    unsigned long long add[2] = {carry[0], carry[1]}, all[2] = {0, 0};
    for (int w = 0; w < 32; w++) {
#pragma unroll
      for (int q = 0; q < 2; q++) {
        if (w < warp) add[q] += s[q][w];
        all[q] += s[q][w];
      }
    }
    if (i < blocks) {
      count_a[i] = uint32_t(x[0] - v[0] + add[0]);
      count_b[i] = uint32_t(x[1] - v[1] + add[1]);
    }
    __syncthreads();
    if (t == 0) {
      carry[0] += all[0];
      carry[1] += all[1];
    }
    __syncthreads();
  }
  if (t == 0) {
    count_a[blocks] = uint32_t(carry[0]);
    count_b[blocks] = uint32_t(carry[1]);
  }
}

// The ordered writes: row numbers (and keys, when asked) of the taken entries at their places.
template <typename KeyT>
__global__ void __launch_bounds__(SEL_THREADS) compact_write_kernel(const __grid_constant__ Source<KeyT> src,
                                                                    const __grid_constant__ Compact c,
                                                                    const uint32_t* __restrict__ off_a,
                                                                    const uint32_t* __restrict__ off_b,
                                                                    KeyT* __restrict__ out_keys,
                                                                    uint32_t* __restrict__ out_rows, uint64_t out_cap,
                                                                    uint32_t* __restrict__ err) {
  __shared__ uint32_t s_warp[SEL_THREADS / 32];
  uint32_t a[SEL_ITEMS], b[SEL_ITEMS], row[SEL_ITEMS];
  KeyT key[SEL_ITEMS];
  classify<KeyT>(src, c, uint64_t(blockIdx.x) * SEL_CHUNK, a, b, key, row);
  const unsigned long long limit = c.mode == PRED_THRESHOLD ? c.st->k_rem : c.limit;
  uint32_t cb = 0;
#pragma unroll
  for (int i = 0; i < SEL_ITEMS; i++) cb += b[i];
  const uint32_t eb = block_scan(cb, s_warp, nullptr);    // B entries before this thread's, in the block
  const unsigned long long b_before = off_b[blockIdx.x];
  uint32_t take[SEL_ITEMS];
  uint32_t cp = 0, rb = 0;
#pragma unroll
  for (int i = 0; i < SEL_ITEMS; i++) {
    take[i] = a[i] || (b[i] && (b_before + eb + rb) < limit);
    rb += b[i];
    cp += take[i];
  }
  const uint32_t ep = block_scan(cp, s_warp, nullptr);
  const unsigned long long dst0 = off_a[blockIdx.x] + (b_before < limit ? b_before : limit) + ep;
  uint32_t r = 0;
#pragma unroll
  for (int i = 0; i < SEL_ITEMS; i++) {
    if (!take[i]) continue;
    const unsigned long long d = dst0 + r++;
    if (d >= out_cap) {
      atomicOr(err, ERR_BOUNDS);
      continue;
    }
    out_rows[d] = row[i];
    if (out_keys) out_keys[d] = key[i];
  }
}

// out[i] = rows[order[i]] for i < m.
__global__ void __launch_bounds__(256) gather_rows_kernel(const uint32_t* __restrict__ order, const uint32_t* __restrict__ rows,
                                                          uint64_t m, uint32_t* __restrict__ out) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x)
    out[i] = rows[order[i]];
}

// Every row at its place: class A rows (in row order) first, then class B rows, then the rest.
template <typename KeyT>
__global__ void __launch_bounds__(SEL_THREADS) partition_write_kernel(const __grid_constant__ Source<KeyT> src,
                                                                      const __grid_constant__ Compact c,
                                                                      const uint32_t* __restrict__ off_a,
                                                                      const uint32_t* __restrict__ off_b,
                                                                      uint32_t blocks, uint32_t* __restrict__ out,
                                                                      uint32_t* __restrict__ err) {
  __shared__ uint32_t s_warp[SEL_THREADS / 32];
  uint32_t a[SEL_ITEMS], b[SEL_ITEMS], row[SEL_ITEMS];
  KeyT key[SEL_ITEMS];
  const uint64_t base = uint64_t(blockIdx.x) * SEL_CHUNK;
  classify<KeyT>(src, c, base, a, b, key, row);
  uint32_t ca = 0, cb = 0;
#pragma unroll
  for (int i = 0; i < SEL_ITEMS; i++) {
    ca += a[i];
    cb += b[i];
  }
  const uint32_t ea = block_scan(ca, s_warp, nullptr);
  const uint32_t eb = block_scan(cb, s_warp, nullptr);
  const uint64_t total_a = off_a[blocks], total_b = off_b[blocks];
  uint64_t a_before = uint64_t(off_a[blockIdx.x]) + ea, b_before = uint64_t(off_b[blockIdx.x]) + eb;
#pragma unroll
  for (int i = 0; i < SEL_ITEMS; i++) {
    const uint64_t g = base + uint64_t(threadIdx.x) * SEL_ITEMS + i;
    if (g >= src.n) break;
    uint64_t d;
    if (a[i]) d = a_before;
    else if (b[i]) d = total_a + b_before;
    else d = total_a + total_b + (g - a_before - b_before);
    a_before += a[i];
    b_before += b[i];
    if (d >= src.n) {
      atomicOr(err, ERR_BOUNDS);
      continue;
    }
    out[d] = row[i];
  }
}

// Per-block counts of a compaction's two classes: blocks + 1 words each (the totals at [blocks]).
inline size_t compact_count_words(uint64_t n) { return 2 * (size_t((n + SEL_CHUNK - 1) / SEL_CHUNK) + 1); }

template <typename KeyT>
void compact(const Source<KeyT>& src, const Compact& c, KeyT* out_keys, uint32_t* out_rows, uint64_t cap,
             uint32_t* counts, uint32_t* err, cudaStream_t s) {
  const uint32_t blocks = uint32_t((src.n + SEL_CHUNK - 1) / SEL_CHUNK);
  if (blocks == 0) return;
  uint32_t* count_a = counts;
  uint32_t* count_b = counts + blocks + 1;
  KernelTimer kt("topk_compact", s);
  compact_count_kernel<KeyT><<<blocks, SEL_THREADS, 0, s>>>(src, c, count_a, count_b);
  AM_CUDA(cudaGetLastError());
  compact_scan_kernel<<<1, 1024, 0, s>>>(count_a, count_b, blocks);
  AM_CUDA(cudaGetLastError());
  compact_write_kernel<KeyT><<<blocks, SEL_THREADS, 0, s>>>(src, c, count_a, count_b, out_keys, out_rows, cap, err);
  AM_CUDA(cudaGetLastError());
}

// The leading digits of the k-th smallest value key (1-based), read off the key statistics' digit
// histograms: the digits that are constant over the value keys, then the first digit that is not
// (dv; -1 when every value key is the same), whose histogram is exact for the rows that share the
// constant ones. k_rem is the wanted key's rank among the keys with those digits; below and bucket
// count the keys under the chosen digit dv and on it.
struct Leading {
  unsigned long long prefix = 0, k_rem = 0;
  int dv = -1;
  uint64_t below = 0, bucket = 0;
};
Leading leading_digits(const KeyStats& st, int D, uint64_t k) {
  Leading r;
  r.k_rem = k;
  for (int d = D - 1; d >= 0; d--) {
    const uint32_t* h = st.hist[d];
    int only = -1, nonzero = 0;
    for (int b = 0; b < 256; b++)
      if (h[b]) { nonzero++; only = b; }
    if (nonzero == 1) {
      r.prefix |= (unsigned long long)only << (8 * d);
      continue;
    }
    uint64_t run = 0;
    for (int b = 0; b < 256; b++) {
      if (h[b] && run < r.k_rem && r.k_rem <= run + h[b]) {
        r.prefix |= (unsigned long long)b << (8 * d);
        r.k_rem -= run;
        r.below = run;
        r.bucket = h[b];
        break;
      }
      run += h[b];
    }
    r.dv = d;
    break;
  }
  return r;
}

template <typename KeyT>
am_array* top_k_of(const SortKey& key, int64_t k, cudaStream_t s) {
  const uint64_t n = uint64_t(key.col->length);
  constexpr int D = int(sizeof(KeyT));
  const Source<KeyT> column{make_view(key), nullptr, nullptr, n};
  const uint32_t blocks = uint32_t((n + SEL_CHUNK - 1) / SEL_CHUNK);

  // Scratch: statistics, selection state, per-digit histograms, compaction counts.
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t off_state = up(sizeof(KeyStats));
  const size_t off_hist = up(off_state + sizeof(SelState));
  const size_t off_counts = up(off_hist + sizeof(uint32_t) * 256 * D);
  const size_t bytes = up(off_counts + sizeof(uint32_t) * compact_count_words(n));
  char* base = static_cast<char*>(dmalloc(bytes, s));
  struct Free { char* p; cudaStream_t s; ~Free() { dfree(p, s); } } guard{base, s};
  KeyStats* st = reinterpret_cast<KeyStats*>(base);
  SelState* state = reinterpret_cast<SelState*>(base + off_state);
  uint32_t* hist = reinterpret_cast<uint32_t*>(base + off_hist);
  uint32_t* counts = reinterpret_cast<uint32_t*>(base + off_counts);
  key_statistics(key, st, s);

  // The statistics on the host: the category counts shape the answer, the digit histograms fix the
  // threshold's leading digits.
  static thread_local KeyStats* host = nullptr;
  if (!host) host = static_cast<KeyStats*>(pinned_alloc(sizeof(KeyStats)));
  AM_CUDA(cudaMemcpyAsync(host, st, sizeof(KeyStats), cudaMemcpyDeviceToHost, s));
  AM_CUDA(cudaStreamSynchronize(s));
  const uint64_t n_value = host->n_value, n_null = host->n_null, n_nan = host->n_nan;
  const uint64_t m = std::min<uint64_t>(uint64_t(k), n);
  uint64_t kv, k_nan, k_null;
  if (!key.nulls_first) {
    kv = std::min(m, n_value);
    k_nan = std::min(m - kv, n_nan);
    k_null = m - kv - k_nan;
  } else {
    k_null = std::min(m, n_null);
    k_nan = std::min(m - k_null, n_nan);
    kv = m - k_null - k_nan;
  }
  // Selection pays while the taken value rows are a small share of them.
  if (kv > n_value / 4) return nullptr;

  am_array* out = new_array(PT_U32, "I", int64_t(m));
  try {
    out->values = DevBuffer::alloc(size_t(std::max<uint64_t>(m, 1)) * 4 + 16, s);
    out->null_count = 0;
    out->perm_of = int64_t(n);
    out->last_stream = s;
    uint32_t* res = static_cast<uint32_t*>(out->values->ptr);
    uint32_t* err = stream_scratch(s, 0).err;
    const uint64_t v_at = key.nulls_first ? k_null + k_nan : 0;
    const uint64_t nan_at = key.nulls_first ? k_null : kv;
    const uint64_t null_at = key.nulls_first ? 0 : kv + k_nan;
    if (k_null) compact<KeyT>(column, Compact{PRED_CATEGORY, 2, 0, 0, k_null, nullptr}, nullptr, res + null_at, k_null,
                              counts, err, s);
    if (k_nan) compact<KeyT>(column, Compact{PRED_CATEGORY, 1, 0, 0, k_nan, nullptr}, nullptr, res + nan_at, k_nan,
                             counts, err, s);
    if (kv) {
      // 1. Leading digits on the host: constant ones, then the first that varies (digit dv).
      const Leading lead = leading_digits(*host, D, kv);
      const int dv = lead.dv;
      const unsigned long long prefix = lead.prefix;
      const uint64_t below = lead.below, bucket = lead.bucket;
      const SelState init{prefix, lead.k_rem};
      AM_CUDA(cudaMemcpyAsync(state, &init, sizeof(SelState), cudaMemcpyHostToDevice, s));
      BufPtr cand_keys = DevBuffer::alloc(size_t(kv) * sizeof(KeyT) + 16, s);
      BufPtr cand_rows = DevBuffer::alloc(size_t(kv) * 4 + 16, s);
      BufPtr order = DevBuffer::alloc(size_t(kv) * 4 + 16, s);
      if (dv < 0) {
        // Every value key is the same: the first kv value rows, in row order.
        compact<KeyT>(column, Compact{PRED_THRESHOLD, 0, 0, 0, 0, state}, static_cast<KeyT*>(cand_keys->ptr),
                      static_cast<uint32_t*>(cand_rows->ptr), kv, counts, err, s);
      } else {
        // 2. The rows at or below the threshold's bucket of digit dv, as (key, row) pairs in row order.
        const uint64_t n1 = below + bucket;
        BufPtr keys1 = DevBuffer::alloc(size_t(n1) * sizeof(KeyT) + 16, s);
        BufPtr rows1 = DevBuffer::alloc(size_t(n1) * 4 + 16, s);
        compact<KeyT>(column, Compact{PRED_PREFIX, 0, 8 * dv, prefix >> (8 * dv), ~0ull, nullptr},
                      static_cast<KeyT*>(keys1->ptr), static_cast<uint32_t*>(rows1->ptr), n1, counts, err, s);
        const Source<KeyT> cand{column.col, static_cast<const KeyT*>(keys1->ptr),
                                static_cast<const uint32_t*>(rows1->ptr), n1};
        // 3. The lower digits on the pairs.
        if (dv > 0) {
          AM_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 256 * D, s));
          KernelTimer kt("topk_select", s);
          const int grid = int(std::min<uint64_t>((n1 + SEL_CHUNK - 1) / SEL_CHUNK, uint64_t(device().sm_count) * 8));
          for (int d = dv - 1; d >= 0; d--) {
            uint32_t* hd = hist + 256 * d;
            select_histogram_kernel<KeyT><<<std::max(grid, 1), SEL_THREADS, 0, s>>>(cand, 8 * d, state, hd);
            AM_CUDA(cudaGetLastError());
            select_step_kernel<<<1, 256, 0, s>>>(hd, 8 * d, state);
            AM_CUDA(cudaGetLastError());
          }
        }
        // 4. Keys below the threshold and the first `need` equal to it: the kv candidates.
        const uint32_t blocks1 = uint32_t((n1 + SEL_CHUNK - 1) / SEL_CHUNK);
        if (blocks1 > blocks) throw Error("top_k: candidate buffer larger than its column");
        compact<KeyT>(cand, Compact{PRED_THRESHOLD, 0, 0, 0, 0, state}, static_cast<KeyT*>(cand_keys->ptr),
                      static_cast<uint32_t*>(cand_rows->ptr), kv, counts, err, s);
        keys1->stream = s;
        rows1->stream = s;
      }
      // 5. The candidates in key order (stable: equal keys stay in row order).
      am_array* tmp = new_array(D == 8 ? PT_U64 : PT_U32, D == 8 ? "L" : "I", int64_t(kv));
      tmp->values = cand_keys;
      tmp->null_count = 0;
      tmp->last_stream = s;
      try {
        radix_argsort({SortKey{tmp, false, false, 0}}, int64_t(kv), order->ptr, 4, s, nullptr);
      } catch (...) {
        release(tmp);
        throw;
      }
      release(tmp);
      KernelTimer kt("topk_gather", s);
      const int grid = int(std::min<uint64_t>((kv + 255) / 256, uint64_t(device().sm_count) * 8));
      gather_rows_kernel<<<std::max(grid, 1), 256, 0, s>>>(static_cast<const uint32_t*>(order->ptr),
                                                           static_cast<const uint32_t*>(cand_rows->ptr), kv, res + v_at);
      AM_CUDA(cudaGetLastError());
      cand_keys->stream = s;
      cand_rows->stream = s;
      order->stream = s;
    }
  } catch (...) {
    release(out);
    throw;
  }
  return out;
}

// Arrow partition_nth_indices (include/arrowmetal.h:1060-1069, :1335; the reference selects the pivot by
// radix select and compacts, Kernels/PartitionNth.swift:229): a permutation whose position `pivot`
// holds the row the stable argsort (ascending, the given null placement) puts there, with no row
// after it ordered before it and none before it ordered after it. By radix selection, reading the
// column a few times and sorting nothing:
//   1. the key statistics give the category counts, so the pivot's block ([values][NaN][nulls], or
//      [nulls][NaN][values]), and for the value block the leading digits of the pivot key T;
//   2. the lower digits of T, one histogram pass over the column per digit (only the keys that share
//      the digits chosen so far count);
//   3. one ordered three-way partition: the rows before the pivot's in the arrangement, in row order,
//      then the rows equal to it, then the rest.
template <typename KeyT>
am_array* partition_of(const SortKey& key, int64_t pivot, cudaStream_t s) {
  const uint64_t n = uint64_t(key.col->length);
  constexpr int D = int(sizeof(KeyT));
  const Source<KeyT> column{make_view(key), nullptr, nullptr, n};

  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t off_state = up(sizeof(KeyStats));
  const size_t off_hist = up(off_state + sizeof(SelState));
  const size_t off_counts = up(off_hist + sizeof(uint32_t) * 256 * D);
  const size_t bytes = up(off_counts + sizeof(uint32_t) * compact_count_words(n));
  char* base = static_cast<char*>(dmalloc(bytes, s));
  struct Free { char* p; cudaStream_t s; ~Free() { dfree(p, s); } } guard{base, s};
  KeyStats* st = reinterpret_cast<KeyStats*>(base);
  SelState* state = reinterpret_cast<SelState*>(base + off_state);
  uint32_t* hist = reinterpret_cast<uint32_t*>(base + off_hist);
  uint32_t* counts = reinterpret_cast<uint32_t*>(base + off_counts);
  key_statistics(key, st, s);
  static thread_local KeyStats* host = nullptr;
  if (!host) host = static_cast<KeyStats*>(pinned_alloc(sizeof(KeyStats)));
  AM_CUDA(cudaMemcpyAsync(host, st, sizeof(KeyStats), cudaMemcpyDeviceToHost, s));
  AM_CUDA(cudaStreamSynchronize(s));

  // 1. The pivot's block: sizes of the arrangement's three blocks in order.
  const uint64_t p = std::min<uint64_t>(uint64_t(pivot), n - 1);   // pivot == n: any permutation will do
  const uint64_t sizes[3] = {key.nulls_first ? host->n_null : host->n_value, host->n_nan,
                             key.nulls_first ? host->n_value : host->n_null};
  const int value_place = key.nulls_first ? 2 : 0;
  int place = 0;
  uint64_t before = 0;
  while (place < 2 && p >= before + sizes[place]) before += sizes[place++];
  SelState init{0, 0};
  int dv = -1;
  if (place == value_place) {
    const Leading lead = leading_digits(*host, D, p - before + 1);
    init = SelState{lead.prefix, lead.k_rem};
    dv = lead.dv;
  }
  AM_CUDA(cudaMemcpyAsync(state, &init, sizeof(SelState), cudaMemcpyHostToDevice, s));

  am_array* out = new_array(PT_U32, "I", int64_t(n));
  try {
    out->values = DevBuffer::alloc(size_t(n) * 4 + 16, s);
    out->null_count = 0;
    out->perm_of = int64_t(n);
    out->last_stream = s;
    // 2. The lower digits of T.
    if (dv > 0) {
      AM_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 256 * D, s));
      KernelTimer kt("partition_select", s);
      const int grid = int(std::min<uint64_t>((n + SEL_CHUNK - 1) / SEL_CHUNK, uint64_t(device().sm_count) * 8));
      for (int d = dv - 1; d >= 0; d--) {
        uint32_t* hd = hist + 256 * d;
        select_histogram_kernel<KeyT><<<std::max(grid, 1), SEL_THREADS, 0, s>>>(column, 8 * d, state, hd);
        AM_CUDA(cudaGetLastError());
        select_step_kernel<<<1, 256, 0, s>>>(hd, 8 * d, state);
        AM_CUDA(cudaGetLastError());
      }
    }
    // 3. The three-way partition.
    const uint32_t blocks = uint32_t((n + SEL_CHUNK - 1) / SEL_CHUNK);
    const Compact c{PRED_PARTITION, place, 0, 0, 0, state, key.nulls_first ? 1 : 0};
    uint32_t* count_a = counts;
    uint32_t* count_b = counts + blocks + 1;
    KernelTimer kt("partition_write", s);
    compact_count_kernel<KeyT><<<blocks, SEL_THREADS, 0, s>>>(column, c, count_a, count_b);
    AM_CUDA(cudaGetLastError());
    compact_scan_kernel<<<1, 1024, 0, s>>>(count_a, count_b, blocks);
    AM_CUDA(cudaGetLastError());
    partition_write_kernel<KeyT><<<blocks, SEL_THREADS, 0, s>>>(column, c, count_a, count_b, blocks,
                                                                static_cast<uint32_t*>(out->values->ptr),
                                                                stream_scratch(s, 0).err);
    AM_CUDA(cudaGetLastError());
  } catch (...) {
    release(out);
    throw;
  }
  return out;
}

}  // namespace
}  // namespace rs

// A dictionary column selects on its rank column, which orders and ties as its values.
template <typename F>
am_array* on_dictionary_key(const SortKey& key, cudaStream_t s, F&& f) {
  am_array* c = dictionary_key_column(key, s);
  am_array* r = nullptr;
  try {
    r = f(SortKey{c, key.descending, key.nulls_first, rs::FO_IEEE});
  } catch (...) {
    release(c);
    throw;
  }
  release(c);
  return r;
}

am_array* radix_partition_nth(const SortKey& key, int64_t pivot, cudaStream_t s) {
  if (key.col->length > 0 && key.col->dictionary)
    return on_dictionary_key(key, s, [&](const SortKey& k) { return radix_partition_nth(k, pivot, s); });
  if (key.col->length <= 0 || pt_var(key.col->pt)) return nullptr;
  return pt_key_bytes(key.col->pt) == 8 ? rs::partition_of<uint64_t>(key, pivot, s)
                                        : rs::partition_of<uint32_t>(key, pivot, s);
}

am_array* radix_top_k(const SortKey& key, int64_t k, cudaStream_t s) {
  if (key.col->length > 0 && k > 0 && key.col->dictionary)
    return on_dictionary_key(key, s, [&](const SortKey& kk) { return radix_top_k(kk, k, s); });
  if (key.col->length <= 0 || k <= 0 || pt_var(key.col->pt)) return nullptr;
  return pt_key_bytes(key.col->pt) == 8 ? rs::top_k_of<uint64_t>(key, k, s) : rs::top_k_of<uint32_t>(key, k, s);
}

}  // namespace am
