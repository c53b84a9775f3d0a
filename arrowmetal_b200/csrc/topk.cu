// Top-k by radix selection: the first k indices of the stable argsort without sorting every row.
//
// am_top_k_ex answers with the first k indices am_argsort_ex2 gives with the same options
// (include/arrowmetal.h:1345-1350; the reference's TopK.swift / RadixSelect.swift select on the same
// key maps). In the argsort's arrangement the value rows come in key order and the NaN-block and null
// rows in row order ([values][NaN][nulls] with nulls at the end, [nulls][NaN][values] at the start),
// so the answer is some leading category rows in row order plus the kv smallest value keys, ties in
// row order. On the order-preserving unsigned keys of the sort:
//   1. the key statistics (one read) give the category counts and the most significant digit's
//      histogram;
//   2. one histogram per lower digit over the value rows that share the digits chosen so far narrows
//      the threshold key T down to the digit at which the kv-th smallest key sits;
//   3. a stable two-phase compaction (per-block counts, one scan, ordered writes) takes every value row
//      with key < T and the first `need` rows with key == T, in row order: exactly kv candidates;
//   4. those kv (key, row) pairs are argsorted by the radix sort and their rows written out;
//   5. the category rows needed before or after them are compacted in row order the same way.
// The output is bit-identical to the prefix of the full argsort.
#include <algorithm>

#include "am_internal.h"
#include "key_encode.cuh"
#include "radix_sort.cuh"

namespace am {
namespace rs {
namespace {

constexpr int SEL_THREADS = 256, SEL_ITEMS = 8;
constexpr uint64_t SEL_CHUNK = uint64_t(SEL_THREADS) * SEL_ITEMS;   // rows per block in the compaction

struct SelState {
  unsigned long long prefix;    // the threshold key's digits chosen so far
  unsigned long long k_rem;     // rank of the wanted key among the rows that share them (1-based)
};

// Digit `shift` of the value keys whose digits above it equal the state's prefix.
template <typename KeyT>
__global__ void __launch_bounds__(SEL_THREADS) select_histogram_kernel(const __grid_constant__ ColView col, uint64_t n,
                                                                       int shift, const SelState* __restrict__ st,
                                                                       uint32_t* __restrict__ hist) {
  __shared__ uint32_t sh[256];
  for (int i = threadIdx.x; i < 256; i += SEL_THREADS) sh[i] = 0;
  __syncthreads();
  const KeyT want = KeyT(st->prefix >> (shift + 8));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint64_t base = uint64_t(blockIdx.x) * SEL_CHUNK; base < n; base += uint64_t(gridDim.x) * SEL_CHUNK) {
    uint32_t row[SEL_ITEMS];
    uint32_t ok = 0;
#pragma unroll
    for (int i = 0; i < SEL_ITEMS; i++) {
      const uint64_t g = base + uint64_t(warp) * (SEL_ITEMS * 32) + uint64_t(i) * 32 + lane;
      row[i] = uint32_t(g);
      if (g < n) ok |= 1u << i;
    }
    KeyT key[SEL_ITEMS];
    int cat[SEL_ITEMS];
    encode_rows<KeyT, SEL_ITEMS>(col, row, ok, key, cat);
#pragma unroll
    for (int i = 0; i < SEL_ITEMS; i++) {
      if (!((ok >> i) & 1u) || cat[i] != 0) continue;
      const KeyT hi = (shift + 8 >= int(8 * sizeof(KeyT))) ? KeyT(0) : KeyT(key[i] >> (shift + 8));
      if (hi == want) atomicAdd(&sh[uint32_t(key[i] >> shift) & 255u], 1u);
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
  __shared__ uint32_t incl[256];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  __shared__ uint32_t wsum[8];
  const unsigned long long k = st->k_rem;     // read by every thread before the one writer below
  uint32_t v = hist[t];
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
  incl[t] = x + add;
  __syncthreads();
  const uint32_t before = incl[t] - v;
  if (v > 0 && before < k && k <= incl[t]) {
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

// The rows a compaction takes: every row of class A, and class-B rows up to `limit` in row order.
//   mode 0: A = value rows with key < T, B = value rows with key == T (T = the state's prefix);
//   mode 1: A = none, B = rows of category `cat` (1 NaN block, 2 null).
struct Compact {
  int mode;
  int cat;
  unsigned long long limit;     // mode 1; mode 0 reads the state's k_rem
  const SelState* st;
};

template <typename KeyT>
__device__ __forceinline__ void classify(const ColView& col, const Compact& c, uint64_t base, uint64_t n,
                                         uint32_t (&a)[SEL_ITEMS], uint32_t (&b)[SEL_ITEMS], KeyT (&key)[SEL_ITEMS]) {
  uint32_t row[SEL_ITEMS];
  uint32_t ok = 0;
#pragma unroll
  for (int i = 0; i < SEL_ITEMS; i++) {
    const uint64_t g = base + uint64_t(threadIdx.x) * SEL_ITEMS + i;   // consecutive rows per thread
    row[i] = uint32_t(g);
    if (g < n) ok |= 1u << i;
  }
  int cat[SEL_ITEMS];
  encode_rows<KeyT, SEL_ITEMS>(col, row, ok, key, cat);
  const KeyT T = KeyT(c.st ? c.st->prefix : 0);
#pragma unroll
  for (int i = 0; i < SEL_ITEMS; i++) {
    const bool live = (ok >> i) & 1u;
    if (c.mode == 0) {
      a[i] = live && cat[i] == 0 && key[i] < T;
      b[i] = live && cat[i] == 0 && key[i] == T;
    } else {
      a[i] = 0;
      b[i] = live && cat[i] == c.cat;
    }
  }
}

template <typename KeyT>
__global__ void __launch_bounds__(SEL_THREADS) compact_count_kernel(const __grid_constant__ ColView col, uint64_t n,
                                                                    const __grid_constant__ Compact c,
                                                                    uint32_t* __restrict__ count_a,
                                                                    uint32_t* __restrict__ count_b) {
  __shared__ uint32_t s_warp[SEL_THREADS / 32];
  uint32_t a[SEL_ITEMS], b[SEL_ITEMS];
  KeyT key[SEL_ITEMS];
  classify<KeyT>(col, c, uint64_t(blockIdx.x) * SEL_CHUNK, n, a, b, key);
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

// One block: exclusive scans of the per-block counts, in place.
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
}

// The ordered writes: row ids (and, in mode 0, keys) of the taken rows at their places.
template <typename KeyT>
__global__ void __launch_bounds__(SEL_THREADS) compact_write_kernel(const __grid_constant__ ColView col, uint64_t n,
                                                                    const __grid_constant__ Compact c,
                                                                    const uint32_t* __restrict__ off_a,
                                                                    const uint32_t* __restrict__ off_b,
                                                                    KeyT* __restrict__ out_keys,
                                                                    uint32_t* __restrict__ out_rows, uint64_t out_cap,
                                                                    uint32_t* __restrict__ err) {
  __shared__ uint32_t s_warp[SEL_THREADS / 32];
  uint32_t a[SEL_ITEMS], b[SEL_ITEMS];
  KeyT key[SEL_ITEMS];
  const uint64_t base = uint64_t(blockIdx.x) * SEL_CHUNK;
  classify<KeyT>(col, c, base, n, a, b, key);
  const unsigned long long limit = c.mode == 0 ? c.st->k_rem : c.limit;
  uint32_t cb = 0;
#pragma unroll
  for (int i = 0; i < SEL_ITEMS; i++) cb += b[i];
  const uint32_t eb = block_scan(cb, s_warp, nullptr);    // B rows before this thread's, in the block
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
    out_rows[d] = uint32_t(base + uint64_t(threadIdx.x) * SEL_ITEMS + i);
    if (out_keys) out_keys[d] = key[i];
  }
}

// out[i] = rows[order[i]] for i < m.
__global__ void __launch_bounds__(256) gather_rows_kernel(const uint32_t* __restrict__ order, const uint32_t* __restrict__ rows,
                                                          uint64_t m, uint32_t* __restrict__ out) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x)
    out[i] = rows[order[i]];
}

template <typename KeyT>
void compact(const ColView& cv, uint64_t n, const Compact& c, KeyT* out_keys, uint32_t* out_rows, uint64_t cap,
             uint32_t* counts, uint32_t* err, cudaStream_t s) {
  const uint32_t blocks = uint32_t((n + SEL_CHUNK - 1) / SEL_CHUNK);
  uint32_t* count_a = counts;
  uint32_t* count_b = counts + blocks;
  {
    KernelTimer kt("topk_compact", s);
    compact_count_kernel<KeyT><<<blocks, SEL_THREADS, 0, s>>>(cv, n, c, count_a, count_b);
    AM_CUDA(cudaGetLastError());
    compact_scan_kernel<<<1, 1024, 0, s>>>(count_a, count_b, blocks);
    AM_CUDA(cudaGetLastError());
    compact_write_kernel<KeyT><<<blocks, SEL_THREADS, 0, s>>>(cv, n, c, count_a, count_b, out_keys, out_rows, cap, err);
    AM_CUDA(cudaGetLastError());
  }
}

template <typename KeyT>
am_array* top_k_of(const SortKey& key, int64_t k, cudaStream_t s) {
  const uint64_t n = uint64_t(key.col->length);
  constexpr int D = int(sizeof(KeyT));
  const ColView cv = make_view(key);
  const uint32_t blocks = uint32_t((n + SEL_CHUNK - 1) / SEL_CHUNK);

  // Scratch: statistics, state, per-digit histograms, compaction counts.
  auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t off_state = up(sizeof(KeyStats));
  const size_t off_hist = up(off_state + sizeof(SelState));
  const size_t off_counts = up(off_hist + sizeof(uint32_t) * 256 * D);
  const size_t bytes = up(off_counts + sizeof(uint32_t) * 2 * size_t(blocks));
  char* base = static_cast<char*>(dmalloc(bytes, s));
  struct Free { char* p; cudaStream_t s; ~Free() { dfree(p, s); } } guard{base, s};
  KeyStats* st = reinterpret_cast<KeyStats*>(base);
  SelState* state = reinterpret_cast<SelState*>(base + off_state);
  uint32_t* hist = reinterpret_cast<uint32_t*>(base + off_hist);
  uint32_t* counts = reinterpret_cast<uint32_t*>(base + off_counts);
  key_statistics(key, st, s);

  // The category counts decide the shape of the answer.
  static thread_local uint32_t* host = nullptr;
  if (!host) host = static_cast<uint32_t*>(pinned_alloc(16));
  AM_CUDA(cudaMemcpyAsync(host, &st->n_value, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  AM_CUDA(cudaStreamSynchronize(s));
  const uint64_t n_value = host[0], n_null = host[1], n_nan = host[2];
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
    if (k_null) compact<KeyT>(cv, n, Compact{1, 2, k_null, nullptr}, nullptr, res + null_at, k_null, counts, err, s);
    if (k_nan) compact<KeyT>(cv, n, Compact{1, 1, k_nan, nullptr}, nullptr, res + nan_at, k_nan, counts, err, s);
    if (kv) {
      // Threshold: digit by digit from the most significant (whose histogram the statistics hold).
      const SelState init{0ull, (unsigned long long)kv};
      AM_CUDA(cudaMemcpyAsync(state, &init, sizeof(SelState), cudaMemcpyHostToDevice, s));
      AM_CUDA(cudaMemsetAsync(hist, 0, sizeof(uint32_t) * 256 * D, s));
      {
        KernelTimer kt("topk_select", s);
        for (int d = D - 1; d >= 0; d--) {
          const uint32_t* h = st->hist[d];
          if (d < D - 1) {
            uint32_t* hd = hist + 256 * d;
            const int grid = int(std::min<uint64_t>((n + SEL_CHUNK - 1) / SEL_CHUNK, uint64_t(device().sm_count) * 8));
            select_histogram_kernel<KeyT><<<std::max(grid, 1), SEL_THREADS, 0, s>>>(cv, n, 8 * d, state, hd);
            AM_CUDA(cudaGetLastError());
            h = hd;
          }
          select_step_kernel<<<1, 256, 0, s>>>(h, 8 * d, state);
          AM_CUDA(cudaGetLastError());
        }
      }
      // The kv candidates in row order, then their stable argsort.
      BufPtr cand_keys = DevBuffer::alloc(size_t(kv) * sizeof(KeyT) + 16, s);
      BufPtr cand_rows = DevBuffer::alloc(size_t(kv) * 4 + 16, s);
      BufPtr order = DevBuffer::alloc(size_t(kv) * 4 + 16, s);
      compact<KeyT>(cv, n, Compact{0, 0, 0, state}, static_cast<KeyT*>(cand_keys->ptr),
                    static_cast<uint32_t*>(cand_rows->ptr), kv, counts, err, s);
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

}  // namespace
}  // namespace rs

am_array* radix_top_k(const SortKey& key, int64_t k, cudaStream_t s) {
  if (key.col->length <= 0 || k <= 0) return nullptr;
  return pt_key_bytes(key.col->pt) == 8 ? rs::top_k_of<uint64_t>(key, k, s) : rs::top_k_of<uint32_t>(key, k, s);
}

}  // namespace am
