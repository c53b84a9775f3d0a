// Shared sorts of the sort server: several queued requests that sort rows of the same table by the
// same keys and options are answered from one sort of the rows they cover together.
//
// A stable sort orders tied rows by row number, so the order of any subset of rows under it is the
// full order restricted to that subset: request q's permutation is the covering sort's permutation
// with every row outside [lo_q, hi_q) dropped, in the same order. One pass over the covering
// permutation keeps, for each of up to MAX_SHARED requests, its rows in order (a ballot per warp and
// request gives each row's place within its block; block counts are scanned per request), so the
// requests' results equal their own sorts exactly.
#include <algorithm>

#include "am_internal.h"

namespace am {
namespace {

constexpr int CMP_THREADS = 256, CMP_ITEMS = 16;
constexpr uint32_t CMP_CHUNK = uint32_t(CMP_THREADS) * CMP_ITEMS;

struct Ranges {
  uint32_t lo[MAX_SHARED], hi[MAX_SHARED];
  uint32_t* out[MAX_SHARED];
  int k;
};

// counts[q * blocks + b]: rows of block b's chunk inside request q's range.
__global__ void __launch_bounds__(CMP_THREADS) range_count_kernel(const uint32_t* __restrict__ perm, uint64_t n,
                                                                  const __grid_constant__ Ranges r,
                                                                  uint32_t* __restrict__ counts) {
  __shared__ uint32_t s_cnt[MAX_SHARED];
  for (int q = threadIdx.x; q < r.k; q += CMP_THREADS) s_cnt[q] = 0;
  __syncthreads();
  const uint64_t base = uint64_t(blockIdx.x) * CMP_CHUNK;
  uint32_t v[CMP_ITEMS];
#pragma unroll
  for (int i = 0; i < CMP_ITEMS; i++) {
    const uint64_t j = base + uint64_t(i) * CMP_THREADS + threadIdx.x;
    v[i] = j < n ? perm[j] : 0xFFFFFFFFu;
  }
  for (int q = 0; q < r.k; q++) {
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < CMP_ITEMS; i++) c += (v[i] >= r.lo[q] && v[i] < r.hi[q]) ? 1u : 0u;
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&s_cnt[q], c);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < r.k; q += CMP_THREADS) counts[size_t(q) * gridDim.x + blockIdx.x] = s_cnt[q];
}

// One block per request: exclusive scan of its block counts, in place.
__global__ void __launch_bounds__(1024) range_scan_kernel(uint32_t* __restrict__ counts, uint32_t blocks) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_carry;
  uint32_t* c = counts + size_t(blockIdx.x) * blocks;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (uint32_t b0 = 0; b0 < blocks; b0 += 1024) {
    const uint32_t b = b0 + threadIdx.x;
    const uint32_t x = b < blocks ? c[b] : 0u;
    uint32_t inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = s_warp[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t before = s_carry + (warp ? s_warp[warp - 1] : 0u) + inc - x;
    if (b < blocks) c[b] = before;
    __syncthreads();
    if (threadIdx.x == 0) s_carry += s_warp[31];
    __syncthreads();
  }
}

// Each request's rows of block b's chunk, in order, from its scanned offset. Row j of the chunk is
// item i = j / CMP_THREADS of thread j % CMP_THREADS, so the chunk's order is item-major: a warp's
// rows of one item are 32 consecutive rows, and the items follow one another.
__global__ void __launch_bounds__(CMP_THREADS) range_write_kernel(const uint32_t* __restrict__ perm, uint64_t n,
                                                                  const __grid_constant__ Ranges r,
                                                                  const uint32_t* __restrict__ offsets) {
  constexpr int WARPS = CMP_THREADS / 32;
  __shared__ uint32_t s_item[CMP_ITEMS][WARPS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint64_t base = uint64_t(blockIdx.x) * CMP_CHUNK;
  uint32_t v[CMP_ITEMS];
#pragma unroll
  for (int i = 0; i < CMP_ITEMS; i++) {
    const uint64_t j = base + uint64_t(i) * CMP_THREADS + threadIdx.x;
    v[i] = j < n ? perm[j] : 0xFFFFFFFFu;
  }
  for (int q = 0; q < r.k; q++) {
    uint32_t m[CMP_ITEMS];
#pragma unroll
    for (int i = 0; i < CMP_ITEMS; i++) {
      m[i] = __ballot_sync(0xffffffffu, v[i] >= r.lo[q] && v[i] < r.hi[q]);
      if (lane == 0) s_item[i][warp] = __popc(m[i]);
    }
    __syncthreads();
    // Rows before (item i, warp w) in chunk order: all earlier items, then this item's earlier warps.
    if (threadIdx.x == 0) {
      uint32_t run = 0;
      for (int i = 0; i < CMP_ITEMS; i++)
        for (int w = 0; w < WARPS; w++) {
          const uint32_t c = s_item[i][w];
          s_item[i][w] = run;
          run += c;
        }
    }
    __syncthreads();
    const uint32_t off = offsets[size_t(q) * gridDim.x + blockIdx.x];
#pragma unroll
    for (int i = 0; i < CMP_ITEMS; i++)
      if ((m[i] >> lane) & 1u) r.out[q][off + s_item[i][warp] + __popc(m[i] & lt)] = v[i];
    __syncthreads();
  }
}

// The columns of the covered rows in the shared order, copied for each request q into its own sorted
// columns: the entries of block b's chunk whose row lies in q's range, in order, at the same places
// the index compaction gives them. Validity bits of one warp item land in at most two output words
// (the item's kept rows are consecutive), OR-ed together and added with one atomic each.
__global__ void __launch_bounds__(CMP_THREADS) range_write_cols_kernel(const uint32_t* __restrict__ perm, uint64_t n,
                                                                       const __grid_constant__ Ranges r,
                                                                       const __grid_constant__ CompactSrc src,
                                                                       const CompactDst* __restrict__ dst,
                                                                       const uint32_t* __restrict__ offsets) {
  constexpr int WARPS = CMP_THREADS / 32;
  __shared__ uint32_t s_item[CMP_ITEMS][WARPS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint64_t base = uint64_t(blockIdx.x) * CMP_CHUNK;
  uint32_t v[CMP_ITEMS];
#pragma unroll
  for (int i = 0; i < CMP_ITEMS; i++) {
    const uint64_t j = base + uint64_t(i) * CMP_THREADS + threadIdx.x;
    v[i] = j < n ? perm[j] : 0xFFFFFFFFu;
  }
  for (int q = 0; q < r.k; q++) {
    uint32_t m[CMP_ITEMS];
#pragma unroll
    for (int i = 0; i < CMP_ITEMS; i++) {
      m[i] = __ballot_sync(0xffffffffu, v[i] >= r.lo[q] && v[i] < r.hi[q]);
      if (lane == 0) s_item[i][warp] = __popc(m[i]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t run = 0;
      for (int i = 0; i < CMP_ITEMS; i++)
        for (int w = 0; w < WARPS; w++) {
          const uint32_t c = s_item[i][w];
          s_item[i][w] = run;
          run += c;
        }
    }
    __syncthreads();
    const uint32_t off = offsets[size_t(q) * gridDim.x + blockIdx.x];
    const CompactDst& d = dst[q];
    for (int c = 0; c < src.ncols; c++) {
      const int w = src.width[c];
      const uint8_t* sv = src.src_valid[c];
      uint32_t nulls = 0;
#pragma unroll
      for (int i = 0; i < CMP_ITEMS; i++) {
        const bool keep = (m[i] >> lane) & 1u;
        const uint64_t row = base + uint64_t(i) * CMP_THREADS + threadIdx.x;
        const uint32_t first = off + s_item[i][warp];          // the item's first kept place
        const uint32_t pos = first + __popc(m[i] & lt);
        if (keep) {
          switch (w) {
            case 8: static_cast<uint64_t*>(d.dst[c])[pos] = static_cast<const uint64_t*>(src.src[c])[row]; break;
            case 4: static_cast<uint32_t*>(d.dst[c])[pos] = static_cast<const uint32_t*>(src.src[c])[row]; break;
            case 2: static_cast<uint16_t*>(d.dst[c])[pos] = static_cast<const uint16_t*>(src.src[c])[row]; break;
            default: static_cast<uint8_t*>(d.dst[c])[pos] = static_cast<const uint8_t*>(src.src[c])[row]; break;
          }
        }
        if (sv && m[i]) {                                       // warp-uniform
          const int64_t b = src.src_voff[c] + int64_t(row);
          const bool valid = keep && ((sv[b >> 3] >> (b & 7)) & 1u);
          if (keep && !valid) nulls++;
          const uint32_t w0 = first >> 5;
          const uint32_t bit = valid ? (1u << (pos & 31)) : 0u;
          const uint32_t lo_w = __reduce_or_sync(0xffffffffu, (pos >> 5) == w0 ? bit : 0u);
          const uint32_t hi_w = __reduce_or_sync(0xffffffffu, (pos >> 5) != w0 ? bit : 0u);
          if (lane == 0) {
            if (lo_w) atomicOr(&d.dst_valid[c][w0], lo_w);
            if (hi_w) atomicOr(&d.dst_valid[c][w0 + 1], hi_w);
          }
        }
      }
      if (sv) {
        nulls = __reduce_add_sync(0xffffffffu, nulls);
        if (lane == 0 && nulls) atomicAdd(d.nulls[c], (unsigned long long)nulls);
      }
    }
    __syncthreads();
  }
}

}  // namespace

void compact_columns(const uint32_t* perm, uint64_t n, const std::vector<uint32_t>& lo, const std::vector<uint32_t>& hi,
                     const CompactSrc& src, const std::vector<CompactDst>& dsts, cudaStream_t s) {
  const int k = int(lo.size());
  if (k == 0 || n == 0) return;
  if (k > MAX_SHARED || hi.size() != lo.size() || dsts.size() != lo.size() || src.ncols < 1 || src.ncols > MAX_CCOLS)
    throw invalid("compact_columns: 1 to " + std::to_string(MAX_SHARED) + " ranges of 1 to " +
                  std::to_string(MAX_CCOLS) + " columns");
  Ranges r{};
  r.k = k;
  for (int q = 0; q < k; q++) {
    r.lo[q] = lo[size_t(q)];
    r.hi[q] = hi[size_t(q)];
  }
  const uint32_t blocks = uint32_t((n + CMP_CHUNK - 1) / CMP_CHUNK);
  uint32_t* counts = static_cast<uint32_t*>(dmalloc(sizeof(uint32_t) * size_t(blocks) * size_t(k), s));
  CompactDst* d = static_cast<CompactDst*>(dmalloc(sizeof(CompactDst) * size_t(k), s));
  copy_h2d(d, dsts.data(), sizeof(CompactDst) * size_t(k), s);
  KernelTimer kt("server_shared_columns", s);
  range_count_kernel<<<blocks, CMP_THREADS, 0, s>>>(perm, n, r, counts);
  AM_CUDA(cudaGetLastError());
  range_scan_kernel<<<k, 1024, 0, s>>>(counts, blocks);
  AM_CUDA(cudaGetLastError());
  range_write_cols_kernel<<<blocks, CMP_THREADS, 0, s>>>(perm, n, r, src, d, counts);
  AM_CUDA(cudaGetLastError());
  dfree(d, s);
  dfree(counts, s);
}

void compact_ranges(const uint32_t* perm, uint64_t n, const std::vector<uint32_t>& lo, const std::vector<uint32_t>& hi,
                    const std::vector<uint32_t*>& outs, cudaStream_t s) {
  const int k = int(lo.size());
  if (k == 0 || n == 0) return;
  if (k > MAX_SHARED || hi.size() != lo.size() || outs.size() != lo.size())
    throw invalid("compact_ranges: 1 to " + std::to_string(MAX_SHARED) + " ranges");
  Ranges r{};
  r.k = k;
  for (int q = 0; q < k; q++) {
    r.lo[q] = lo[size_t(q)];
    r.hi[q] = hi[size_t(q)];
    r.out[q] = outs[size_t(q)];
  }
  const uint32_t blocks = uint32_t((n + CMP_CHUNK - 1) / CMP_CHUNK);
  uint32_t* counts = static_cast<uint32_t*>(dmalloc(sizeof(uint32_t) * size_t(blocks) * size_t(k), s));
  KernelTimer kt("server_shared_compact", s);
  range_count_kernel<<<blocks, CMP_THREADS, 0, s>>>(perm, n, r, counts);
  AM_CUDA(cudaGetLastError());
  range_scan_kernel<<<k, 1024, 0, s>>>(counts, blocks);
  AM_CUDA(cudaGetLastError());
  range_write_kernel<<<blocks, CMP_THREADS, 0, s>>>(perm, n, r, counts);
  AM_CUDA(cudaGetLastError());
  dfree(counts, s);
}

}  // namespace am
