// String and binary columns (Arrow utf8 / binary with int32 offsets, large_utf8 / large_binary with
// int64 offsets): sort keys and take.
//
// Sort order is Arrow's for these types: bytes compared lexicographically, a string that is a prefix
// of another first (the reference's StringSort.swift sorts by prefix keys the same way). A string key
// becomes derived unsigned keys for the radix sort: its bytes in big-endian 8-byte chunks, zero-padded
// (chunk j holds bytes [8j, 8j + 8)), then its length. The tuple (chunk 0, ..., chunk m-1, length) orders
// strings exactly as the byte comparison does: two strings first differ in the chunk that holds their
// first differing byte, and when one is a prefix of the other their padded chunks tie and the shorter
// length comes first. Null rows are routed by the first chunk, which carries the column's validity; a
// descending sort reverses every derived key.
//
// Take gathers the rows' lengths, scans them into the output offsets and copies each row's bytes.
#include <algorithm>

#include "am_internal.h"
#include "radix_sort.cuh"

namespace am {
namespace {

__device__ __forceinline__ bool bit_at(const uint8_t* p, int64_t i) { return (p[i >> 3] >> (i & 7)) & 1; }

template <typename OffT>
__device__ __forceinline__ void row_span(const OffT* off, int64_t row, uint64_t& start, uint64_t& len) {
  const uint64_t a = uint64_t(off[row]), b = uint64_t(off[row + 1]);
  start = a;
  len = b > a ? b - a : 0;
}

// The longest valid row's length.
template <typename OffT>
__global__ void __launch_bounds__(256) max_length_kernel(const OffT* __restrict__ off, const uint8_t* __restrict__ valid,
                                                         int64_t voff, uint64_t n, unsigned long long* __restrict__ out) {
  unsigned long long m = 0;
  for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += uint64_t(gridDim.x) * blockDim.x) {
    if (valid && !bit_at(valid, voff + int64_t(r))) continue;
    uint64_t s, l;
    row_span(off, int64_t(r), s, l);
    m = l > m ? l : m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long y = __shfl_xor_sync(0xffffffffu, m, o);
    m = y > m ? y : m;
  }
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// chunk[j][r]: bytes [8 (first + j), 8 (first + j) + 8) of row r, big-endian, zero-padded, for j < m;
// length[r] (when asked). A null row is the empty string here, whatever its slot spans, so the null
// rows tie on every derived key and keep their row order.
template <typename OffT, typename LenT>
__global__ void __launch_bounds__(256) chunk_kernel(const OffT* __restrict__ off, const uint8_t* __restrict__ bytes,
                                                    const uint8_t* __restrict__ valid, int64_t voff, uint64_t n,
                                                    int first, int m, uint64_t* const* __restrict__ chunks,
                                                    LenT* __restrict__ length) {
  for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += uint64_t(gridDim.x) * blockDim.x) {
    uint64_t s, l;
    row_span(off, int64_t(r), s, l);
    if (valid && !bit_at(valid, voff + int64_t(r))) l = 0;
    for (int j = 0; j < m; j++) {
      uint64_t v = 0;
#pragma unroll
      for (int b = 0; b < 8; b++) {
        const uint64_t p = uint64_t(first + j) * 8 + b;
        v = (v << 8) | (p < l ? uint64_t(bytes[s + p]) : 0u);
      }
      chunks[j][r] = v;
    }
    if (length) length[r] = LenT(l);
  }
}

// ---- take

template <typename IdxT>
__device__ __forceinline__ bool index_of(const void* idx, const uint8_t* idx_valid, int64_t idx_voff, uint64_t i,
                                         uint64_t src_len, int64_t& out) {
  if (idx_valid && !bit_at(idx_valid, idx_voff + int64_t(i))) return false;
  const int64_t v = int64_t(static_cast<const IdxT*>(idx)[i]);
  out = v;
  return v >= 0 && uint64_t(v) < src_len;
}

struct StrTake {
  const void* idx;
  const uint8_t* idx_valid;
  int64_t idx_voff;
  int idx_kind;              // 0 uint32, 1 int32, 2 int64, 3 uint64
  uint64_t n;                // output rows
  uint64_t src_len;
  const void* src_off;       // source offsets at its row 0
  const uint8_t* src_valid;
  int64_t src_voff;
  const uint8_t* src_bytes;
  int check;
  uint32_t* err;
};

template <typename OffT>
__device__ __forceinline__ bool gathered(const StrTake& t, uint64_t i, uint64_t& start, uint64_t& len) {
  int64_t r = 0;
  bool ok;
  switch (t.idx_kind) {
    case 0: ok = index_of<uint32_t>(t.idx, t.idx_valid, t.idx_voff, i, t.src_len, r); break;
    case 1: ok = index_of<int32_t>(t.idx, t.idx_valid, t.idx_voff, i, t.src_len, r); break;
    case 2: ok = index_of<int64_t>(t.idx, t.idx_valid, t.idx_voff, i, t.src_len, r); break;
    default: ok = index_of<uint64_t>(t.idx, t.idx_valid, t.idx_voff, i, t.src_len, r); break;
  }
  if (!ok) {
    const bool null_index = t.idx_valid && !bit_at(t.idx_valid, t.idx_voff + int64_t(i));
    if (!null_index && t.check) atomicOr(t.err, rs::ERR_TAKE_RANGE);
    start = len = 0;
    return false;
  }
  if (t.src_valid && !bit_at(t.src_valid, t.src_voff + r)) {
    start = len = 0;
    return false;
  }
  row_span(static_cast<const OffT*>(t.src_off), r, start, len);
  return true;
}

// Lengths of the gathered rows and the output's validity words (32 rows a warp) and null count.
template <typename OffT>
__global__ void __launch_bounds__(256) take_lengths_kernel(const __grid_constant__ StrTake t, uint64_t* __restrict__ lens,
                                                           uint32_t* __restrict__ out_valid,
                                                           unsigned long long* __restrict__ nulls) {
  const int lane = threadIdx.x & 31;
  const uint64_t words = (t.n + 31) / 32;
  unsigned long long z = 0;
  for (uint64_t w = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; w < words;
       w += uint64_t(gridDim.x) * blockDim.x / 32) {
    const uint64_t i = w * 32 + lane;
    bool valid = false;
    if (i < t.n) {
      uint64_t s, l;
      valid = gathered<OffT>(t, i, s, l);
      lens[i] = l;
    }
    const uint32_t b = __ballot_sync(0xffffffffu, valid);
    const uint32_t live = __ballot_sync(0xffffffffu, i < t.n);
    if (lane == 0) {
      out_valid[w] = b;
      z += __popc(live & ~b);
    }
  }
  if (lane == 0 && z) atomicAdd(nulls, z);
}

// Exclusive scan of 64-bit values in chunks of 1024 (three launches: chunk sums, one-block scan of
// the sums, scan within the chunks); out[i] = sum of in[0..i), out[n] = the total.
__global__ void __launch_bounds__(1024) chunk_sums_kernel(const uint64_t* __restrict__ in, uint64_t n,
                                                          uint64_t* __restrict__ sums) {
  __shared__ unsigned long long s[32];
  const uint64_t i = uint64_t(blockIdx.x) * 1024 + threadIdx.x;
  unsigned long long v = i < n ? in[i] : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    unsigned long long x = s[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (threadIdx.x == 0) sums[blockIdx.x] = x;
  }
}

__global__ void __launch_bounds__(1024) scan_sums_kernel(uint64_t* __restrict__ sums, uint64_t chunks,
                                                         uint64_t* __restrict__ total) {
  __shared__ unsigned long long s[32];
  __shared__ unsigned long long carry;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t == 0) carry = 0;
  __syncthreads();
  for (uint64_t base = 0; base < chunks; base += 1024) {
    const uint64_t i = base + uint64_t(t);
    const unsigned long long v = i < chunks ? sums[i] : 0;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s[warp] = x;
    __syncthreads();
    unsigned long long add = carry, all = 0;
    for (int w = 0; w < 32; w++) {
      if (w < warp) add += s[w];
      all += s[w];
    }
    if (i < chunks) sums[i] = x - v + add;
    __syncthreads();
    if (t == 0) carry += all;
    __syncthreads();
  }
  if (t == 0) *total = carry;
}

template <typename OffT>
__global__ void __launch_bounds__(1024) scan_chunks_kernel(const uint64_t* __restrict__ in, uint64_t n,
                                                           const uint64_t* __restrict__ sums, const uint64_t* __restrict__ total,
                                                           OffT* __restrict__ out) {
  __shared__ unsigned long long s[32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint64_t i = uint64_t(blockIdx.x) * 1024 + uint64_t(t);
  const unsigned long long v = i < n ? in[i] : 0;
  unsigned long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s[warp] = x;
  __syncthreads();
  unsigned long long add = sums[blockIdx.x];
  for (int w = 0; w < warp; w++) add += s[w];
  if (i < n) out[i] = OffT(x - v + add);
  if (blockIdx.x == 0 && t == 0) out[n] = OffT(*total);
}

// Each output row's bytes, one thread a row.
template <typename OffT>
__global__ void __launch_bounds__(256) take_bytes_kernel(const __grid_constant__ StrTake t, const OffT* __restrict__ out_off,
                                                         uint8_t* __restrict__ out_bytes, uint64_t out_cap) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < t.n; i += uint64_t(gridDim.x) * blockDim.x) {
    uint64_t s, l;
    if (!gathered<OffT>(t, i, s, l)) continue;
    const uint64_t d = uint64_t(out_off[i]);
    if (d + l > out_cap) {
      atomicOr(t.err, rs::ERR_BOUNDS);
      continue;
    }
    for (uint64_t b = 0; b < l; b++) out_bytes[d + b] = t.src_bytes[s + b];
  }
}

int grid_for(uint64_t n, int per_block) {
  return int(std::max<uint64_t>(1, std::min<uint64_t>((n + per_block - 1) / per_block, uint64_t(device().sm_count) * 8)));
}

template <typename OffT>
const OffT* offsets_at_row0(const am_array* a) {
  return static_cast<const OffT*>(a->values->ptr) + a->value_offset;
}

template <typename OffT>
uint64_t max_length(const am_array* a, cudaStream_t s) {
  static thread_local unsigned long long* host = nullptr;
  if (!host) host = static_cast<unsigned long long*>(pinned_alloc(16));
  unsigned long long* dev = static_cast<unsigned long long*>(dmalloc(16, s));
  AM_CUDA(cudaMemsetAsync(dev, 0, 8, s));
  const uint64_t n = uint64_t(a->length);
  max_length_kernel<OffT><<<grid_for(n, 256), 256, 0, s>>>(offsets_at_row0<OffT>(a),
                                                          a->null_count != 0 ? a->valid_bits() : nullptr,
                                                          a->validity_offset, n, dev);
  AM_CUDA(cudaGetLastError());
  AM_CUDA(cudaMemcpyAsync(host, dev, 8, cudaMemcpyDeviceToHost, s));
  AM_CUDA(cudaStreamSynchronize(s));
  dfree(dev, s);
  return *host;
}

template <typename OffT, typename LenT>
std::vector<am_array*> key_columns(const am_array* a, int first, int m, bool with_length, cudaStream_t s) {
  const uint64_t n = uint64_t(a->length);
  std::vector<am_array*> cols;
  std::vector<uint64_t*> ptrs;
  try {
    for (int j = 0; j < m; j++) {
      am_array* c = new_array(PT_U64, "L", int64_t(n));
      cols.push_back(c);
      c->values = DevBuffer::alloc(size_t(std::max<uint64_t>(n, 1)) * 8 + 16, s);
      c->null_count = 0;
      c->last_stream = s;
      ptrs.push_back(static_cast<uint64_t*>(c->values->ptr));
    }
    const bool wide = sizeof(LenT) == 8;
    LenT* len_ptr = nullptr;
    if (with_length) {
      am_array* len = new_array(wide ? PT_U64 : PT_U32, wide ? "L" : "I", int64_t(n));
      cols.push_back(len);
      len->values = DevBuffer::alloc(size_t(std::max<uint64_t>(n, 1)) * sizeof(LenT) + 16, s);
      len->null_count = 0;
      len->last_stream = s;
      len_ptr = static_cast<LenT*>(len->values->ptr);
    }
    BufPtr table = DevBuffer::alloc(sizeof(uint64_t*) * std::max(m, 1), s);
    if (m > 0) AM_CUDA(cudaMemcpyAsync(table->ptr, ptrs.data(), sizeof(uint64_t*) * m, cudaMemcpyHostToDevice, s));
    const uint8_t* valid = a->null_count != 0 ? a->valid_bits() : nullptr;
    chunk_kernel<OffT, LenT><<<grid_for(n, 256), 256, 0, s>>>(offsets_at_row0<OffT>(a),
                                                             a->bytes ? static_cast<const uint8_t*>(a->bytes->ptr) : nullptr,
                                                             valid, a->validity_offset, n, first, m,
                                                             static_cast<uint64_t* const*>(table->ptr), len_ptr);
    AM_CUDA(cudaGetLastError());
    // Chunk 0 carries the column's nulls (routed or folded by the sort).
    if (first == 0 && m > 0) {
      am_array* c0 = cols.front();
      c0->validity = a->validity;
      c0->validity_offset = a->validity_offset;
      c0->null_count = a->null_count;
      c0->null_count_dev = a->null_count_dev;
      if (a->null_count < 0) c0->null_count = -1;
    }
  } catch (...) {
    for (am_array* c : cols) release(c);
    throw;
  }
  return cols;
}

template <typename OffT>
void take_strings_t(am_array* src, am_array* idx, am_array* out, bool check, cudaStream_t s) {
  const uint64_t n = uint64_t(idx->length);
  StrTake t{};
  t.idx = idx->data();
  t.idx_valid = idx->null_count != 0 ? idx->valid_bits() : nullptr;
  t.idx_voff = idx->validity_offset;
  switch (idx->pt) {
    case PT_U32: t.idx_kind = 0; break;
    case PT_I32: t.idx_kind = 1; break;
    case PT_I64: t.idx_kind = 2; break;
    case PT_U64: t.idx_kind = 3; break;
    default: throw unsupported("take indices must be int32, int64 or uint32");
  }
  t.n = n;
  t.src_len = uint64_t(src->length);
  t.src_off = offsets_at_row0<OffT>(src);
  t.src_valid = src->null_count != 0 ? src->valid_bits() : nullptr;
  t.src_voff = src->validity_offset;
  t.src_bytes = static_cast<const uint8_t*>(src->bytes->ptr);
  t.check = check ? 1 : 0;
  t.err = stream_scratch(s, 0).err;

  const uint64_t words = (n + 31) / 32;
  const uint64_t chunks = (n + 1023) / 1024;
  char* scratch = static_cast<char*>(dmalloc(size_t(std::max<uint64_t>(n, 1)) * 8 + size_t(chunks + 1) * 8 + 16, s));
  uint64_t* lens = reinterpret_cast<uint64_t*>(scratch);
  uint64_t* sums = lens + std::max<uint64_t>(n, 1);
  uint64_t* total = sums + chunks;
  out->validity = DevBuffer::alloc(std::max<uint64_t>(words, 1) * 4 + 16, s);
  out->null_count_dev = DevBuffer::alloc(sizeof(unsigned long long), s);
  AM_CUDA(cudaMemsetAsync(out->null_count_dev->ptr, 0, sizeof(unsigned long long), s));
  out->null_count = -1;
  out->values = DevBuffer::alloc((n + 1) * sizeof(OffT) + 16, s);
  OffT* out_off = static_cast<OffT*>(out->values->ptr);
  {
    KernelTimer kt("take_strings", s);
    if (n > 0) {
      take_lengths_kernel<OffT><<<grid_for(words * 32, 256), 256, 0, s>>>(t, lens, static_cast<uint32_t*>(out->validity->ptr),
                                                                         static_cast<unsigned long long*>(out->null_count_dev->ptr));
      AM_CUDA(cudaGetLastError());
      chunk_sums_kernel<<<uint32_t(chunks), 1024, 0, s>>>(lens, n, sums);
      AM_CUDA(cudaGetLastError());
    }
    scan_sums_kernel<<<1, 1024, 0, s>>>(sums, chunks, total);
    AM_CUDA(cudaGetLastError());
    if (n > 0) {
      scan_chunks_kernel<OffT><<<uint32_t(chunks), 1024, 0, s>>>(lens, n, sums, total, out_off);
    } else {
      AM_CUDA(cudaMemsetAsync(out_off, 0, sizeof(OffT), s));
    }
    AM_CUDA(cudaGetLastError());
  }
  // The output's byte count sizes its data buffer.
  static thread_local unsigned long long* host = nullptr;
  if (!host) host = static_cast<unsigned long long*>(pinned_alloc(16));
  AM_CUDA(cudaMemcpyAsync(host, total, 8, cudaMemcpyDeviceToHost, s));
  AM_CUDA(cudaStreamSynchronize(s));
  const uint64_t bytes = *host;
  if (sizeof(OffT) == 4 && bytes > uint64_t(INT32_MAX))
    throw invalid("take: " + std::to_string(bytes) + " bytes of strings do not fit int32 offsets (use large_utf8)");
  out->bytes = DevBuffer::alloc(bytes + 16, s);
  if (n > 0 && bytes > 0) {
    KernelTimer kt("take_strings", s);
    take_bytes_kernel<OffT><<<grid_for(n, 256), 256, 0, s>>>(t, out_off, static_cast<uint8_t*>(out->bytes->ptr), bytes);
    AM_CUDA(cudaGetLastError());
  }
  dfree(scratch, s);
  out->value_offset = 0;
  out->validity_offset = 0;
  out->last_stream = s;
}

}  // namespace

int string_chunk_count(const am_array* a, cudaStream_t s) {
  if (!pt_var(a->pt)) throw Error("string_chunk_count: not a string column");
  if (a->length <= 0) return 1;
  const uint64_t maxlen = a->pt == PT_LSTR ? max_length<int64_t>(a, s) : max_length<int32_t>(a, s);
  const uint64_t m = std::max<uint64_t>(1, (maxlen + 7) / 8);
  if (m > (uint64_t(1) << 24)) throw unsupported("string keys longer than 128 MiB");
  return int(m);
}

std::vector<am_array*> string_key_columns(const am_array* a, int first, int count, bool with_length, cudaStream_t s) {
  if (!pt_var(a->pt)) throw Error("string_key_columns: not a string column");
  if (a->length <= 0) throw Error("string_key_columns: empty column");
  return a->pt == PT_LSTR ? key_columns<int64_t, uint64_t>(a, first, count, with_length, s)
                          : key_columns<int32_t, uint32_t>(a, first, count, with_length, s);
}

void take_strings(am_array* src, am_array* idx, am_array* out, bool check_range, cudaStream_t s) {
  use_on(src, s);
  use_on(idx, s);
  if (src->pt == PT_LSTR) take_strings_t<int64_t>(src, idx, out, check_range, s);
  else take_strings_t<int32_t>(src, idx, out, check_range, s);
}

}  // namespace am
