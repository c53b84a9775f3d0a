// Arrow `take` for sm_100a: every column of a batch gathered through one read of the index array.
//
// Semantics are the reference's take (Sources/ArrowMetal/Kernels/Take.swift:41-79 and `take_kernel`,
// Sources/ArrowMetal/Kernels/KernelSource.swift:209-228): out[i] = values[indices[i]]; a null index
// gives a null row; a row is null when its source row is; an index outside [0, length) is an error
// reported after the launch; int32, int64 and uint32 indices. The reference runs one launch per
// column, one row per thread, writes a validity byte per row and packs the bytes in a second kernel
// (BitmapOps.packBits, Take.swift:75). Here one launch serves up to kMaxTakeCols columns: each lane
// owns four consecutive rows, loads their indices with one 128-bit load, gathers each column's four
// values and writes them with 128-bit stores, and the four validity bits of eight lanes are OR-ed
// into one 32-bit bitmap word with three shuffles, so the bitmap is written packed and the null count
// comes from its popcount.
#include "am_internal.h"
#include "radix_sort.cuh"
#include "take.cuh"

namespace am {
namespace tk {

__device__ __forceinline__ bool bit_at(const uint8_t* p, int64_t i) { return (p[i >> 3] >> (i & 7)) & 1; }

template <int KIND> struct IdxT;
template <> struct IdxT<IDX_U32> { using T = uint32_t; };
template <> struct IdxT<IDX_I32> { using T = int32_t; };
template <> struct IdxT<IDX_I64> { using T = int64_t; };
template <> struct IdxT<IDX_U64> { using T = uint64_t; };

template <int KIND>
__device__ __forceinline__ void load4(const void* base, uint64_t row0, bool vec, uint64_t n, int64_t (&out)[4]) {
  using T = typename IdxT<KIND>::T;
  const T* p = static_cast<const T*>(base) + row0;
  if (vec && row0 + 4 <= n) {
    if constexpr (sizeof(T) == 4) {
      const uint4 v = *reinterpret_cast<const uint4*>(p);
      out[0] = int64_t(T(v.x)); out[1] = int64_t(T(v.y)); out[2] = int64_t(T(v.z)); out[3] = int64_t(T(v.w));
    } else {
      const longlong2 a = reinterpret_cast<const longlong2*>(p)[0];
      const longlong2 b = reinterpret_cast<const longlong2*>(p)[1];
      out[0] = int64_t(T(a.x)); out[1] = int64_t(T(a.y)); out[2] = int64_t(T(b.x)); out[3] = int64_t(T(b.y));
    }
  } else {
#pragma unroll
    for (int j = 0; j < 4; j++) out[j] = (row0 + j < n) ? int64_t(p[j]) : 0;
  }
}

// OR of the 4-bit groups of the 8 lanes that share a 32-row bitmap word, delivered to all 8.
__device__ __forceinline__ uint32_t gather_word(uint32_t nib, int lane) {
  uint32_t w = nib << (4 * (lane & 7));
  w |= __shfl_xor_sync(0xffffffffu, w, 1);
  w |= __shfl_xor_sync(0xffffffffu, w, 2);
  w |= __shfl_xor_sync(0xffffffffu, w, 4);
  return w;
}

template <int KIND>
__global__ void __launch_bounds__(256) take_kernel(const __grid_constant__ TakeArgs a) {
  const int lane = threadIdx.x & 31;
  const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
  const uint64_t chunks = (a.n + 127) / 128;
  unsigned long long nulls[kMaxTakeCols];
#pragma unroll
  for (int c = 0; c < kMaxTakeCols; c++) nulls[c] = 0;

  for (uint64_t ch = uint64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); ch < chunks; ch += warps) {
    const uint64_t row0 = ch * 128 + uint64_t(lane) * 4;
    int64_t ix[4];
    load4<KIND>(a.idx, row0, a.idx_vec, a.n, ix);
    uint32_t ok = 0;          // bit j: row j exists, its index is valid and in range
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const uint64_t r = row0 + j;
      if (r >= a.n) continue;
      if (a.idx_valid && !bit_at(a.idx_valid, a.idx_voff + int64_t(r))) continue;
      if (ix[j] < 0 || uint64_t(ix[j]) >= a.src_len) {
        if (a.check) atomicOr(a.err, rs::ERR_TAKE_RANGE);
        continue;
      }
      ok |= 1u << j;
    }
    const bool full = row0 + 4 <= a.n;
    const uint32_t rows_mask = full ? 0xFu : ((1u << uint32_t(a.n > row0 ? a.n - row0 : 0)) - 1u);
    const uint64_t word = ch * 4 + (lane >> 3);

    for (int c = 0; c < a.ncols; c++) {
      const TakeCol& col = a.col[c];
      uint32_t vb = ok;
      if (col.src_valid) {
#pragma unroll
        for (int j = 0; j < 4; j++)
          if ((ok >> j) & 1u && !bit_at(col.src_valid, col.src_voff + ix[j])) vb &= ~(1u << j);
      }
      switch (col.width) {
        case 8: {
          const uint64_t* s = static_cast<const uint64_t*>(col.src);
          uint64_t v[4];
#pragma unroll
          for (int j = 0; j < 4; j++) v[j] = ((ok >> j) & 1u) ? s[ix[j]] : 0ull;
          uint64_t* d = static_cast<uint64_t*>(col.dst) + row0;
          if (full) {
            reinterpret_cast<ulonglong2*>(d)[0] = make_ulonglong2(v[0], v[1]);
            reinterpret_cast<ulonglong2*>(d)[1] = make_ulonglong2(v[2], v[3]);
          } else {
            for (int j = 0; j < 4; j++) if (row0 + j < a.n) d[j] = v[j];
          }
          break;
        }
        case 4: {
          const uint32_t* s = static_cast<const uint32_t*>(col.src);
          uint32_t v[4];
#pragma unroll
          for (int j = 0; j < 4; j++) v[j] = ((ok >> j) & 1u) ? s[ix[j]] : 0u;
          uint32_t* d = static_cast<uint32_t*>(col.dst) + row0;
          if (full) *reinterpret_cast<uint4*>(d) = make_uint4(v[0], v[1], v[2], v[3]);
          else for (int j = 0; j < 4; j++) if (row0 + j < a.n) d[j] = v[j];
          break;
        }
        case 2: {
          const uint16_t* s = static_cast<const uint16_t*>(col.src);
          uint16_t v[4];
#pragma unroll
          for (int j = 0; j < 4; j++) v[j] = ((ok >> j) & 1u) ? s[ix[j]] : uint16_t(0);
          uint16_t* d = static_cast<uint16_t*>(col.dst) + row0;
          if (full) *reinterpret_cast<uint2*>(d) = make_uint2(uint32_t(v[0]) | (uint32_t(v[1]) << 16), uint32_t(v[2]) | (uint32_t(v[3]) << 16));
          else for (int j = 0; j < 4; j++) if (row0 + j < a.n) d[j] = v[j];
          break;
        }
        case 1: {
          const uint8_t* s = static_cast<const uint8_t*>(col.src);
          uint8_t v[4];
#pragma unroll
          for (int j = 0; j < 4; j++) v[j] = ((ok >> j) & 1u) ? s[ix[j]] : uint8_t(0);
          uint8_t* d = static_cast<uint8_t*>(col.dst) + row0;
          if (full) *reinterpret_cast<uint32_t*>(d) = uint32_t(v[0]) | (uint32_t(v[1]) << 8) | (uint32_t(v[2]) << 16) | (uint32_t(v[3]) << 24);
          else for (int j = 0; j < 4; j++) if (row0 + j < a.n) d[j] = v[j];
          break;
        }
        default: {  // boolean: bit-packed values, gathered like the validity
          const uint8_t* s = static_cast<const uint8_t*>(col.src);
          uint32_t bits = 0;
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (((ok >> j) & 1u) && bit_at(s, col.src_bit_off + ix[j])) bits |= 1u << j;
          const uint32_t w = gather_word(bits, lane);
          if ((lane & 7) == 0) static_cast<uint32_t*>(col.dst)[word] = w;
          break;
        }
      }
      if (col.dst_valid) {
        const uint32_t w = gather_word(vb, lane);
        if ((lane & 7) == 0) col.dst_valid[word] = w;
        nulls[c] += __popc(rows_mask & ~vb);
      }
    }
  }
  // One atomic per warp and column for the null counts.
  for (int c = 0; c < a.ncols; c++) {
    if (!a.col[c].dst_valid) continue;
    unsigned long long v = nulls[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0 && v) atomicAdd(a.col[c].dst_nulls, v);
  }
}

}  // namespace tk

void launch_take(const tk::TakeArgs& a, cudaStream_t s) {
  if (a.n == 0) return;
  const uint64_t chunks = (a.n + 127) / 128;
  const int grid = int(std::min<uint64_t>((chunks + 7) / 8, uint64_t(device().sm_count) * 8));
  KernelTimer kt("take_gather", s);
  switch (a.idx_kind) {
    case tk::IDX_U32: tk::take_kernel<tk::IDX_U32><<<grid, 256, 0, s>>>(a); break;
    case tk::IDX_I32: tk::take_kernel<tk::IDX_I32><<<grid, 256, 0, s>>>(a); break;
    case tk::IDX_I64: tk::take_kernel<tk::IDX_I64><<<grid, 256, 0, s>>>(a); break;
    default: tk::take_kernel<tk::IDX_U64><<<grid, 256, 0, s>>>(a); break;
  }
  AM_CUDA(cudaGetLastError());
}

void take_columns(am_array* const* cols, int count, am_array* indices, am_array** outs, bool check_range,
                  cudaStream_t s) {
  using namespace tk;
  const int64_t n = indices->length;
  int kind;
  switch (indices->pt) {
    case PT_U32: kind = IDX_U32; break;
    case PT_I32: kind = IDX_I32; break;
    case PT_I64: kind = IDX_I64; break;
    case PT_U64: kind = IDX_U64; break;
    default: throw unsupported("take indices must be int32, int64 or uint32");
  }
  use_on(indices, s);
  for (int base = 0; base < count; base += kMaxTakeCols) {
    const int m0 = std::min(kMaxTakeCols, count - base);
    for (int c = 1; c < m0; c++)
      if (cols[base + c]->length != cols[base]->length) throw length_mismatch(cols[base]->length, cols[base + c]->length);
    const int m = std::min(kMaxTakeCols, count - base);
    TakeArgs a{};
    a.ncols = m;
    a.idx = indices->data();
    a.idx_kind = kind;
    a.idx_vec = (reinterpret_cast<uintptr_t>(a.idx) % 16) == 0;
    a.idx_valid = indices->null_count != 0 ? indices->valid_bits() : nullptr;
    a.idx_voff = indices->validity_offset;
    a.n = uint64_t(n);
    a.check = check_range ? 1 : 0;
    a.err = stream_scratch(s, 0).err;
    // Every column of one launch must have the same length (the index range check is shared).
    const int64_t src_len = cols[base]->length;
    a.src_len = uint64_t(src_len);
    const size_t words = size_t((n + 127) / 128) * 4;   // bitmap words, whole 128-row chunks
    for (int c = 0; c < m; c++) {
      am_array* src = cols[base + c];
      if (src->length != src_len) throw length_mismatch(src_len, src->length);
      use_on(src, s);
      am_array* o = outs[base + c];
      TakeCol& tc = a.col[c];
      tc.src = src->data();
      tc.src_valid = src->null_count != 0 ? src->valid_bits() : nullptr;
      tc.src_voff = src->validity_offset;
      tc.src_bit_off = src->pt == PT_BOOL ? src->value_offset : 0;
      tc.width = pt_bytes(src->pt);
      const size_t vbytes = tc.width == 0 ? words * 4 : size_t(std::max<int64_t>(n, 1)) * tc.width + 16;
      o->values = DevBuffer::alloc(vbytes, s);
      tc.dst = o->values->ptr;
      const bool nullable = tc.src_valid || a.idx_valid;
      if (nullable) {
        o->validity = DevBuffer::alloc(words * 4, s);
        o->null_count_dev = DevBuffer::alloc(sizeof(unsigned long long), s);
        AM_CUDA(cudaMemsetAsync(o->null_count_dev->ptr, 0, sizeof(unsigned long long), s));
        tc.dst_valid = static_cast<uint32_t*>(o->validity->ptr);
        tc.dst_nulls = static_cast<unsigned long long*>(o->null_count_dev->ptr);
        o->null_count = -1;
      } else {
        o->null_count = 0;
      }
      o->last_stream = s;
    }
    launch_take(a, s);
  }
}

}  // namespace am
