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
#include <algorithm>
#include <type_traits>

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

// ---- row records

// Each thread packs H rows of a block's H x 256 consecutive rows, their loads in flight together.
template <int W>
__global__ void __launch_bounds__(256) pack_records_kernel(const __grid_constant__ RecArgs r) {
  constexpr int H = pack_rows_per_thread(W);
  const uint64_t step = uint64_t(gridDim.x) * (256 * H);
  for (uint64_t base = uint64_t(blockIdx.x) * (256 * H); base < r.n; base += step)
    pack_records_rows<W, H>(r, base + threadIdx.x);
}

template <int W>
__device__ __forceinline__ void load_record(const uint64_t* rec, uint64_t row, uint64_t (&w)[W / 8]) {
  const uint64_t* p = rec + row * (W / 8);
  if constexpr (W == 8) {
    w[0] = p[0];
  } else {
#pragma unroll
    for (int k = 0; k < W / 8; k += 2) {
      const ulonglong2 v = reinterpret_cast<const ulonglong2*>(p)[k / 2];
      w[k] = v.x;
      w[k + 1] = v.y;
    }
  }
}

// take_kernel with every column read from the packed records: per gathered row one record load. The
// index array is one this library produced (no nulls, in range).
// Bytes [o, o + bytes) of a record held in registers (o a multiple of bytes, so never across words).
template <int WORDS>
__device__ __forceinline__ uint64_t record_field(const uint64_t (&w)[WORDS], int o, int bytes) {
  const int k = o >> 3;
  uint64_t x = w[0];
#pragma unroll
  for (int q = 1; q < WORDS; q++) x = (k == q) ? w[q] : x;
  x >>= 8 * (o & 7);
  return bytes == 8 ? x : (x & ((uint64_t(1) << (8 * bytes)) - 1));
}

template <int KIND, int W>
__global__ void __launch_bounds__(256) take_records_kernel(const __grid_constant__ TakeArgs a,
                                                           const __grid_constant__ RecArgs r) {
  constexpr int WORDS = W / 8;
  const int lane = threadIdx.x & 31;
  const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
  const uint64_t chunks = (a.n + 127) / 128;
  const uint64_t* rec = static_cast<const uint64_t*>(r.rec);
  unsigned long long nulls[kMaxTakeCols];
#pragma unroll
  for (int c = 0; c < kMaxTakeCols; c++) nulls[c] = 0;

  for (uint64_t ch = uint64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); ch < chunks; ch += warps) {
    const uint64_t row0 = ch * 128 + uint64_t(lane) * 4;
    int64_t ix[4];
    load4<KIND>(a.idx, row0, a.idx_vec, a.n, ix);
    uint32_t ok = 0;
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (row0 + j < a.n && ix[j] >= 0 && uint64_t(ix[j]) < a.src_len) ok |= 1u << j;
    uint64_t w[4][WORDS];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if ((ok >> j) & 1u) load_record<W>(rec, uint64_t(ix[j]), w[j]);
      else {
#pragma unroll
        for (int k = 0; k < WORDS; k++) w[j][k] = 0;
      }
    }
    const bool full = row0 + 4 <= a.n;
    const uint32_t rows_mask = full ? 0xFu : ((1u << uint32_t(a.n > row0 ? a.n - row0 : 0)) - 1u);
    const uint64_t word = ch * 4 + (lane >> 3);
#define AM_FIELD(j, o, bytes) record_field<WORDS>(w[j], (o), (bytes))
    for (int c = 0; c < a.ncols; c++) {
      const TakeCol& col = a.col[c];
      uint32_t vb = ok;
      if (r.valid_off >= 0 && col.dst_valid) {
#pragma unroll
        for (int j = 0; j < 4; j++)
          if (!((AM_FIELD(j, r.valid_off, 1) >> c) & 1u)) vb &= ~(1u << j);
      }
      const int o = r.rec_off[c];
      switch (col.width) {
        case 8: {
          uint64_t* d = static_cast<uint64_t*>(col.dst) + row0;
          if (full) {
            reinterpret_cast<ulonglong2*>(d)[0] = make_ulonglong2(AM_FIELD(0, o, 8), AM_FIELD(1, o, 8));
            reinterpret_cast<ulonglong2*>(d)[1] = make_ulonglong2(AM_FIELD(2, o, 8), AM_FIELD(3, o, 8));
          } else {
#pragma unroll
            for (int j = 0; j < 4; j++) if (row0 + j < a.n) d[j] = AM_FIELD(j, o, 8);
          }
          break;
        }
        case 4: {
          uint32_t* d = static_cast<uint32_t*>(col.dst) + row0;
          if (full) *reinterpret_cast<uint4*>(d) = make_uint4(uint32_t(AM_FIELD(0, o, 4)), uint32_t(AM_FIELD(1, o, 4)),
                                                             uint32_t(AM_FIELD(2, o, 4)), uint32_t(AM_FIELD(3, o, 4)));
          else _Pragma("unroll") for (int j = 0; j < 4; j++) if (row0 + j < a.n) d[j] = uint32_t(AM_FIELD(j, o, 4));
          break;
        }
        case 2: {
          uint16_t* d = static_cast<uint16_t*>(col.dst) + row0;
          if (full) *reinterpret_cast<uint2*>(d) = make_uint2(uint32_t(AM_FIELD(0, o, 2)) | (uint32_t(AM_FIELD(1, o, 2)) << 16),
                                                             uint32_t(AM_FIELD(2, o, 2)) | (uint32_t(AM_FIELD(3, o, 2)) << 16));
          else _Pragma("unroll") for (int j = 0; j < 4; j++) if (row0 + j < a.n) d[j] = uint16_t(AM_FIELD(j, o, 2));
          break;
        }
        case 1: {
          uint8_t* d = static_cast<uint8_t*>(col.dst) + row0;
          if (full) *reinterpret_cast<uint32_t*>(d) = uint32_t(AM_FIELD(0, o, 1)) | (uint32_t(AM_FIELD(1, o, 1)) << 8) |
                                                      (uint32_t(AM_FIELD(2, o, 1)) << 16) | (uint32_t(AM_FIELD(3, o, 1)) << 24);
          else _Pragma("unroll") for (int j = 0; j < 4; j++) if (row0 + j < a.n) d[j] = uint8_t(AM_FIELD(j, o, 1));
          break;
        }
        default: {  // boolean: the record's 0/1 byte
          uint32_t bits = 0;
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (((ok >> j) & 1u) && AM_FIELD(j, o, 1)) bits |= 1u << j;
          const uint32_t wd = gather_word(bits, lane);
          if ((lane & 7) == 0) static_cast<uint32_t*>(col.dst)[word] = wd;
          break;
        }
      }
      if (col.dst_valid) {
        const uint32_t wd = gather_word(vb, lane);
        if ((lane & 7) == 0) col.dst_valid[word] = wd;
        nulls[c] += __popc(rows_mask & ~vb);
      }
    }
  }
  for (int c = 0; c < a.ncols; c++) {
    if (!a.col[c].dst_valid) continue;
    unsigned long long v = nulls[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0 && v) atomicAdd(a.col[c].dst_nulls, v);
  }
}
#undef AM_FIELD

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

// Gathers through row records pay off when the sources are far larger than L2 (each random read then
// costs a DRAM burst) and most of their rows are gathered (the records are built from every row).
constexpr uint64_t kRecordMinSourceBytes = uint64_t(256) << 20;

// Record width (8, 16 or 32) for gathering these columns through row records, or 0 for the direct
// gather: at least two columns, indices that need no checks, rows that fit 32 bytes.
static int record_bytes(am_array* const* cols, int m, bool checked, int64_t n) {
  if (m < 2 || checked) return 0;
  const int64_t src_len = cols[0]->length;
  if (n < src_len / 2) return 0;
  int bytes = 0;
  bool nullable = false;
  for (int c = 0; c < m; c++) {
    bytes += std::max(pt_bytes(cols[c]->pt), 1);
    if (cols[c]->null_count != 0) nullable = true;
  }
  if (uint64_t(src_len) * uint64_t(bytes) < kRecordMinSourceBytes) return 0;
  bytes += nullable ? 1 : 0;
  return bytes <= 8 ? 8 : bytes <= 16 ? 16 : bytes <= 32 ? 32 : 0;
}

// The record layout of a TakeArgs' columns: widest first, so every field sits at a multiple of its
// width; the validity byte last when any column has nulls.
static void layout_records(const tk::TakeArgs& a, tk::RecArgs& r) {
  using namespace tk;
  r.ncols = a.ncols;
  r.n = a.src_len;
  int order[kMaxTakeCols];
  for (int c = 0; c < a.ncols; c++) order[c] = c;
  std::stable_sort(order, order + a.ncols, [&](int x, int y) { return a.col[x].width > a.col[y].width; });
  int off = 0;
  bool nullable = false;
  for (int k = 0; k < a.ncols; k++) {
    const int c = order[k];
    r.rec_off[c] = off;
    off += std::max(a.col[c].width, 1);
  }
  for (int c = 0; c < a.ncols; c++) {
    r.src[c] = a.col[c].src;
    r.src_valid[c] = a.col[c].src_valid;
    r.src_voff[c] = a.col[c].src_voff;
    r.src_bit_off[c] = a.col[c].src_bit_off;
    r.width[c] = a.col[c].width;
    if (a.col[c].src_valid) nullable = true;
  }
  r.valid_off = nullable ? off : -1;
}

static void take_through_records(const tk::TakeArgs& a, int rec_w, cudaStream_t s) {
  using namespace tk;
  RecArgs r{};
  layout_records(a, r);
  r.rec = dmalloc(size_t(a.src_len) * size_t(rec_w), s);
  const uint64_t pack_chunk = 256 * uint64_t(pack_rows_per_thread(rec_w));
  const int pack_grid = int(std::min<uint64_t>((a.src_len + pack_chunk - 1) / pack_chunk, uint64_t(device().sm_count) * 16));
  const uint64_t chunks = (a.n + 127) / 128;
  const int grid = int(std::min<uint64_t>((chunks + 7) / 8, uint64_t(device().sm_count) * 8));
  {
    KernelTimer kt("take_pack_records", s);
    switch (rec_w) {
      case 8: pack_records_kernel<8><<<std::max(pack_grid, 1), 256, 0, s>>>(r); break;
      case 16: pack_records_kernel<16><<<std::max(pack_grid, 1), 256, 0, s>>>(r); break;
      default: pack_records_kernel<32><<<std::max(pack_grid, 1), 256, 0, s>>>(r); break;
    }
    AM_CUDA(cudaGetLastError());
  }
  {
    KernelTimer kt("take_gather_records", s);
    auto go = [&](auto kind_tag) {
      constexpr int KIND = decltype(kind_tag)::value;
      switch (rec_w) {
        case 8: take_records_kernel<KIND, 8><<<std::max(grid, 1), 256, 0, s>>>(a, r); break;
        case 16: take_records_kernel<KIND, 16><<<std::max(grid, 1), 256, 0, s>>>(a, r); break;
        default: take_records_kernel<KIND, 32><<<std::max(grid, 1), 256, 0, s>>>(a, r); break;
      }
    };
    switch (a.idx_kind) {
      case IDX_U32: go(std::integral_constant<int, IDX_U32>{}); break;
      case IDX_I32: go(std::integral_constant<int, IDX_I32>{}); break;
      case IDX_I64: go(std::integral_constant<int, IDX_I64>{}); break;
      default: go(std::integral_constant<int, IDX_U64>{}); break;
    }
    AM_CUDA(cudaGetLastError());
  }
  dfree(r.rec, s);
}

void take_columns(am_array* const* cols_in, int count_in, am_array* indices, am_array** outs_in, bool check_range,
                  cudaStream_t s) {
  using namespace tk;
  // String columns have their own gather; the fixed-width ones share the launches below.
  std::vector<am_array*> fixed_cols, fixed_outs;
  for (int c = 0; c < count_in; c++) {
    if (cols_in[c]->pt == PT_STRUCT) throw unsupported("+s: a struct result is exported, not computed on");
    if (cols_in[c]->dictionary && !outs_in[c]->dictionary) {
      // The codes move; the dictionary is shared.
      retain(cols_in[c]->dictionary);
      outs_in[c]->dictionary = cols_in[c]->dictionary;
    }
    if (pt_var(cols_in[c]->pt)) {
      take_strings(cols_in[c], indices, outs_in[c], check_range, s);
    } else {
      fixed_cols.push_back(cols_in[c]);
      fixed_outs.push_back(outs_in[c]);
    }
  }
  am_array* const* cols = fixed_cols.data();
  am_array** outs = fixed_outs.data();
  const int count = int(fixed_cols.size());
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
    const int rec_w = record_bytes(cols + base, m, check_range || a.idx_valid != nullptr, n);
    if (rec_w) take_through_records(a, rec_w, s);
    else launch_take(a, s);
  }
}

}  // namespace am
