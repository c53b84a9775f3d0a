// Launch layout of the take/gather kernel (take.cu).
#pragma once

#include <stdint.h>

namespace am {
namespace tk {

constexpr int kMaxTakeCols = 8;
constexpr int IDX_U32 = 0, IDX_I32 = 1, IDX_I64 = 2, IDX_U64 = 3;

struct TakeCol {
  const void* src;
  const uint8_t* src_valid;       // NULL: the source has no nulls
  int64_t src_voff;               // bit of source row 0 in src_valid
  int64_t src_bit_off;            // boolean sources: bit of row 0 in src
  int32_t width;                  // bytes per value; 0 for boolean
  void* dst;
  uint32_t* dst_valid;            // NULL: the output has no nulls
  unsigned long long* dst_nulls;  // null count of the output, accumulated
};

struct TakeArgs {
  TakeCol col[kMaxTakeCols];
  int32_t ncols;
  int32_t idx_kind;
  int32_t idx_vec;                // index array 16-byte aligned: 128-bit loads
  int32_t check;                  // flag an out-of-range index in *err
  const void* idx;
  const uint8_t* idx_valid;
  int64_t idx_voff;
  uint64_t n;
  uint64_t src_len;
  uint32_t* err;
};

// Row records: the columns of a multi-column gather packed row by row, so that one random read of a
// record (8, 16 or 32 bytes: one DRAM burst) fetches every column of a gathered row instead of one
// burst per column. Column c sits at byte rec_off[c] (booleans as a 0/1 byte); bit c of the byte at
// valid_off is the row's validity of column c.
struct RecArgs {
  const void* src[kMaxTakeCols];
  const uint8_t* src_valid[kMaxTakeCols];
  int64_t src_voff[kMaxTakeCols];
  int64_t src_bit_off[kMaxTakeCols];
  int32_t width[kMaxTakeCols];    // bytes per value; 0 for boolean (a byte in the record)
  int32_t rec_off[kMaxTakeCols];
  int32_t ncols;
  int32_t valid_off;              // -1: no column has nulls
  uint64_t n;                     // source rows
  void* rec;
};

#ifdef __CUDACC__
__device__ __forceinline__ bool rec_bit(const uint8_t* p, int64_t i) { return (p[i >> 3] >> (i & 7)) & 1; }

// Rows a thread packs per grid-stride step, 256 rows apart: a W-byte record per row.
__host__ __device__ constexpr int pack_rows_per_thread(int w) { return w == 8 ? 8 : 4; }

// Records of rows j0, j0 + 256, ..., j0 + 256 (H - 1): every column's value at its offset and the
// validity byte. All H rows of a column are loaded before anything is stored, so each thread keeps H
// loads in flight: a store between rows would order the next row's loads after it (the record buffer
// is not known to be apart from the columns), one DRAM round trip per row.
template <int W, int H>
__device__ __forceinline__ void pack_records_rows(const RecArgs& r, uint64_t j0) {
  constexpr int WORDS = W / 8;
  uint64_t w[H][WORDS];
  uint32_t valid[H];
  bool in[H];
#pragma unroll
  for (int h = 0; h < H; h++) {
    in[h] = j0 + uint64_t(h) * 256 < r.n;
    valid[h] = 0;
#pragma unroll
    for (int k = 0; k < WORDS; k++) w[h][k] = 0;
  }
#pragma unroll 1
  for (int c = 0; c < kMaxTakeCols; c++) {
    if (c >= r.ncols) break;
    uint64_t v[H];
    switch (r.width[c]) {
      case 8: {
        const uint64_t* src = static_cast<const uint64_t*>(r.src[c]);
#pragma unroll
        for (int h = 0; h < H; h++) v[h] = in[h] ? src[j0 + uint64_t(h) * 256] : 0;
        break;
      }
      case 4: {
        const uint32_t* src = static_cast<const uint32_t*>(r.src[c]);
#pragma unroll
        for (int h = 0; h < H; h++) v[h] = in[h] ? src[j0 + uint64_t(h) * 256] : 0;
        break;
      }
      case 2: {
        const uint16_t* src = static_cast<const uint16_t*>(r.src[c]);
#pragma unroll
        for (int h = 0; h < H; h++) v[h] = in[h] ? src[j0 + uint64_t(h) * 256] : 0;
        break;
      }
      case 1: {
        const uint8_t* src = static_cast<const uint8_t*>(r.src[c]);
#pragma unroll
        for (int h = 0; h < H; h++) v[h] = in[h] ? src[j0 + uint64_t(h) * 256] : 0;
        break;
      }
      default: {   // boolean: bit-packed values, a 0/1 byte in the record
        const uint8_t* src = static_cast<const uint8_t*>(r.src[c]);
#pragma unroll
        for (int h = 0; h < H; h++)
          v[h] = (in[h] && rec_bit(src, r.src_bit_off[c] + int64_t(j0 + uint64_t(h) * 256))) ? 1u : 0u;
        break;
      }
    }
    const int o = r.rec_off[c];
    const uint8_t* vb = r.src_valid[c];
    // Word masks instead of a branch per word: the record stays in registers.
    uint64_t wm[WORDS];
#pragma unroll
    for (int k = 0; k < WORDS; k++) wm[k] = uint64_t(0) - uint64_t((o >> 3) == k);
#pragma unroll
    for (int h = 0; h < H; h++) {
      const uint64_t sh = v[h] << (8 * (o & 7));
#pragma unroll
      for (int k = 0; k < WORDS; k++) w[h][k] |= sh & wm[k];
      if (!vb || (in[h] && rec_bit(vb, r.src_voff[c] + int64_t(j0 + uint64_t(h) * 256)))) valid[h] |= 1u << c;
    }
  }
  if (r.valid_off >= 0) {
    uint64_t wm[WORDS];
#pragma unroll
    for (int k = 0; k < WORDS; k++) wm[k] = uint64_t(0) - uint64_t((r.valid_off >> 3) == k);
#pragma unroll
    for (int h = 0; h < H; h++)
#pragma unroll
      for (int k = 0; k < WORDS; k++) w[h][k] |= (uint64_t(valid[h]) << (8 * (r.valid_off & 7))) & wm[k];
  }
  uint64_t* rec = static_cast<uint64_t*>(r.rec);
#pragma unroll
  for (int h = 0; h < H; h++) {
    if (!in[h]) continue;
    uint64_t* dst = rec + (j0 + uint64_t(h) * 256) * WORDS;
    if constexpr (WORDS == 1) {
      dst[0] = w[h][0];
    } else {
#pragma unroll
      for (int k = 0; k < WORDS; k += 2) reinterpret_cast<ulonglong2*>(dst)[k / 2] = make_ulonglong2(w[h][k], w[h][k + 1]);
    }
  }
}
#endif

}  // namespace tk

void launch_take(const tk::TakeArgs& a, cudaStream_t s);

}  // namespace am
