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

// Column c's value of row j, zero-extended (booleans as 0/1).
__device__ __forceinline__ uint64_t record_value(const RecArgs& r, int c, uint64_t j) {
  switch (r.width[c]) {
    case 8: return static_cast<const uint64_t*>(r.src[c])[j];
    case 4: return static_cast<const uint32_t*>(r.src[c])[j];
    case 2: return static_cast<const uint16_t*>(r.src[c])[j];
    case 1: return static_cast<const uint8_t*>(r.src[c])[j];
    default: return rec_bit(static_cast<const uint8_t*>(r.src[c]), r.src_bit_off[c] + int64_t(j)) ? 1u : 0u;
  }
}

// Row j's W-byte record: every column's value at its offset and the validity byte.
template <int W>
__device__ __forceinline__ void pack_record(const RecArgs& r, uint64_t j) {
  constexpr int WORDS = W / 8;
  uint64_t w[WORDS];
#pragma unroll
  for (int k = 0; k < WORDS; k++) w[k] = 0;
  uint32_t valid = 0;
#pragma unroll
  for (int c = 0; c < kMaxTakeCols; c++) {
    if (c >= r.ncols) break;
    const uint64_t v = record_value(r, c, j);
    const int o = r.rec_off[c];
#pragma unroll
    for (int k = 0; k < WORDS; k++)
      if ((o >> 3) == k) w[k] |= v << (8 * (o & 7));
    if (!r.src_valid[c] || rec_bit(r.src_valid[c], r.src_voff[c] + int64_t(j))) valid |= 1u << c;
  }
  if (r.valid_off >= 0) {
#pragma unroll
    for (int k = 0; k < WORDS; k++)
      if ((r.valid_off >> 3) == k) w[k] |= uint64_t(valid) << (8 * (r.valid_off & 7));
  }
  uint64_t* dst = static_cast<uint64_t*>(r.rec) + j * WORDS;
  if constexpr (WORDS == 1) {
    dst[0] = w[0];
  } else {
#pragma unroll
    for (int k = 0; k < WORDS; k += 2) reinterpret_cast<ulonglong2*>(dst)[k / 2] = make_ulonglong2(w[k], w[k + 1]);
  }
}
#endif

}  // namespace tk

void launch_take(const tk::TakeArgs& a, cudaStream_t s);

}  // namespace am
