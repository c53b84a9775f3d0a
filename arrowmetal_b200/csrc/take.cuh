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

}  // namespace tk

void launch_take(const tk::TakeArgs& a, cudaStream_t s);

}  // namespace am
