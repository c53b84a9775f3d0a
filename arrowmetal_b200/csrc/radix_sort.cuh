// Shared layouts of the radix sort's kernels (radix_sort.cu) and the segmented form (segmented.cu).
#pragma once

#include <stdint.h>

namespace am {
namespace rs {

constexpr int RADIX = 256;                 // 8-bit digits: 4 passes for a 32-bit key, 8 for a 64-bit one
constexpr int NAN_BIN = 256;               // routing bins of the most significant key's first pass
constexpr int NULL_BIN = 257;
constexpr int NBINS = 258;
constexpr uint32_t INVALID_DIGIT = 0xFFFFu;
constexpr int MAX_KEYS = 16;
constexpr int MAX_SLOTS = MAX_KEYS * 9;

constexpr int FO_IEEE = 0, FO_TOTAL = 1, FO_NANLARGEST = 2;

// Pass flags.
constexpr uint32_t PF_ENCODE = 1;          // first pass of a key: read the column (through the ids)
constexpr uint32_t PF_ROUTE = 2;           // most significant key: null / NaN rows go straight out
constexpr uint32_t PF_CATPASS = 4;         // a lower key's null category, looked up by row id
constexpr uint32_t PF_WIDE_OUT = 8;        // the output index array is uint64
constexpr uint32_t PF_LAST = 16;           // the last pass: rows reach their final places
constexpr uint32_t PF_BUCKETS = 32;        // two-level sort's second pass: count its (digit, lower digit) buckets

// Look-back status word: epoch (30 bits) | flag (2 bits) | count (32 bits).
constexpr uint32_t ST_AGG = 1, ST_INCL = 2;
constexpr uint64_t LOOKBACK_TIMEOUT_NS = 1000000000ull;   // 1 s, then the pass reports an error

// Device error word bits.
constexpr uint32_t ERR_LOOKBACK_TIMEOUT = 1;
constexpr uint32_t ERR_TAKE_RANGE = 2;
constexpr uint32_t ERR_BOUNDS = 4;                        // a kernel computed a destination outside its array
constexpr uint32_t ERR_DICT_CODE = 8;                     // a dictionary code outside its dictionary

// One key column as the kernels read it.
struct ColView {
  const void* values;        // row 0 (bool: the bitmap, row 0 at bit bool_off)
  const uint8_t* valid;      // NULL: no nulls
  int64_t valid_off;         // bit of row 0 in `valid`
  int64_t bool_off;
  int32_t pt;                // am::PhysType
  uint8_t desc;
  uint8_t nulls_first;
  uint8_t float_order;
  uint8_t nan_cat;           // ieee float: NaN rows form their own block
};

struct KeyStats {
  uint32_t hist[8][256];     // per digit position, counts of the value keys
  uint32_t n_value, n_null, n_nan, pad;
  unsigned long long vmax, vmin_inv;
};

struct KeyPlan {
  unsigned long long fold_nan, fold_null;   // keys given to a lower key's NaN / null rows
  uint32_t fold_mode;                       // 1: no room in the key range, a category pass follows
  uint32_t pad;
};

struct PassDesc {
  uint32_t active, flags, count, shift;
  int32_t src_keys, src_ids, dst_keys, dst_ids;   // -1: none / identity / the output array
  uint32_t value_base, key;
  uint32_t buf_rows, out_rows;                    // bounds of the key / id buffers and of the output
  uint32_t bucket_shift;                          // PF_BUCKETS: the lower bucket digit's shift
  uint32_t pad2;
  uint32_t bin_base[NBINS];
};

struct SortSummary {
  uint32_t value_rows, null_rows, nan_rows, passes_run, passes_total, pad[3];
};

struct PlanArgs {
  uint64_t n;
  uint64_t hyb_min_rows;                    // value rows from which one 8-byte key takes the two-level sort
  int32_t nkeys, nslots, slot_key0_first, index_wide;
  uint8_t key_bytes[MAX_KEYS];
  uint8_t nulls_first[MAX_KEYS];
  int8_t slot_key[MAX_SLOTS];
  int8_t slot_digit[MAX_SLOTS];             // -1: category pass
};

// One array of a segmented (batched) sort. The batch's arrays of one key width share one launch per
// digit pass; each has its own plan and pass descriptors, and its rows sit at `row_off` in the group's
// ping-pong buffers.
struct SegDesc {
  ColView col;
  uint64_t row_off;
  void* out;                 // its uint32 index array
  uint32_t n;
  uint32_t pad;
};

// Payload columns that ride through the sort with their rows (instead of a gather through the
// permutation afterwards). A row's record is 16 bytes: word 0 its row id, bytes 4-15 its payload
// fields, each at a multiple of its width (at most one 8-byte field, at byte 4). The first pass builds
// each row's record from the columns; every later pass moves records; whatever writes a row to its
// final place (the last pass, the local sorts, the first pass for null rows) unpacks its record into
// the sorted payload columns. Payload columns are fixed-width without nulls.
constexpr int REC_MAX_COLS = 4;
constexpr int REC_PAYLOAD_BYTES = 12;
struct RecLayout {
  const void* src[REC_MAX_COLS];      // row 0 of each payload column
  void* dst[REC_MAX_COLS];            // row 0 of each sorted payload column
  int32_t width[REC_MAX_COLS];        // 1, 2, 4 or 8 bytes
  int32_t off[REC_MAX_COLS];          // byte offset within the payload (0-11)
  int32_t ncols;
  int32_t pair;                       // 1: exactly an 8-byte column (wide) and a 4-byte one (narrow)
  int32_t wide, narrow;               // their column numbers, when `pair`
};

// key_out modes: the sorted key column itself, produced by inverting the key map in the last pass.
constexpr int KEY_OUT_NONE = 0, KEY_OUT_UNKEY = 1;

struct PassArgs {
  const PassDesc* desc;
  const KeyPlan* kplan;
  void* keys[2];
  uint32_t* ids[2];
  void* final_out;            // the index output (NULL: none wanted)
  void* status;
  uint32_t* tile_counter;
  uint32_t* err;
  uint32_t epoch;
  int32_t carry_ids;          // 0: row ids are never stored (a sorted copy only)
  int32_t key_out_mode;
  int32_t key_out_pt;         // physical type of the key column (for the inverse map)
  int32_t key_desc;
  int32_t key_float_order;
  void* key_out;              // sorted key values
  // PF_BUCKETS passes: 65,536 row counts, one per (this pass's digit, lower digit) bucket.
  uint32_t* bucket_count;
  // Segmented passes: `desc` and `kplan` are per-segment arrays (desc[seg * nslots + slot]); tile T of
  // the launch belongs to the segment s with tile_start[s] <= T < tile_start[s + 1].
  const SegDesc* segs;
  const uint32_t* tile_start;
  uint32_t nsegs, total_tiles, slot, nslots;
  // Record passes (`ids` then hold 16-byte records, see RecLayout): the payload's layout.
  int32_t rec_mode;
  int32_t pad_rec;
  RecLayout rec;
};

}  // namespace rs
}  // namespace am
