// Internal declarations of libArrowMetalC for B200: the device runtime (one CUDA device, a stream per
// calling thread, stream-ordered allocation from the device memory pool, a pinned host pool), the
// HBM-resident array handle behind `am_array*`, and the entry points of the sort and take engines.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <array>
#include <vector>

#include "../../include/arrowmetal.h"

#ifdef __CUDACC__
#define AM_HD __host__ __device__
#else
#define AM_HD
#endif

namespace am {

// ---------------------------------------------------------------------------------------------
// Errors. Internal code throws; every extern "C" entry point catches and turns the exception into
// the reference's return-code convention (Sources/ArrowMetalC/ArrowMetalC.swift:9-34).

struct Error : std::runtime_error {
  int code;
  explicit Error(const std::string& m, int c = 1) : std::runtime_error(m), code(c) {}
};

// The reference's ArrowMetalError descriptions (Sources/ArrowMetal/MetalContext.swift:19-27).
inline Error invalid(const std::string& m) { return Error("Invalid ArrowArray: " + m); }
inline Error unsupported(const std::string& m) { return Error("Unsupported Arrow type: " + m); }
inline Error length_mismatch(int64_t a, int64_t b) {
  return Error("Array length mismatch: " + std::to_string(a) + " vs " + std::to_string(b));
}

void cuda_check(cudaError_t e, const char* what);
#define AM_CUDA(x) ::am::cuda_check((x), #x)

void set_last_error(const std::string& m);

// ---------------------------------------------------------------------------------------------
// Device runtime.

struct Device {
  int ordinal = 0;
  int sm_count = 0;
  std::string name;
  cudaMemPool_t pool = nullptr;
};
Device& device();                       // initialises on first use; throws when no CUDA device
cudaStream_t stream();                  // the calling thread's stream (override or its own)
cudaStream_t copy_stream();             // the calling thread's stream for asynchronous host copies
cudaStream_t d2h_stream();              // the calling thread's stream for exports that need not wait
// An event recorded when an array's contents were complete; copies of the array wait for it alone.
struct ReadyEvent {
  cudaEvent_t ev = nullptr;
  explicit ReadyEvent(cudaStream_t s);
  ~ReadyEvent();
};
// Runs `fn` on a library thread once `ev` (recorded by the caller) has completed, then destroys `ev`:
// a producer's buffers are released as soon as the copies reading them are done.
void release_after(cudaEvent_t ev, std::function<void()> fn);
void set_stream_override(cudaStream_t s);
cudaStream_t stream_override();

// Stream-ordered device allocation from the device's memory pool (kept reserved between calls).
void* dmalloc(size_t bytes, cudaStream_t s);
void dfree(void* p, cudaStream_t s);
void debug_fail_alloc_after(int64_t n);
void debug_skip_first_tile(bool on);
bool debug_skip_first_tile();

// A device allocation, or a borrowed device range with a custom release.
struct DevBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;          // the stream its last writer / reader used
  // A library stream the memory goes back to the pool on (after the last user's work): imports are
  // allocated on the copy stream, and their memory freed there is what the next imports reuse.
  cudaStream_t home = nullptr;
  std::function<void()> on_release;       // borrowed memory: runs the producer's release
  bool owned = false;
  // Set once a low-cardinality probe of rows in this buffer found more than 256 distinct keys: later
  // sorts of it, or of slices of it, skip the probe (and its readback).
  std::atomic<bool> many_values{false};
  DevBuffer() = default;
  DevBuffer(const DevBuffer&) = delete;
  DevBuffer& operator=(const DevBuffer&) = delete;
  ~DevBuffer();
  static std::shared_ptr<DevBuffer> alloc(size_t bytes, cudaStream_t s);
};
using BufPtr = std::shared_ptr<DevBuffer>;

// Pinned host memory from a caching pool (export buffers and staging).
void* pinned_alloc(size_t bytes);
void pinned_free(void* p);

// Host threads used by the staged host copies (am_set_import_threads).
int import_threads();
void set_import_threads(int n);
// Host <-> device copies of user memory: pinned sources copy directly; pageable ones go through a
// ring of pinned staging slots filled by `import_threads()` host threads. copy_h2d returns true when
// the copy may still read `src` after it returns (a pinned source): the caller keeps it alive.
bool copy_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s);
bool is_pinned(const void* p);          // page-locked host memory the GPU reads directly
void copy_d2h(void* dst, const void* src, size_t bytes, cudaStream_t s);

// Per-thread state.
struct ThreadState {
  std::string last_error;
  int batch_depth = 0;
  cudaStream_t override_stream = nullptr;
  cudaStream_t own_stream = nullptr;
  cudaStream_t copy_stream = nullptr;                    // asynchronous imports from pinned memory
  cudaStream_t d2h_stream = nullptr;                     // exports of arrays that carry a ready event
  am_sort_stats last_stats{};
  cudaStream_t stats_stream = nullptr;                   // the last sort's counters are copied here
  std::vector<std::function<void()>> deferred_checks;   // run at the batch's end
  std::string scratch_text;                              // am_plan_explain result
};
ThreadState& tls();

// Per-stream persistent scratch: the radix sort's look-back status words (zeroed once when grown,
// then told apart by a per-stream epoch), and a device error word kernels OR into.
struct StreamScratch {
  uint64_t* status = nullptr;
  size_t status_words = 0;
  uint32_t epoch = 0;
  uint32_t* err = nullptr;
  // The sorts' working buffers, kept for the stream's next sort (up to kArenaMax bytes): repeated sorts
  // neither return them to the pool nor ask it again, so the pool's blocks are not split between the
  // sort's scratch and the results allocated after it.
  void* arena = nullptr;
  size_t arena_bytes = 0;
  std::atomic<bool> arena_busy{false};   // held by one sort at a time (threads may share a stream)
};
constexpr size_t kArenaMax = size_t(4) << 30;
StreamScratch& stream_scratch(cudaStream_t s, size_t status_words);
// A stream's sort scratch of `bytes`: its arena when free and large enough (grown when it is not),
// else a block of its own; released (back to the arena, or freed) on the stream when it goes away.
class ScratchBlock {
 public:
  ScratchBlock(cudaStream_t s, size_t bytes);
  ~ScratchBlock();
  ScratchBlock(const ScratchBlock&) = delete;
  ScratchBlock& operator=(const ScratchBlock&) = delete;
  char* data() const { return p_; }
 private:
  cudaStream_t s_;
  char* p_ = nullptr;
  StreamScratch* arena_ = nullptr;
};
// Reads and clears the stream's device error word (synchronises the stream); throws on an error.
void check_device_errors(cudaStream_t s);
void sync_stream(cudaStream_t s);

// Kernel timing (am_cuda_profile).
bool profiling();
void set_profiling(bool on);
struct KernelTimer {
  const char* name;
  cudaStream_t s;
  cudaEvent_t a = nullptr, b = nullptr;
  KernelTimer(const char* n, cudaStream_t st);
  ~KernelTimer();
};
void profile_collect();
struct ProfileEntry { std::string name; int64_t launches; double total_ms; };
std::vector<ProfileEntry> profile_entries();
void profile_reset();

// ---------------------------------------------------------------------------------------------
// Arrow types the sort path carries.

enum PhysType : int32_t {
  PT_BOOL = 0, PT_I8, PT_U8, PT_I16, PT_U16, PT_I32, PT_U32, PT_I64, PT_U64, PT_F16, PT_F32, PT_F64,
  PT_STR,    // variable-size bytes (utf8 "u", binary "z") with int32 offsets
  PT_LSTR,   // the same with int64 offsets (large_utf8 "U", large_binary "Z")
  PT_STRUCT, // a struct of child arrays ("+s"): value_counts' result, exported only
};
// Bytes per value; for the variable-size types, bytes per offset.
AM_HD inline int pt_bytes(int pt) {
  switch (pt) {
    case PT_BOOL: return 0;   // bit-packed
    case PT_I8: case PT_U8: return 1;
    case PT_I16: case PT_U16: case PT_F16: return 2;
    case PT_I32: case PT_U32: case PT_F32: case PT_STR: return 4;
    default: return 8;
  }
}
AM_HD inline bool pt_var(int pt) { return pt == PT_STR || pt == PT_LSTR; }
AM_HD inline bool pt_float(int pt) { return pt == PT_F16 || pt == PT_F32 || pt == PT_F64; }
AM_HD inline int pt_key_bytes(int pt) { return pt_bytes(pt) == 8 ? 8 : 4; }
// Parses an Arrow C Data Interface format string; throws unsupported for the types this build does
// not carry (strings, nested, dictionary, decimal, intervals).
int parse_format(const char* fmt);

// ---------------------------------------------------------------------------------------------
// The array handle.

}  // namespace am

struct am_array {
  std::atomic<int64_t> refs{1};
  int32_t pt = 0;
  std::string format;
  int64_t length = 0;
  int64_t null_count = 0;             // -1: being counted on the device (null_count_dev)
  am::BufPtr values;                  // element 0 sits at values->ptr + value_offset * width (strings: offsets)
  am::BufPtr bytes;                   // strings: the bytes the offsets point into
  int64_t value_offset = 0;           // elements (bits for bool)
  am::BufPtr validity;                // may be null: no nulls
  int64_t validity_offset = 0;        // bits
  am::BufPtr null_count_dev;          // unsigned long long, when null_count == -1
  cudaStream_t last_stream = nullptr;
  // >= 0 when this is an index array this library produced: no nulls and every index < perm_of.
  int64_t perm_of = -1;
  // Settled and read by many streams at once (a served table's columns): its contents are complete,
  // so readers neither wait for nor record a stream; its buffers outlive every reader, which holds
  // them through its own slices.
  bool shared_read = false;
  // Recorded on last_stream when the contents were complete (optional): an export waits for it alone,
  // not for later work on that stream.
  std::shared_ptr<am::ReadyEvent> ready;
  // A dictionary-encoded array: `pt` / `format` / `values` are its integer codes and this is the
  // dictionary they index (a flat array, one reference owned). Sorts order by the values; takes and
  // slices move the codes and share the dictionary.
  am_array* dictionary = nullptr;
  // PT_STRUCT: the fields, owned (one reference each), and their names.
  std::vector<am_array*> children;
  std::vector<std::string> child_names;

  const void* data() const {
    if (!values) return nullptr;
    int w = am::pt_bytes(pt);
    if (w == 0) return values->ptr;
    return static_cast<const char*>(values->ptr) + value_offset * w;
  }
  const uint8_t* valid_bits() const {
    return validity ? static_cast<const uint8_t*>(validity->ptr) : nullptr;
  }
};

namespace am {

am_array* new_array(int pt, const std::string& format, int64_t length);
void retain(am_array* a);
void release(am_array* a);
// Orders the calling stream after the last work that touched `a` (when it ran on another stream).
void use_on(am_array* a, cudaStream_t s);
int64_t resolve_null_count(am_array* a);     // waits for a pending device count
std::string format_of(int pt);

// ---------------------------------------------------------------------------------------------
// Engines.

// Key options of one sort key (the reference's descending / NullPlacement / FloatOrder,
// Sources/ArrowMetal/ComputeOptions.swift:15-60).
struct SortKey {
  am_array* col = nullptr;
  bool descending = false;
  bool nulls_first = false;
  int float_order = 0;                 // 0 ieee, 1 total, 2 nan_largest
};
// Stable multi-key argsort; keys[0] is the most significant. Writes n row numbers of `index_width`
// bytes (4 or 8) into `out` (device memory) on stream `s`.
void radix_argsort(const std::vector<SortKey>& keys, int64_t n, void* out, int index_width,
                   cudaStream_t s, am_sort_stats* stats);

namespace rs { struct KeyStats; struct ColView; struct RecLayout; ColView make_view(const SortKey& k); }
// The key column's statistics (all digit histograms of its value keys, null / NaN / value counts)
// into `st` on the device.
void key_statistics(const SortKey& k, rs::KeyStats* st, cudaStream_t s);
// The first min(k, rows) indices of the stable argsort of `key`, by radix selection; NULL when a full
// sort is the better way (k close to the number of value rows).
am_array* radix_top_k(const SortKey& key, int64_t k, cudaStream_t s);

// A dense-rank column (uint8) of an integer key with at most 256 distinct value keys and at least 4M
// rows, ranked in the key's own order (its direction included; nulls kept), or NULL. Sorting it
// ascending orders the rows as the key does.
am_array* low_cardinality_ranks(const SortKey& k, cudaStream_t s);
// True when the key column can be rebuilt from its sorted keys (the key map is a bijection).
bool key_invertible(const SortKey& k);
// The sort engine. `out` (may be NULL) receives the index array; `key_dst` (may be NULL; one
// key_invertible key only) receives the sorted key column, rebuilt from the sorted keys by the last
// pass, so a sorted copy of the key needs no gather. `payload` (may be NULL; one key only): payload
// columns carried through the sort in row records and written, sorted, to their destinations.
void radix_sort(const std::vector<SortKey>& keys, int64_t n, void* out, int index_width, am_array* key_dst,
                cudaStream_t s, am_sort_stats* stats, const rs::RecLayout* payload = nullptr);
// The row-record layout of payload columns (RecLayout without its destinations), or false when they
// cannot ride in a record: at most four fixed-width columns without nulls, twelve bytes in all.
bool payload_record_layout(const std::vector<am_array*>& cols, rs::RecLayout* L);
// The sort server's shared sorts: for each range q, the entries of `perm` (n row numbers) that lie in
// [lo[q], hi[q]), in order, into outs[q] (device memory holding hi[q] - lo[q] entries).
constexpr int MAX_SHARED = 32;
// The same for columns: `src` holds the covered rows' columns in the shared order (fixed width), and
// dsts[q] receives request q's rows of each, in order (values; validity bits OR-ed into zeroed words,
// null counts added), so a request needs no gather of its own.
constexpr int MAX_CCOLS = 8;
struct CompactSrc {
  const void* src[MAX_CCOLS];
  const uint8_t* src_valid[MAX_CCOLS];   // NULL: no nulls
  int64_t src_voff[MAX_CCOLS];
  int32_t width[MAX_CCOLS];              // 1, 2, 4 or 8 bytes
  int32_t ncols;
};
struct CompactDst {
  void* dst[MAX_CCOLS];
  uint32_t* dst_valid[MAX_CCOLS];        // zeroed bitmap words (when the source has nulls)
  unsigned long long* nulls[MAX_CCOLS];  // zeroed null counters (when the source has nulls)
};
void compact_columns(const uint32_t* perm, uint64_t n, const std::vector<uint32_t>& lo, const std::vector<uint32_t>& hi,
                     const CompactSrc& src, const std::vector<CompactDst>& dsts, cudaStream_t s);
void compact_ranges(const uint32_t* perm, uint64_t n, const std::vector<uint32_t>& lo, const std::vector<uint32_t>& hi,
                    const std::vector<uint32_t*>& outs, cudaStream_t s);
// Segmented argsort: outs[i] (a uint32 array of keys[i].col->length rows) receives the argsort of
// keys[i], one key per array; the arrays of a key width share every launch.
void radix_argsort_batch(const std::vector<SortKey>& keys, const std::vector<void*>& outs, cudaStream_t s);
// The segmented sort's chosen shapes: {key bytes, size class, the class's largest array (-1: none),
// method (-1 not measured yet, 0 digit passes, 1 one CTA per array), threads, rows per thread, digit bits}.
std::vector<std::array<int32_t, 7>> batch_tuning();
// Test hook: the segmented sort uses shape `shape` (an index into its shape table) for every size class
// it can serve instead of the tuned one; -1 restores the tuning.
void debug_force_batch_shape(int shape);
// Single-key argsort of a device column into a caller's uint32 array with no allocation: all
// scratch sits in a fixed device block of the library (radix_sort.cu). Waits for its work.
uint64_t noalloc_max_rows();
void argsort_noalloc(int pt, const void* values, const uint8_t* validity, int64_t offset, int64_t length,
                     bool descending, bool nulls_first, int float_order, uint32_t* indices, cudaStream_t s);

// Partition around position `pivot` of the ascending stable argsort (Arrow partition_nth_indices), by
// radix selection; NULL for a string column (the caller sorts instead).
am_array* radix_partition_nth(const SortKey& key, int64_t pivot, cudaStream_t s);

// Sort consumers (consumers.cu). rank_of's functions: Arrow's rank tiebreakers in the C ABI's numbering
// (0 min, 1 max, 2 first, 3 dense), then rank_quantile, rank_normal in float64 and float32, and the SQL
// percent_rank and cume_dist. `merge_nan`: the NaN rows tie with the nulls (Arrow's rank functions).
enum RankFn : int {
  RANK_MIN = 0, RANK_MAX, RANK_FIRST, RANK_DENSE, RANK_QUANTILE, RANK_NORMAL64, RANK_NORMAL32, RANK_PERCENT, RANK_CUME
};
am_array* rank_of(am_array* a, int fn, bool desc, bool nulls_first, bool merge_nan, cudaStream_t s,
                  int float_order = 0);
// The distinct values, ascending or in order of first appearance; `counts_out` (may be NULL) receives
// each one's row count (int64).
am_array* unique_of(am_array* a, bool first_appearance, am_array** counts_out, cudaStream_t s);
// The sort key of a dictionary column: per row the rank of its value among the dictionary's distinct
// values under `k`'s float order (a float, so a NaN value stays NaN), null where the code or the value
// is null. Sorting it with k's direction and null placement (float order ieee) sorts the column.
am_array* dictionary_key_column(const SortKey& k, cudaStream_t s);
// Stable argsort over any sort keys: string keys of any length (their chunk and length keys),
// dictionary keys (their rank columns) and plain columns. Up to MAX_KEYS derived keys sort in one
// radix sort; more are sorted in groups of MAX_KEYS, least significant group first, each group's
// keys gathered through the order so far and the orders composed. `out` gets n indices of `width`.
void argsort_any(const std::vector<SortKey>& keys, int64_t n, void* out, int width, cudaStream_t s,
                 am_sort_stats* stats);

// Copies a host Arrow array (a dictionary array with its dictionary) into HBM on stream `s`; the caller
// keeps and releases the struct.
am_array* import_copy(const ArrowSchema* schema, const ArrowArray* array, cudaStream_t s);

// String and binary columns: the derived unsigned keys that sort like the strings (big-endian 8-byte
// chunks, then the length; the first carries the nulls), and the take of one string column.
// A string key is the tuple (chunk 0, ..., chunk m-1, length) with m = string_chunk_count; a call
// derives chunks [first, first + count) and, when asked, the length (chunk 0 carries the nulls).
int string_chunk_count(const am_array* a, cudaStream_t s);
std::vector<am_array*> string_key_columns(const am_array* a, int first, int count, bool with_length, cudaStream_t s);
void take_strings(am_array* src, am_array* idx, am_array* out, bool check_range, cudaStream_t s);

// Gathers `count` columns through one index array. outs[i] must be new arrays of indices' length.
// `check_range` asks the kernel to flag an index outside [0, src length) in the stream's error word.
void take_columns(am_array* const* cols, int count, am_array* indices, am_array** outs,
                  bool check_range, cudaStream_t s);

void fill_last_sort_stats(am_sort_stats* out);   // waits for the calling thread's last sort

int64_t max_row_index();
void set_max_row_index(int64_t v);
void check_index_rows(int64_t rows, const char* op);

}  // namespace am
