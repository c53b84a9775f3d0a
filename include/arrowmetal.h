/* ArrowMetal C ABI, sort path, for NVIDIA B200 (sm_100a).
 *
 * Drop-in for the full-sort surface of ArrowMetal's include/arrowmetal.h (version 0.6.1): the same
 * names, argument meanings, return codes and Arrow C Data Interface arrays, so the callers of that
 * header (the Python ctypes binding, the DataFusion rule, the Polars engine and plugin) link against
 * libArrowMetalC.so unchanged. Each declaration cites the reference declaration it replaces as
 * include/arrowmetal.h:<line> (paths relative to the ArrowMetal source tree).
 *
 * Conventions (reference include/arrowmetal.h:1-3, Sources/ArrowMetalC/ArrowMetalC.swift:9-34):
 *   return 0  success
 *   return 1  the operation failed; am_last_error() holds the message (thread-local)
 *   return 2  invalid argument (a NULL handle or pointer)
 *   return 3  am_import_chunks: the type is not taken by the chunked import
 * Handles are reference counted. Every `out` handle is new (+1) and the caller releases it with
 * am_release; input handles are borrowed. Index arrays are uint32 ("I") holding row numbers up to
 * 2^32 - 1; a call whose row numbers would pass that returns 1 with
 * "<op>: row N does not fit the UInt32 index type (row numbers go up to M)".
 *
 * Arrays live in B200 HBM. Calls enqueue work on the calling thread's CUDA stream and return without
 * waiting for the GPU; a call that must see a result (am_export, am_null_count of a fresh gather,
 * am_take with indices this library did not produce, am_batch_end) waits for it. */
#ifndef ARROWMETAL_H
#define ARROWMETAL_H

#include <stdint.h>
#include "arrow_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct am_array am_array;                 /* opaque, HBM-resident Arrow array */
typedef struct am_plan_source_t am_plan_source;   /* include/arrowmetal.h:1419 */
typedef struct am_plan_result_t am_plan_result;   /* include/arrowmetal.h:1420 */

/* ---- library ---------------------------------------------------------------------------------- */
const char* am_version(void);                     /* include/arrowmetal.h:15 */
const char* am_device_name(void);                 /* include/arrowmetal.h:16 */
const char* am_last_error(void);                  /* include/arrowmetal.h:17 */

/* ---- lifecycle and interop -------------------------------------------------------------------- */
/* Moves `array` (its release is NULL on success) and copies its buffers into HBM. Primitive, boolean,
 * temporal, utf8 / binary (and their large forms) arrays, and dictionary arrays of those with integer
 * codes: am_format then reports the codes' format, every sort orders the column by its values, and
 * take / slice / sorted copies keep the dictionary. include/arrowmetal.h:20, :124-130 */
int  am_import(const struct ArrowSchema* schema, struct ArrowArray* array, am_array** out);
/* ARROW_DEVICE_CUDA arrays on this library's device are wrapped without a copy (the producer's
 * release runs when the last handle goes); ARROW_DEVICE_CPU / CUDA_HOST arrays are copied.
 * include/arrowmetal.h:21 */
int  am_import_device(const struct ArrowSchema* schema, struct ArrowDeviceArray* array, am_array** out);
/* n chunks of one type imported as one array; every chunk is moved on success.
 * include/arrowmetal.h:34-35 */
int  am_import_chunks(const struct ArrowSchema* schema, struct ArrowArray* arrays, int64_t n, am_array** out);
int  am_import_chunks_supported(const struct ArrowSchema* schema);
/* Host threads of the chunked import and of the staged host copies (0 = the built-in policy).
 * include/arrowmetal.h:46-47 */
int  am_set_import_threads(int n);
int  am_get_import_threads(void);
/* Copies the array into pinned host memory owned by the exported structs' release callbacks.
 * include/arrowmetal.h:48 */
int  am_export(am_array* a, struct ArrowSchema* schema, struct ArrowArray* array);
/* Zero-copy export of the HBM buffers with device_type ARROW_DEVICE_CUDA (the reference exports
 * ARROW_DEVICE_METAL). include/arrowmetal.h:49 */
int  am_export_device(am_array* a, struct ArrowSchema* schema, struct ArrowDeviceArray* array);
void am_release(am_array* a);                     /* include/arrowmetal.h:50 */
int64_t     am_length(am_array* a);               /* include/arrowmetal.h:51 */
int64_t     am_null_count(am_array* a);           /* include/arrowmetal.h:52 */
const char* am_format(am_array* a);               /* include/arrowmetal.h:53 */
const char* am_compute_format(am_array* a);       /* include/arrowmetal.h:58 */

/* ---- selection -------------------------------------------------------------------------------- */
/* Arrow `take`: indices int32, int64 or uint32; a null index gives a null row; an index out of range
 * returns 1 ("take: index out of range (array length N)"). include/arrowmetal.h:93 */
int  am_take(am_array* a, am_array* indices, am_array** out);
int  am_slice(am_array* a, int64_t offset, int64_t length, am_array** out);   /* include/arrowmetal.h:94 */

/* ---- sorting ---------------------------------------------------------------------------------- */
/* Stable; nulls last; float -0.0 ties +0.0 and NaN sits next to the nulls in both directions.
 * include/arrowmetal.h:96-110 */
int  am_argsort(am_array* a, int descending, am_array** out);                 /* :108 */
int  am_sort(am_array* a, int descending, am_array** out);                    /* :109 */
int  am_top_k(am_array* a, int64_t k, int largest, am_array** out);           /* :110 */

/* Option-carrying forms. null_placement: 0 at_end, 1 at_start. float_order: 0 ieee (Arrow C++),
 * 1 total (IEEE 754 totalOrder, arrow-rs), 2 nan_largest (Polars). include/arrowmetal.h:1302-1352 */
int  am_argsort_ex(am_array* a, int descending, int null_placement, am_array** out);          /* :1331 */
int  am_sort_ex(am_array* a, int descending, int null_placement, am_array** out);             /* :1332 */
int  am_lexsort_ex(am_array** columns, const int* descending, int64_t count,
                   int null_placement, am_array** out);                                      /* :1333 */
int  am_argsort_ex2(am_array* a, int descending, int null_placement, int float_order,
                    am_array** out);                                                         /* :1348 */
int  am_sort_ex2(am_array* a, int descending, int null_placement, int float_order,
                 am_array** out);                                                            /* :1349 */
int  am_top_k_ex(am_array* a, int64_t k, int largest, int null_placement, int float_order,
                 am_array** out);                                                            /* :1350 */
int  am_lexsort_ex2(am_array** columns, const int* descending, const int* null_placement,
                    const int* float_order, int64_t count, am_array** out);                  /* :1352 */
/* Multi-column sort, first column most significant. include/arrowmetal.h:458 */
int  am_lexsort(am_array** columns, const int* descending, int64_t count, am_array** out);

/* ---- sort consumers --------------------------------------------------------------------------- */
/* partition_nth_indices: uint32 indices whose position `pivot` holds the row the ascending stable sort
 * (null_placement as above) puts there; no row before it orders after it, none after it before it, and
 * each of the three blocks keeps row order. 0 <= pivot <= length, else 1 ("partition index P is outside
 * 0...N"). A radix select and one three-way partition, not a sort. include/arrowmetal.h:1069, :1335 */
int  am_partition_nth_indices(am_array* a, int64_t n, am_array** out);                       /* :1069 */
int  am_partition_nth_ex(am_array* a, int64_t pivot, int null_placement, am_array** out);    /* :1335 */
/* Arrow rank, uint32 (pyarrow returns uint64 with the same values). tiebreaker: 0 min, 1 max, 2 first,
 * 3 dense. The nulls and the NaN rows are one tie group at the null_placement end; -0.0 ties +0.0.
 * include/arrowmetal.h:1306, :1355 */
int  am_rank_ex(am_array* a, int tiebreaker, int descending, int null_placement, am_array** out);
/* op 0 rank_quantile (float64: (s + e) / 2n over the row's tie group [s, e) of sorted positions),
 * op 1 rank_normal (float64: the standard normal quantile of that), op 2 rank_normal in float32.
 * am_rank is ascending with nulls at the end. include/arrowmetal.h:1001-1014, :1356 */
int  am_rank(am_array* a, int op, am_array** out);                                           /* :1014 */
int  am_rank_quantile_ex(am_array* a, int op, int descending, int null_placement, am_array** out);
/* The ranking ops of am_window: 0 row_number, 1 rank, 2 dense_rank (uint32), 3 percent_rank
 * ((rank - 1) / (n - 1)), 4 cume_dist (rows at or before the value / n) (float64); ascending, nulls last
 * and one tie group, every NaN one value after +inf. p1, p2 and scalar_or_null are unused by these ops;
 * ops 5-12 (shifts, differences, running and rolling windows) return 1, unsupported.
 * include/arrowmetal.h:415-452 */
int  am_window(am_array* a, int op, int64_t p1, int64_t p2, const void* scalar_or_null, am_array** out);
/* Distinct values. order 0 first_appearance (Arrow's order; a fixed-width column keeps one null entry
 * at the first null's place), 1 sorted (ascending, nulls dropped). String columns drop the null in
 * both orders. -0.0 matches 0.0 and every NaN is one value; the representative is the earliest row.
 * am_unique and am_value_counts are the sorted order. value_counts returns a struct array ("+s") of
 * `values` and int64 `counts`, exported with am_export (it takes part in no other call).
 * include/arrowmetal.h:1060-1068, :1359-1360 */
int  am_unique(am_array* a, am_array** out);                                                 /* :1067 */
int  am_value_counts(am_array* a, am_array** out);                                           /* :1068 */
int  am_unique_ex(am_array* a, int order, am_array** out);                                   /* :1359 */
int  am_value_counts_ex(am_array* a, int order, am_array** out);                             /* :1360 */

/* ---- batching --------------------------------------------------------------------------------- */
/* Between begin and end the calls of this thread do not wait for the GPU; deferred errors (a take
 * out of range) surface from am_batch_end. include/arrowmetal.h:184-185 */
int  am_batch_begin(void);
int  am_batch_end(void);

/* ---- plan engine (the subset the DataFusion rule and the Polars engine emit for a sort) -------- */
/* Grammar taken: scan {source, columns?}; select / with_columns of [name, "(col \"x\")"] pairs;
 * sort {by: [KEY...], nulls?, float_order?}; limit {count, offset?}. include/arrowmetal.h:1369-1433 */
int  am_plan_source_create(const char* name, am_array** columns, const char** names,
                           int64_t n_columns, am_plan_source** out);                         /* :1422 */
void am_plan_source_release(am_plan_source* s);                                              /* :1424 */
int  am_plan_run(const char* plan_json, am_plan_source** sources, int64_t n_sources, int optimize,
                 am_plan_result** out);                                                      /* :1425 */
const char* am_plan_explain(const char* plan_json, am_plan_source** sources, int64_t n_sources,
                            int optimize);                                                   /* :1427 */
int64_t     am_plan_column_count(am_plan_result* r);                                         /* :1428 */
int64_t     am_plan_row_count(am_plan_result* r);                                            /* :1429 */
const char* am_plan_column_name(am_plan_result* r, int64_t i);                               /* :1430 */
int         am_plan_column(am_plan_result* r, int64_t i, am_array** out);                    /* :1431 */
void        am_plan_result_release(am_plan_result* r);                                       /* :1432 */

/* ---- router ------------------------------------------------------------------------------------ */
/* Modes 0 auto, 1 gpu, 2 cpu are recorded (2 returned for an unknown mode); the sort is never routed
 * to the CPU (include/arrowmetal.h:1785-1797), so the mode changes nothing on this path. The
 * binding's test set-up calls it. include/arrowmetal.h:1799-1800 */
int  am_router_set_mode(int mode);
int  am_router_get_mode(void);

/* ---- out-of-core sort of a record-batch stream ------------------------------------------------ */
/* A stream handle wraps a producer of Arrow record batches (the Arrow C Stream Interface: pyarrow's
 * RecordBatchReader and dataset scanners, Polars, DuckDB) and is consumed by one terminal call.
 * Errors: a NULL handle or a non-zero return, with the message in am_stream_last_error().
 * include/arrowmetal.h:1515-1547 */
typedef struct am_stream am_stream;                               /* :1528 */
typedef struct am_stream_result am_stream_result;                 /* :1529 */
const char* am_stream_last_error(void);                           /* :1538 */
/* Takes ownership of `in` (its release is NULL afterwards); prefetch_depth batches are read ahead on
 * a reader thread (0: read on the calling thread). include/arrowmetal.h:1546 */
am_stream* am_stream_from_c_stream(struct ArrowArrayStream* in, int prefetch_depth);
/* An Arrow IPC file (file or stream format) or a directory of them (.arrow, .arrows, .ipc, .feather, in
 * name order), memory-mapped and read on the reader thread. Uncompressed bodies of flat columns;
 * dictionary-encoded, nested and compressed IPC data return NULL with the reason. `readers` is
 * accepted and the files are read in order. include/arrowmetal.h:1544 */
am_stream* am_stream_open_ipc(const char* path, int prefetch_depth, int readers);
void       am_stream_release(am_stream* s);                       /* :1547 */
/* Keeps the named columns, in this order, in the terminal's output. include/arrowmetal.h:1551 */
int am_stream_select(am_stream* s, const char** names, int64_t n);
/* Hands the stream's batches (the selected columns) to a consumer as an Arrow C stream; a terminal,
 * the handle is consumed. include/arrowmetal.h:1595 */
int am_stream_export_c(am_stream* s, struct ArrowArrayStream* out);
/* External sort: batches gather in HBM up to a run budget (a sixth of the free device memory, or
 * ARROWMETAL_STREAM_RUN_BYTES), each run is sorted on the GPU and, when more than one is needed,
 * spilled under scratch_dir (NULL: a new directory under the system's temporary directory) and
 * merged on the GPU in windows. The output is in full sort order, ties in stream order (stable).
 * limit 0 means all rows. sink_path NULL collects the rows into the result's columns; otherwise they
 * are written to that path as an Arrow IPC stream. include/arrowmetal.h:1576-1584 */
int am_stream_sort(am_stream* s, const char** columns, const int* descending, int64_t n_keys,
                   int64_t limit, const char* scratch_dir, const char* sink_path, am_stream_result** out);
int am_stream_sort_ex(am_stream* s, const char** columns, const int* descending,
                      const int* null_placement, const int* float_order, int64_t n_keys,
                      int64_t limit, const char* scratch_dir, const char* sink_path,
                      am_stream_result** out);
/* Results. A sort has columns and no scalars. include/arrowmetal.h:1597-1611 */
int64_t     am_stream_result_column_count(am_stream_result* r);
const char* am_stream_result_column_name(am_stream_result* r, int64_t i);
int         am_stream_result_column(am_stream_result* r, int64_t i, am_array** out);
int64_t     am_stream_result_scalar_count(am_stream_result* r);
const char* am_stream_result_scalar_name(am_stream_result* r, int64_t i);
int         am_stream_result_scalar(am_stream_result* r, int64_t i, int64_t* out_i64, double* out_f64,
                                    int* out_kind, int* is_null);
int64_t     am_stream_result_rows_out(am_stream_result* r);
/* batches and rows read, bytes imported, wall time and the time each stage was busy (read: the
 * producer's get_next; gpu: the run sorts; merge: the merge windows); overlap = (read + gpu + merge)
 * / wall. */
int         am_stream_result_stats(am_stream_result* r, int64_t* batches, int64_t* rows,
                                   int64_t* bytes_read, double* wall_s, double* read_s,
                                   double* gpu_s, double* merge_s, double* overlap);
int         am_stream_result_stalls(am_stream_result* r, double* read_stall_s, double* merge_stall_s);
void        am_stream_result_release(am_stream_result* r);

/* ================================================================================================
 * Additions with no counterpart in the reference header. They stand beside the drop-in surface and
 * change nothing in it.
 * ============================================================================================== */

/* The CUDA stream the calling thread's calls enqueue on (a cudaStream_t). NULL restores the
 * library's own non-blocking stream for this thread. Lets a host that already owns a stream (a
 * PyTorch program, a server worker) order the sort with its own work. */
int   am_cuda_set_stream(void* stream);
void* am_cuda_get_stream(void);
/* Waits for every call this thread has enqueued, then reports any deferred device error. */
int   am_cuda_synchronize(void);
/* CUDA device ordinal the library runs on (the ARROWMETAL_DEVICE variable, else the current one). */
int   am_cuda_device(void);

/* am_argsort_ex2 with the index width chosen: 4 gives uint32 ("I", as am_argsort_ex2), 8 gives
 * uint64 ("L", the type pyarrow's sort_indices returns). */
int  am_argsort_ex3(am_array* a, int descending, int null_placement, int float_order,
                    int index_width, am_array** out);

/* Multi-column take with one index read: outs[i] = take(columns[i], indices). Same rules as
 * am_take; one gather kernel serves every column. */
int  am_take_columns(am_array** columns, int64_t count, am_array* indices, am_array** outs);

/* Segmented (batched) argsort: `count` independent arrays sorted in one pipeline, each with its own
 * options (descending / null_placement / float_order hold `count` entries or are NULL). outs[i]
 * receives uint32 indices into arrays[i], identical to am_argsort_ex2 on that array alone. */
int  am_argsort_batch(am_array** arrays, const int* descending, const int* null_placement,
                      const int* float_order, int64_t count, am_array** outs);

/* The segmented sort's shapes as its autotuner chose them, one entry per key width (4 or 8 bytes) and
 * size class (0: arrays of up to 4,096 rows, 1: up to 16,384, 2: larger; `max_rows` -1: no bound):
 * the method (-1: not measured yet, 0: digit passes over tiles of threads x items rows, 1: one CTA of
 * `threads` threads and `items` rows a thread per array), and the digit width in bits. Writes up to
 * `capacity` entries and their number to `count`. */
typedef struct am_batch_shape {
  int32_t key_bytes;
  int32_t size_class;
  int32_t max_rows;
  int32_t method;
  int32_t threads;
  int32_t items;
  int32_t digit_bits;
} am_batch_shape;
int  am_cuda_batch_tuning(am_batch_shape* out, int64_t capacity, int64_t* count);

/* Per-call counters of the calling thread's last sort: rows, radix passes run and skipped, the device
 * time of the sort's kernels in microseconds (0 unless am_cuda_profile(1) is on), and whether the
 * payload columns rode through the sort in row records (1) instead of a gather afterwards (0). */
typedef struct am_sort_stats {
  int64_t rows;
  int64_t value_rows;
  int32_t passes_run;
  int32_t passes_skipped;
  double  kernel_us;
  int32_t payload_in_records;
  int32_t reserved;
} am_sort_stats;
int  am_last_sort_stats(am_sort_stats* out);
/* Kernel timing with CUDA events around every launch of this library (1 on, 0 off), and the
 * accumulated per-kernel totals: name, launches, total milliseconds. */
int  am_cuda_profile(int on);
int64_t am_cuda_profile_count(void);
int  am_cuda_profile_entry(int64_t i, const char** name, int64_t* launches, double* total_ms);
int  am_cuda_profile_reset(void);

/* Test hooks: the largest row number an index array may hold (2^32 - 1 by default; tests lower it to
 * reach the refusal at small sizes), and a host allocation failure after `n` more device
 * allocations (-1 disables it). */
int  am_debug_set_max_row_index(int64_t max_row);
int  am_debug_fail_alloc_after(int64_t n);
/* Test hook: am_argsort_batch sorts with candidate shape `shape` (0-2: digit passes over tiles of 512 x 8,
 * 512 x 4 and 384 x 12 rows; 3-6: one CTA per array of up to 4,096 rows, 256 x 16 or 512 x 8 rows
 * with 8- or 4-bit digits) for every size class it can serve, instead of the autotuner's choice; -1
 * restores the autotuner. */
int  am_debug_force_batch_shape(int shape);
/* Test hook for the bounded look-back: with `on` set, the calling process's next sorts never process
 * their first tile, so the tiles after it wait on a status nothing writes; each such wait gives up
 * after one second and the call returns 1 ("look-back wait timed out"). No GPU fault is involved. */
int  am_debug_skip_first_tile(int on);

/* Sort server: continuous batching of sort requests over tables resident in HBM. No counterpart in
 * the reference, whose callers make one call per query (include/arrowmetal.h:1419-1433 is the call a
 * request stands for). A request sorts rows [offset, offset + length) of a plan source by `nkeys`
 * key columns (options per key as in am_lexsort_ex2) and returns an am_plan_result holding the sorted
 * key columns followed by the `npayload` payload columns taken through the same permutation: the
 * same result am_plan_run gives for select(sort(limit(scan))). `workers` threads, each with its own
 * CUDA stream, take requests in arrival order as long as their estimated HBM footprint fits under
 * `hbm_cap_bytes` beside the work in flight; single-key requests of at most `batch_rows` rows that
 * are waiting together are sorted as one segmented batch. The table must stay alive until every
 * request on it has been waited for. am_server_wait blocks until the request is done, hands its
 * result to the caller and gives the latency from submission to completion. */
typedef struct am_server_t am_server;
typedef struct am_server_stats {
  int64_t requests;               /* completed */
  int64_t solo_requests;          /* run alone through the plan path */
  int64_t batches;                /* segmented batches run */
  int64_t batched_requests;       /* requests served inside those batches */
  int64_t rows;                   /* rows of the completed, successful requests */
  int64_t peak_in_flight_bytes;   /* largest admitted footprint on the GPU at once */
  int64_t in_flight_bytes;
  int64_t queued;
  int64_t shared_sorts;           /* sorts shared by several queued requests of one table and key */
  int64_t shared_requests;        /* requests answered from those sorts */
} am_server_stats;
int  am_server_create(int workers, int64_t hbm_cap_bytes, int64_t batch_rows, am_server** out);
int  am_server_submit(am_server* server, am_plan_source* table, int64_t offset, int64_t length,
                      const char** keys, const int* descending, const int* null_placement,
                      const int* float_order, int64_t nkeys, const char** payload, int64_t npayload,
                      int64_t* ticket);
int  am_server_wait(am_server* server, int64_t ticket, am_plan_result** out, double* latency_ms);
int  am_server_get_stats(am_server* server, am_server_stats* out);
/* Finishes the queued requests, stops the workers and frees the server. */
int  am_server_release(am_server* server);

/* Argsort that allocates no device memory. No counterpart in the reference.
 * For callers that cannot allocate on the device when they sort: a process whose device memory
 * belongs to its own pool allocator (a framework's caching allocator, an RMM pool), or a serving loop
 * that cannot afford cudaFree's wait for the whole device. The column and the output are the caller's
 * device memory: `values` (Arrow values buffer; a bitmap for "b"), `validity` (bitmap, or NULL for no
 * nulls), row i at element / bit offset + i, `format` an Arrow format string of a fixed-width type.
 * `indices` receives `length` uint32 row numbers, the same as am_argsort_ex2 gives for that array.
 * All scratch lives in one fixed block inside the library (about 6.1 MiB on each GPU the library is
 * loaded on, held until exit), so one call sorts at most 262,144 rows; longer inputs return 2 with an
 * error naming the limit. The work runs on `stream` (NULL: the default stream) on the calling thread's
 * current device, and the call is synchronous: it waits for that stream before it returns. The first
 * call on each device looks up the block's device address and sets up the kernels; make that first
 * call before any stream capture.
 * Calls share the block: they take turns inside this process, and work that overlapped on the GPU
 * would race on it. */
int  am_argsort_device_noalloc(const char* format, const void* values, const void* validity,
                               int64_t offset, int64_t length, int descending, int null_placement,
                               int float_order, uint32_t* indices, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ARROWMETAL_H */
