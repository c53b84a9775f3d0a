// Entry points of ArrowMetal's C ABI that lie outside the sort path this library serves.
//
// The reference's callers bind every symbol of include/arrowmetal.h when they load the library (the
// Python binding resolves them all at import, python/arrowmetal/__init__.py:80-1230), so a library that
// answers only the sort path must still export the rest for those callers to load it unchanged. Each
// symbol here does no work: it records "<name>: not served by this library" as the thread's last error
// and returns the failure value of its kind. Only the names and the return kinds follow the reference
// header (include/arrowmetal.h); a C symbol carries no parameter types, and a callee that reads none of
// its arguments may be called with any of them.
//
//   status entry points (int / int32_t)  -> 1, the operation-error status
//   count entry points (int64_t)          -> -1
//   text entry points (const char*)       -> NULL
//   entry points without a result (void)  -> nothing
#include <string>

#include "am_internal.h"

namespace {

void not_served(const char* name) {
  am::set_last_error(std::string(name) + ": not served by this library (it serves ArrowMetal's sort path)");
}

}  // namespace

#define AM_UNSERVED_STATUS(X) \
  X(am_add_interval) X(am_and_kleene) X(am_arith_array) X(am_arith_scalar) X(am_assume_timezone) \
  X(am_binary) X(am_binary_checked) X(am_binary_join) X(am_bool_and) X(am_bool_not) X(am_bool_or) \
  X(am_byte_transform) X(am_case_when) X(am_cast) X(am_cast_ex) X(am_cast_float16) X(am_child) X(am_choose) \
  X(am_coalesce) X(am_compare_array) X(am_compare_scalar) X(am_csv_batch_column) X(am_csv_open) \
  X(am_csv_read) X(am_cumulative) X(am_cumulative_checked) X(am_decimal_narrow) X(am_decimal_op) \
  X(am_decimal_widen) X(am_delta_read) X(am_dictionary_decode) X(am_dictionary_encode) \
  X(am_dictionary_encode_ex) X(am_drop_null) X(am_extension_storage) X(am_extension_wrap) \
  X(am_extract_struct) X(am_fill_null) X(am_fill_null_direction) X(am_filter) X(am_filter_where) \
  X(am_first_last) X(am_fixed_binary_compare) X(am_fixed_binary_hash64) X(am_float_class) \
  X(am_group_agg_ex) X(am_group_by) X(am_group_by_ids) X(am_group_by_keys) X(am_group_by_keys_result) \
  X(am_group_pivot_wider) X(am_hash64) X(am_iceberg_current_snapshot) X(am_iceberg_read) X(am_if_else) \
  X(am_index_in) X(am_index_in_ex) X(am_indices_nonzero) X(am_interval_between) X(am_interval_field) \
  X(am_inverse_permutation) X(am_is_in) X(am_is_in_ex) X(am_is_null) X(am_is_valid) X(am_join) \
  X(am_join_element_wise) X(am_json_batch_column) X(am_json_open) X(am_json_open_buffer) X(am_json_read) \
  X(am_json_read_named) X(am_lakehouse_batch_column) X(am_lakehouse_batch_stats) X(am_list_element) \
  X(am_list_flatten) X(am_list_parent_indices) X(am_list_parent_indices64) X(am_list_slice) \
  X(am_list_value_length) X(am_local_timestamp) X(am_logical) X(am_low_latency_wait) X(am_make_struct) \
  X(am_map_lookup) X(am_math_extra) X(am_null_array) X(am_or_kleene) X(am_parquet_batch_column) \
  X(am_parquet_open) X(am_parquet_read) X(am_parquet_read_ex) X(am_parquet_set_bloom_filters) \
  X(am_parquet_set_page_index) X(am_parquet_write) X(am_parse) X(am_pivot_wider) X(am_query) \
  X(am_query_column) X(am_query_scalar) X(am_random) X(am_reduce) X(am_reduce_ex) X(am_reduce_ex2) \
  X(am_regex) X(am_replace_with_mask) X(am_resident_mode) X(am_resident_mode_available) \
  X(am_round_temporal_ex) X(am_router_decide) X(am_router_get_thread_mode) X(am_router_last) \
  X(am_router_load_table) X(am_router_set_thread_mode) X(am_run_end_decode) X(am_run_end_encode) \
  X(am_scatter) X(am_split) X(am_str_concat) X(am_str_dictionary_encode) X(am_str_equals_array) \
  X(am_str_extra) X(am_str_match) X(am_str_transform) X(am_str_unary) X(am_stream_aggregate) \
  X(am_stream_filter) X(am_stream_group_by) X(am_stream_join_aggregate) X(am_stream_join_broadcast) \
  X(am_stream_join_grace) X(am_stream_join_group_by) X(am_stream_project) X(am_stream_quantiles) \
  X(am_stream_query) X(am_stream_set_progress) X(am_stream_sink_ipc) X(am_stream_top_k) \
  X(am_string_index_in) X(am_string_is_in) X(am_string_layout) X(am_string_predicate) \
  X(am_string_transform) X(am_string_view_info) X(am_struct_field) X(am_temporal_cast_unit) \
  X(am_temporal_extra) X(am_temporal_extract) X(am_temporal_math) X(am_to_strings) X(am_to_timezone) \
  X(am_trig) X(am_true_unless_null) X(am_unary) X(am_unary_checked) X(am_utc_offset) X(am_winsorize)

#define AM_UNSERVED_COUNT(X) \
  X(am_child_count) X(am_count_all) X(am_csv_batch_column_name_length) X(am_csv_batch_columns) \
  X(am_csv_batch_rows) X(am_delta_latest_version) X(am_group_by_group_count) X(am_json_batch_column_names) \
  X(am_json_batch_columns) X(am_json_batch_rows) X(am_json_last_error) X(am_lakehouse_batch_columns) \
  X(am_lakehouse_batch_rows) X(am_parquet_batch_columns) X(am_parquet_batch_rows) \
  X(am_parquet_column_null_count) X(am_parquet_field_metadata) X(am_parquet_last_read_stats) \
  X(am_parquet_num_columns) X(am_parquet_num_row_groups) X(am_parquet_num_rows) \
  X(am_parquet_row_group_rows) X(am_parquet_schema_metadata) X(am_parquet_selected_row_groups) \
  X(am_query_column_count) X(am_query_scalar_count) X(am_router_crossover) X(am_router_multiply_crossover) \
  X(am_spin_microseconds)

#define AM_UNSERVED_TEXT(X) \
  X(am_csv_batch_column_name) X(am_csv_last_error) X(am_extension_metadata) X(am_extension_name) \
  X(am_json_batch_column_name) X(am_lakehouse_batch_column_name) X(am_parquet_batch_column_name) \
  X(am_parquet_codec) X(am_parquet_column_name) X(am_parquet_column_type) X(am_parquet_encodings) \
  X(am_query_canonical) X(am_query_column_name) X(am_query_scalar_name) X(am_resident_mode_reason) \
  X(am_router_explain) X(am_router_last_reason) X(am_router_table_info)

#define AM_UNSERVED_NOTHING(X) \
  X(am_csv_batch_release) X(am_csv_close) X(am_csv_options_init) X(am_group_by_release) \
  X(am_json_batch_release) X(am_json_close) X(am_lakehouse_batch_release) X(am_parquet_batch_release) \
  X(am_parquet_close) X(am_query_result_release) X(am_router_clear_last) X(am_string_view_conversions)

extern "C" {

#define AM_STATUS_STUB(name) int name(void) { not_served(#name); return 1; }
#define AM_COUNT_STUB(name) int64_t name(void) { not_served(#name); return -1; }
#define AM_TEXT_STUB(name) const char* name(void) { not_served(#name); return nullptr; }
#define AM_NOTHING_STUB(name) void name(void) { not_served(#name); }

AM_UNSERVED_STATUS(AM_STATUS_STUB)
AM_UNSERVED_COUNT(AM_COUNT_STUB)
AM_UNSERVED_TEXT(AM_TEXT_STUB)
AM_UNSERVED_NOTHING(AM_NOTHING_STUB)

}  // extern "C"
