// The extern "C" surface of libArrowMetalC for B200: the sort path of ArrowMetal's C ABI
// (include/arrowmetal.h), served from HBM-resident arrays.
//
// Reference: Sources/ArrowMetalC/ArrowMetalC.swift (handles, errors, import / export, am_take,
// am_argsort, am_sort, am_top_k, am_batch_*), Sources/ArrowMetalC/ArrowMetalC_Options.swift:49-228
// (the option-carrying sorts), Sources/ArrowMetalC/ArrowMetalC_Window.swift:106-118 (am_lexsort) and
// Sources/ArrowMetal/CInterop.swift:136-425 (import and export).
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <mutex>
#include <set>

#include "am_internal.h"
#include "radix_sort.cuh"

using namespace am;

namespace {

// Return-code convention: 0 ok, 1 operation error (message in am_last_error), 2 invalid argument.
template <class F>
int guard(F&& f) {
  try {
    return f();
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return 1;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 1;
  }
}

const char* intern(const std::string& s) {
  static std::mutex mu;
  static std::set<std::string> pool;
  std::lock_guard<std::mutex> g(mu);
  return pool.insert(s).first->c_str();
}

bool in_batch() { return tls().batch_depth > 0; }

// After a kernel that may set the stream's error word: check now, or at the batch's end.
void checkpoint(cudaStream_t s) {
  if (in_batch()) {
    tls().deferred_checks.push_back([s] { check_device_errors(s); });
  } else {
    check_device_errors(s);
  }
}

int64_t host_null_count(const uint8_t* bits, int64_t off, int64_t n) {
  int64_t valid = 0;
  int64_t i = 0;
  for (; i < n && ((off + i) & 7); i++) valid += (bits[(off + i) >> 3] >> ((off + i) & 7)) & 1;
  const uint8_t* p = bits + ((off + i) >> 3);
  for (; i + 64 <= n; i += 64, p += 8) {
    uint64_t w;
    std::memcpy(&w, p, 8);
    valid += __builtin_popcountll(w);
  }
  for (; i < n; i++) valid += (bits[(off + i) >> 3] >> ((off + i) & 7)) & 1;
  return n - valid;
}

// Copies bits [off, off + n) of `src` to a fresh bitmap starting at bit 0.
std::vector<uint8_t> realign_bits(const uint8_t* src, int64_t off, int64_t n) {
  std::vector<uint8_t> out(size_t((n + 7) / 8), 0);
  for (int64_t i = 0; i < n; i++)
    if ((src[(off + i) >> 3] >> ((off + i) & 7)) & 1) out[size_t(i >> 3)] |= uint8_t(1u << (i & 7));
  return out;
}

// Uploads bits [off, off + n) of a host bitmap as a device bitmap starting at bit 0.
BufPtr upload_bits(const uint8_t* src, int64_t off, int64_t n, cudaStream_t s) {
  const size_t bytes = size_t((n + 7) / 8);
  BufPtr b = DevBuffer::alloc(bytes + 16, s);
  if (bytes == 0) return b;
  if ((off & 7) == 0) {
    if (copy_h2d(b->ptr, src + (off >> 3), bytes, s)) AM_CUDA(cudaStreamSynchronize(s));
  } else {
    std::vector<uint8_t> v = realign_bits(src, off, n);
    copy_h2d(b->ptr, v.data(), bytes, s);
    AM_CUDA(cudaStreamSynchronize(s));   // the temporary must outlive the copy
  }
  return b;
}

bool is_index_format(const char* f) {
  static const char* idx[] = {"c", "C", "s", "S", "i", "I", "l", "L"};
  for (const char* x : idx)
    if (std::strcmp(f, x) == 0) return true;
  return false;
}

// The fields of one flat array (no children) that its buffers are read by: length, offset and the
// buffer count its format needs.
void check_flat_struct(const ArrowSchema* schema, const ArrowArray* array, const char* what) {
  if (schema->n_children != 0 || array->n_children != 0)
    throw unsupported(std::string("nested arrays are not carried by this build (a nested ") + what + ")");
  if (array->length < 0 || array->offset < 0) throw invalid(std::string("negative length or offset in ") + what);
  const int want = pt_var(parse_format(schema->format)) ? 3 : 2;
  if (array->n_buffers != want || (array->n_buffers > 0 && !array->buffers))
    throw invalid(std::string(want == 3 ? "a string or binary " : "a primitive ") + what + " has " +
                  std::to_string(want) + " buffers, got " + std::to_string(array->n_buffers));
}

void check_array_struct(const ArrowSchema* schema, const ArrowArray* array) {
  if (!schema->dictionary != !array->dictionary) throw invalid("the schema and the array disagree on a dictionary");
  if (schema->dictionary) {
    // A dictionary array: integer codes, and a flat dictionary (not itself dictionary-encoded), checked
    // like any array before its buffers are read.
    if (!is_index_format(schema->format))
      throw invalid(std::string("dictionary codes of type ") + schema->format + " (an integer type is required)");
    if (schema->dictionary->dictionary || array->dictionary->dictionary)
      throw unsupported("a dictionary whose values are themselves dictionary-encoded");
    check_flat_struct(schema->dictionary, array->dictionary, "dictionary");
  }
  check_flat_struct(schema, array, "array");
}

// A host string or binary array's offsets must exist and never decrease: the device kernels read each
// row's bytes between its two offsets, so a bad offset would send them outside the copied bytes. One
// host pass over the offsets, before anything is allocated on the device.
void check_host_offsets(const char* format, const ArrowArray* arr) {
  const int pt = parse_format(format);
  if (!pt_var(pt)) return;
  const int64_t n = arr->length, off = arr->offset;
  const void* vals = arr->buffers[1];
  if (!vals) {
    if (n == 0) return;
    throw invalid("a string or binary array without an offsets buffer");
  }
  int64_t prev = 0;
  for (int64_t i = 0; i <= n; i++) {
    const int64_t o = pt == PT_LSTR ? static_cast<const int64_t*>(vals)[off + i] : static_cast<const int32_t*>(vals)[off + i];
    if (o < 0 || (i > 0 && o < prev)) throw invalid("string offsets that are negative or decrease");
    prev = o;
  }
}

void check_host_array(const ArrowSchema* schema, const ArrowArray* array) {
  check_array_struct(schema, array);
  check_host_offsets(schema->format, array);
  if (schema->dictionary) check_host_offsets(schema->dictionary->format, array->dictionary);
}

// Fills `a` from a host ArrowArray (the caller still owns the struct).
void import_host(am_array* a, const ArrowArray* arr, cudaStream_t s) {
  const int64_t n = arr->length, off = arr->offset;
  const uint8_t* vbits = static_cast<const uint8_t*>(arr->buffers[0]);
  const void* vals = arr->buffers[1];
  int64_t nulls = 0;
  if (vbits) nulls = arr->null_count >= 0 ? arr->null_count : host_null_count(vbits, off, n);
  a->null_count = nulls;
  if (nulls > 0) a->validity = upload_bits(vbits, off, n, s);
  const int w = pt_bytes(a->pt);
  bool reads_later = false;
  if (pt_var(a->pt)) {
    // Offsets rebased to the first row's start, and exactly the bytes the rows span.
    const bool large = a->pt == PT_LSTR;
    std::vector<char> offs(size_t(n + 1) * w);
    int64_t first = 0, last = 0;
    for (int64_t i = 0; vals && i <= n; i++) {     // no offsets buffer: an empty array (checked)
      const int64_t o = large ? static_cast<const int64_t*>(vals)[off + i] : static_cast<const int32_t*>(vals)[off + i];
      if (i == 0) first = o;
      if (i == n) last = o;
      if (large) reinterpret_cast<int64_t*>(offs.data())[i] = o - first;
      else reinterpret_cast<int32_t*>(offs.data())[i] = int32_t(o - first);
    }
    if (last < first) throw invalid("string offsets decrease");
    a->values = DevBuffer::alloc(offs.size() + 16, s);
    copy_h2d(a->values->ptr, offs.data(), offs.size(), s);
    a->bytes = DevBuffer::alloc(size_t(last - first) + 16, s);
    if (last > first) {
      const void* bytes = arr->buffers[2];
      if (!bytes) throw invalid("string array without a data buffer");
      reads_later = copy_h2d(a->bytes->ptr, static_cast<const char*>(bytes) + first, size_t(last - first), s);
    }
    AM_CUDA(cudaStreamSynchronize(s));   // the rebased offsets are a temporary
  } else if (w == 0) {
    if (n > 0 && !vals) throw invalid("boolean array without a values buffer");
    a->values = n > 0 ? upload_bits(static_cast<const uint8_t*>(vals), off, n, s) : DevBuffer::alloc(16, s);
  } else {
    const size_t bytes = size_t(n) * w;
    a->values = DevBuffer::alloc(bytes + 16, s);
    if (bytes) {
      if (!vals) throw invalid("array without a values buffer");
      reads_later = copy_h2d(a->values->ptr, static_cast<const char*>(vals) + size_t(off) * w, bytes, s);
    }
  }
  // The producer's buffers are released right after the import: a pinned source must be read first.
  if (reads_later) AM_CUDA(cudaStreamSynchronize(s));
  a->last_stream = s;
}

// A primitive array whose buffers are pinned host memory: its copies are enqueued on the calling
// thread's copy stream and the import returns at once; the array records that stream, so its first use
// on another stream waits for the copies, and the producer's buffers are released once they are done.
// The ArrowArray is moved into the pending release. Returns false (nothing done) for other arrays.
bool import_pinned_async(am_array* a, ArrowArray* arr) {
  const int64_t n = arr->length, off = arr->offset;
  const int w = pt_bytes(a->pt);
  const uint8_t* vbits = static_cast<const uint8_t*>(arr->buffers[0]);
  const void* vals = arr->buffers[1];
  if (w == 0 || pt_var(a->pt) || n <= 0 || !vals || !is_pinned(vals)) return false;
  int64_t nulls = 0;
  if (vbits) nulls = arr->null_count >= 0 ? arr->null_count : host_null_count(vbits, off, n);
  if (nulls > 0 && ((off & 7) != 0 || !is_pinned(vbits))) return false;
  cudaStream_t cs = copy_stream();
  const size_t bytes = size_t(n) * w;
  a->values = DevBuffer::alloc(bytes + 16, cs);
  a->values->home = cs;
  AM_CUDA(cudaMemcpyAsync(a->values->ptr, static_cast<const char*>(vals) + size_t(off) * w, bytes,
                          cudaMemcpyHostToDevice, cs));
  a->null_count = nulls;
  if (nulls > 0) {
    const size_t vb = size_t((n + 7) / 8);
    a->validity = DevBuffer::alloc(vb + 16, cs);
    a->validity->home = cs;
    AM_CUDA(cudaMemcpyAsync(a->validity->ptr, vbits + (off >> 3), vb, cudaMemcpyHostToDevice, cs));
  }
  a->last_stream = cs;
  a->ready = std::make_shared<ReadyEvent>(cs);      // readers wait for these copies, not later ones
  cudaEvent_t ev;
  AM_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  AM_CUDA(cudaEventRecord(ev, cs));
  auto* moved = new ArrowArray(*arr);
  arr->release = nullptr;
  release_after(ev, [moved] {
    if (moved->release) moved->release(moved);
    delete moved;
  });
  return true;
}

void move_release(ArrowArray* arr) {
  if (arr->release) arr->release(arr);
  arr->release = nullptr;
}

// ---- export

struct ExportHold {
  std::vector<void*> pinned;      // am_export: pinned host buffers
  am_array* keep = nullptr;       // am_export_device: the array whose HBM the buffers point into
  const void* buffers[3] = {nullptr, nullptr, nullptr};
  std::string format, name;
  ArrowArray* dict_array = nullptr;     // a dictionary array's exported dictionary (owned)
  ArrowSchema* dict_schema = nullptr;
};

void release_schema(ArrowSchema* s) {
  if (!s || !s->release) return;
  auto* h = static_cast<ExportHold*>(s->private_data);
  if (h->dict_schema) {
    if (h->dict_schema->release) h->dict_schema->release(h->dict_schema);
    delete h->dict_schema;
  }
  delete h;
  s->release = nullptr;
  s->private_data = nullptr;
}
void release_array(ArrowArray* a) {
  if (!a || !a->release) return;
  auto* h = static_cast<ExportHold*>(a->private_data);
  for (void* p : h->pinned) pinned_free(p);
  if (h->keep) am::release(h->keep);
  if (h->dict_array) {
    if (h->dict_array->release) h->dict_array->release(h->dict_array);
    delete h->dict_array;
  }
  delete h;
  a->release = nullptr;
  a->private_data = nullptr;
}

void fill_schema(am_array* a, ArrowSchema* schema) {
  auto* h = new ExportHold();
  h->format = a->format;
  schema->format = h->format.c_str();
  schema->name = h->name.c_str();
  schema->metadata = nullptr;
  schema->flags = ARROW_FLAG_NULLABLE;
  schema->n_children = 0;
  schema->children = nullptr;
  schema->dictionary = nullptr;
  schema->release = release_schema;
  schema->private_data = h;
}

// A struct array (value_counts' result): one child array and schema per field, exported the way
// am_export exports a flat array, and no buffer of its own but an absent validity bitmap.
struct StructArrayHold {
  std::vector<ArrowArray> arrays;
  std::vector<ArrowArray*> ptrs;
  const void* buffers[1] = {nullptr};
};
struct StructSchemaHold {
  std::vector<ArrowSchema> schemas;
  std::vector<ArrowSchema*> ptrs;
  std::vector<std::string> names;
  std::string format = "+s", name;
};
void release_struct_array(ArrowArray* a) {
  if (!a || !a->release) return;
  auto* h = static_cast<StructArrayHold*>(a->private_data);
  for (ArrowArray& c : h->arrays)
    if (c.release) c.release(&c);
  delete h;
  a->release = nullptr;
  a->private_data = nullptr;
}
void release_struct_schema(ArrowSchema* s) {
  if (!s || !s->release) return;
  auto* h = static_cast<StructSchemaHold*>(s->private_data);
  for (ArrowSchema& c : h->schemas)
    if (c.release) c.release(&c);
  delete h;
  s->release = nullptr;
  s->private_data = nullptr;
}

am_array* make_index_array(int64_t n, int width, cudaStream_t s) {
  am_array* o = new_array(width == 8 ? PT_U64 : PT_U32, width == 8 ? "L" : "I", n);
  o->values = DevBuffer::alloc(size_t(std::max<int64_t>(n, 1)) * width + 16, s);
  o->null_count = 0;
  o->perm_of = n;
  o->last_stream = s;
  return o;
}

int float_order_ok(int fo) {
  if (fo < 0 || fo > 2) throw invalid("unknown float_order " + std::to_string(fo));
  return fo;
}

// One call of the sort engine: argsort of `keys` into a fresh index array.
am_array* argsort_keys(std::vector<SortKey>& keys, int width, const char* op) {
  const int64_t n = keys[0].col->length;
  for (auto& k : keys) {
    if (k.col->length != n) throw length_mismatch(n, k.col->length);
    float_order_ok(k.float_order);
  }
  check_index_rows(n, op);
  cudaStream_t s = stream();
  for (auto& k : keys) use_on(k.col, s);
  am_array* out = make_index_array(n, width, s);
  try {
    // String keys sort as their derived chunk and length keys, dictionary keys as their rank columns.
    argsort_any(keys, n, out->values->ptr, width, s, &tls().last_stats);
  } catch (...) {
    am::release(out);
    throw;
  }
  if (!in_batch() && std::getenv("ARROWMETAL_SYNC_EVERY_CALL")) check_device_errors(s);
  return out;
}

am_array* take_one(am_array* a, am_array* idx) {
  cudaStream_t s = stream();
  am_array* out = new_array(a->pt, a->format, idx->length);
  const bool trusted = idx->perm_of >= 0 && idx->perm_of <= a->length;
  try {
    take_columns(&a, 1, idx, &out, !trusted, s);   // string columns go through take_strings
    if (!trusted) checkpoint(s);
  } catch (...) {
    am::release(out);
    throw;
  }
  return out;
}

am_array* slice_of(am_array* a, int64_t offset, int64_t length) {
  if (a->pt == PT_STRUCT) throw unsupported("+s: a struct result is exported, not computed on");
  am_array* o = new_array(a->pt, a->format, length);
  if (a->dictionary) {
    retain(a->dictionary);
    o->dictionary = a->dictionary;
  }
  o->values = a->values;
  o->bytes = a->bytes;
  o->value_offset = a->value_offset + offset;
  o->validity = a->validity;
  o->validity_offset = a->validity_offset + offset;
  o->last_stream = a->last_stream;
  o->shared_read = a->shared_read;
  o->ready = a->ready;
  if (a->perm_of >= 0) o->perm_of = a->perm_of;
  if (a->null_count == 0 || !a->validity) {
    o->null_count = 0;
    o->validity.reset();
  } else if (offset == 0 && length == a->length && a->null_count >= 0) {
    o->null_count = a->null_count;
  } else {
    // Count the slice's nulls from the host copy of its bitmap bits.
    const int64_t nb = (o->validity_offset + length + 7) / 8 - o->validity_offset / 8;
    std::vector<uint8_t> h(size_t(std::max<int64_t>(nb, 1)));
    if (a->null_count < 0) resolve_null_count(a);
    if (!a->validity) { o->null_count = 0; o->validity.reset(); return o; }
    cudaStream_t s = (a->last_stream && !a->shared_read) ? a->last_stream : stream();
    AM_CUDA(cudaMemcpyAsync(h.data(), static_cast<const uint8_t*>(a->validity->ptr) + o->validity_offset / 8, size_t(nb),
                            cudaMemcpyDeviceToHost, s));
    AM_CUDA(cudaStreamSynchronize(s));
    o->null_count = host_null_count(h.data(), o->validity_offset & 7, length);
    if (o->null_count == 0) o->validity.reset();
  }
  return o;
}

}  // namespace

namespace am {
// A host array (or a dictionary array) copied into HBM on stream `s`; the caller keeps the struct and
// releases it (the copies are complete, or staged, when this returns).
am_array* import_copy(const ArrowSchema* schema, const ArrowArray* array, cudaStream_t s) {
  const int pt = parse_format(schema->format);
  check_host_array(schema, array);
  am_array* a = new_array(pt, schema->format, array->length);
  try {
    import_host(a, array, s);
    if (schema->dictionary) {
      am_array* d = new_array(parse_format(schema->dictionary->format), schema->dictionary->format,
                              array->dictionary->length);
      a->dictionary = d;
      import_host(d, array->dictionary, s);
    }
  } catch (...) {
    am::release(a);
    throw;
  }
  return a;
}
}  // namespace am

extern "C" {

const char* am_version(void) { return "0.6.1"; }

const char* am_device_name(void) {
  try {
    return intern(device().name);
  } catch (const Error& e) {
    set_last_error(e.what());
    return intern(std::string("unavailable: ") + e.what());
  }
}

const char* am_last_error(void) { return tls().last_error.c_str(); }

// ---- import

int am_import(const ArrowSchema* schema, ArrowArray* array, am_array** out) {
  if (!schema || !array || !out) return 2;
  return guard([&] {
    const int pt = parse_format(schema->format);
    check_host_array(schema, array);
    cudaStream_t s = stream();
    am_array* a = new_array(pt, schema->format, array->length);
    try {
      if (schema->dictionary) {
        // The codes, then the dictionary (both copied before the producer's release).
        import_host(a, array, s);
        am_array* d = new_array(parse_format(schema->dictionary->format), schema->dictionary->format,
                                array->dictionary->length);
        a->dictionary = d;
        import_host(d, array->dictionary, s);
        move_release(array);
        *out = a;
        return 0;
      }
      if (import_pinned_async(a, array)) {
        *out = a;
        return 0;
      }
      import_host(a, array, s);
    } catch (...) {
      am::release(a);
      throw;
    }
    move_release(array);
    *out = a;
    return 0;
  });
}

int am_import_device(const ArrowSchema* schema, ArrowDeviceArray* darr, am_array** out) {
  if (!schema || !darr || !out) return 2;
  return guard([&] {
    ArrowArray* array = &darr->array;
    const int pt = parse_format(schema->format);
    const int dt0 = darr->device_type;
    if ((pt_var(pt) || schema->dictionary) && dt0 == ARROW_DEVICE_CUDA)
      throw unsupported("am_import_device takes fixed-width CUDA arrays; import string and dictionary arrays from host memory");
    check_array_struct(schema, array);
    const int dt = darr->device_type;
    if (dt == ARROW_DEVICE_CPU || dt == ARROW_DEVICE_CUDA_HOST) return am_import(schema, array, out);
    if (dt != ARROW_DEVICE_CUDA) throw unsupported("device type " + std::to_string(dt) + " (CUDA, CUDA host and CPU are taken)");
    Device& d = device();
    if (darr->device_id != d.ordinal)
      throw invalid("array on CUDA device " + std::to_string(darr->device_id) + ", the library runs on " + std::to_string(d.ordinal));
    cudaStream_t s = stream();
    if (darr->sync_event) AM_CUDA(cudaStreamWaitEvent(s, *static_cast<cudaEvent_t*>(darr->sync_event), 0));
    // Zero copy: the producer's buffers stay where they are; its release runs with the last handle.
    auto held = std::shared_ptr<ArrowArray>(new ArrowArray(*array), [](ArrowArray* p) {
      if (p->release) p->release(p);
      delete p;
    });
    array->release = nullptr;
    const int64_t n = held->length, off = held->offset;
    am_array* a = new_array(pt, schema->format, n);
    auto wrap = [&](const void* p) {
      auto b = std::make_shared<DevBuffer>();
      b->ptr = const_cast<void*>(p);
      b->owned = false;
      b->stream = s;
      b->on_release = [held] {};
      return b;
    };
    a->values = wrap(held->buffers[1]);
    a->value_offset = off;
    a->validity_offset = off;
    const uint8_t* vb = static_cast<const uint8_t*>(held->buffers[0]);
    if (vb && held->null_count != 0) {
      a->validity = wrap(vb);
      if (held->null_count > 0) {
        a->null_count = held->null_count;
      } else {
        const int64_t nb = (off + n + 7) / 8 - off / 8;
        std::vector<uint8_t> h(size_t(std::max<int64_t>(nb, 1)));
        AM_CUDA(cudaMemcpyAsync(h.data(), vb + off / 8, size_t(nb), cudaMemcpyDeviceToHost, s));
        AM_CUDA(cudaStreamSynchronize(s));
        a->null_count = host_null_count(h.data(), off & 7, n);
        if (a->null_count == 0) a->validity.reset();
      }
    } else {
      a->null_count = 0;
    }
    a->last_stream = s;
    *out = a;
    return 0;
  });
}

int am_import_chunks_supported(const ArrowSchema* schema) {
  if (!schema || !schema->format || schema->dictionary || schema->n_children) return 0;
  try {
    return pt_var(parse_format(schema->format)) ? 0 : 1;
  } catch (...) {
    return 0;
  }
}

int am_import_chunks(const ArrowSchema* schema, ArrowArray* arrays, int64_t n, am_array** out) {
  if (!schema || n < 0 || (n > 0 && !arrays) || !out) return 2;
  if (!am_import_chunks_supported(schema)) {
    set_last_error(std::string("Unsupported Arrow type: am_import_chunks does not take ") +
                   (schema->format ? schema->format : "(null format)") + " arrays; import their concatenation");
    return 3;
  }
  if (n == 1) return am_import(schema, arrays, out);
  return guard([&] {
    const int pt = parse_format(schema->format);
    int64_t total = 0, nulls = 0;
    for (int64_t i = 0; i < n; i++) {
      check_array_struct(schema, &arrays[i]);
      total += arrays[i].length;
      const uint8_t* vb = static_cast<const uint8_t*>(arrays[i].buffers[0]);
      if (vb) nulls += arrays[i].null_count >= 0 ? arrays[i].null_count : host_null_count(vb, arrays[i].offset, arrays[i].length);
    }
    cudaStream_t s = stream();
    am_array* a = new_array(pt, schema->format, total);
    try {
      const int w = pt_bytes(pt);
      a->null_count = nulls;
      auto bits_of = [&](int buf) {
        std::vector<uint8_t> h(size_t((total + 7) / 8 + 8), 0);
        int64_t at = 0;
        for (int64_t i = 0; i < n; i++) {
          const ArrowArray& c = arrays[i];
          const uint8_t* b = static_cast<const uint8_t*>(c.buffers[buf]);
          for (int64_t r = 0; r < c.length; r++, at++) {
            const bool v = b ? ((b[(c.offset + r) >> 3] >> ((c.offset + r) & 7)) & 1) : true;
            if (v) h[size_t(at >> 3)] |= uint8_t(1u << (at & 7));
          }
        }
        BufPtr d = DevBuffer::alloc(h.size() + 16, s);
        copy_h2d(d->ptr, h.data(), h.size(), s);
        AM_CUDA(cudaStreamSynchronize(s));
        return d;
      };
      if (nulls > 0) a->validity = bits_of(0);
      if (w == 0) {
        a->values = bits_of(1);
      } else {
        a->values = DevBuffer::alloc(size_t(total) * w + 16, s);
        int64_t at = 0;
        for (int64_t i = 0; i < n; i++) {
          const ArrowArray& c = arrays[i];
          const size_t bytes = size_t(c.length) * w;
          if (bytes && copy_h2d(static_cast<char*>(a->values->ptr) + size_t(at) * w,
                                static_cast<const char*>(c.buffers[1]) + size_t(c.offset) * w, bytes, s))
            AM_CUDA(cudaStreamSynchronize(s));
          at += c.length;
        }
      }
      a->last_stream = s;
    } catch (...) {
      am::release(a);
      throw;
    }
    for (int64_t i = 0; i < n; i++) move_release(&arrays[i]);
    *out = a;
    return 0;
  });
}

int am_set_import_threads(int n) {
  if (n < 0) return 2;
  set_import_threads(n);
  return 0;
}
int am_get_import_threads(void) { return import_threads(); }

// ---- export

int am_export(am_array* a, ArrowSchema* schema, ArrowArray* array) {
  if (!a || !array) return 2;
  if (a->pt == PT_STRUCT) {
    auto* ah = new StructArrayHold();
    auto* sh = schema ? new StructSchemaHold() : nullptr;
    const size_t k = a->children.size();
    ah->arrays.resize(k);
    if (sh) {
      sh->schemas.resize(k);
      sh->names = a->child_names;
    }
    for (size_t i = 0; i < k; i++) {
      std::memset(&ah->arrays[i], 0, sizeof(ArrowArray));
      if (sh) std::memset(&sh->schemas[i], 0, sizeof(ArrowSchema));
    }
    int rc = 0;
    for (size_t i = 0; i < k && rc == 0; i++) {
      rc = am_export(a->children[i], sh ? &sh->schemas[i] : nullptr, &ah->arrays[i]);
      if (rc == 0 && sh) sh->schemas[i].name = sh->names[i].c_str();
    }
    ArrowArray tmp_a{};
    tmp_a.release = release_struct_array;
    tmp_a.private_data = ah;
    if (rc != 0) {
      release_struct_array(&tmp_a);
      if (sh) {
        ArrowSchema tmp_s{};
        tmp_s.release = release_struct_schema;
        tmp_s.private_data = sh;
        release_struct_schema(&tmp_s);
      }
      return rc;
    }
    for (ArrowArray& c : ah->arrays) ah->ptrs.push_back(&c);
    array->length = a->length;
    array->null_count = 0;
    array->offset = 0;
    array->n_buffers = 1;
    array->n_children = int64_t(k);
    array->buffers = ah->buffers;
    array->children = ah->ptrs.data();
    array->dictionary = nullptr;
    array->release = release_struct_array;
    array->private_data = ah;
    if (sh) {
      for (ArrowSchema& c : sh->schemas) sh->ptrs.push_back(&c);
      schema->format = sh->format.c_str();
      schema->name = sh->name.c_str();
      schema->metadata = nullptr;
      schema->flags = 0;
      schema->n_children = int64_t(k);
      schema->children = sh->ptrs.data();
      schema->dictionary = nullptr;
      schema->release = release_struct_schema;
      schema->private_data = sh;
    }
    return 0;
  }
  return guard([&] {
    cudaStream_t s = a->last_stream ? a->last_stream : stream();
    const int64_t nulls = resolve_null_count(a);
    if (a->ready) {
      // The contents are complete at the ready event: copy on the export stream after it, without
      // waiting for the work enqueued since on the producing stream.
      s = d2h_stream();
      AM_CUDA(cudaStreamWaitEvent(s, a->ready->ev, 0));
    }
    const int64_t n = a->length;
    auto* h = new ExportHold();
    try {
      const int w = pt_bytes(a->pt);
      void* vals = nullptr;
      auto bits_down = [&](const BufPtr& b, int64_t off) -> void* {
        const int64_t nb = (n + 7) / 8;
        const int64_t first = off / 8;
        const int64_t span = (off + n + 7) / 8 - first;
        void* p = pinned_alloc(size_t(std::max<int64_t>(span, 1)) + 8);
        h->pinned.push_back(p);
        if (span > 0) copy_d2h(p, static_cast<const uint8_t*>(b->ptr) + first, size_t(span), s);
        if (off & 7) {
          std::vector<uint8_t> r = realign_bits(static_cast<const uint8_t*>(p), off & 7, n);
          std::memcpy(p, r.data(), size_t(nb));
        }
        return p;
      };
      if (pt_var(a->pt)) {
        // Offsets rebased to 0 and the bytes they span.
        const bool large = a->pt == PT_LSTR;
        const size_t ob = size_t(n + 1) * w;
        vals = pinned_alloc(ob);
        h->pinned.push_back(vals);
        copy_d2h(vals, static_cast<const char*>(a->values->ptr) + size_t(a->value_offset) * w, ob, s);
        const int64_t first = large ? static_cast<int64_t*>(vals)[0] : static_cast<int32_t*>(vals)[0];
        const int64_t last = large ? static_cast<int64_t*>(vals)[n] : static_cast<int32_t*>(vals)[n];
        for (int64_t i = 0; i <= n; i++) {
          if (large) static_cast<int64_t*>(vals)[i] -= first;
          else static_cast<int32_t*>(vals)[i] -= int32_t(first);
        }
        void* bytes = pinned_alloc(size_t(std::max<int64_t>(last - first, 1)));
        h->pinned.push_back(bytes);
        if (last > first) copy_d2h(bytes, static_cast<const char*>(a->bytes->ptr) + first, size_t(last - first), s);
        h->buffers[2] = bytes;
      } else if (w == 0) {
        vals = bits_down(a->values, a->value_offset);
      } else {
        const size_t bytes = size_t(n) * w;
        vals = pinned_alloc(std::max<size_t>(bytes, 1));
        h->pinned.push_back(vals);
        if (bytes) copy_d2h(vals, a->data(), bytes, s);
      }
      void* valid = nullptr;
      if (nulls > 0 && a->validity) valid = bits_down(a->validity, a->validity_offset);
      AM_CUDA(cudaStreamSynchronize(s));
      h->buffers[0] = valid;
      h->buffers[1] = vals;
    } catch (...) {
      for (void* p : h->pinned) pinned_free(p);
      delete h;
      throw;
    }
    ArrowSchema* dict_schema = nullptr;
    if (a->dictionary) {
      // A dictionary array: the codes above, and the dictionary exported beside them.
      h->dict_array = new ArrowArray{};
      dict_schema = schema ? new ArrowSchema{} : nullptr;
      const int rc = am_export(a->dictionary, dict_schema, h->dict_array);
      if (rc != 0) {
        const std::string why = am_last_error();
        delete dict_schema;
        delete h->dict_array;
        for (void* p : h->pinned) pinned_free(p);
        delete h;
        throw Error(why, rc);
      }
    }
    if (schema) {
      fill_schema(a, schema);
      if (dict_schema) {
        static_cast<ExportHold*>(schema->private_data)->dict_schema = dict_schema;
        schema->dictionary = dict_schema;
      }
    }
    array->length = n;
    array->null_count = nulls;
    array->offset = 0;
    array->n_buffers = pt_var(a->pt) ? 3 : 2;
    array->n_children = 0;
    array->buffers = h->buffers;
    array->children = nullptr;
    array->dictionary = h->dict_array;
    array->release = release_array;
    array->private_data = h;
    return 0;
  });
}

int am_export_device(am_array* a, ArrowSchema* schema, ArrowDeviceArray* darr) {
  if (!a || !darr) return 2;
  return guard([&] {
    if (a->pt == PT_STRUCT || a->dictionary)
      throw unsupported("am_export_device takes flat arrays; export struct and dictionary arrays with am_export");
    if (pt_var(a->pt)) throw unsupported("am_export_device takes fixed-width arrays; export string arrays with am_export");
    const int64_t nulls = resolve_null_count(a);
    if (a->validity && a->validity_offset != a->value_offset)
      throw invalid("export_device: the validity and value offsets differ");
    auto* h = new ExportHold();
    retain(a);
    h->keep = a;
    h->buffers[0] = (nulls > 0 && a->validity) ? a->validity->ptr : nullptr;
    h->buffers[1] = a->values ? a->values->ptr : nullptr;
    if (schema) fill_schema(a, schema);
    ArrowArray* array = &darr->array;
    array->length = a->length;
    array->null_count = nulls;
    array->offset = a->value_offset;
    array->n_buffers = 2;
    array->n_children = 0;
    array->buffers = h->buffers;
    array->children = nullptr;
    array->dictionary = nullptr;
    array->release = release_array;
    array->private_data = h;
    darr->device_id = device().ordinal;
    darr->device_type = ARROW_DEVICE_CUDA;
    // The buffers are ready once the producing stream reaches this point.
    sync_stream(a->last_stream ? a->last_stream : stream());
    darr->sync_event = nullptr;
    std::memset(darr->reserved, 0, sizeof(darr->reserved));
    return 0;
  });
}

void am_release(am_array* a) {
  try {
    am::release(a);
  } catch (...) {
  }
}
int64_t am_length(am_array* a) { return a ? a->length : -1; }
int64_t am_null_count(am_array* a) {
  if (!a) return -1;
  try {
    return resolve_null_count(a);
  } catch (const Error& e) {
    set_last_error(e.what());
    return -1;
  }
}
const char* am_format(am_array* a) { return a ? intern(a->format) : nullptr; }
const char* am_compute_format(am_array* a) { return am_format(a); }

// ---- selection

int am_take(am_array* a, am_array* indices, am_array** out) {
  if (!a || !indices || !out) return 2;
  return guard([&] {
    *out = take_one(a, indices);
    return 0;
  });
}

int am_take_columns(am_array** columns, int64_t count, am_array* indices, am_array** outs) {
  if (!columns || !indices || !outs || count <= 0) return 2;
  for (int64_t i = 0; i < count; i++) if (!columns[i]) return 2;
  return guard([&] {
    cudaStream_t s = stream();
    std::vector<am_array*> res(size_t(count), nullptr);
    try {
      bool trusted = indices->perm_of >= 0;
      for (int64_t i = 0; i < count; i++) {
        res[size_t(i)] = new_array(columns[i]->pt, columns[i]->format, indices->length);
        if (indices->perm_of > columns[i]->length) trusted = false;
      }
      // Columns of one length share a launch.
      size_t i = 0;
      while (i < size_t(count)) {
        size_t j = i + 1;
        while (j < size_t(count) && columns[j]->length == columns[i]->length) j++;
        take_columns(columns + i, int(j - i), indices, res.data() + i, !trusted, s);
        i = j;
      }
      if (!trusted) checkpoint(s);
    } catch (...) {
      for (am_array* r : res) am::release(r);
      throw;
    }
    for (int64_t i = 0; i < count; i++) outs[i] = res[size_t(i)];
    return 0;
  });
}

int am_slice(am_array* a, int64_t offset, int64_t length, am_array** out) {
  if (!a || !out) return 2;
  if (offset < 0 || length < 0 || offset + length > a->length) {
    set_last_error("Invalid ArrowArray: slice out of range");
    return 1;
  }
  return guard([&] {
    *out = slice_of(a, offset, length);
    return 0;
  });
}

// ---- sorting

int am_argsort_ex3(am_array* a, int descending, int null_placement, int float_order, int index_width, am_array** out) {
  if (!a || !out) return 2;
  return guard([&] {
    if (index_width != 4 && index_width != 8) throw invalid("index_width must be 4 or 8");
    std::vector<SortKey> k(1);
    k[0] = SortKey{a, descending != 0, null_placement == 1, float_order};
    *out = argsort_keys(k, index_width, "argsort");
    return 0;
  });
}
int am_argsort_device_noalloc(const char* format, const void* values, const void* validity, int64_t offset,
                              int64_t length, int descending, int null_placement, int float_order,
                              uint32_t* indices, void* stream) {
  return guard([&] {
    const int pt = parse_format(format);
    argsort_noalloc(pt, values, static_cast<const uint8_t*>(validity), offset, length, descending != 0,
                    null_placement == 1, float_order, indices, static_cast<cudaStream_t>(stream));
    return 0;
  });
}
int am_argsort_ex2(am_array* a, int descending, int null_placement, int float_order, am_array** out) {
  return am_argsort_ex3(a, descending, null_placement, float_order, 4, out);
}
int am_argsort_ex(am_array* a, int descending, int null_placement, am_array** out) {
  return am_argsort_ex2(a, descending, null_placement, 0, out);
}
int am_argsort(am_array* a, int descending, am_array** out) { return am_argsort_ex2(a, descending, 0, 0, out); }

int am_sort_ex2(am_array* a, int descending, int null_placement, int float_order, am_array** out) {
  if (!a || !out) return 2;
  return guard([&] {
    std::vector<SortKey> k(1);
    k[0] = SortKey{a, descending != 0, null_placement == 1, float_order};
    // A key map that is a bijection: the sorted column is rebuilt from the sorted keys, no gather
    // (the reference's sortedByInvertingKeys, Sources/ArrowMetal/Kernels/Sort.swift:509-619).
    if (a->length > 0 && float_order_ok(float_order) >= 0 && key_invertible(k[0])) {
      check_index_rows(a->length, "sort");
      cudaStream_t s = stream();
      use_on(a, s);
      am_array* sorted = new_array(a->pt, a->format, a->length);
      try {
        radix_sort(k, a->length, nullptr, 4, sorted, s, &tls().last_stats);
      } catch (...) {
        am::release(sorted);
        throw;
      }
      *out = sorted;
      return 0;
    }
    am_array* idx = argsort_keys(k, 4, "sort");
    am_array* r = nullptr;
    try {
      r = take_one(a, idx);
    } catch (...) {
      am::release(idx);
      throw;
    }
    am::release(idx);
    *out = r;
    return 0;
  });
}
int am_sort_ex(am_array* a, int descending, int null_placement, am_array** out) {
  return am_sort_ex2(a, descending, null_placement, 0, out);
}
int am_sort(am_array* a, int descending, am_array** out) { return am_sort_ex2(a, descending, 0, 0, out); }

int am_top_k_ex(am_array* a, int64_t k, int largest, int null_placement, int float_order, am_array** out) {
  if (!a || !out) return 2;
  if (k < 0) {
    set_last_error("Invalid ArrowArray: top_k needs k >= 0");
    return 1;
  }
  return guard([&] {
    std::vector<SortKey> key(1);
    key[0] = SortKey{a, largest != 0, null_placement == 1, float_order};
    if (k == 0 || a->length == 0) {
      float_order_ok(float_order);
      *out = make_index_array(0, 4, stream());
      return 0;
    }
    // k below the rows: radix selection, unless it would take most of the value rows anyway.
    if (k < a->length) {
      float_order_ok(float_order);
      check_index_rows(a->length, "top_k");
      cudaStream_t s = stream();
      use_on(a, s);
      if (am_array* r = radix_top_k(key[0], k, s)) {
        checkpoint(s);
        *out = r;
        return 0;
      }
    }
    am_array* idx = argsort_keys(key, 4, "top_k");
    const int64_t m = std::min<int64_t>(k, idx->length);
    if (m == idx->length) {
      *out = idx;
      return 0;
    }
    am_array* r = slice_of(idx, 0, m);
    am::release(idx);
    *out = r;
    return 0;
  });
}
int am_top_k(am_array* a, int64_t k, int largest, am_array** out) { return am_top_k_ex(a, k, largest, 0, 0, out); }

// ---- sort consumers (Sources/ArrowMetalC/ArrowMetalC_Options.swift:134-143, :228-320)

int am_partition_nth_ex(am_array* a, int64_t pivot, int null_placement, am_array** out) {
  if (!a || !out) return 2;
  return guard([&] {
    if (a->pt == PT_STRUCT) throw unsupported("+s: a struct result is exported, not computed on");
    if (pivot < 0 || pivot > a->length)
      throw invalid("partition index " + std::to_string(pivot) + " is outside 0..." + std::to_string(a->length));
    check_index_rows(a->length, "partition_nth_indices");
    SortKey key{a, false, null_placement == 1, 0};
    if (a->length == 0) {
      *out = make_index_array(0, 4, stream());
      return 0;
    }
    cudaStream_t s = stream();
    use_on(a, s);
    if (am_array* r = radix_partition_nth(key, pivot, s)) {
      checkpoint(s);
      *out = r;
      return 0;
    }
    // A string column: the stable argsort is itself such a partition.
    std::vector<SortKey> k{key};
    *out = argsort_keys(k, 4, "partition_nth_indices");
    return 0;
  });
}
int am_partition_nth_indices(am_array* a, int64_t n, am_array** out) { return am_partition_nth_ex(a, n, 0, out); }

int am_rank_ex(am_array* a, int tiebreaker, int descending, int null_placement, am_array** out) {
  if (!a || !out) return 2;
  return guard([&] {
    if (tiebreaker < 0 || tiebreaker > 3) throw invalid("unknown rank tiebreaker " + std::to_string(tiebreaker));
    check_index_rows(a->length, "rank");
    *out = rank_of(a, tiebreaker, descending != 0, null_placement == 1, true, stream());
    return 0;
  });
}

int am_rank_quantile_ex(am_array* a, int op, int descending, int null_placement, am_array** out) {
  if (!a || !out) return 2;
  return guard([&] {
    if (op < 0 || op > 2) throw invalid("unknown rank op " + std::to_string(op));
    check_index_rows(a->length, "rank");
    *out = rank_of(a, RANK_QUANTILE + op, descending != 0, null_placement == 1, true, stream());
    return 0;
  });
}
int am_rank(am_array* a, int op, am_array** out) { return am_rank_quantile_ex(a, op, 0, 0, out); }

// The ranking ops of am_window (0 row_number, 1 rank, 2 dense_rank, 3 percent_rank, 4 cume_dist):
// ascending, nulls last and one tie group, every NaN one value after +inf.
int am_window(am_array* a, int op, int64_t p1, int64_t p2, const void* scalar_or_null, am_array** out) {
  (void)p1;
  (void)p2;
  (void)scalar_or_null;
  if (!a || !out) return 2;
  return guard([&] {
    static const int fn[] = {RANK_FIRST, RANK_MIN, RANK_DENSE, RANK_PERCENT, RANK_CUME};
    if (op < 0 || op > 12) throw invalid("unknown window op " + std::to_string(op));
    if (op > 4) throw unsupported("window op " + std::to_string(op) + " (shifts, differences, running and rolling windows are not on the sort path)");
    check_index_rows(a->length, "window");
    *out = rank_of(a, fn[op], false, false, false, stream());
    return 0;
  });
}

int am_unique_ex(am_array* a, int order, am_array** out) {
  if (!a || !out) return 2;
  return guard([&] {
    check_index_rows(a->length, "unique");
    *out = unique_of(a, order != 1, nullptr, stream());
    return 0;
  });
}
int am_unique(am_array* a, am_array** out) { return am_unique_ex(a, 1, out); }

int am_value_counts_ex(am_array* a, int order, am_array** out) {
  if (!a || !out) return 2;
  return guard([&] {
    check_index_rows(a->length, "value_counts");
    am_array* counts = nullptr;
    am_array* values = unique_of(a, order != 1, &counts, stream());
    am_array* st = new_array(PT_STRUCT, "+s", values->length);
    st->null_count = 0;
    st->children = {values, counts};
    st->child_names = {"values", "counts"};
    *out = st;
    return 0;
  });
}
int am_value_counts(am_array* a, am_array** out) { return am_value_counts_ex(a, 1, out); }

int am_lexsort_ex2(am_array** columns, const int* descending, const int* null_placement, const int* float_order,
                   int64_t count, am_array** out) {
  if (!columns || count <= 0 || !out) return 2;
  for (int64_t i = 0; i < count; i++) if (!columns[i]) return 2;
  return guard([&] {
    std::vector<SortKey> keys(static_cast<size_t>(count));
    for (int64_t i = 0; i < count; i++) {
      keys[size_t(i)] = SortKey{columns[i], descending ? descending[i] != 0 : false,
                                null_placement ? null_placement[i] == 1 : false, float_order ? float_order[i] : 0};
    }
    const int64_t n = columns[0]->length;
    for (auto& k : keys) if (k.col->length != n) throw length_mismatch(n, k.col->length);
    if (count > rs::MAX_KEYS) throw invalid("lexsort takes at most " + std::to_string(rs::MAX_KEYS) + " key columns");
    if (n == 0) {
      for (auto& k : keys) float_order_ok(k.float_order);
      *out = make_index_array(0, 4, stream());
      return 0;
    }
    *out = argsort_keys(keys, 4, "lexsort");
    return 0;
  });
}
int am_lexsort_ex(am_array** columns, const int* descending, int64_t count, int null_placement, am_array** out) {
  if (!columns || count <= 0 || !out) return 2;
  std::vector<int> np(size_t(count), null_placement);
  return am_lexsort_ex2(columns, descending, np.data(), nullptr, count, out);
}
int am_lexsort(am_array** columns, const int* descending, int64_t count, am_array** out) {
  return am_lexsort_ex2(columns, descending, nullptr, nullptr, count, out);
}

// ---- batching

int am_batch_begin(void) {
  tls().batch_depth++;
  return 0;
}
int am_batch_end(void) {
  ThreadState& t = tls();
  if (t.batch_depth == 0) {
    set_last_error("am_batch_end without am_batch_begin");
    return 1;
  }
  if (--t.batch_depth > 0) return 0;
  std::vector<std::function<void()>> checks;
  checks.swap(t.deferred_checks);
  return guard([&] {
    for (auto& c : checks) c();
    sync_stream(stream());
    return 0;
  });
}

// ---- router

static std::atomic<int> g_router_mode{0};
int am_router_set_mode(int mode) {
  if (mode < 0 || mode > 2) return 2;
  g_router_mode.store(mode);
  return 0;
}
int am_router_get_mode(void) { return g_router_mode.load(); }

// ---- CUDA additions

int am_cuda_set_stream(void* s) {
  return guard([&] {
    device();
    set_stream_override(static_cast<cudaStream_t>(s));
    return 0;
  });
}
void* am_cuda_get_stream(void) {
  try {
    return stream();
  } catch (const Error& e) {
    set_last_error(e.what());
    return nullptr;
  }
}
int am_cuda_synchronize(void) {
  return guard([&] {
    check_device_errors(stream());
    return 0;
  });
}
int am_cuda_device(void) {
  try {
    return device().ordinal;
  } catch (const Error& e) {
    set_last_error(e.what());
    return -1;
  }
}

int am_last_sort_stats(am_sort_stats* out) {
  if (!out) return 2;
  return guard([&] {
    fill_last_sort_stats(out);
    return 0;
  });
}

int am_cuda_batch_tuning(am_batch_shape* out, int64_t capacity, int64_t* count) {
  if (!count || capacity < 0 || (capacity > 0 && !out)) return 2;
  return guard([&] {
    const auto v = batch_tuning();
    *count = int64_t(v.size());
    for (size_t i = 0; i < v.size() && int64_t(i) < capacity; i++)
      out[i] = am_batch_shape{v[i][0], v[i][1], v[i][2], v[i][3], v[i][4], v[i][5], v[i][6]};
    return 0;
  });
}

int am_cuda_profile(int on) {
  set_profiling(on != 0);
  return 0;
}
int64_t am_cuda_profile_count(void) {
  try {
    return int64_t(profile_entries().size());
  } catch (const Error& e) {
    set_last_error(e.what());
    return -1;
  }
}
int am_cuda_profile_entry(int64_t i, const char** name, int64_t* launches, double* total_ms) {
  return guard([&] {
    auto v = profile_entries();
    if (i < 0 || i >= int64_t(v.size())) throw invalid("profile entry out of range");
    if (name) *name = intern(v[size_t(i)].name);
    if (launches) *launches = v[size_t(i)].launches;
    if (total_ms) *total_ms = v[size_t(i)].total_ms;
    return 0;
  });
}
int am_cuda_profile_reset(void) {
  return guard([&] {
    profile_reset();
    return 0;
  });
}

int am_debug_set_max_row_index(int64_t max_row) {
  if (max_row < 0) return 2;
  set_max_row_index(max_row);
  return 0;
}
int am_debug_force_batch_shape(int shape) {
  return guard([&] {
    debug_force_batch_shape(shape);
    return 0;
  });
}
int am_debug_fail_alloc_after(int64_t n) {
  debug_fail_alloc_after(n);
  return 0;
}
int am_debug_skip_first_tile(int on) {
  debug_skip_first_tile(on != 0);
  return 0;
}

}  // extern "C"
