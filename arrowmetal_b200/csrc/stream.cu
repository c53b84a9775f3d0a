// Out-of-core sort of a stream of Arrow record batches: the reference's am_stream_* sort terminal
// (include/arrowmetal.h:1515-1611, Sources/ArrowMetal/Stream/StreamingSort.swift) on a B200.
//
// Runs. Batches are read ahead on a reader thread, copied into HBM and gathered until a run budget
// (a sixth of the free device memory by default). A run is sorted on the GPU as one table: the
// columns concatenated, one argsort over the keys (argsort_any: every key type the sort path takes)
// and one gather of every column. When the whole stream fits one run, that sorted run is the answer
// and nothing leaves HBM. Otherwise each sorted run is exported and written to a file under the
// scratch directory.
//
// Merge. The reference merges on the CPU with a heap of cursors; here the merge runs on the GPU in
// windows. A window holds the next block of every unfinished run, concatenated in run order, and is
// argsorted stably -- so equal keys keep run order, then row order, the stream's order. A row of the
// window may be emitted once no row still on disk can sort before it: every run j with rows left
// bounds that by its last loaded row (all of run j's unloaded rows sort after it). So the window's
// sorted prefix up to the earliest such bound row is final; it is gathered and emitted, each run's
// cursor advances by its rows in that prefix (a prefix of its block, the sort being stable), and the
// run that attains the bound has emitted its whole block, so every window makes progress.
#include <cuda_runtime.h>
#include <dirent.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <thread>

#include "am_internal.h"
#include "radix_sort.cuh"

using namespace am;

struct am_stream {
  ArrowArrayStream in{};
  ArrowSchema schema{};
  std::vector<int> select;          // output columns (schema child indices); empty: all of them
  int prefetch = 3;
  bool consumed = false;
  ~am_stream() {
    if (schema.release) schema.release(&schema);
    if (in.release) in.release(&in);
  }
};

struct am_stream_result {
  std::vector<std::string> names;
  std::vector<am_array*> cols;
  int64_t rows_out = 0, batches = 0, rows = 0, bytes_read = 0;
  double wall_s = 0, read_s = 0, gpu_s = 0, merge_s = 0, read_stall_s = 0, merge_stall_s = 0;
  ~am_stream_result() {
    for (am_array* c : cols) release(c);
  }
};

namespace {

thread_local std::string t_stream_error;

template <class F>
int stream_guard(F&& f) {
  try {
    return f();
  } catch (const Error& e) {
    t_stream_error = e.what();
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    t_stream_error = e.what();
    set_last_error(e.what());
    return 1;
  }
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// ---- device kernels of the merge

// q[r] = the sorted position of run r's bound row (its last loaded row), for the runs with rows left.
__global__ void __launch_bounds__(256) bound_positions_kernel(const uint32_t* __restrict__ perm, uint64_t w,
                                                              const uint32_t* __restrict__ bound_row, int k,
                                                              const uint32_t* __restrict__ run_start,
                                                              uint32_t* __restrict__ q) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < w; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t p = perm[i];
    int lo = 0, hi = k;                       // the run whose window range holds p
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (run_start[mid] <= p) lo = mid;
      else hi = mid;
    }
    if (bound_row[lo] == p) q[lo] = uint32_t(i);
  }
}

// counts[r] = rows of run r among the first e sorted positions.
__global__ void __launch_bounds__(256) emitted_per_run_kernel(const uint32_t* __restrict__ perm, uint64_t e,
                                                              const uint32_t* __restrict__ run_start, int k,
                                                              unsigned long long* __restrict__ counts) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < e; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t p = perm[i];
    int lo = 0, hi = k;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (run_start[mid] <= p) lo = mid;
      else hi = mid;
    }
    atomicAdd(&counts[lo], 1ull);
  }
}

// Bits [src_off, src_off + n) of `src` to bits [dst_off, ...) of `dst` (dst zeroed beforehand).
__global__ void __launch_bounds__(256) copy_bits_kernel(const uint8_t* __restrict__ src, int64_t src_off, uint64_t n,
                                                        uint32_t* __restrict__ dst, int64_t dst_off) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const int64_t s = src_off + int64_t(i);
    if ((src[s >> 3] >> (s & 7)) & 1) {
      const int64_t d = dst_off + int64_t(i);
      atomicOr(&dst[d >> 5], 1u << (d & 31));
    }
  }
}

__global__ void __launch_bounds__(256) set_bits_kernel(uint64_t n, uint32_t* __restrict__ dst, int64_t dst_off) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const int64_t d = dst_off + int64_t(i);
    atomicOr(&dst[d >> 5], 1u << (d & 31));
  }
}

// out[i] = src[i] - src[0] + base for i <= n.
template <typename OffT>
__global__ void __launch_bounds__(256) rebase_offsets_kernel(const OffT* __restrict__ src, uint64_t n, int64_t base,
                                                             OffT* __restrict__ out) {
  const OffT first = src[0];
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i <= n; i += uint64_t(gridDim.x) * blockDim.x)
    out[i] = OffT(int64_t(src[i] - first) + base);
}

int grid_of(uint64_t n) {
  return int(std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, uint64_t(device().sm_count) * 8)));
}

// ---- arrays

am_array* empty_like(int pt, const std::string& format, cudaStream_t s) {
  am_array* a = new_array(pt, format, 0);
  a->null_count = 0;
  a->values = DevBuffer::alloc(16, s);
  AM_CUDA(cudaMemsetAsync(a->values->ptr, 0, 16, s));
  if (pt_var(pt)) a->bytes = DevBuffer::alloc(16, s);
  a->last_stream = s;
  return a;
}

template <typename OffT>
void offsets_ends(const am_array* a, int64_t& first, int64_t& last, cudaStream_t s) {
  OffT h[2];
  const OffT* off = static_cast<const OffT*>(a->values->ptr) + a->value_offset;
  AM_CUDA(cudaMemcpyAsync(&h[0], off, sizeof(OffT), cudaMemcpyDeviceToHost, s));
  AM_CUDA(cudaMemcpyAsync(&h[1], off + a->length, sizeof(OffT), cudaMemcpyDeviceToHost, s));
  AM_CUDA(cudaStreamSynchronize(s));
  first = int64_t(h[0]);
  last = int64_t(h[1]);
}

// The parts end to end, one new array (same type; a dictionary column is not concatenated).
am_array* concat(const std::vector<am_array*>& parts, cudaStream_t s) {
  const am_array* p0 = parts.front();
  if (p0->dictionary) throw unsupported("an external sort of a dictionary column");
  if (parts.size() == 1) {
    retain(parts[0]);
    return parts[0];
  }
  int64_t n = 0, nulls = 0;
  for (am_array* p : parts) {
    use_on(p, s);
    n += p->length;
    nulls += resolve_null_count(p);
  }
  am_array* a = new_array(p0->pt, p0->format, n);
  try {
    a->last_stream = s;
    a->null_count = nulls;
    const uint64_t words = uint64_t(n + 31) / 32;
    if (nulls > 0) {
      a->validity = DevBuffer::alloc(size_t(words) * 4 + 16, s);
      AM_CUDA(cudaMemsetAsync(a->validity->ptr, 0, size_t(words) * 4 + 16, s));
      int64_t at = 0;
      for (am_array* p : parts) {
        uint32_t* dst = static_cast<uint32_t*>(a->validity->ptr);
        if (p->length == 0) continue;
        if (p->null_count != 0 && p->validity)
          copy_bits_kernel<<<grid_of(p->length), 256, 0, s>>>(p->valid_bits(), p->validity_offset, uint64_t(p->length), dst, at);
        else set_bits_kernel<<<grid_of(p->length), 256, 0, s>>>(uint64_t(p->length), dst, at);
        AM_CUDA(cudaGetLastError());
        at += p->length;
      }
    }
    const int w = pt_bytes(p0->pt);
    if (pt_var(p0->pt)) {
      const bool large = p0->pt == PT_LSTR;
      a->values = DevBuffer::alloc(size_t(n + 1) * w + 16, s);
      std::vector<std::pair<int64_t, int64_t>> spans;
      int64_t total = 0;
      for (am_array* p : parts) {
        int64_t f = 0, l = 0;
        if (p->length > 0) {
          if (large) offsets_ends<int64_t>(p, f, l, s);
          else offsets_ends<int32_t>(p, f, l, s);
        }
        spans.push_back({f, l});
        total += l - f;
      }
      if (!large && total > int64_t(INT32_MAX)) throw invalid("concatenated strings do not fit int32 offsets");
      a->bytes = DevBuffer::alloc(size_t(total) + 16, s);
      int64_t at = 0, base = 0;
      for (size_t i = 0; i < parts.size(); i++) {
        am_array* p = parts[i];
        if (p->length == 0) continue;
        char* out_off = static_cast<char*>(a->values->ptr) + size_t(at) * w;
        const char* src_off = static_cast<const char*>(p->values->ptr) + size_t(p->value_offset) * w;
        if (large)
          rebase_offsets_kernel<int64_t><<<grid_of(p->length + 1), 256, 0, s>>>(
              reinterpret_cast<const int64_t*>(src_off), uint64_t(p->length), base, reinterpret_cast<int64_t*>(out_off));
        else
          rebase_offsets_kernel<int32_t><<<grid_of(p->length + 1), 256, 0, s>>>(
              reinterpret_cast<const int32_t*>(src_off), uint64_t(p->length), base, reinterpret_cast<int32_t*>(out_off));
        AM_CUDA(cudaGetLastError());
        const int64_t len = spans[i].second - spans[i].first;
        if (len > 0)
          AM_CUDA(cudaMemcpyAsync(static_cast<char*>(a->bytes->ptr) + base,
                                  static_cast<const char*>(p->bytes->ptr) + spans[i].first, size_t(len),
                                  cudaMemcpyDeviceToDevice, s));
        at += p->length;
        base += len;
      }
      if (n == 0) AM_CUDA(cudaMemsetAsync(a->values->ptr, 0, size_t(w), s));
    } else if (w == 0) {
      a->values = DevBuffer::alloc(size_t(words) * 4 + 16, s);
      AM_CUDA(cudaMemsetAsync(a->values->ptr, 0, size_t(words) * 4 + 16, s));
      int64_t at = 0;
      for (am_array* p : parts) {
        if (p->length == 0) continue;
        copy_bits_kernel<<<grid_of(p->length), 256, 0, s>>>(static_cast<const uint8_t*>(p->values->ptr), p->value_offset,
                                                             uint64_t(p->length), static_cast<uint32_t*>(a->values->ptr), at);
        AM_CUDA(cudaGetLastError());
        at += p->length;
      }
    } else {
      a->values = DevBuffer::alloc(size_t(std::max<int64_t>(n, 1)) * w + 16, s);
      int64_t at = 0;
      for (am_array* p : parts) {
        if (p->length > 0)
          AM_CUDA(cudaMemcpyAsync(static_cast<char*>(a->values->ptr) + size_t(at) * w, p->data(), size_t(p->length) * w,
                                  cudaMemcpyDeviceToDevice, s));
        at += p->length;
      }
    }
  } catch (...) {
    release(a);
    throw;
  }
  return a;
}

// ---- runs on disk

// A sorted run spilled to a file: per column its validity bits (when it has nulls), its values (bits
// for boolean, offsets for strings) and, for strings, its bytes, each 64-byte aligned.
struct RunColumn {
  int pt = 0;
  std::string format;
  int64_t null_count = 0;
  size_t valid_at = 0, values_at = 0, bytes_at = 0, values_len = 0, bytes_len = 0;
};
struct Run {
  std::string path;
  int64_t rows = 0;
  std::vector<RunColumn> cols;
  const char* map = nullptr;
  size_t map_len = 0;
  ~Run() {
    if (map) munmap(const_cast<char*>(map), map_len);
    if (!path.empty()) std::remove(path.c_str());
  }
};

void write_all(FILE* f, const void* p, size_t n, size_t& at, const std::string& path) {
  if (n && std::fwrite(p, 1, n, f) != n) throw Error("external sort: writing " + path + " failed");
  at += n;
  static const char zero[64] = {0};
  const size_t pad = (64 - (at & 63)) & 63;
  if (pad && std::fwrite(zero, 1, pad, f) != pad) throw Error("external sort: writing " + path + " failed");
  at += pad;
}

std::unique_ptr<Run> spill(const std::vector<am_array*>& cols, const std::string& path) {
  auto run = std::make_unique<Run>();
  run->rows = cols.front()->length;
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw Error("external sort: cannot create " + path);
  run->path = path;
  size_t at = 0;
  try {
    for (am_array* c : cols) {
      ArrowArray arr{};
      if (am_export(c, nullptr, &arr) != 0) throw Error(am_last_error());
      RunColumn rc;
      rc.pt = c->pt;
      rc.format = c->format;
      rc.null_count = arr.null_count;
      const int64_t n = arr.length;
      const int w = pt_bytes(c->pt);
      try {
        if (arr.null_count > 0 && arr.buffers[0]) {
          rc.valid_at = at;
          write_all(f, arr.buffers[0], size_t((n + 7) / 8), at, path);
        }
        rc.values_at = at;
        if (pt_var(c->pt)) {
          rc.values_len = size_t(n + 1) * w;
          write_all(f, arr.buffers[1], rc.values_len, at, path);
          const int64_t last = c->pt == PT_LSTR ? static_cast<const int64_t*>(arr.buffers[1])[n]
                                                : static_cast<const int32_t*>(arr.buffers[1])[n];
          rc.bytes_at = at;
          rc.bytes_len = size_t(last);
          write_all(f, arr.buffers[2], rc.bytes_len, at, path);
        } else {
          rc.values_len = w == 0 ? size_t((n + 7) / 8) : size_t(n) * w;
          write_all(f, arr.buffers[1], rc.values_len, at, path);
        }
      } catch (...) {
        arr.release(&arr);
        throw;
      }
      arr.release(&arr);
      run->cols.push_back(rc);
    }
  } catch (...) {
    std::fclose(f);
    throw;
  }
  if (std::fclose(f) != 0) throw Error("external sort: writing " + path + " failed");
  const int fd = open(path.c_str(), O_RDONLY);
  if (fd < 0) throw Error("external sort: cannot open " + path);
  run->map_len = std::max<size_t>(at, 1);
  void* m = mmap(nullptr, run->map_len, PROT_READ, MAP_PRIVATE, fd, 0);
  close(fd);
  if (m == MAP_FAILED) throw Error("external sort: cannot map " + path);
  run->map = static_cast<const char*>(m);
  return run;
}

void append_bits(std::vector<uint8_t>& dst, int64_t dst_off, const uint8_t* src, int64_t src_off, int64_t n) {
  for (int64_t i = 0; i < n; i++) {
    const bool v = src ? ((src[(src_off + i) >> 3] >> ((src_off + i) & 7)) & 1) : true;
    if (v) dst[size_t((dst_off + i) >> 3)] |= uint8_t(1u << ((dst_off + i) & 7));
  }
}

// Rows [start[j], start[j] + len[j]) of every run j, end to end, of column c, as one HBM array.
am_array* load_window_column(const std::vector<std::unique_ptr<Run>>& runs, size_t c, const std::vector<int64_t>& start,
                             const std::vector<int64_t>& len, cudaStream_t s) {
  const RunColumn& c0 = runs.front()->cols[c];
  const int w = pt_bytes(c0.pt);
  int64_t n = 0;
  bool nulls = false;
  for (size_t j = 0; j < runs.size(); j++) {
    n += len[j];
    if (len[j] > 0 && runs[j]->cols[c].null_count > 0) nulls = true;
  }
  std::vector<uint8_t> valid(nulls ? size_t((n + 7) / 8 + 8) : 0, 0);
  std::vector<uint8_t> values, bytes;
  const bool large = c0.pt == PT_LSTR;
  if (pt_var(c0.pt)) values.resize(size_t(n + 1) * w);
  else values.resize(w == 0 ? size_t((n + 7) / 8 + 8) : size_t(std::max<int64_t>(n, 1)) * w, 0);
  int64_t at = 0, base = 0;
  for (size_t j = 0; j < runs.size(); j++) {
    if (len[j] == 0) continue;
    const Run& r = *runs[j];
    const RunColumn& rc = r.cols[c];
    const char* vals = r.map + rc.values_at;
    if (nulls) append_bits(valid, at, rc.null_count > 0 ? reinterpret_cast<const uint8_t*>(r.map + rc.valid_at) : nullptr,
                           start[j], len[j]);
    if (pt_var(c0.pt)) {
      auto off = [&](int64_t i) -> int64_t {
        return large ? reinterpret_cast<const int64_t*>(vals)[i] : reinterpret_cast<const int32_t*>(vals)[i];
      };
      const int64_t f = off(start[j]);
      for (int64_t i = 0; i < len[j]; i++) {
        const int64_t o = off(start[j] + i) - f + base;
        if (large) reinterpret_cast<int64_t*>(values.data())[at + i] = o;
        else reinterpret_cast<int32_t*>(values.data())[at + i] = int32_t(o);
      }
      const int64_t l = off(start[j] + len[j]) - f;
      bytes.insert(bytes.end(), r.map + rc.bytes_at + f, r.map + rc.bytes_at + f + l);
      base += l;
    } else if (w == 0) {
      append_bits(values, at, reinterpret_cast<const uint8_t*>(vals), start[j], len[j]);
    } else {
      std::memcpy(values.data() + size_t(at) * w, vals + size_t(start[j]) * w, size_t(len[j]) * w);
    }
    at += len[j];
  }
  if (pt_var(c0.pt)) {
    if (!large && base > int64_t(INT32_MAX)) throw invalid("a merge window's strings do not fit int32 offsets");
    if (large) reinterpret_cast<int64_t*>(values.data())[n] = base;
    else reinterpret_cast<int32_t*>(values.data())[n] = int32_t(base);
  }
  const void* bufs[3] = {nulls ? valid.data() : nullptr, values.data(), bytes.data()};
  ArrowArray arr{};
  arr.length = n;
  arr.null_count = -1;
  arr.offset = 0;
  arr.n_buffers = pt_var(c0.pt) ? 3 : 2;
  arr.buffers = bufs;
  ArrowSchema sch{};
  sch.format = c0.format.c_str();
  return import_copy(&sch, &arr, s);
}

// ---- IPC stream output

// An Arrow IPC stream writer (https://arrow.apache.org/docs/format/Columnar.html#ipc-streaming-format)
// for the flat types the sort path carries: a Schema message, one RecordBatch message per emitted
// batch, and the end-of-stream marker. The flatbuffer messages are built by FlatBuilder below.
struct FlatBuilder {
  // Flatbuffers are built back to front; `buf` holds the tail, `buf.size()` is the current offset from
  // the end.
  std::vector<uint8_t> buf;
  std::vector<std::pair<uint16_t, uint32_t>> fields;   // (slot, offset-from-end of the field's value)
  uint32_t table_start = 0;

  uint32_t size() const { return uint32_t(buf.size()); }
  void pad_to(size_t align, size_t extra = 0) {
    while ((buf.size() + extra) % align) buf.insert(buf.begin(), 0);
  }
  template <typename T>
  uint32_t push(T v) {
    pad_to(sizeof(T));
    uint8_t b[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));
    buf.insert(buf.begin(), b, b + sizeof(T));
    return size();
  }
  // An offset (uoffset_t) to something `target` from the end: relative to where it is written.
  uint32_t push_offset(uint32_t target) {
    pad_to(4);
    const uint32_t here = size() + 4;
    return push<uint32_t>(here - target);
  }
  uint32_t string(const std::string& s) {
    pad_to(4, s.size() + 1);
    buf.insert(buf.begin(), 0);
    buf.insert(buf.begin(), s.begin(), s.end());
    return push<uint32_t>(uint32_t(s.size()));
  }
  uint32_t offset_vector(const std::vector<uint32_t>& targets) {
    pad_to(4, targets.size() * 4);
    for (size_t i = targets.size(); i-- > 0;) push_offset(targets[i]);
    return push<uint32_t>(uint32_t(targets.size()));
  }
  // A vector of structs of `elem` bytes each, given as raw little-endian bytes.
  uint32_t struct_vector(const std::vector<uint8_t>& raw, size_t elem, size_t align) {
    pad_to(std::max<size_t>(align, 4), raw.size());
    buf.insert(buf.begin(), raw.begin(), raw.end());
    return push<uint32_t>(uint32_t(raw.size() / elem));
  }
  void start() {
    fields.clear();
    table_start = size();
  }
  template <typename T>
  void add(uint16_t slot, T v) {
    fields.push_back({slot, push<T>(v)});
  }
  void add_offset(uint16_t slot, uint32_t target) { fields.push_back({slot, push_offset(target)}); }
  uint32_t end() {
    // The table: its soffset to the vtable, then the fields already pushed.
    const uint32_t obj = push<int32_t>(0);
    uint16_t max_slot = 0;
    for (auto& f : fields) max_slot = std::max<uint16_t>(max_slot, uint16_t(f.first + 1));
    std::vector<uint16_t> vt(size_t(max_slot) + 2, 0);
    vt[0] = uint16_t((max_slot + 2) * 2);
    vt[1] = uint16_t(obj - table_start);
    for (auto& f : fields) vt[size_t(f.first) + 2] = uint16_t(obj - f.second);
    for (size_t i = vt.size(); i-- > 0;) {
      uint8_t b[2];
      std::memcpy(b, &vt[i], 2);
      buf.insert(buf.begin(), b, b + 2);
    }
    const uint32_t vt_pos = size();
    // soffset from the table to its vtable: table position minus vtable position (as addresses).
    const int32_t soff = int32_t(vt_pos) - int32_t(obj);
    std::memcpy(&buf[buf.size() - obj], &soff, 4);
    return obj;
  }
  std::vector<uint8_t> finish(uint32_t root) {
    pad_to(8, 4);
    push_offset(root);
    return buf;
  }
};

// The Arrow type of one column as a flatbuffer Type union (type code, table).
std::pair<uint8_t, uint32_t> ipc_type(FlatBuilder& b, const std::string& f) {
  auto int_type = [&](int bits, bool sgn) {
    b.start();
    b.add<int32_t>(0, bits);
    b.add<uint8_t>(1, sgn ? 1 : 0);
    return std::make_pair(uint8_t(2), b.end());
  };
  auto fp = [&](int16_t prec) {
    b.start();
    b.add<int16_t>(0, prec);
    return std::make_pair(uint8_t(3), b.end());
  };
  auto empty = [&](uint8_t code) {
    b.start();
    return std::make_pair(code, b.end());
  };
  auto unit_of = [](char c) -> int16_t { return c == 's' ? 0 : c == 'm' ? 1 : c == 'u' ? 2 : 3; };
  if (f == "c") return int_type(8, true);
  if (f == "C") return int_type(8, false);
  if (f == "s") return int_type(16, true);
  if (f == "S") return int_type(16, false);
  if (f == "i") return int_type(32, true);
  if (f == "I") return int_type(32, false);
  if (f == "l") return int_type(64, true);
  if (f == "L") return int_type(64, false);
  if (f == "e") return fp(0);
  if (f == "f") return fp(1);
  if (f == "g") return fp(2);
  if (f == "b") return empty(6);
  if (f == "z") return empty(4);
  if (f == "u") return empty(5);
  if (f == "Z") return empty(19);
  if (f == "U") return empty(20);
  if (f == "tdD" || f == "tdm") {
    b.start();
    b.add<int16_t>(0, f == "tdD" ? 0 : 1);
    return std::make_pair(uint8_t(8), b.end());
  }
  if (f.size() == 3 && f[0] == 't' && f[1] == 't') {
    b.start();
    b.add<int16_t>(0, unit_of(f[2]));
    b.add<int32_t>(1, (f[2] == 's' || f[2] == 'm') ? 32 : 64);
    return std::make_pair(uint8_t(9), b.end());
  }
  if (f.size() == 3 && f[0] == 't' && f[1] == 'D') {
    b.start();
    b.add<int16_t>(0, unit_of(f[2]));
    return std::make_pair(uint8_t(18), b.end());
  }
  if (f.size() >= 4 && f[0] == 't' && f[1] == 's' && f[3] == ':') {
    const std::string tz = f.substr(4);
    const uint32_t tzs = tz.empty() ? 0 : b.string(tz);
    b.start();
    b.add<int16_t>(0, unit_of(f[2]));
    if (!tz.empty()) b.add_offset(1, tzs);
    return std::make_pair(uint8_t(10), b.end());
  }
  throw unsupported("an IPC stream of " + f + " columns");
}

struct IpcWriter {
  FILE* f = nullptr;
  std::string path;
  std::vector<std::string> names;
  std::vector<std::string> formats;
  std::vector<bool> nullable;

  void message(const std::vector<uint8_t>& meta, const std::vector<std::vector<uint8_t>>& body) {
    const uint32_t cont = 0xFFFFFFFFu;
    std::vector<uint8_t> m = meta;
    while ((m.size() + 8) % 8) m.push_back(0);
    const int32_t len = int32_t(m.size());
    put(&cont, 4);
    put(&len, 4);
    put(m.data(), m.size());
    for (auto& b : body) put(b.data(), b.size());
  }
  void put(const void* p, size_t n) {
    if (n && std::fwrite(p, 1, n, f) != n) throw Error("external sort: writing " + path + " failed");
  }
  // Message { version: V5, header_type, header, bodyLength }.
  std::vector<uint8_t> wrap(FlatBuilder& b, uint8_t header_type, uint32_t header, int64_t body_len) {
    b.start();
    b.add<int64_t>(3, body_len);
    b.add_offset(2, header);
    b.add<uint8_t>(1, header_type);
    b.add<int16_t>(0, 4);
    return b.finish(b.end());
  }
  void open(const std::string& p, const std::vector<std::string>& n, const std::vector<std::string>& fmt) {
    path = p;
    names = n;
    formats = fmt;
    f = std::fopen(p.c_str(), "wb");
    if (!f) throw Error("external sort: cannot create " + p);
    FlatBuilder b;
    std::vector<uint32_t> fields;
    for (size_t i = 0; i < names.size(); i++) {
      const uint32_t nm = b.string(names[i]);
      const auto ty = ipc_type(b, formats[i]);
      const uint32_t children = b.offset_vector({});
      b.start();
      b.add_offset(0, nm);
      b.add<uint8_t>(1, 1);
      b.add<uint8_t>(2, ty.first);
      b.add_offset(3, ty.second);
      b.add_offset(5, children);
      fields.push_back(b.end());
    }
    const uint32_t fv = b.offset_vector(fields);
    b.start();
    b.add_offset(1, fv);
    const uint32_t schema = b.end();
    message(wrap(b, 1, schema, 0), {});
  }
  void batch(const std::vector<am_array*>& cols) {
    const int64_t n = cols.empty() ? 0 : cols.front()->length;
    std::vector<std::vector<uint8_t>> body;
    std::vector<int64_t> nodes, bufs;   // (length, null_count) pairs; (offset, length) pairs
    int64_t at = 0;
    auto add_buf = [&](const void* p, size_t len) {
      std::vector<uint8_t> v(static_cast<const uint8_t*>(p), static_cast<const uint8_t*>(p) + len);
      const size_t padded = (len + 7) / 8 * 8;
      v.resize(padded, 0);
      bufs.push_back(at);
      bufs.push_back(int64_t(len));
      at += int64_t(padded);
      body.push_back(std::move(v));
    };
    for (am_array* c : cols) {
      ArrowArray arr{};
      if (am_export(c, nullptr, &arr) != 0) throw Error(am_last_error());
      nodes.push_back(arr.length);
      nodes.push_back(arr.null_count);
      const int w = pt_bytes(c->pt);
      if (arr.null_count > 0 && arr.buffers[0]) add_buf(arr.buffers[0], size_t((n + 7) / 8));
      else add_buf(nullptr, 0);
      if (pt_var(c->pt)) {
        add_buf(arr.buffers[1], size_t(n + 1) * w);
        const int64_t last = c->pt == PT_LSTR ? static_cast<const int64_t*>(arr.buffers[1])[n]
                                              : static_cast<const int32_t*>(arr.buffers[1])[n];
        add_buf(arr.buffers[2], size_t(last));
      } else {
        add_buf(arr.buffers[1], w == 0 ? size_t((n + 7) / 8) : size_t(n) * w);
      }
      arr.release(&arr);
    }
    FlatBuilder b;
    std::vector<uint8_t> rn(nodes.size() * 8), rb(bufs.size() * 8);
    std::memcpy(rn.data(), nodes.data(), rn.size());
    std::memcpy(rb.data(), bufs.data(), rb.size());
    const uint32_t bv = b.struct_vector(rb, 16, 8);
    const uint32_t nv = b.struct_vector(rn, 16, 8);
    b.start();
    b.add<int64_t>(0, n);
    b.add_offset(1, nv);
    b.add_offset(2, bv);
    const uint32_t rec = b.end();
    message(wrap(b, 3, rec, at), body);
  }
  void close() {
    if (!f) return;
    const uint32_t eos[2] = {0xFFFFFFFFu, 0};
    put(eos, 8);
    const int rc = std::fclose(f);
    f = nullptr;
    if (rc != 0) throw Error("external sort: writing " + path + " failed");
  }
  ~IpcWriter() {
    if (f) std::fclose(f);
  }
};

// ---- IPC input

// Reading side of the flatbuffer format, bounds-checked against the message.
struct FlatReader {
  const uint8_t* p;
  size_t n;
  void need(size_t at, size_t len) const {
    if (at > n || len > n - at) throw invalid("a malformed Arrow IPC message");
  }
  template <typename T>
  T get(size_t at) const {
    need(at, sizeof(T));
    T v;
    std::memcpy(&v, p + at, sizeof(T));
    return v;
  }
  size_t deref(size_t at) const { return at + get<uint32_t>(at); }
  size_t root() const { return deref(0); }
  // The address of field `slot` of the table at `t`, or 0 when absent.
  size_t field(size_t t, int slot) const {
    const size_t vt = size_t(int64_t(t) - int64_t(get<int32_t>(t)));
    const uint16_t vsize = get<uint16_t>(vt);
    const size_t at = 4 + 2 * size_t(slot);
    if (at + 2 > vsize) return 0;
    const uint16_t off = get<uint16_t>(vt + at);
    return off ? t + off : 0;
  }
  template <typename T>
  T scalar(size_t t, int slot, T dflt) const {
    const size_t a = field(t, slot);
    return a ? get<T>(a) : dflt;
  }
  size_t table(size_t t, int slot) const {
    const size_t a = field(t, slot);
    return a ? deref(a) : 0;
  }
  std::string string(size_t t, int slot) const {
    const size_t a = table(t, slot);
    if (!a) return "";
    const uint32_t len = get<uint32_t>(a);
    need(a + 4, len);
    return std::string(reinterpret_cast<const char*>(p + a + 4), len);
  }
  // (element address, count) of a vector field.
  std::pair<size_t, uint32_t> vec(size_t t, int slot) const {
    const size_t a = table(t, slot);
    if (!a) return {0, 0};
    return {a + 4, get<uint32_t>(a)};
  }
};

// The C Data format string of an IPC Field's type.
std::string ipc_format(const FlatReader& r, size_t field) {
  const uint8_t code = r.scalar<uint8_t>(field, 2, 0);
  const size_t t = r.table(field, 3);
  static const char* units[] = {"s", "m", "u", "n"};
  auto unit = [&](int slot, int16_t dflt) {
    const int16_t u = t ? r.scalar<int16_t>(t, slot, dflt) : dflt;
    if (u < 0 || u > 3) throw invalid("an IPC time unit out of range");
    return std::string(units[u]);
  };
  switch (code) {
    case 2: {
      const int32_t bits = t ? r.scalar<int32_t>(t, 0, 0) : 0;
      const bool sgn = t ? r.scalar<uint8_t>(t, 1, 0) != 0 : false;
      if (bits == 8) return sgn ? "c" : "C";
      if (bits == 16) return sgn ? "s" : "S";
      if (bits == 32) return sgn ? "i" : "I";
      if (bits == 64) return sgn ? "l" : "L";
      break;
    }
    case 3: {
      const int16_t prec = t ? r.scalar<int16_t>(t, 0, 0) : 0;
      return prec == 0 ? "e" : prec == 1 ? "f" : "g";
    }
    case 4: return "z";
    case 5: return "u";
    case 6: return "b";
    case 8: return (t ? r.scalar<int16_t>(t, 0, 1) : 1) == 0 ? "tdD" : "tdm";
    case 9: return "tt" + unit(0, 1);
    case 10: return "ts" + unit(0, 0) + ":" + (t ? r.string(t, 1) : "");
    case 18: return "tD" + unit(0, 1);
    case 19: return "Z";
    case 20: return "U";
    default: break;
  }
  throw unsupported("an Arrow IPC column of type code " + std::to_string(code) +
                    " (primitive, boolean, temporal, string and binary columns are read)");
}

struct IpcMap {
  const uint8_t* data = nullptr;
  size_t size = 0;
  ~IpcMap() {
    if (data) munmap(const_cast<uint8_t*>(data), size);
  }
};

// One record batch handed out by the IPC source: the struct array and its children, pointing into the
// mapped file (held until the batch is released).
struct IpcBatch {
  std::shared_ptr<IpcMap> map;
  std::vector<ArrowArray> children;
  std::vector<ArrowArray*> child_ptrs;
  std::vector<std::vector<const void*>> buffers;
  const void* top_buffers[1] = {nullptr};
};

void release_ipc_batch(ArrowArray* a) {
  if (!a || !a->release) return;
  delete static_cast<IpcBatch*>(a->private_data);
  a->release = nullptr;
}

// A column of an IPC record batch must fit its buffers before anything reads it (on the host, or on
// the device after its import): the bitmap and the values cover `length` rows, and the offsets of a
// string or binary column rise from 0 or more to at most the size of its data buffer.
void check_ipc_buffers(int pt, int64_t length, int64_t null_count, const uint64_t (&lens)[3],
                       const void* const* bufs) {
  const uint64_t n = uint64_t(length);
  if (n == 0) return;
  const uint64_t bitmap = (n + 7) / 8;
  if (lens[0] != 0 && lens[0] < bitmap) throw invalid("an IPC validity bitmap shorter than its column");
  if (null_count > 0 && lens[0] == 0) throw invalid("an IPC column with nulls and no validity bitmap");
  // Each size is compared by division, so a row count near 2^64 / width cannot wrap the product
  // that a multiplication would form and pass as a small buffer.
  if (!pt_var(pt)) {
    if (pt == PT_BOOL) {
      if (lens[1] < bitmap) throw invalid("an IPC values buffer shorter than its column");
    } else if (n > lens[1] / uint64_t(pt_bytes(pt))) {
      throw invalid("an IPC values buffer shorter than its column");
    }
    return;
  }
  const uint64_t ow = uint64_t(pt_bytes(pt));
  if (n >= lens[1] / ow) throw invalid("an IPC offsets buffer shorter than its column");
  int64_t prev = 0;
  for (uint64_t i = 0; i <= n; i++) {
    int64_t o;
    if (ow == 4) {
      int32_t v;
      std::memcpy(&v, static_cast<const uint8_t*>(bufs[1]) + 4 * i, 4);
      o = v;
    } else {
      std::memcpy(&o, static_cast<const uint8_t*>(bufs[1]) + 8 * i, 8);
    }
    if (o < (i == 0 ? 0 : prev)) throw invalid("IPC string offsets that are negative or decreasing");
    prev = o;
  }
  if (uint64_t(prev) > lens[2]) throw invalid("IPC string offsets past the end of their data");
}

struct IpcSource {
  std::vector<std::string> files;
  size_t file = 0;
  std::shared_ptr<IpcMap> map;
  size_t pos = 0, end = 0;
  bool have_schema = false;
  std::vector<std::string> names, formats;
  std::vector<int> nbuf;          // buffers per column
  std::vector<int> pts;           // physical type per column
  std::string error;
  std::vector<std::string> owned_strings;   // schema strings handed out

  // Maps the next file, reads its schema (the first file's fixes the stream's; later ones must match).
  bool open_next() {
    map.reset();
    while (file < files.size()) {
      const std::string& path = files[file++];
      const int fd = ::open(path.c_str(), O_RDONLY);
      if (fd < 0) throw Error("cannot open " + path);
      struct stat stt;
      if (fstat(fd, &stt) != 0) {
        close(fd);
        throw Error("cannot stat " + path);
      }
      auto m = std::make_shared<IpcMap>();
      m->size = size_t(stt.st_size);
      if (m->size == 0) {
        close(fd);
        continue;
      }
      void* d = mmap(nullptr, m->size, PROT_READ, MAP_PRIVATE, fd, 0);
      close(fd);
      if (d == MAP_FAILED) throw Error("cannot map " + path);
      m->data = static_cast<const uint8_t*>(d);
      map = m;
      pos = 0;
      end = m->size;
      if (m->size >= 8 && std::memcmp(m->data, "ARROW1", 6) == 0) {
        // The file format: magic, the stream's messages, the footer, its length and the magic again.
        pos = 8;
        if (m->size >= 18) {
          int32_t flen = 0;
          std::memcpy(&flen, m->data + m->size - 10, 4);
          if (flen > 0 && size_t(flen) + 18 <= m->size) end = m->size - 10 - size_t(flen);
        }
      }
      // The schema message.
      size_t body = 0, body_len = 0;
      FlatReader r{};
      if (!message(r, body, body_len)) continue;
      const size_t msg = r.root();
      if (r.scalar<uint8_t>(msg, 1, 0) != 1) throw invalid(path + ": an Arrow IPC stream starts with its schema");
      schema_of(r, r.table(msg, 2), path);
      return true;
    }
    return false;
  }
  // The next message of the current file: its flatbuffer, and its body's position and length.
  bool message(FlatReader& r, size_t& body, size_t& body_len) {
    for (;;) {
      if (pos + 4 > end) return false;
      int32_t len = 0;
      std::memcpy(&len, map->data + pos, 4);
      size_t at = pos + 4;
      if (uint32_t(len) == 0xFFFFFFFFu) {
        if (at + 4 > end) return false;
        std::memcpy(&len, map->data + at, 4);
        at += 4;
      }
      if (len == 0) return false;                       // end of stream
      if (len < 0 || at + size_t(len) > end) throw invalid("a truncated Arrow IPC message");
      r = FlatReader{map->data + at, size_t(len)};
      const size_t msg = r.root();
      const int64_t blen = r.scalar<int64_t>(msg, 3, 0);
      body = at + size_t(len);
      if (blen < 0 || body + size_t(blen) > map->size) throw invalid("a truncated Arrow IPC message body");
      body_len = size_t(blen);
      pos = body + body_len;
      return true;
    }
  }
  void schema_of(const FlatReader& r, size_t sch, const std::string& path) {
    if (!sch) throw invalid(path + ": an Arrow IPC schema message without a schema");
    const auto fv = r.vec(sch, 1);
    std::vector<std::string> nm, fm;
    std::vector<int> nb, pt;
    for (uint32_t i = 0; i < fv.second; i++) {
      const size_t f = r.deref(fv.first + 4 * size_t(i));
      if (r.field(f, 4)) throw unsupported("dictionary-encoded columns in an Arrow IPC file");
      if (r.vec(f, 5).second != 0) throw unsupported("nested columns in an Arrow IPC file");
      nm.push_back(r.string(f, 0));
      fm.push_back(ipc_format(r, f));
      pt.push_back(parse_format(fm.back().c_str()));
      nb.push_back(pt_var(pt.back()) ? 3 : 2);
    }
    if (have_schema) {
      if (nm != names || fm != formats) throw invalid(path + ": its schema differs from the first file's");
      return;
    }
    names = nm;
    formats = fm;
    nbuf = nb;
    pts = pt;
    have_schema = true;
  }
  // The next record batch, or false at the end of the last file.
  bool next(ArrowArray* out) {
    for (;;) {
      if (!map && !open_next()) return false;
      FlatReader r{};
      size_t body = 0, body_len = 0;
      if (!message(r, body, body_len)) {
        map.reset();
        continue;
      }
      const size_t msg = r.root();
      const uint8_t type = r.scalar<uint8_t>(msg, 1, 0);
      if (type == 2) throw unsupported("dictionary batches in an Arrow IPC file");
      if (type != 3) continue;
      const size_t rb = r.table(msg, 2);
      if (!rb) throw invalid("a record batch message without its batch");
      if (r.field(rb, 3)) throw unsupported("compressed Arrow IPC bodies (write them uncompressed)");
      const int64_t length = r.scalar<int64_t>(rb, 0, 0);
      if (length < 0) throw invalid("an IPC record batch of negative length");
      const auto nodes = r.vec(rb, 1);
      const auto bufs = r.vec(rb, 2);
      if (nodes.second != names.size()) throw invalid("a record batch with the wrong number of columns");
      auto* b = new IpcBatch();
      b->map = map;
      b->children.resize(names.size());
      b->buffers.resize(names.size());
      size_t bi = 0;
      try {
        for (size_t c = 0; c < names.size(); c++) {
          ArrowArray& a = b->children[c];
          a = ArrowArray{};
          a.length = r.get<int64_t>(nodes.first + 16 * c);
          a.null_count = r.get<int64_t>(nodes.first + 16 * c + 8);
          a.n_buffers = nbuf[c];
          if (a.length != length || a.null_count < 0 || a.null_count > a.length)
            throw invalid("an IPC column whose length or null count does not fit its record batch");
          uint64_t lens[3] = {0, 0, 0};
          for (int k = 0; k < nbuf[c]; k++, bi++) {
            if (bi >= bufs.second) throw invalid("a record batch with too few buffers");
            const int64_t off = r.get<int64_t>(bufs.first + 16 * bi);
            const int64_t len = r.get<int64_t>(bufs.first + 16 * bi + 8);
            if (off < 0 || len < 0 || uint64_t(off) > body_len || uint64_t(len) > body_len - uint64_t(off))
              throw invalid("an IPC buffer outside its body");
            lens[k] = uint64_t(len);
            b->buffers[c].push_back(len > 0 ? map->data + body + size_t(off) : nullptr);
          }
          check_ipc_buffers(pts[c], a.length, a.null_count, lens, b->buffers[c].data());
          a.buffers = b->buffers[c].data();
          a.release = [](ArrowArray* x) { x->release = nullptr; };   // the parent owns the memory
          b->child_ptrs.push_back(&a);
        }
      } catch (...) {
        delete b;
        throw;
      }
      *out = ArrowArray{};
      out->length = length;
      out->null_count = 0;
      out->n_buffers = 1;
      out->buffers = b->top_buffers;
      out->n_children = int64_t(names.size());
      out->children = b->child_ptrs.data();
      out->release = release_ipc_batch;
      out->private_data = b;
      return true;
    }
  }
};

// The IPC source as an Arrow C stream, so the sort reads it like any other producer.
struct IpcStreamState {
  IpcSource src;
};
int ipc_get_schema(ArrowArrayStream* st, ArrowSchema* out) {
  auto* s = static_cast<IpcStreamState*>(st->private_data);
  struct Hold {
    std::vector<ArrowSchema> kids;
    std::vector<ArrowSchema*> ptrs;
    std::vector<std::string> names, formats;
  };
  auto* h = new Hold();
  h->names = s->src.names;
  h->formats = s->src.formats;
  h->kids.resize(h->names.size());
  for (size_t i = 0; i < h->names.size(); i++) {
    ArrowSchema& k = h->kids[i];
    k = ArrowSchema{};
    k.format = h->formats[i].c_str();
    k.name = h->names[i].c_str();
    k.flags = ARROW_FLAG_NULLABLE;
    k.release = [](ArrowSchema* x) { x->release = nullptr; };
    h->ptrs.push_back(&k);
  }
  *out = ArrowSchema{};
  out->format = "+s";
  out->name = "";
  out->n_children = int64_t(h->names.size());
  out->children = h->ptrs.data();
  out->private_data = h;
  out->release = [](ArrowSchema* x) {
    delete static_cast<Hold*>(x->private_data);
    x->release = nullptr;
  };
  return 0;
}
int ipc_get_next(ArrowArrayStream* st, ArrowArray* out) {
  auto* s = static_cast<IpcStreamState*>(st->private_data);
  try {
    if (!s->src.next(out)) *out = ArrowArray{};
    return 0;
  } catch (const std::exception& e) {
    s->src.error = e.what();
    return 5;   // EIO
  }
}
const char* ipc_last_error(ArrowArrayStream* st) {
  return static_cast<IpcStreamState*>(st->private_data)->src.error.c_str();
}
void ipc_release(ArrowArrayStream* st) {
  delete static_cast<IpcStreamState*>(st->private_data);
  st->release = nullptr;
}

// ---- projection of a C stream (am_stream_export_c with selected columns)

// The selected children are moved out of each schema / batch the inner stream gives (their structs
// copied, the originals marked released), so the inner parent releases only what was not taken.
struct ProjectState {
  ArrowArrayStream inner{};
  std::vector<int> select;
  std::string error;
};
struct ProjectHold {
  std::vector<ArrowSchema> schemas;
  std::vector<ArrowArray> arrays;
  std::vector<ArrowSchema*> sptrs;
  std::vector<ArrowArray*> aptrs;
  ArrowSchema parent_schema{};
  ArrowArray parent_array{};
  const void* top_buffers[1] = {nullptr};
};
int project_get_schema(ArrowArrayStream* st, ArrowSchema* out) {
  auto* ps = static_cast<ProjectState*>(st->private_data);
  auto* h = new ProjectHold();
  int rc = ps->inner.get_schema(&ps->inner, &h->parent_schema);
  if (rc != 0) {
    delete h;
    return rc;
  }
  for (int ci : ps->select) {
    ArrowSchema* c = h->parent_schema.children[ci];
    h->schemas.push_back(*c);
    c->release = nullptr;
  }
  for (ArrowSchema& c : h->schemas) h->sptrs.push_back(&c);
  *out = ArrowSchema{};
  out->format = "+s";
  out->name = "";
  out->n_children = int64_t(h->sptrs.size());
  out->children = h->sptrs.data();
  out->private_data = h;
  out->release = [](ArrowSchema* x) {
    auto* hh = static_cast<ProjectHold*>(x->private_data);
    for (ArrowSchema& c : hh->schemas)
      if (c.release) c.release(&c);
    if (hh->parent_schema.release) hh->parent_schema.release(&hh->parent_schema);
    delete hh;
    x->release = nullptr;
  };
  return 0;
}
int project_get_next(ArrowArrayStream* st, ArrowArray* out) {
  auto* ps = static_cast<ProjectState*>(st->private_data);
  auto* h = new ProjectHold();
  int rc = ps->inner.get_next(&ps->inner, &h->parent_array);
  if (rc != 0 || !h->parent_array.release) {
    delete h;
    *out = ArrowArray{};
    return rc;
  }
  ArrowArray& p = h->parent_array;
  for (int ci : ps->select) {
    ArrowArray* c = p.children[ci];
    h->arrays.push_back(*c);
    c->release = nullptr;
    if (p.offset != 0) {
      h->arrays.back().offset += p.offset;
      h->arrays.back().length = p.length;
      h->arrays.back().null_count = -1;
    }
  }
  for (ArrowArray& c : h->arrays) h->aptrs.push_back(&c);
  *out = ArrowArray{};
  out->length = p.length;
  out->null_count = 0;
  out->n_buffers = 1;
  out->buffers = h->top_buffers;
  out->n_children = int64_t(h->aptrs.size());
  out->children = h->aptrs.data();
  out->private_data = h;
  out->release = [](ArrowArray* x) {
    auto* hh = static_cast<ProjectHold*>(x->private_data);
    for (ArrowArray& c : hh->arrays)
      if (c.release) c.release(&c);
    if (hh->parent_array.release) hh->parent_array.release(&hh->parent_array);
    delete hh;
    x->release = nullptr;
  };
  return 0;
}
const char* project_last_error(ArrowArrayStream* st) {
  auto* ps = static_cast<ProjectState*>(st->private_data);
  return ps->inner.get_last_error ? ps->inner.get_last_error(&ps->inner) : nullptr;
}
void project_release(ArrowArrayStream* st) {
  auto* ps = static_cast<ProjectState*>(st->private_data);
  if (ps->inner.release) ps->inner.release(&ps->inner);
  delete ps;
  st->release = nullptr;
}

// ---- the reader

// Pulls record batches from the C stream, `depth` ahead on its own thread (depth 0: on the caller's).
class Reader {
 public:
  Reader(ArrowArrayStream* in, int depth) : in_(in), depth_(depth) {
    if (depth_ > 0) th_ = std::thread([this] { loop(); });
  }
  ~Reader() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    if (th_.joinable()) th_.join();
    for (ArrowArray& a : q_)
      if (a.release) a.release(&a);
  }
  // The next batch (caller releases it), or false at the end of the stream.
  bool next(ArrowArray* out) {
    if (depth_ == 0) return pull(out);
    const auto t0 = std::chrono::steady_clock::now();
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return !q_.empty() || done_; });
    stall_s += seconds_since(t0);
    if (q_.empty()) {
      if (!error_.empty()) throw Error(error_);
      return false;
    }
    *out = q_.front();
    q_.pop_front();
    cv_.notify_all();
    return true;
  }
  double read_s = 0, stall_s = 0;

 private:
  bool pull(ArrowArray* out) {
    const auto t0 = std::chrono::steady_clock::now();
    *out = ArrowArray{};
    const int rc = in_->get_next(in_, out);
    read_s += seconds_since(t0);
    if (rc != 0) {
      const char* e = in_->get_last_error ? in_->get_last_error(in_) : nullptr;
      throw Error(std::string("the record batch stream failed: ") + (e ? e : std::strerror(rc)));
    }
    return out->release != nullptr;
  }
  void loop() {
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || int(q_.size()) < depth_; });
        if (stop_) return;
      }
      ArrowArray a{};
      bool more = false;
      std::string err;
      try {
        more = pull(&a);
      } catch (const std::exception& e) {
        err = e.what();
      }
      std::lock_guard<std::mutex> g(mu_);
      if (!err.empty() || !more) {
        error_ = err;
        done_ = true;
        cv_.notify_all();
        return;
      }
      q_.push_back(a);
      cv_.notify_all();
    }
  }
  ArrowArrayStream* in_;
  int depth_;
  std::thread th_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<ArrowArray> q_;
  bool done_ = false, stop_ = false;
  std::string error_;
};

// ---- the sort

struct SortSpec {
  std::vector<int> key_cols;        // indices into the batch columns
  std::vector<SortKey> options;     // descending / nulls_first / float_order per key (col unset)
};

std::vector<SortKey> keys_of(const SortSpec& spec, const std::vector<am_array*>& cols) {
  std::vector<SortKey> ks;
  for (size_t i = 0; i < spec.key_cols.size(); i++) {
    SortKey k = spec.options[i];
    k.col = cols[size_t(spec.key_cols[i])];
    ks.push_back(k);
  }
  return ks;
}

// The rows of `cols` in the order of `perm`'s first `m` entries.
std::vector<am_array*> gather(const std::vector<am_array*>& cols, am_array* perm, int64_t m, cudaStream_t s) {
  am_array* idx = perm;
  if (m != perm->length) {
    idx = new_array(PT_U32, "I", m);
    idx->values = perm->values;
    idx->null_count = 0;
    idx->perm_of = perm->perm_of;
    idx->last_stream = s;
  } else {
    retain(idx);
  }
  std::vector<am_array*> out(cols.size(), nullptr);
  try {
    for (size_t c = 0; c < cols.size(); c++) out[c] = new_array(cols[c]->pt, cols[c]->format, m);
    take_columns(cols.data(), int(cols.size()), idx, out.data(), false, s);
  } catch (...) {
    for (am_array* o : out) if (o) release(o);
    release(idx);
    throw;
  }
  release(idx);
  return out;
}

am_array* argsort_of(const std::vector<SortKey>& keys, int64_t n, cudaStream_t s) {
  check_index_rows(n, "external sort");
  am_array* perm = new_array(PT_U32, "I", n);
  perm->values = DevBuffer::alloc(size_t(std::max<int64_t>(n, 1)) * 4 + 16, s);
  perm->null_count = 0;
  perm->perm_of = n;
  perm->last_stream = s;
  try {
    argsort_any(keys, n, perm->values->ptr, 4, s, nullptr);
  } catch (...) {
    release(perm);
    throw;
  }
  return perm;
}

void release_all(std::vector<am_array*>& v) {
  for (am_array* a : v) if (a) release(a);
  v.clear();
}

struct Output {
  IpcWriter* ipc = nullptr;
  std::vector<std::vector<am_array*>> batches;     // collected (column order of `out_cols`)
  int64_t rows = 0;
};

void emit(Output& o, std::vector<am_array*>& cols) {
  if (cols.empty() || cols.front()->length == 0) {
    release_all(cols);
    return;
  }
  o.rows += cols.front()->length;
  if (o.ipc) {
    o.ipc->batch(cols);
    release_all(cols);
  } else {
    o.batches.push_back(cols);
    cols.clear();
  }
}

void external_sort(am_stream* st, const SortSpec& spec_in, const std::vector<std::string>& key_names, int64_t limit,
                   const char* scratch_dir, const char* sink_path, am_stream_result* res) {
  const auto t_wall = std::chrono::steady_clock::now();
  cudaStream_t s = stream();
  const ArrowSchema& sch = st->schema;
  if (!sch.format || std::strcmp(sch.format, "+s") != 0) throw invalid("a record batch stream's schema is a struct");
  // The columns a batch carries: the output columns, then any key column not among them.
  std::vector<int> out_idx = st->select;
  if (out_idx.empty())
    for (int64_t i = 0; i < sch.n_children; i++) out_idx.push_back(int(i));
  std::vector<int> need = out_idx;
  SortSpec spec = spec_in;
  for (size_t k = 0; k < key_names.size(); k++) {
    int ci = -1;
    for (int64_t i = 0; i < sch.n_children; i++)
      if (sch.children[i]->name && key_names[k] == sch.children[i]->name) ci = int(i);
    if (ci < 0) throw invalid("external sort: no column named \"" + key_names[k] + "\"");
    auto it = std::find(need.begin(), need.end(), ci);
    if (it == need.end()) {
      need.push_back(ci);
      spec.key_cols.push_back(int(need.size()) - 1);
    } else {
      spec.key_cols.push_back(int(it - need.begin()));
    }
  }
  for (int ci : need) {
    const ArrowSchema* c = sch.children[ci];
    parse_format(c->format);
    if (c->n_children) throw unsupported(std::string("an external sort of nested columns (") + c->format + ")");
    if (c->dictionary) throw unsupported("an external sort of a dictionary column");
  }
  for (int ci : out_idx) res->names.push_back(sch.children[ci]->name ? sch.children[ci]->name : "");
  const size_t n_out = out_idx.size();

  // The run budget: device bytes of gathered batches before a run is sorted (sorting a run holds about
  // three times its bytes: the batches, the concatenated columns and the sorted copy).
  size_t free_b = 0, total_b = 0;
  AM_CUDA(cudaMemGetInfo(&free_b, &total_b));
  size_t budget = free_b / 6;
  if (const char* e = std::getenv("ARROWMETAL_STREAM_RUN_BYTES")) budget = size_t(std::max<long long>(1, std::atoll(e)));

  IpcWriter ipc;
  Output out;
  if (sink_path) {
    std::vector<std::string> fmts;
    for (int ci : out_idx) fmts.push_back(sch.children[ci]->format);
    ipc.open(sink_path, res->names, fmts);
    out.ipc = &ipc;
  }

  // Scratch directory for spilled runs.
  std::string dir;
  bool made_dir = false;
  auto scratch = [&]() -> const std::string& {
    if (dir.empty()) {
      if (scratch_dir) {
        dir = scratch_dir;
        mkdir(dir.c_str(), 0700);
      } else {
        const char* tmp = std::getenv("TMPDIR");
        std::string tmpl = std::string(tmp ? tmp : "/tmp") + "/arrowmetal-sort-XXXXXX";
        std::vector<char> b(tmpl.begin(), tmpl.end());
        b.push_back(0);
        if (!mkdtemp(b.data())) throw Error("external sort: cannot create a scratch directory under " + tmpl);
        dir = b.data();
        made_dir = true;
      }
    }
    return dir;
  };

  std::vector<std::unique_ptr<Run>> runs;
  std::vector<std::vector<am_array*>> pending;   // gathered batches of the current run
  size_t pending_bytes = 0;
  std::vector<am_array*> last_run;               // the sorted run, while it may still be the only one
  auto device_bytes = [](const am_array* a) {
    size_t b = 0;
    for (const BufPtr* p : {&a->values, &a->bytes, &a->validity})
      if (*p) b += (*p)->bytes;
    return b;
  };

  auto sort_pending = [&]() {
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<am_array*> cols(need.size(), nullptr);
    try {
      for (size_t c = 0; c < need.size(); c++) {
        std::vector<am_array*> parts;
        for (auto& b : pending) parts.push_back(b[c]);
        cols[c] = concat(parts, s);
      }
    } catch (...) {
      release_all(cols);
      throw;
    }
    for (auto& b : pending) release_all(b);
    pending.clear();
    pending_bytes = 0;
    const int64_t n = cols.front()->length;
    am_array* perm = nullptr;
    std::vector<am_array*> sorted;
    try {
      perm = argsort_of(keys_of(spec, cols), n, s);
      sorted = gather(cols, perm, limit > 0 ? std::min<int64_t>(limit, n) : n, s);
    } catch (...) {
      if (perm) release(perm);
      release_all(cols);
      throw;
    }
    release(perm);
    release_all(cols);
    sync_stream(s);
    res->gpu_s += seconds_since(t0);
    return sorted;
  };
  auto spill_last = [&]() {
    // Unique within the machine: sorts of several threads or processes may share a scratch directory.
    static std::atomic<uint64_t> seq{0};
    const std::string path = scratch() + "/run-" + std::to_string(getpid()) + "-" + std::to_string(seq.fetch_add(1)) + ".amrun";
    runs.push_back(spill(last_run, path));
    release_all(last_run);
  };

  {
    Reader reader(&st->in, st->prefetch);
    try {
      ArrowArray batch{};
      while (reader.next(&batch)) {
        struct Rel { ArrowArray* a; ~Rel() { if (a->release) a->release(a); } } rel{&batch};
        res->batches++;
        res->rows += batch.length;
        if (batch.n_children != sch.n_children) throw invalid("a record batch does not match its stream's schema");
        std::vector<am_array*> cols;
        try {
          for (int ci : need) {
            ArrowArray child = *batch.children[ci];
            if (batch.offset != 0) {
              child.offset += batch.offset;
              child.length = batch.length;
              child.null_count = -1;
            }
            cols.push_back(import_copy(sch.children[ci], &child, s));
            res->bytes_read += int64_t(device_bytes(cols.back()));
          }
        } catch (...) {
          release_all(cols);
          throw;
        }
        for (am_array* c : cols) pending_bytes += device_bytes(c);
        pending.push_back(cols);
        if (pending_bytes >= budget) {
          if (!last_run.empty()) spill_last();
          last_run = sort_pending();
        }
      }
      if (!pending.empty()) {
        if (!last_run.empty()) spill_last();
        last_run = sort_pending();
      }
    } catch (...) {
      for (auto& b : pending) release_all(b);
      release_all(last_run);
      res->read_s = reader.read_s;
      throw;
    }
    res->read_s = reader.read_s;
    res->read_stall_s = reader.stall_s;
  }

  try {
    if (runs.empty()) {
      // One run: it is the answer, already in HBM.
      if (!last_run.empty()) {
        std::vector<am_array*> o(last_run.begin(), last_run.begin() + long(n_out));
        for (size_t c = n_out; c < last_run.size(); c++) release(last_run[c]);
        last_run.clear();
        emit(out, o);
      }
    } else {
      if (!last_run.empty()) spill_last();
      // The merge, in windows.
      const auto t0 = std::chrono::steady_clock::now();
      const int k = int(runs.size());
      size_t row_bytes = 0;
      for (const RunColumn& rc : runs.front()->cols) row_bytes += size_t(std::max(pt_bytes(rc.pt), 1)) + 1;
      for (auto& r : runs)
        for (const RunColumn& rc : r->cols)
          if (pt_var(rc.pt) && r->rows > 0) row_bytes += rc.bytes_len / size_t(r->rows) / size_t(k) + 1;
      const int64_t window_rows = std::max<int64_t>(int64_t(k), int64_t(budget / std::max<size_t>(row_bytes * 4, 1)));
      const int64_t block = std::max<int64_t>(1, window_rows / k);
      std::vector<int64_t> cursor(size_t(k), 0);
      BufPtr dev = DevBuffer::alloc(size_t(k) * 12 + 16, s);
      uint32_t* d_bound = static_cast<uint32_t*>(dev->ptr);
      uint32_t* d_start = d_bound + k;
      uint32_t* d_q = d_start + k;
      BufPtr dev_counts = DevBuffer::alloc(size_t(k) * 8 + 16, s);
      auto* d_counts = static_cast<unsigned long long*>(dev_counts->ptr);
      const size_t ks = static_cast<size_t>(k);
      std::vector<uint32_t> h_bound(ks), h_start(ks), h_q(ks);
      std::vector<unsigned long long> h_counts(ks);
      for (;;) {
        if (limit > 0 && out.rows >= limit) break;
        std::vector<int64_t> len(size_t(k), 0);
        int64_t w = 0;
        bool any_left = false;
        for (int j = 0; j < k; j++) {
          len[size_t(j)] = std::min<int64_t>(block, runs[size_t(j)]->rows - cursor[size_t(j)]);
          h_start[size_t(j)] = uint32_t(w);
          w += len[size_t(j)];
        }
        if (w == 0) break;
        for (int j = 0; j < k; j++) {
          const bool left = cursor[size_t(j)] + len[size_t(j)] < runs[size_t(j)]->rows;
          h_bound[size_t(j)] = left ? uint32_t(h_start[size_t(j)] + len[size_t(j)] - 1) : 0xFFFFFFFFu;
          any_left = any_left || left;
        }
        std::vector<am_array*> cols;
        am_array* perm = nullptr;
        try {
          for (size_t c = 0; c < need.size(); c++) cols.push_back(load_window_column(runs, c, cursor, len, s));
          perm = argsort_of(keys_of(spec, cols), w, s);
          int64_t e = w;
          if (any_left) {
            AM_CUDA(cudaMemcpyAsync(d_bound, h_bound.data(), size_t(k) * 4, cudaMemcpyHostToDevice, s));
            AM_CUDA(cudaMemcpyAsync(d_start, h_start.data(), size_t(k) * 4, cudaMemcpyHostToDevice, s));
            bound_positions_kernel<<<grid_of(uint64_t(w)), 256, 0, s>>>(static_cast<const uint32_t*>(perm->values->ptr),
                                                                        uint64_t(w), d_bound, k, d_start, d_q);
            AM_CUDA(cudaGetLastError());
            AM_CUDA(cudaMemcpyAsync(h_q.data(), d_q, size_t(k) * 4, cudaMemcpyDeviceToHost, s));
            AM_CUDA(cudaStreamSynchronize(s));
            for (int j = 0; j < k; j++)
              if (h_bound[size_t(j)] != 0xFFFFFFFFu) e = std::min<int64_t>(e, int64_t(h_q[size_t(j)]) + 1);
          } else {
            AM_CUDA(cudaMemcpyAsync(d_start, h_start.data(), size_t(k) * 4, cudaMemcpyHostToDevice, s));
          }
          if (limit > 0) e = std::min<int64_t>(e, limit - out.rows);
          AM_CUDA(cudaMemsetAsync(d_counts, 0, size_t(k) * 8, s));
          emitted_per_run_kernel<<<grid_of(uint64_t(e)), 256, 0, s>>>(static_cast<const uint32_t*>(perm->values->ptr),
                                                                      uint64_t(e), d_start, k, d_counts);
          AM_CUDA(cudaGetLastError());
          std::vector<am_array*> outc(cols.begin(), cols.begin() + long(n_out));
          std::vector<am_array*> emitted = gather(outc, perm, e, s);
          AM_CUDA(cudaMemcpyAsync(h_counts.data(), d_counts, size_t(k) * 8, cudaMemcpyDeviceToHost, s));
          AM_CUDA(cudaStreamSynchronize(s));
          for (int j = 0; j < k; j++) cursor[size_t(j)] += int64_t(h_counts[size_t(j)]);
          emit(out, emitted);
        } catch (...) {
          release_all(cols);
          if (perm) release(perm);
          throw;
        }
        release_all(cols);
        release(perm);
      }
      res->merge_s += seconds_since(t0);
    }
  } catch (...) {
    release_all(last_run);
    for (auto& b : out.batches) release_all(b);
    runs.clear();
    if (made_dir) rmdir(dir.c_str());
    throw;
  }
  runs.clear();
  if (made_dir) rmdir(dir.c_str());

  res->rows_out = out.rows;
  if (out.ipc) {
    ipc.close();
  } else {
    // Collected: one array per output column.
    for (size_t c = 0; c < n_out; c++) {
      if (out.batches.empty()) {
        const ArrowSchema* cs = sch.children[out_idx[c]];
        res->cols.push_back(empty_like(parse_format(cs->format), cs->format, s));
        continue;
      }
      std::vector<am_array*> parts;
      for (auto& b : out.batches) parts.push_back(b[c]);
      res->cols.push_back(concat(parts, s));
    }
    for (auto& b : out.batches) release_all(b);
    sync_stream(s);
  }
  res->wall_s = seconds_since(t_wall);
}

int sort_terminal(am_stream* st, const char** columns, const int* descending, const int* null_placement,
                  const int* float_order, int64_t n_keys, int64_t limit, const char* scratch_dir,
                  const char* sink_path, am_stream_result** out) {
  if (!st || !columns || n_keys <= 0 || !out) return 2;
  for (int64_t i = 0; i < n_keys; i++) if (!columns[i]) return 2;
  return stream_guard([&] {
    if (st->consumed) throw invalid("this stream has already been consumed");
    st->consumed = true;
    if (limit < 0) throw invalid("limit must be >= 0");
    SortSpec spec;
    std::vector<std::string> names;
    for (int64_t i = 0; i < n_keys; i++) {
      names.push_back(columns[i]);
      const int fo = float_order ? float_order[i] : 0;
      if (fo < 0 || fo > 2) throw invalid("unknown float_order " + std::to_string(fo));
      spec.options.push_back(SortKey{nullptr, descending ? descending[i] != 0 : false,
                                     null_placement ? null_placement[i] == 1 : false, fo});
    }
    auto* r = new am_stream_result();
    try {
      external_sort(st, spec, names, limit, scratch_dir, sink_path, r);
    } catch (...) {
      delete r;
      throw;
    }
    *out = r;
    return 0;
  });
}

}  // namespace

extern "C" {

const char* am_stream_last_error(void) { return t_stream_error.c_str(); }

am_stream* am_stream_from_c_stream(ArrowArrayStream* in, int prefetch_depth) {
  if (!in || !in->release) {
    t_stream_error = "Invalid ArrowArray: a released or NULL ArrowArrayStream";
    return nullptr;
  }
  auto* st = new am_stream();
  st->in = *in;
  in->release = nullptr;
  st->prefetch = std::max(0, prefetch_depth);
  const int rc = st->in.get_schema(&st->in, &st->schema);
  if (rc != 0) {
    const char* e = st->in.get_last_error ? st->in.get_last_error(&st->in) : nullptr;
    t_stream_error = std::string("the record batch stream has no schema: ") + (e ? e : std::strerror(rc));
    delete st;
    return nullptr;
  }
  return st;
}

am_stream* am_stream_open_ipc(const char* path, int prefetch_depth, int readers) {
  (void)readers;   // files are read one after another, so batch order is always the source's
  if (!path) {
    t_stream_error = "Invalid ArrowArray: a NULL path";
    return nullptr;
  }
  try {
    auto* state = new IpcStreamState();
    std::unique_ptr<IpcStreamState> guard(state);
    struct stat stt;
    if (stat(path, &stt) != 0) throw Error(std::string("cannot open ") + path);
    if (S_ISDIR(stt.st_mode)) {
      // A directory: its Arrow IPC files in name order.
      std::vector<std::string> names;
      if (DIR* d = opendir(path)) {
        while (dirent* e = readdir(d)) {
          const std::string n = e->d_name;
          auto ends = [&](const char* x) { return n.size() > std::strlen(x) && n.compare(n.size() - std::strlen(x), std::string::npos, x) == 0; };
          if (ends(".arrow") || ends(".arrows") || ends(".ipc") || ends(".feather")) names.push_back(n);
        }
        closedir(d);
      }
      std::sort(names.begin(), names.end());
      for (auto& n : names) state->src.files.push_back(std::string(path) + "/" + n);
      if (state->src.files.empty()) throw Error(std::string("no Arrow IPC files (.arrow, .arrows, .ipc, .feather) in ") + path);
    } else {
      state->src.files.push_back(path);
    }
    if (!state->src.open_next()) throw invalid(std::string("no Arrow IPC schema in ") + path);
    ArrowArrayStream in{};
    in.get_schema = ipc_get_schema;
    in.get_next = ipc_get_next;
    in.get_last_error = ipc_last_error;
    in.release = ipc_release;
    in.private_data = guard.release();
    return am_stream_from_c_stream(&in, prefetch_depth);
  } catch (const std::exception& e) {
    t_stream_error = e.what();
    set_last_error(e.what());
    return nullptr;
  }
}

void am_stream_release(am_stream* s) { delete s; }

int am_stream_export_c(am_stream* st, ArrowArrayStream* out) {
  if (!st || !out) return 2;
  return stream_guard([&] {
    if (st->consumed) throw invalid("this stream has already been consumed");
    st->consumed = true;
    if (st->select.empty()) {
      *out = st->in;
      st->in.release = nullptr;
      return 0;
    }
    auto* ps = new ProjectState();
    ps->inner = st->in;
    st->in.release = nullptr;
    ps->select = st->select;
    *out = ArrowArrayStream{};
    out->get_schema = project_get_schema;
    out->get_next = project_get_next;
    out->get_last_error = project_last_error;
    out->release = project_release;
    out->private_data = ps;
    return 0;
  });
}

int am_stream_select(am_stream* st, const char** names, int64_t n) {
  if (!st || (!names && n > 0) || n < 0) return 2;
  return stream_guard([&] {
    std::vector<int> sel;
    for (int64_t i = 0; i < n; i++) {
      if (!names[i]) throw invalid("a NULL column name");
      int ci = -1;
      for (int64_t c = 0; c < st->schema.n_children; c++)
        if (st->schema.children[c]->name && std::strcmp(st->schema.children[c]->name, names[i]) == 0) ci = int(c);
      if (ci < 0) throw invalid(std::string("no column named \"") + names[i] + "\"");
      sel.push_back(ci);
    }
    st->select = sel;
    return 0;
  });
}

int am_stream_sort(am_stream* s, const char** columns, const int* descending, int64_t n_keys, int64_t limit,
                   const char* scratch_dir, const char* sink_path, am_stream_result** out) {
  return sort_terminal(s, columns, descending, nullptr, nullptr, n_keys, limit, scratch_dir, sink_path, out);
}

int am_stream_sort_ex(am_stream* s, const char** columns, const int* descending, const int* null_placement,
                      const int* float_order, int64_t n_keys, int64_t limit, const char* scratch_dir,
                      const char* sink_path, am_stream_result** out) {
  return sort_terminal(s, columns, descending, null_placement, float_order, n_keys, limit, scratch_dir, sink_path, out);
}

int64_t am_stream_result_column_count(am_stream_result* r) { return r ? int64_t(r->cols.size()) : -1; }
const char* am_stream_result_column_name(am_stream_result* r, int64_t i) {
  if (!r || i < 0 || i >= int64_t(r->names.size())) return nullptr;
  return r->names[size_t(i)].c_str();
}
int am_stream_result_column(am_stream_result* r, int64_t i, am_array** out) {
  if (!r || !out || i < 0 || i >= int64_t(r->cols.size())) return 2;
  retain(r->cols[size_t(i)]);
  *out = r->cols[size_t(i)];
  return 0;
}
int64_t am_stream_result_scalar_count(am_stream_result* r) { return r ? 0 : -1; }
const char* am_stream_result_scalar_name(am_stream_result* r, int64_t i) {
  (void)r;
  (void)i;
  return nullptr;
}
int am_stream_result_scalar(am_stream_result* r, int64_t i, int64_t* out_i64, double* out_f64, int* out_kind,
                            int* is_null) {
  (void)i;
  (void)out_i64;
  (void)out_f64;
  (void)out_kind;
  (void)is_null;
  if (!r) return 2;
  t_stream_error = "a sort result has no scalars";
  return 2;
}
int64_t am_stream_result_rows_out(am_stream_result* r) { return r ? r->rows_out : -1; }
int am_stream_result_stats(am_stream_result* r, int64_t* batches, int64_t* rows, int64_t* bytes_read, double* wall_s,
                           double* read_s, double* gpu_s, double* merge_s, double* overlap) {
  if (!r) return 2;
  if (batches) *batches = r->batches;
  if (rows) *rows = r->rows;
  if (bytes_read) *bytes_read = r->bytes_read;
  if (wall_s) *wall_s = r->wall_s;
  if (read_s) *read_s = r->read_s;
  if (gpu_s) *gpu_s = r->gpu_s;
  if (merge_s) *merge_s = r->merge_s;
  if (overlap) *overlap = r->wall_s > 0 ? (r->read_s + r->gpu_s + r->merge_s) / r->wall_s : 0.0;
  return 0;
}
int am_stream_result_stalls(am_stream_result* r, double* read_stall_s, double* merge_stall_s) {
  if (!r) return 2;
  if (read_stall_s) *read_stall_s = r->read_stall_s;
  if (merge_stall_s) *merge_stall_s = r->merge_stall_s;
  return 0;
}
void am_stream_result_release(am_stream_result* r) { delete r; }

}  // extern "C"
