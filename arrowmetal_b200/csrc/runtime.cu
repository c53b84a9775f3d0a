// Device runtime of libArrowMetalC for B200: one CUDA device per process, a CUDA stream per calling
// thread, stream-ordered allocation from the device's memory pool, a caching pinned host pool, staged
// host copies, per-stream look-back scratch, and kernel timing.
//
// It replaces the reference's Metal runtime (Sources/ArrowMetal/MetalContext.swift: command buffers,
// `run` / `commitAndWait` at :102-115 and :216-231, the per-thread batch at :245-312 and `BufferPool`
// at :361-437). Where the reference commits and waits after every call, calls here enqueue on the
// thread's stream and only the calls that must read a result wait.
#include <cuda_runtime.h>

#include <condition_variable>
#include <deque>
#include <cstdlib>
#include <cstring>
#include <map>
#include <thread>
#include <unordered_map>

#include "am_internal.h"
#include "radix_sort.cuh"

namespace am {

void cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  (void)cudaGetLastError();
  throw Error(std::string("CUDA error: ") + cudaGetErrorString(e) + " (" + what + ")");
}

ThreadState& tls() {
  static thread_local ThreadState t;
  return t;
}
void set_last_error(const std::string& m) { tls().last_error = m; }

// ------------------------------------------------------------------------------------------------
// Device.

static std::once_flag g_dev_once;
static Device g_dev;
static std::string g_dev_error;

Device& device() {
  std::call_once(g_dev_once, [] {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
      (void)cudaGetLastError();
      g_dev_error = std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "none found");
      return;
    }
    int ord = 0;
    if (const char* env = std::getenv("ARROWMETAL_DEVICE")) ord = std::atoi(env);
    else (void)cudaGetDevice(&ord);
    if (ord < 0 || ord >= count) {
      g_dev_error = "ARROWMETAL_DEVICE=" + std::to_string(ord) + " is not a CUDA device";
      return;
    }
    if (cudaSetDevice(ord) != cudaSuccess) { g_dev_error = "cudaSetDevice failed"; return; }
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, ord) != cudaSuccess) { g_dev_error = "cudaGetDeviceProperties failed"; return; }
    g_dev.ordinal = ord;
    g_dev.sm_count = prop.multiProcessorCount;
    g_dev.name = prop.name;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, ord) == cudaSuccess) {
      uint64_t keep = ~uint64_t(0);   // keep freed memory reserved: repeated sorts reuse it
      (void)cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      g_dev.pool = pool;
    }
  });
  if (!g_dev_error.empty()) throw Error(g_dev_error);
  return g_dev;
}

cudaStream_t copy_stream() {
  Device& d = device();
  ThreadState& t = tls();
  if (!t.copy_stream) {
    AM_CUDA(cudaSetDevice(d.ordinal));
    AM_CUDA(cudaStreamCreateWithFlags(&t.copy_stream, cudaStreamNonBlocking));
  }
  return t.copy_stream;
}

cudaStream_t d2h_stream() {
  Device& d = device();
  ThreadState& t = tls();
  if (!t.d2h_stream) {
    AM_CUDA(cudaSetDevice(d.ordinal));
    AM_CUDA(cudaStreamCreateWithFlags(&t.d2h_stream, cudaStreamNonBlocking));
  }
  return t.d2h_stream;
}

ReadyEvent::ReadyEvent(cudaStream_t s) {
  AM_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  AM_CUDA(cudaEventRecord(ev, s));
}
ReadyEvent::~ReadyEvent() {
  if (ev) (void)cudaEventDestroy(ev);
}

namespace {
// The releaser: one library thread that waits for copy events and then runs their releases, in order.
struct Releaser {
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::pair<cudaEvent_t, std::function<void()>>> q;
  Releaser() {
    std::thread([this] {
      for (;;) {
        std::pair<cudaEvent_t, std::function<void()>> job;
        {
          std::unique_lock<std::mutex> lk(mu);
          cv.wait(lk, [&] { return !q.empty(); });
          job = std::move(q.front());
          q.pop_front();
        }
        (void)cudaEventSynchronize(job.first);
        (void)cudaEventDestroy(job.first);
        job.second();
      }
    }).detach();
  }
};
Releaser& releaser() {
  static Releaser* r = new Releaser();   // lives for the process: its thread never exits
  return *r;
}
}  // namespace

void release_after(cudaEvent_t ev, std::function<void()> fn) {
  Releaser& r = releaser();
  {
    std::lock_guard<std::mutex> lk(r.mu);
    r.q.emplace_back(ev, std::move(fn));
  }
  r.cv.notify_one();
}

cudaStream_t stream() {
  Device& d = device();
  ThreadState& t = tls();
  if (!t.own_stream) {
    AM_CUDA(cudaSetDevice(d.ordinal));
    AM_CUDA(cudaStreamCreateWithFlags(&t.own_stream, cudaStreamNonBlocking));
  }
  return t.override_stream ? t.override_stream : t.own_stream;
}
void set_stream_override(cudaStream_t s) { tls().override_stream = s; }
cudaStream_t stream_override() { return tls().override_stream; }

// ------------------------------------------------------------------------------------------------
// Device memory.

static std::atomic<int64_t> g_fail_after{-1};
void debug_fail_alloc_after(int64_t n) { g_fail_after.store(n); }
static std::atomic<bool> g_skip_first_tile{false};
void debug_skip_first_tile(bool on) { g_skip_first_tile.store(on); }
bool debug_skip_first_tile() { return g_skip_first_tile.load(); }

void* dmalloc(size_t bytes, cudaStream_t s) {
  int64_t f = g_fail_after.load();
  if (f >= 0) {
    if (f == 0) throw Error("device allocation of " + std::to_string(bytes) + " bytes failed (injected)");
    g_fail_after.store(f - 1);
  }
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMallocAsync(&p, bytes, s);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw Error("device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
  }
  return p;
}
void dfree(void* p, cudaStream_t s) {
  if (p) (void)cudaFreeAsync(p, s);
}

DevBuffer::~DevBuffer() {
  if (owned && ptr) {
    cudaEvent_t e = nullptr;
    if (home && stream && stream != home && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess) {
      // Back to its home stream's part of the pool, once the last user's work is done.
      if (cudaEventRecord(e, stream) == cudaSuccess && cudaStreamWaitEvent(home, e, 0) == cudaSuccess) dfree(ptr, home);
      else dfree(ptr, stream);
      (void)cudaEventDestroy(e);
    } else {
      dfree(ptr, stream ? stream : home);
    }
  }
  if (on_release) on_release();
}
std::shared_ptr<DevBuffer> DevBuffer::alloc(size_t bytes, cudaStream_t s) {
  auto b = std::make_shared<DevBuffer>();
  b->ptr = dmalloc(bytes, s);
  b->bytes = bytes;
  b->stream = s;
  b->owned = true;
  return b;
}

// ------------------------------------------------------------------------------------------------
// Pinned host pool: export buffers and staging slots. Blocks are cached by size and reused.

namespace {
std::mutex g_pin_mu;
std::multimap<size_t, void*> g_pin_free;
std::unordered_map<void*, size_t> g_pin_size;
}  // namespace

void* pinned_alloc(size_t bytes) {
  const size_t gran = bytes >= (size_t(1) << 21) ? (size_t(1) << 21) : 4096;
  const size_t want = (std::max<size_t>(bytes, 1) + gran - 1) / gran * gran;
  {
    std::lock_guard<std::mutex> g(g_pin_mu);
    auto it = g_pin_free.lower_bound(want);
    if (it != g_pin_free.end() && it->first <= want * 2) {
      void* p = it->second;
      g_pin_free.erase(it);
      return p;
    }
  }
  device();
  void* p = nullptr;
  cudaError_t e = cudaMallocHost(&p, want);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw Error("pinned host allocation of " + std::to_string(want) + " bytes failed: " + cudaGetErrorString(e));
  }
  std::lock_guard<std::mutex> g(g_pin_mu);
  g_pin_size[p] = want;
  return p;
}
void pinned_free(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> g(g_pin_mu);
  auto it = g_pin_size.find(p);
  if (it == g_pin_size.end()) return;
  g_pin_free.emplace(it->second, p);
}

// ------------------------------------------------------------------------------------------------
// Host worker pool for the staged copies.

namespace {
class Workers {
 public:
  explicit Workers(int n) {
    for (int i = 0; i < n; i++) threads_.emplace_back([this] { loop(); });
  }
  ~Workers() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }
  int size() const { return int(threads_.size()); }
  // Runs fn(0..n-1) on the workers and the calling thread; returns when all are done.
  void parallel_for(int n, const std::function<void(int)>& fn) {
    if (n <= 1 || threads_.empty()) {
      for (int i = 0; i < n; i++) fn(i);
      return;
    }
    std::atomic<int> next{0}, done{0};
    auto body = [&] {
      for (int i; (i = next.fetch_add(1)) < n;) {
        fn(i);
        done.fetch_add(1);
      }
    };
    {
      std::lock_guard<std::mutex> g(mu_);
      for (int i = 0; i < int(threads_.size()); i++) jobs_.push_back(body);
    }
    cv_.notify_all();
    body();
    while (done.load() < n) std::this_thread::yield();
    // Jobs that never started still reference this frame: drain them before returning.
    std::unique_lock<std::mutex> g(mu_);
    idle_cv_.wait(g, [&] { return jobs_.empty() && running_ == 0; });
  }

 private:
  void loop() {
    for (;;) {
      std::function<void()> job;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return stop_ || !jobs_.empty(); });
        if (stop_) return;
        job = std::move(jobs_.back());
        jobs_.pop_back();
        running_++;
      }
      job();
      {
        std::lock_guard<std::mutex> g(mu_);
        running_--;
      }
      idle_cv_.notify_all();
    }
  }
  std::vector<std::thread> threads_;
  std::vector<std::function<void()>> jobs_;
  std::mutex mu_;
  std::condition_variable cv_, idle_cv_;
  int running_ = 0;
  bool stop_ = false;
};

std::atomic<int> g_import_threads{0};
std::mutex g_workers_mu;
std::unique_ptr<Workers> g_workers;
int g_workers_n = 0;

int effective_threads() {
  int n = g_import_threads.load();
  if (n <= 0) {
    unsigned hc = std::thread::hardware_concurrency();
    n = int(std::min<unsigned>(hc ? hc : 4, 16));
  }
  return n;
}
Workers& workers() {
  std::lock_guard<std::mutex> g(g_workers_mu);
  int want = effective_threads() - 1;
  if (!g_workers || g_workers_n != want) {
    g_workers.reset();
    g_workers.reset(new Workers(want));
    g_workers_n = want;
  }
  return *g_workers;
}

// Ring of pinned staging slots for pageable host memory.
constexpr size_t kSlotBytes = size_t(32) << 20;
constexpr int kSlots = 4;
struct Staging {
  std::mutex mu;
  void* slot[kSlots] = {};
  cudaEvent_t ev[kSlots] = {};
  bool ready = false;
  void init() {
    if (ready) return;
    for (int i = 0; i < kSlots; i++) {
      slot[i] = pinned_alloc(kSlotBytes);
      AM_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
    }
    ready = true;
  }
};
Staging g_stage;

bool staged_copies() {
  const char* e = std::getenv("ARROWMETAL_STAGED_COPY");
  return !(e && e[0] == '0');
}

void parallel_memcpy(void* dst, const void* src, size_t bytes) {
  Workers& w = workers();
  const int parts = std::max(1, std::min<int>(w.size() + 1, int(bytes / (size_t(2) << 20))));
  const size_t step = (bytes + parts - 1) / parts;
  w.parallel_for(parts, [&](int i) {
    const size_t off = size_t(i) * step;
    if (off < bytes) std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, std::min(step, bytes - off));
  });
}
}  // namespace

bool is_pinned(const void* p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

int import_threads() { return g_import_threads.load(); }
void set_import_threads(int n) { g_import_threads.store(n); }

bool copy_h2d(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return false;
  const bool pinned = is_pinned(src);
  if (bytes < (size_t(1) << 20) || !staged_copies() || pinned) {
    // A pageable source is consumed by the time the call returns; a pinned one is read later.
    AM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return pinned;
  }
  std::lock_guard<std::mutex> g(g_stage.mu);
  g_stage.init();
  int i = 0;
  for (size_t off = 0; off < bytes; off += kSlotBytes, i = (i + 1) % kSlots) {
    const size_t len = std::min(kSlotBytes, bytes - off);
    AM_CUDA(cudaEventSynchronize(g_stage.ev[i]));
    parallel_memcpy(g_stage.slot[i], static_cast<const char*>(src) + off, len);
    AM_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + off, g_stage.slot[i], len, cudaMemcpyHostToDevice, s));
    AM_CUDA(cudaEventRecord(g_stage.ev[i], s));
  }
  return false;
}

void copy_d2h(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return;
  if (bytes < (size_t(1) << 20) || !staged_copies() || is_pinned(dst)) {
    AM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    AM_CUDA(cudaStreamSynchronize(s));
    return;
  }
  std::lock_guard<std::mutex> g(g_stage.mu);
  g_stage.init();
  int i = 0;
  std::vector<std::pair<size_t, size_t>> pending(kSlots, {0, 0});
  auto drain = [&](int slot) {
    if (pending[slot].second == 0) return;
    AM_CUDA(cudaEventSynchronize(g_stage.ev[slot]));
    parallel_memcpy(static_cast<char*>(dst) + pending[slot].first, g_stage.slot[slot], pending[slot].second);
    pending[slot] = {0, 0};
  };
  for (size_t off = 0; off < bytes; off += kSlotBytes, i = (i + 1) % kSlots) {
    drain(i);
    const size_t len = std::min(kSlotBytes, bytes - off);
    AM_CUDA(cudaMemcpyAsync(g_stage.slot[i], static_cast<const char*>(src) + off, len, cudaMemcpyDeviceToHost, s));
    AM_CUDA(cudaEventRecord(g_stage.ev[i], s));
    pending[i] = {off, len};
  }
  for (int k = 0; k < kSlots; k++) drain((i + k) % kSlots);
}

// ------------------------------------------------------------------------------------------------
// Per-stream scratch and device errors.

namespace {
std::mutex g_scratch_mu;
std::unordered_map<cudaStream_t, StreamScratch*> g_scratch;
}  // namespace

StreamScratch& stream_scratch(cudaStream_t s, size_t status_words) {
  StreamScratch* sc;
  {
    std::lock_guard<std::mutex> g(g_scratch_mu);
    auto& slot = g_scratch[s];
    if (!slot) slot = new StreamScratch();
    sc = slot;
  }
  if (!sc->err) {
    sc->err = static_cast<uint32_t*>(dmalloc(sizeof(uint32_t) * 4, s));
    AM_CUDA(cudaMemsetAsync(sc->err, 0, sizeof(uint32_t) * 4, s));
  }
  if (status_words > sc->status_words) {
    if (sc->status) dfree(sc->status, s);
    const size_t words = std::max(status_words, sc->status_words * 2);
    sc->status = static_cast<uint64_t*>(dmalloc(words * sizeof(uint64_t), s));
    AM_CUDA(cudaMemsetAsync(sc->status, 0, words * sizeof(uint64_t), s));
    sc->status_words = words;
    sc->epoch = 0;
  }
  return *sc;
}

namespace {
// Bytes held in all streams' arenas (a stream outlives its thread, and so does its arena): past
// kArenaTotal, sorts take blocks of their own instead of growing an arena.
std::atomic<size_t> g_arena_total{0};
constexpr size_t kArenaTotal = size_t(16) << 30;
}  // namespace

ScratchBlock::ScratchBlock(cudaStream_t s, size_t bytes) : s_(s) {
  StreamScratch& sc = stream_scratch(s, 0);
  bool expected = false;
  if (bytes <= kArenaMax && sc.arena_busy.compare_exchange_strong(expected, true)) {
    if (sc.arena_bytes < bytes && g_arena_total.load() - sc.arena_bytes + bytes > kArenaTotal) {
      sc.arena_busy = false;
      p_ = static_cast<char*>(dmalloc(bytes, s));
      return;
    }
    if (sc.arena_bytes < bytes) {
      g_arena_total -= sc.arena_bytes;
      if (sc.arena) dfree(sc.arena, s);
      sc.arena = nullptr;
      sc.arena_bytes = 0;
      try {
        sc.arena = dmalloc(bytes, s);
      } catch (...) {
        sc.arena_busy = false;
        throw;
      }
      sc.arena_bytes = bytes;
      g_arena_total += bytes;
    }
    arena_ = &sc;
    p_ = static_cast<char*>(sc.arena);
  } else {
    p_ = static_cast<char*>(dmalloc(bytes, s));
  }
}
ScratchBlock::~ScratchBlock() {
  if (arena_) arena_->arena_busy = false;
  else dfree(p_, s_);
}

void sync_stream(cudaStream_t s) { AM_CUDA(cudaStreamSynchronize(s)); }

void check_device_errors(cudaStream_t s) {
  StreamScratch& sc = stream_scratch(s, 0);
  static thread_local uint32_t* host = nullptr;
  if (!host) host = static_cast<uint32_t*>(pinned_alloc(16));
  AM_CUDA(cudaMemcpyAsync(host, sc.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  AM_CUDA(cudaStreamSynchronize(s));
  const uint32_t e = *host;
  if (e == 0) return;
  AM_CUDA(cudaMemsetAsync(sc.err, 0, sizeof(uint32_t), s));
  if (e & rs::ERR_TAKE_RANGE) throw invalid("take: index out of range");
  if (e & rs::ERR_LOOKBACK_TIMEOUT) throw Error("radix sort: a look-back wait timed out on the device");
  if (e & rs::ERR_BOUNDS) throw Error("radix sort: a destination fell outside its array (write skipped)");
  if (e & rs::ERR_DICT_CODE) throw invalid("dictionary code out of range of its dictionary");
  throw Error("device error word " + std::to_string(e));
}

// ------------------------------------------------------------------------------------------------
// Kernel timing.

namespace {
std::atomic<bool> g_prof{false};
std::mutex g_prof_mu;
struct Pending { std::string name; cudaEvent_t a, b; };
std::vector<Pending> g_pending;
std::map<std::string, std::pair<int64_t, double>> g_totals;
std::vector<cudaEvent_t> g_event_pool;
cudaEvent_t get_event() {
  {
    std::lock_guard<std::mutex> g(g_prof_mu);
    if (!g_event_pool.empty()) {
      cudaEvent_t e = g_event_pool.back();
      g_event_pool.pop_back();
      return e;
    }
  }
  cudaEvent_t e;
  AM_CUDA(cudaEventCreate(&e));
  return e;
}
}  // namespace

bool profiling() { return g_prof.load(std::memory_order_relaxed); }
void set_profiling(bool on) { g_prof.store(on); }

KernelTimer::KernelTimer(const char* n, cudaStream_t st) : name(n), s(st) {
  if (!profiling()) return;
  a = get_event();
  b = get_event();
  AM_CUDA(cudaEventRecord(a, s));
}
KernelTimer::~KernelTimer() {
  if (!a) return;
  if (cudaEventRecord(b, s) != cudaSuccess) { (void)cudaGetLastError(); return; }
  std::lock_guard<std::mutex> g(g_prof_mu);
  g_pending.push_back({name, a, b});
}

void profile_collect() {
  std::vector<Pending> p;
  {
    std::lock_guard<std::mutex> g(g_prof_mu);
    p.swap(g_pending);
  }
  for (auto& e : p) {
    AM_CUDA(cudaEventSynchronize(e.b));
    float ms = 0.f;
    AM_CUDA(cudaEventElapsedTime(&ms, e.a, e.b));
    std::lock_guard<std::mutex> g(g_prof_mu);
    auto& t = g_totals[e.name];
    t.first += 1;
    t.second += ms;
    g_event_pool.push_back(e.a);
    g_event_pool.push_back(e.b);
  }
}
std::vector<ProfileEntry> profile_entries() {
  profile_collect();
  std::lock_guard<std::mutex> g(g_prof_mu);
  std::vector<ProfileEntry> v;
  for (auto& kv : g_totals) v.push_back({kv.first, kv.second.first, kv.second.second});
  return v;
}
void profile_reset() {
  profile_collect();
  std::lock_guard<std::mutex> g(g_prof_mu);
  g_totals.clear();
}

// ------------------------------------------------------------------------------------------------
// Types and handles.

int parse_format(const char* f) {
  if (!f) throw invalid("schema without a format");
  const std::string s(f);
  if (s == "b") return PT_BOOL;
  if (s == "c") return PT_I8;
  if (s == "C") return PT_U8;
  if (s == "s") return PT_I16;
  if (s == "S") return PT_U16;
  if (s == "i") return PT_I32;
  if (s == "I") return PT_U32;
  if (s == "l") return PT_I64;
  if (s == "L") return PT_U64;
  if (s == "e") return PT_F16;
  if (s == "f") return PT_F32;
  if (s == "g") return PT_F64;
  // Temporal types sort and move as their integer storage (MultiSort.swift:96-99).
  if (s == "u" || s == "z") return PT_STR;
  if (s == "U" || s == "Z") return PT_LSTR;
  if (s == "tdD" || s == "tts" || s == "ttm") return PT_I32;
  if (s == "tdm" || s == "ttu" || s == "ttn") return PT_I64;
  if (s.size() >= 4 && s[0] == 't' && s[1] == 's' && s[3] == ':' && std::strchr("smun", s[2])) return PT_I64;
  if (s.size() == 3 && s[0] == 't' && s[1] == 'D' && std::strchr("smun", s[2])) return PT_I64;
  throw unsupported(s + " is not carried by this build (primitive numeric, boolean, temporal, string and binary types are)");
}

std::string format_of(int pt) {
  static const char* names[] = {"b", "c", "C", "s", "S", "i", "I", "l", "L", "e", "f", "g", "u", "U", "+s"};
  return names[pt];
}

am_array* new_array(int pt, const std::string& format, int64_t length) {
  auto* a = new am_array();
  a->pt = pt;
  a->format = format;
  a->length = length;
  return a;
}
void retain(am_array* a) { a->refs.fetch_add(1); }
void release(am_array* a) {
  if (!a) return;
  if (a->refs.fetch_sub(1) == 1) {
    cudaStream_t s = a->last_stream;
    if (s) {
      for (BufPtr* b : {&a->values, &a->bytes, &a->validity, &a->null_count_dev})
        if (*b && b->use_count() == 1) (*b)->stream = s;
    }
    for (am_array* c : a->children) release(c);
    if (a->dictionary) release(a->dictionary);
    delete a;
  }
}

void use_on(am_array* a, cudaStream_t s) {
  if (a && a->pt == PT_STRUCT) throw unsupported("+s: a struct result is exported, not computed on");
  if (!a || a->shared_read) return;
  if (a->ready && a->last_stream != s) {
    // Contents complete at the ready event: wait for it alone, not for later work on its stream.
    AM_CUDA(cudaStreamWaitEvent(s, a->ready->ev, 0));
  } else if (a->last_stream && a->last_stream != s) {
    cudaEvent_t e;
    AM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    AM_CUDA(cudaEventRecord(e, a->last_stream));
    AM_CUDA(cudaStreamWaitEvent(s, e, 0));
    AM_CUDA(cudaEventDestroy(e));
  }
  a->last_stream = s;
}

int64_t resolve_null_count(am_array* a) {
  if (a->null_count >= 0) return a->null_count;
  cudaStream_t s = a->last_stream ? a->last_stream : stream();
  static thread_local unsigned long long* host = nullptr;
  if (!host) host = static_cast<unsigned long long*>(pinned_alloc(16));
  AM_CUDA(cudaMemcpyAsync(host, a->null_count_dev->ptr, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  AM_CUDA(cudaStreamSynchronize(s));
  a->null_count = int64_t(*host);
  a->null_count_dev.reset();
  if (a->null_count == 0) a->validity.reset();
  return a->null_count;
}

static std::atomic<int64_t> g_max_row{int64_t(0xFFFFFFFFll)};
int64_t max_row_index() { return g_max_row.load(); }
void set_max_row_index(int64_t v) { g_max_row.store(v); }
void check_index_rows(int64_t rows, const char* op) {
  // Dispatch.checkIndexRows (Sources/ArrowMetal/Kernels/Dispatch.swift:198-203).
  const int64_t last = rows - 1;
  if (last <= max_row_index()) return;
  throw invalid(std::string(op) + ": row " + std::to_string(last) +
                " does not fit the UInt32 index type (row numbers go up to " + std::to_string(max_row_index()) + ")");
}

}  // namespace am
