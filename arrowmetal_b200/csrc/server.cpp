// Sort server: sort requests over tables resident in HBM, admitted by their HBM footprint and batched
// as they arrive (continuous batching).
//
// A request sorts rows [offset, offset + length) of a resident table by one or more key columns and
// returns the sorted keys with the payload columns taken through the same permutation -- the ORDER BY
// of the plan entry points (include/arrowmetal.h:1419-1433), addressed to a slice of a table. Worker
// threads each own a CUDA stream. A free worker takes, in arrival order, the first queued request
// whose footprint fits under the admission cap beside the work already on the GPU; a single-key request
// of at most `batch_rows` rows takes every other such request that fits with it, and they are sorted as
// one segmented batch (am_argsort_batch) followed by one fused gather per request. When the queue is
// backlogged, queued requests of the same table, keys and options share one sort of the rows they
// cover together: each is answered by keeping, in order, the entries of that sort that fall in its own
// rows (a stable sort restricted to a subset of rows is the subset's own stable sort) and one fused
// gather (shared_sort.cu). Other requests run alone through am_plan_run. Requests that arrive while
// others run are picked up by the next free worker, so their work overlaps on the device.
//
// The reference has no server: its callers make one call per query. Every result equals the same
// request run alone through am_plan_run.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <algorithm>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>
#include <unordered_map>

#include "am_internal.h"
#include "plan_types.h"

using namespace am;

namespace {

using Clock = std::chrono::steady_clock;

struct ServeRequest {
  int64_t id = 0;
  Clock::time_point enqueued;       // host work of the request done, device work in flight
  am_plan_source* table = nullptr;
  int64_t offset = 0, length = 0;
  std::vector<int> key_cols, pay_cols;          // column positions in the table
  std::vector<int> desc, nulls_first, float_order;
  int64_t footprint = 0;
  bool batchable = false;
  Clock::time_point arrival, finished;
  bool done = false;
  int rc = 0;
  std::string error;
  am_plan_result* result = nullptr;
};
using ReqPtr = std::shared_ptr<ServeRequest>;

std::string json_str(const std::string& s) {
  std::string o = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') o += '\\';
    o += c;
  }
  return o + "\"";
}

// select(sort(select(limit(scan)))): the slice, only the columns the request returns, sorted.
std::string plan_of(const ServeRequest& r) {
  const am_plan_source_t& t = *r.table;
  std::ostringstream sel, by;
  std::vector<int> cols = r.key_cols;
  cols.insert(cols.end(), r.pay_cols.begin(), r.pay_cols.end());
  for (size_t i = 0; i < cols.size(); i++) {
    const std::string& n = t.names[size_t(cols[i])];
    const std::string e = "[" + json_str(n) + "," + json_str("(col \"" + n + "\")") + "]";
    sel << (i ? "," : "") << e;
  }
  for (size_t k = 0; k < r.key_cols.size(); k++) {
    static const char* orders[] = {"ieee", "total", "nan_largest"};
    by << (k ? "," : "") << "[" << json_str(t.names[size_t(r.key_cols[k])]) << "," << (r.desc[k] ? "true" : "false")
       << ",{\"nulls\":\"" << (r.nulls_first[k] ? "first" : "last") << "\",\"float_order\":\""
       << orders[r.float_order[k]] << "\"}]";
  }
  std::ostringstream p;
  p << "{\"op\":\"select\",\"exprs\":[" << sel.str() << "],\"input\":{\"op\":\"sort\",\"by\":[" << by.str()
    << "],\"input\":{\"op\":\"select\",\"exprs\":[" << sel.str() << "],\"input\":{\"op\":\"limit\",\"count\":"
    << r.length << ",\"offset\":" << r.offset << ",\"input\":{\"op\":\"scan\",\"source\":" << json_str(t.name)
    << "}}}}}";
  return p.str();
}

int64_t width_of(const am_array* a) { return std::max(pt_bytes(a->pt), 1); }

}  // namespace

struct am_server_t {
  std::mutex mu;
  std::mutex settle_mu;            // settling a table's columns, once, for shared reading
  std::condition_variable work_cv, done_cv;
  std::deque<ReqPtr> queue;
  std::unordered_map<int64_t, ReqPtr> requests;
  int64_t next_id = 1;
  int64_t cap = 0, batch_rows = 0;
  int64_t in_flight = 0;
  bool stop = false;
  bool share = true;               // ARROWMETAL_SERVER_SHARED=0 turns shared sorts off
  am_server_stats stats{};
  std::vector<std::thread> workers;
  Clock::time_point created = Clock::now();
  FILE* trace = nullptr;           // ARROWMETAL_SERVER_TRACE: one line per unit of work
  std::mutex trace_mu;

  void run_worker(int index);
  std::vector<ReqPtr> next_unit(int64_t* footprint, bool* shared);
  bool take_shared(std::vector<ReqPtr>& unit, int64_t* footprint);
  void execute(std::vector<ReqPtr>& unit, bool shared);
  void execute_shared(std::vector<ReqPtr>& unit);
  void finish_now(ServeRequest& r);
};

// A request whose result is complete on the device, handed to its waiter before the rest of its unit.
void am_server_t::finish_now(ServeRequest& r) {
  {
    std::lock_guard<std::mutex> lk(mu);
    r.finished = Clock::now();
    r.done = true;
    stats.requests++;
    if (r.rc == 0) stats.rows += r.length;
  }
  done_cv.notify_all();
}

namespace {

constexpr int kMaxSharedUnit = 32;      // requests answered from one shared sort (at most MAX_SHARED)
static_assert(kMaxSharedUnit <= MAX_SHARED, "one compaction launch serves the unit");

// Requests that one sort can answer: the same table, keys and options.
bool same_sort(const ServeRequest& a, const ServeRequest& b) {
  return a.table == b.table && a.key_cols == b.key_cols && a.desc == b.desc && a.nulls_first == b.nulls_first &&
         a.float_order == b.float_order;
}

}  // namespace

// Under the lock, `unit` holding the first request (already out of the queue): the queued requests that
// share its sort, when sharing saves work. A request joins when it covers at least a 32nd of the rows
// the shared sort covers (its share of the compaction stays small), and the unit is shared when its
// requests' rows add up to at least one and a half times the covered rows.
bool am_server_t::take_shared(std::vector<ReqPtr>& unit, int64_t* footprint) {
  // Only a backlog is shared (two requests queued per worker); under lighter load each request runs on
  // its own. A unit hands each request out when its own take is done, smallest first.
  if (queue.size() < 2 * workers.size()) return false;
  const ServeRequest& r0 = *unit[0];
  std::vector<std::deque<ReqPtr>::iterator> cand;
  for (auto it = queue.begin(); it != queue.end() && cand.size() + 1 < size_t(kMaxSharedUnit); ++it)
    if (same_sort(**it, r0)) cand.push_back(it);
  if (cand.empty()) return false;
  int64_t lo = r0.offset, hi = r0.offset + r0.length;
  for (auto& it : cand) {
    lo = std::min(lo, (*it)->offset);
    hi = std::max(hi, (*it)->offset + (*it)->length);
  }
  std::vector<std::deque<ReqPtr>::iterator> keep;
  int64_t rows = r0.length, fp = r0.footprint;
  int64_t klo = r0.offset, khi = r0.offset + r0.length;
  for (auto& it : cand) {
    const ServeRequest& q = **it;
    if (q.length * 32 < hi - lo) continue;
    if (in_flight > 0 && in_flight + fp + q.footprint > cap) continue;
    keep.push_back(it);
    rows += q.length;
    fp += q.footprint;
    klo = std::min(klo, q.offset);
    khi = std::max(khi, q.offset + q.length);
  }
  if (keep.empty() || r0.length * 32 < khi - klo || 2 * rows < 3 * (khi - klo)) return false;
  std::vector<const ServeRequest*> taken;
  for (auto& it : keep) {
    unit.push_back(*it);
    taken.push_back(it->get());
  }
  queue.erase(std::remove_if(queue.begin(), queue.end(),
                             [&](const ReqPtr& q) { return std::find(taken.begin(), taken.end(), q.get()) != taken.end(); }),
              queue.end());
  *footprint = fp;
  return true;
}

// One sort of the rows the unit's requests cover together, then each request's order by keeping the
// entries within its rows (compact_ranges), then one fused take of its columns.
void am_server_t::execute_shared(std::vector<ReqPtr>& unit) {
  const ServeRequest& r0 = *unit[0];
  int64_t lo = r0.offset, hi = r0.offset + r0.length;
  for (auto& r : unit) {
    lo = std::min(lo, r->offset);
    hi = std::max(hi, r->offset + r->length);
  }
  const int64_t n = hi - lo;
  std::vector<am_array*> temps, kcols, idx;
  std::map<int, am_array*> pcols;
  std::vector<cudaEvent_t> events;
  am_array* perm = nullptr;
  auto cleanup = [&] {
    for (am_array* a : temps) am_release(a);
    for (am_array* a : idx) am_release(a);
    if (perm) am_release(perm);
  };
  int rc = 0;
  std::string err;
  try {
    auto slice = [&](int c) {
      am_array* a = nullptr;
      if (am_slice(r0.table->cols[size_t(c)], lo, n, &a) != 0) throw Error(am_last_error());
      temps.push_back(a);
      return a;
    };
    for (int c : r0.key_cols) kcols.push_back(slice(c));
    const int K = int(kcols.size());
    std::vector<int> desc(r0.desc), np(r0.nulls_first), fo(r0.float_order);
    rc = K == 1 ? am_argsort_ex2(kcols[0], desc[0], np[0], fo[0], &perm)
                : am_lexsort_ex2(kcols.data(), desc.data(), np.data(), fo.data(), K, &perm);
    if (rc != 0) throw Error(am_last_error(), rc);
    cudaStream_t s = stream();
    use_on(perm, s);
    // Requests covering at least an eighth of the covered rows get their columns by compaction of the
    // covered rows' columns in the shared order (one gather for all of them, then one streaming pass);
    // the others by compaction of the order and a take of their own.
    std::vector<int> needed(r0.key_cols);
    for (auto& r : unit)
      for (int c : r->pay_cols)
        if (std::find(needed.begin(), needed.end(), c) == needed.end()) needed.push_back(c);
    bool flat = int(needed.size()) <= MAX_CCOLS;
    for (int c : needed) {
      const am_array* col = r0.table->cols[size_t(c)];
      if (col->dictionary || pt_var(col->pt) || pt_bytes(col->pt) <= 0) flat = false;
    }
    std::vector<size_t> big, small;
    for (size_t i = 0; i < unit.size(); i++) (flat && unit[i]->length * 8 >= n ? big : small).push_back(i);
    if (big.size() < 2) {
      small.insert(small.end(), big.begin(), big.end());
      big.clear();
    }
    std::stable_sort(small.begin(), small.end(), [&](size_t x, size_t y) { return unit[x]->length < unit[y]->length; });
    auto record = [&] {
      cudaEvent_t e;
      AM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      events.push_back(e);
      const cudaError_t rec = cudaEventRecord(e, s);
      if (rec != cudaSuccess) throw Error(std::string("cudaEventRecord: ") + cudaGetErrorString(rec));
    };
    std::vector<std::vector<size_t>> done_at;   // the requests each event completes, in event order
    // 1. The smaller requests: their orders, then their takes, smallest first.
    {
      std::vector<uint32_t> qlo, qhi;
      std::vector<uint32_t*> outs;
      for (size_t i : small) {
        ServeRequest& r = *unit[i];
        am_array* o = new_array(PT_U32, "I", r.length);
        idx.push_back(o);
        o->values = DevBuffer::alloc(size_t(std::max<int64_t>(r.length, 1)) * 4 + 16, s);
        o->null_count = 0;
        o->perm_of = n;                      // entries index the covered rows
        o->last_stream = s;
        qlo.push_back(uint32_t(r.offset - lo));
        qhi.push_back(uint32_t(r.offset - lo + r.length));
        outs.push_back(static_cast<uint32_t*>(o->values->ptr));
      }
      compact_ranges(static_cast<const uint32_t*>(perm->data()), uint64_t(n), qlo, qhi, outs, s);
    }
    for (size_t k = 0; k < small.size(); k++) {
      ServeRequest& r = *unit[small[k]];
      std::vector<am_array*> cols(kcols);
      for (int c : r.pay_cols) {
        if (!pcols.count(c)) pcols[c] = slice(c);
        cols.push_back(pcols[c]);
      }
      auto* res = new am_plan_result_t();
      res->rows = r.length;
      res->cols.assign(cols.size(), nullptr);
      if (am_take_columns(cols.data(), int64_t(cols.size()), idx[k], res->cols.data()) != 0) {
        res->cols.clear();
        delete res;
        throw Error(am_last_error());
      }
      for (int c : r.key_cols) res->names.push_back(r.table->names[size_t(c)]);
      for (int c : r.pay_cols) res->names.push_back(r.table->names[size_t(c)]);
      r.result = res;
      r.enqueued = Clock::now();
      record();
      done_at.push_back({small[k]});
    }
    // 2. The larger requests: the covered rows' columns in the shared order, then one compaction.
    if (!big.empty()) {
      std::vector<am_array*> src_cols;
      for (int c : needed) {
        if (std::find(r0.key_cols.begin(), r0.key_cols.end(), c) != r0.key_cols.end())
          src_cols.push_back(kcols[size_t(std::find(r0.key_cols.begin(), r0.key_cols.end(), c) - r0.key_cols.begin())]);
        else {
          if (!pcols.count(c)) pcols[c] = slice(c);
          src_cols.push_back(pcols[c]);
        }
      }
      std::vector<am_array*> sorted(src_cols.size(), nullptr);
      if (am_take_columns(src_cols.data(), int64_t(src_cols.size()), perm, sorted.data()) != 0)
        throw Error(am_last_error());
      for (am_array* a : sorted) temps.push_back(a);
      CompactSrc cs{};
      cs.ncols = int32_t(sorted.size());
      for (size_t c = 0; c < sorted.size(); c++) {
        am_array* a = sorted[c];
        use_on(a, s);
        cs.src[c] = a->data();
        cs.src_valid[c] = a->null_count != 0 ? a->valid_bits() : nullptr;
        cs.src_voff[c] = a->validity_offset;
        cs.width[c] = pt_bytes(a->pt);
      }
      std::vector<uint32_t> qlo, qhi;
      std::vector<CompactDst> dsts;
      for (size_t i : big) {
        ServeRequest& r = *unit[i];
        auto* res = new am_plan_result_t();
        res->rows = r.length;
        r.result = res;
        CompactDst d{};
        std::vector<am_array*> outs;
        for (size_t c = 0; c < needed.size(); c++) {
          const am_array* srcc = sorted[c];
          am_array* o = new_array(srcc->pt, srcc->format, r.length);
          temps.push_back(o);                   // released below; the request's result holds its own
          o->values = DevBuffer::alloc(size_t(std::max<int64_t>(r.length, 1)) * size_t(pt_bytes(srcc->pt)) + 16, s);
          o->last_stream = s;
          o->null_count = 0;
          if (cs.src_valid[c]) {
            const size_t bytes = size_t((r.length + 127) / 128) * 16;
            o->validity = DevBuffer::alloc(bytes + 16, s);
            o->null_count_dev = DevBuffer::alloc(sizeof(unsigned long long), s);
            AM_CUDA(cudaMemsetAsync(o->validity->ptr, 0, bytes + 16, s));
            AM_CUDA(cudaMemsetAsync(o->null_count_dev->ptr, 0, sizeof(unsigned long long), s));
            o->null_count = -1;
            d.dst_valid[c] = static_cast<uint32_t*>(o->validity->ptr);
            d.nulls[c] = static_cast<unsigned long long*>(o->null_count_dev->ptr);
          }
          d.dst[c] = o->values->ptr;
          outs.push_back(o);
        }
        // The request's columns in its own order: its keys, then its payload.
        std::vector<int> cols(r.key_cols);
        cols.insert(cols.end(), r.pay_cols.begin(), r.pay_cols.end());
        for (int c : cols) {
          am_array* o = outs[size_t(std::find(needed.begin(), needed.end(), c) - needed.begin())];
          retain(o);
          res->cols.push_back(o);
          res->names.push_back(r.table->names[size_t(c)]);
        }
        dsts.push_back(d);
        qlo.push_back(uint32_t(r.offset - lo));
        qhi.push_back(uint32_t(r.offset - lo + r.length));
      }
      compact_columns(static_cast<const uint32_t*>(perm->data()), uint64_t(n), qlo, qhi, cs, dsts, s);
      for (size_t i : big) unit[i]->enqueued = Clock::now();
      record();
      done_at.push_back(big);
    }
    for (size_t k = 0; k < events.size(); k++) {
      const cudaError_t w = cudaEventSynchronize(events[k]);
      if (w != cudaSuccess) throw Error(std::string("shared sort: ") + cudaGetErrorString(w));
      for (size_t i : done_at[k]) finish_now(*unit[i]);
    }
    rc = am_cuda_synchronize();
    if (rc != 0) err = am_last_error();
  } catch (const Error& e) {
    rc = e.code ? e.code : 1;
    err = e.what();
  }
  for (cudaEvent_t e : events) (void)cudaEventDestroy(e);
  if (rc != 0) {
    for (auto& r : unit) {
      if (r->done) continue;
      if (r->result) {
        am_plan_result_release(r->result);
        r->result = nullptr;
      }
      r->rc = rc;
      r->error = err;
    }
  }
  cleanup();
}

// Under the lock: the first queued request that fits, with the requests that share its sort, or else
// the batchable requests that fit beside it.
std::vector<ReqPtr> am_server_t::next_unit(int64_t* footprint, bool* shared) {
  *shared = false;
  std::vector<ReqPtr> unit;
  int64_t fp = 0, rows = 0;
  for (auto it = queue.begin(); it != queue.end(); ++it) {
    const ReqPtr& r = *it;
    if (in_flight > 0 && in_flight + r->footprint > cap) continue;
    unit.push_back(r);
    fp = r->footprint;
    rows = r->length;
    queue.erase(it);
    break;
  }
  if (!unit.empty() && share && take_shared(unit, &fp)) {
    *shared = true;
    *footprint = fp;
    return unit;
  }
  if (!unit.empty() && unit[0]->batchable) {
    for (auto it = queue.begin(); it != queue.end();) {
      const ReqPtr& r = *it;
      if (r->batchable && rows + r->length <= batch_rows * 4 && in_flight + fp + r->footprint <= cap) {
        fp += r->footprint;
        rows += r->length;
        unit.push_back(r);
        it = queue.erase(it);
      } else {
        ++it;
      }
    }
  }
  *footprint = fp;
  return unit;
}

void am_server_t::execute(std::vector<ReqPtr>& unit, bool shared) {
  if (shared) {
    execute_shared(unit);
    return;
  }
  auto fail_all = [&](int rc, const std::string& msg) {
    for (auto& r : unit) {
      if (r->result) {
        am_plan_result_release(r->result);
        r->result = nullptr;
      }
      r->rc = rc;
      r->error = msg;
    }
  };
  if (unit.size() == 1 && !unit[0]->batchable) {
    ServeRequest& r = *unit[0];
    const std::string plan = plan_of(r);
    am_plan_source* src = r.table;
    int rc = am_plan_run(plan.c_str(), &src, 1, 0, &r.result);
    r.enqueued = Clock::now();
    if (rc == 0) rc = am_cuda_synchronize();
    if (rc != 0) fail_all(rc, am_last_error());
    return;
  }
  // A segmented batch: slices of every request's key, one am_argsort_batch, one fused gather each.
  std::vector<am_array*> keys, idx(unit.size(), nullptr), temps;
  std::vector<int> desc, np, fo;
  auto cleanup = [&] {
    for (am_array* a : temps) am_release(a);
    for (am_array* a : idx) if (a) am_release(a);
  };
  int rc = 0;
  for (auto& r : unit) {
    am_array* k = nullptr;
    rc = am_slice(r->table->cols[size_t(r->key_cols[0])], r->offset, r->length, &k);
    if (rc != 0) break;
    temps.push_back(k);
    keys.push_back(k);
    desc.push_back(r->desc[0]);
    np.push_back(r->nulls_first[0]);
    fo.push_back(r->float_order[0]);
  }
  if (rc == 0) rc = am_argsort_batch(keys.data(), desc.data(), np.data(), fo.data(), int64_t(keys.size()), idx.data());
  for (size_t i = 0; rc == 0 && i < unit.size(); i++) {
    ServeRequest& r = *unit[i];
    std::vector<am_array*> cols{keys[i]};
    for (int c : r.pay_cols) {
      am_array* p = nullptr;
      rc = am_slice(r.table->cols[size_t(c)], r.offset, r.length, &p);
      if (rc != 0) break;
      temps.push_back(p);
      cols.push_back(p);
    }
    if (rc != 0) break;
    auto* res = new am_plan_result_t();
    res->rows = r.length;
    res->cols.assign(cols.size(), nullptr);
    rc = am_take_columns(cols.data(), int64_t(cols.size()), idx[i], res->cols.data());
    if (rc != 0) {
      res->cols.clear();
      delete res;
      break;
    }
    res->names.push_back(r.table->names[size_t(r.key_cols[0])]);
    for (int c : r.pay_cols) res->names.push_back(r.table->names[size_t(c)]);
    r.result = res;
  }
  for (auto& r : unit) r->enqueued = Clock::now();
  if (rc == 0) rc = am_cuda_synchronize();
  if (rc != 0) fail_all(rc, am_last_error());
  cleanup();
}

void am_server_t::run_worker(int index) {
  for (;;) {
    std::vector<ReqPtr> unit;
    int64_t fp = 0;
    bool shared = false;
    {
      std::unique_lock<std::mutex> lk(mu);
      work_cv.wait(lk, [&] {
        if (stop && queue.empty()) return true;
        for (auto& r : queue)
          if (in_flight == 0 || in_flight + r->footprint <= cap) return true;
        return false;
      });
      if (stop && queue.empty()) return;
      unit = next_unit(&fp, &shared);
      if (unit.empty()) continue;
      in_flight += fp;
      stats.peak_in_flight_bytes = std::max(stats.peak_in_flight_bytes, in_flight);
      if (shared) {
        stats.shared_sorts++;
        stats.shared_requests += int64_t(unit.size());
      } else if (unit.size() > 1 || unit[0]->batchable) {
        stats.batches++;
        stats.batched_requests += int64_t(unit.size());
      } else {
        stats.solo_requests++;
      }
    }
    const Clock::time_point t_start = Clock::now();
    execute(unit, shared);
    const Clock::time_point t = Clock::now();
    if (trace) {
      // worker, dispatch and finish (ms since the server started), requests, rows, first request's
      // arrival; a unit of several requests is a segmented batch.
      auto ms = [&](Clock::time_point x) { return std::chrono::duration<double, std::milli>(x - created).count(); };
      int64_t rows = 0;
      for (auto& r : unit) rows += r->length;
      std::lock_guard<std::mutex> lk(trace_mu);
      std::fprintf(trace, "worker %d start %.3f enqueued %.3f end %.3f requests %zu rows %lld first_id %lld arrival %.3f "
                   "table %s keys %zu rc %d\n", index, ms(t_start), ms(unit[0]->enqueued), ms(t), unit.size(),
                   (long long)rows, (long long)unit[0]->id, ms(unit[0]->arrival), unit[0]->table->name.c_str(),
                   unit[0]->key_cols.size(), unit[0]->rc);
    }
    {
      std::lock_guard<std::mutex> lk(mu);
      in_flight -= fp;
      for (auto& r : unit) {
        if (r->done) continue;           // finished on its own inside a shared unit
        r->finished = t;
        r->done = true;
        stats.requests++;
        if (r->rc == 0) stats.rows += r->length;
      }
    }
    done_cv.notify_all();
    work_cv.notify_all();
  }
}

extern "C" {

int am_server_create(int workers, int64_t hbm_cap_bytes, int64_t batch_rows, am_server** out) {
  if (!out || workers < 1 || workers > 64 || hbm_cap_bytes <= 0 || batch_rows < 0) return 2;
  try {
    (void)device();
    // Reserve the admission budget in the device's memory pool (allocated, freed and kept: the pool
    // never releases memory), so that the workers' allocations are served from memory already
    // mapped. Growing the pool while other streams keep the GPU busy stalls the allocating thread
    // for up to hundreds of milliseconds.
    {
      size_t free_b = 0, total_b = 0;
      AM_CUDA(cudaMemGetInfo(&free_b, &total_b));
      const int64_t spare = int64_t(free_b) - (int64_t(2) << 30);
      const int64_t reserve = std::min<int64_t>(hbm_cap_bytes, spare);
      if (reserve > 0) {
        cudaStream_t st = stream();
        void* p = dmalloc(size_t(reserve), st);
        dfree(p, st);
        AM_CUDA(cudaStreamSynchronize(st));
      }
    }
    auto* s = new am_server_t();
    s->cap = hbm_cap_bytes;
    s->batch_rows = batch_rows;
    if (const char* e = std::getenv("ARROWMETAL_SERVER_SHARED")) s->share = e[0] != '0';
    if (const char* path = std::getenv("ARROWMETAL_SERVER_TRACE")) {
      s->trace = std::fopen(path, "a");
      if (s->trace) std::fprintf(s->trace, "server workers %d cap %lld batch_rows %lld\n", workers,
                                 (long long)hbm_cap_bytes, (long long)batch_rows);
    }
    for (int i = 0; i < workers; i++) s->workers.emplace_back([s, i] { s->run_worker(i); });
    *out = s;
    return 0;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 1;
  }
}

int am_server_submit(am_server* srv, am_plan_source* table, int64_t offset, int64_t length, const char** keys,
                     const int* descending, const int* null_placement, const int* float_order, int64_t nkeys,
                     const char** payload, int64_t npayload, int64_t* ticket) {
  if (!srv || !table || !keys || nkeys < 1 || npayload < 0 || (npayload > 0 && !payload) || !ticket) return 2;
  if (offset < 0 || length < 0 || offset + length > table->rows) {
    set_last_error("Invalid ArrowArray: request rows [" + std::to_string(offset) + ", " +
                   std::to_string(offset + length) + ") outside the table's " + std::to_string(table->rows));
    return 2;
  }
  try {
    auto r = std::make_shared<ServeRequest>();
    r->table = table;
    r->offset = offset;
    r->length = length;
    auto find = [&](const char* name) {
      if (!name) throw invalid("null column name");
      const std::string n(name);
      if (n.find('"') != std::string::npos || n.find('\\') != std::string::npos)
        throw invalid("column names with quotes or backslashes are not served: " + n);
      for (size_t i = 0; i < table->names.size(); i++) if (table->names[i] == n) return int(i);
      throw invalid("unknown column \"" + n + "\" in table \"" + table->name + "\"");
    };
    int64_t bytes_per_row = 12;                 // ids (two buffers) and the index array
    for (int64_t k = 0; k < nkeys; k++) {
      const int c = find(keys[k]);
      r->key_cols.push_back(c);
      r->desc.push_back(descending && descending[k] ? 1 : 0);
      r->nulls_first.push_back(null_placement && null_placement[k] == 1 ? 1 : 0);
      const int fo = float_order ? float_order[k] : 0;
      if (fo < 0 || fo > 2) throw invalid("unknown float_order " + std::to_string(fo));
      r->float_order.push_back(fo);
      const am_array* col = table->cols[size_t(c)];
      bytes_per_row += 2 * pt_key_bytes(col->pt) + width_of(col);
    }
    for (int64_t p = 0; p < npayload; p++) {
      const int c = find(payload[p]);
      r->pay_cols.push_back(c);
      bytes_per_row += width_of(table->cols[size_t(c)]);
    }
    r->footprint = length * bytes_per_row + (int64_t(1) << 20);
    r->batchable = nkeys == 1 && length <= srv->batch_rows;
    // A served table is read by many streams at once: settle it once (its producer done, null
    // counts known) and let readers skip stream tracking.
    std::lock_guard<std::mutex> settle(srv->settle_mu);
    for (am_array* col : table->cols) {
      if (col->shared_read) continue;
      if (col->last_stream) AM_CUDA(cudaStreamSynchronize(col->last_stream));
      resolve_null_count(col);
      col->shared_read = true;
    }
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      if (srv->stop) throw Error("the server is shutting down");
      r->id = srv->next_id++;
      r->arrival = Clock::now();
      srv->requests[r->id] = r;
      srv->queue.push_back(r);
      *ticket = r->id;
    }
    srv->work_cv.notify_one();
    return 0;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 1;
  }
}

int am_server_wait(am_server* srv, int64_t ticket, am_plan_result** out, double* latency_ms) {
  if (!srv || !out) return 2;
  ReqPtr r;
  {
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->requests.find(ticket);
    if (it == srv->requests.end()) {
      set_last_error("unknown request " + std::to_string(ticket));
      return 2;
    }
    r = it->second;
    srv->done_cv.wait(lk, [&] { return r->done; });
    srv->requests.erase(it);
  }
  if (latency_ms) latency_ms[0] = std::chrono::duration<double, std::milli>(r->finished - r->arrival).count();
  if (r->rc != 0) {
    set_last_error(r->error);
    *out = nullptr;
    return r->rc;
  }
  *out = r->result;
  r->result = nullptr;
  return 0;
}

int am_server_get_stats(am_server* srv, am_server_stats* out) {
  if (!srv || !out) return 2;
  std::lock_guard<std::mutex> lk(srv->mu);
  *out = srv->stats;
  out->in_flight_bytes = srv->in_flight;
  out->queued = int64_t(srv->queue.size());
  return 0;
}

int am_server_release(am_server* srv) {
  if (!srv) return 2;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
  }
  srv->work_cv.notify_all();
  for (auto& t : srv->workers) t.join();
  for (auto& kv : srv->requests)
    if (kv.second->result) am_plan_result_release(kv.second->result);
  if (srv->trace) std::fclose(srv->trace);
  delete srv;
  return 0;
}

}  // extern "C"
