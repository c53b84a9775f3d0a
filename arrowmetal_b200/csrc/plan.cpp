// The plan entry points, reduced to the plans the sort's callers send: the DataFusion rule
// (datafusion/src/gpu.rs:45-66: select_all over sort over scan, optionally under limit) and the
// Polars engine (python/arrowmetal/polars_engine.py:944-998: sort with per-key nulls / float_order,
// optionally with_columns below it and limit above it).
//
// Grammar and key options follow the reference's PlanJSON (Sources/ArrowMetal/Engine/PlanJSON.swift:
// 80-140) and include/arrowmetal.h:1369-1404. A one-key sort of a plain frame on an integer (or
// totalOrder float) key gets its sorted key column from the sort's last pass and the other columns
// from one fused gather; other sorts yield a row permutation, a limit slices it, a select picks
// columns, and only the columns the plan returns are gathered, in one fused take launch.
#include <sstream>

#include "am_internal.h"
#include "json.h"
#include "plan_types.h"
#include "radix_sort.cuh"

using namespace am;

namespace {

struct Frame {
  std::vector<std::string> names;
  std::vector<am_array*> cols;   // retained
  am_array* perm = nullptr;      // retained; rows are cols taken through perm
  int64_t rows = 0;
  Frame() = default;
  Frame(const Frame&) = delete;
  Frame& operator=(const Frame&) = delete;
  Frame(Frame&& o) noexcept { *this = std::move(o); }
  Frame& operator=(Frame&& o) noexcept {
    std::swap(names, o.names);
    std::swap(cols, o.cols);
    std::swap(perm, o.perm);
    std::swap(rows, o.rows);
    return *this;
  }
  ~Frame() {
    for (am_array* c : cols) am::release(c);
    if (perm) am::release(perm);
  }
  int find(const std::string& n) const {
    for (size_t i = 0; i < names.size(); i++) if (names[i] == n) return int(i);
    return -1;
  }
};

std::string str_of(const json::Value* v, const char* what) {
  if (!v || v->kind != json::Value::String) throw invalid(std::string("plan: ") + what + " must be a string");
  return v->str;
}

// The only expression the sort's callers send: (col "name").
std::string column_ref(const std::string& sexpr) {
  size_t i = 0;
  auto ws = [&] { while (i < sexpr.size() && isspace(static_cast<unsigned char>(sexpr[i]))) i++; };
  ws();
  if (i >= sexpr.size() || sexpr[i] != '(') throw invalid("plan: expression " + sexpr + " is not taken by this build (only (col \"name\") is)");
  i++;
  ws();
  if (sexpr.compare(i, 3, "col") != 0) throw invalid("plan: expression " + sexpr + " is not taken by this build (only (col \"name\") is)");
  i += 3;
  ws();
  if (i >= sexpr.size() || sexpr[i] != '"') throw invalid("plan: bad column reference " + sexpr);
  i++;
  std::string name;
  while (i < sexpr.size() && sexpr[i] != '"') {
    if (sexpr[i] == '\\' && i + 1 < sexpr.size()) i++;
    name += sexpr[i++];
  }
  if (i >= sexpr.size()) throw invalid("plan: bad column reference " + sexpr);
  i++;
  ws();
  if (i >= sexpr.size() || sexpr[i] != ')') throw invalid("plan: bad column reference " + sexpr);
  return name;
}

bool nulls_first_of(const json::Value* v, bool fallback) {
  if (!v || v->is_null()) return fallback;
  if (v->kind == json::Value::String && v->str == "first") return true;
  if (v->kind == json::Value::String && v->str == "last") return false;
  throw invalid("plan: sort \"nulls\" must be \"first\" or \"last\"");
}
int float_order_of(const json::Value* v, int fallback) {
  if (!v || v->is_null()) return fallback;
  if (v->kind == json::Value::String) {
    const std::string& s = v->str;
    if (s == "ieee") return 0;
    if (s == "total" || s == "total_order" || s == "totalOrder") return 1;
    if (s == "nan_largest" || s == "nanLargest") return 2;
  }
  throw invalid("plan: sort \"float_order\" must be \"ieee\", \"total\" or \"nan_largest\"");
}
bool flag_of(const json::Value* v) {
  if (!v) return false;
  if (v->kind == json::Value::Bool) return v->b;
  if (v->kind == json::Value::Number) return v->num != 0;
  return false;
}

struct KeySpec { std::string col; bool desc; bool nulls_first; int float_order; };

std::vector<KeySpec> sort_keys(const json::Value& o) {
  const json::Value* by = o.get("by");
  if (!by || by->kind != json::Value::Array || by->arr.empty()) throw invalid("plan: sort needs a non-empty \"by\"");
  const bool dnf = nulls_first_of(o.get("nulls"), false);
  const int dfo = float_order_of(o.get("float_order"), 0);
  std::vector<KeySpec> keys;
  for (const json::Value& k : by->arr) {
    if (k.kind == json::Value::Object) {
      keys.push_back({str_of(k.get("column"), "a sort key's \"column\""), flag_of(k.get("descending")),
                      nulls_first_of(k.get("nulls"), dnf), float_order_of(k.get("float_order"), dfo)});
    } else if (k.kind == json::Value::Array && !k.arr.empty() && k.arr[0].kind == json::Value::String) {
      const json::Value* opts = k.arr.size() > 2 && k.arr[2].kind == json::Value::Object ? &k.arr[2] : nullptr;
      keys.push_back({k.arr[0].str, k.arr.size() > 1 ? flag_of(&k.arr[1]) : false,
                      nulls_first_of(opts ? opts->get("nulls") : nullptr, dnf),
                      float_order_of(opts ? opts->get("float_order") : nullptr, dfo)});
    } else {
      throw invalid("plan: sort keys are [name, descending, options?] or {\"column\": ...}");
    }
  }
  return keys;
}

am_array* gather_index(am_array* perm, am_array* idx) {
  am_array* out = nullptr;
  if (am_take(perm, idx, &out) != 0) throw Error(am_last_error());
  return out;
}

// The frame's columns, gathered through its permutation if it has one.
std::vector<am_array*> materialize(Frame& f, const std::vector<int>& which) {
  std::vector<am_array*> out(which.size(), nullptr);
  if (!f.perm) {
    for (size_t i = 0; i < which.size(); i++) {
      out[i] = f.cols[size_t(which[i])];
      retain(out[i]);
    }
    return out;
  }
  std::vector<am_array*> src;
  for (int w : which) src.push_back(f.cols[size_t(w)]);
  if (src.empty()) return out;
  if (am_take_columns(src.data(), int64_t(src.size()), f.perm, out.data()) != 0) throw Error(am_last_error());
  return out;
}

Frame eval(const json::Value& node, am_plan_source** sources, int64_t nsrc, std::ostringstream* explain, int depth);

// A column whose contents are complete on the device (no upload still running).
bool settled(const am_array* c) {
  return !c->ready || cudaEventQuery(c->ready->ev) == cudaSuccess;
}

// One invertible key over an unpermuted frame whose other columns are complete in device memory and
// fit a 16-byte row record: they ride through the sort with their rows and come out sorted where the
// rows reach their final places, so nothing is gathered afterwards. Columns still uploading (imports
// from host memory) are gathered after the sort instead, which then waits only for the key column.
// Returns false, with the frame untouched, when the frame does not qualify.
bool sort_payload_in_records(Frame& f, int key_col, const SortKey& key, cudaStream_t s) {
  std::vector<am_array*> pay;
  for (size_t c = 0; c < f.cols.size(); c++)
    if (int(c) != key_col) pay.push_back(f.cols[c]);
  rs::RecLayout rl{};
  if (pay.empty() || !payload_record_layout(pay, &rl)) return false;
  for (am_array* c : pay)
    if (c->length != f.rows || !settled(c)) return false;
  for (am_array* c : pay) use_on(c, s);
  am_array* sorted_key = new_array(key.col->pt, key.col->format, f.rows);
  std::vector<am_array*> outs;
  try {
    for (size_t i = 0; i < pay.size(); i++) {
      am_array* o = new_array(pay[i]->pt, pay[i]->format, f.rows);
      outs.push_back(o);
      o->values = DevBuffer::alloc(size_t(f.rows) * size_t(rl.width[i]) + 16, s);
      o->null_count = 0;
      o->last_stream = s;
      rl.dst[i] = o->values->ptr;
    }
    radix_sort({key}, f.rows, nullptr, 4, sorted_key, s, &tls().last_stats, &rl);
  } catch (...) {
    am::release(sorted_key);
    for (am_array* o : outs) am::release(o);
    throw;
  }
  auto ready = std::make_shared<ReadyEvent>(s);
  size_t t = 0;
  for (size_t c = 0; c < f.cols.size(); c++) {
    am::release(f.cols[c]);
    if (int(c) == key_col) {
      f.cols[c] = sorted_key;
    } else {
      outs[t]->ready = ready;
      f.cols[c] = outs[t++];
    }
  }
  return true;
}

// The sort of a frame by `keys`.
Frame sort_frame(Frame f, const std::vector<KeySpec>& keys) {
  std::vector<int> which;
  for (auto& k : keys) {
    const int i = f.find(k.col);
    if (i < 0) throw invalid("plan: unknown sort column \"" + k.col + "\"");
    which.push_back(i);
  }
  // One integer (or totalOrder float) key over an unpermuted frame: the last pass rebuilds the sorted
  // key column from the sorted keys while it writes the permutation, and the other columns come
  // through one fused gather. The key column is never gathered.
  if (keys.size() == 1 && !f.perm && f.rows > 0) {
    SortKey key{f.cols[size_t(which[0])], keys[0].desc, keys[0].nulls_first, keys[0].float_order};
    if (key.float_order < 0 || key.float_order > 2) throw invalid("unknown float_order " + std::to_string(key.float_order));
    if (key_invertible(key)) {
      check_index_rows(f.rows, "sort");
      cudaStream_t s = stream();
      use_on(key.col, s);
      if (sort_payload_in_records(f, which[0], key, s)) return f;
      am_array* sorted_key = new_array(key.col->pt, key.col->format, f.rows);
      am_array* idx = new_array(PT_U32, "I", f.rows);
      std::vector<am_array*> src, taken;
      try {
        idx->values = DevBuffer::alloc(size_t(f.rows) * 4 + 16, s);
        idx->null_count = 0;
        idx->perm_of = f.rows;
        idx->last_stream = s;
        radix_sort({key}, f.rows, idx->values->ptr, 4, sorted_key, s, &tls().last_stats);
        for (size_t c = 0; c < f.cols.size(); c++)
          if (int(c) != which[0]) src.push_back(f.cols[c]);
        taken.assign(src.size(), nullptr);
        bool uploading = false;
        for (am_array* c : src) uploading = uploading || !settled(c);
        if (uploading && src.size() > 1) {
          // Columns still uploading: each is gathered once its own upload is done, in column order (the
          // order of their imports), and carries its own ready event, so its export starts while the
          // later columns still upload or gather.
          for (size_t i = 0; i < src.size(); i++) {
            if (am_take_columns(&src[i], 1, idx, &taken[i]) != 0) throw Error(am_last_error());
            if (taken[i]->pt != PT_STRUCT) taken[i]->ready = std::make_shared<ReadyEvent>(taken[i]->last_stream ? taken[i]->last_stream : s);
          }
        } else if (!src.empty() && am_take_columns(src.data(), int64_t(src.size()), idx, taken.data()) != 0) {
          throw Error(am_last_error());
        }
      } catch (...) {
        am::release(sorted_key);
        am::release(idx);
        for (am_array* t : taken)
          if (t) am::release(t);
        throw;
      }
      am::release(idx);
      size_t t = 0;
      for (size_t c = 0; c < f.cols.size(); c++) {
        am::release(f.cols[c]);
        f.cols[c] = int(c) == which[0] ? sorted_key : taken[t++];
      }
      return f;
    }
  }
  std::vector<am_array*> kc = materialize(f, which);
  std::vector<am_array*> handles = kc;
  std::vector<int> desc, np, fo;
  for (auto& k : keys) {
    desc.push_back(k.desc ? 1 : 0);
    np.push_back(k.nulls_first ? 1 : 0);
    fo.push_back(k.float_order);
  }
  am_array* idx = nullptr;
  int rc = f.rows == 0 ? 0 : am_lexsort_ex2(handles.data(), desc.data(), np.data(), fo.data(), int64_t(keys.size()), &idx);
  for (am_array* c : kc) am::release(c);
  if (rc != 0) throw Error(am_last_error());
  if (f.rows == 0) return f;
  if (f.perm) {
    am_array* composed = gather_index(f.perm, idx);
    am::release(idx);
    am::release(f.perm);
    f.perm = composed;
  } else {
    f.perm = idx;
  }
  return f;
}

// Rows [off, off + count) of a frame.
Frame limit_frame(Frame f, int64_t off, int64_t count) {
  const int64_t start = std::min(off, f.rows);
  const int64_t len = std::min<int64_t>(count, f.rows - start);
  auto cut = [&](am_array*& a) {
    am_array* s = nullptr;
    if (am_slice(a, start, len, &s) != 0) throw Error(am_last_error());
    am::release(a);
    a = s;
  };
  if (f.perm) cut(f.perm);
  else for (am_array*& col : f.cols) cut(col);
  f.rows = len;
  return f;
}


Frame eval(const json::Value& node, am_plan_source** sources, int64_t nsrc, std::ostringstream* explain, int depth) {
  if (node.kind != json::Value::Object) throw invalid("plan: a node must be an object");
  const std::string op = str_of(node.get("op"), "\"op\"");
  const std::string pad(size_t(depth) * 2, ' ');
  if (op == "scan") {
    const std::string name = str_of(node.get("source"), "scan \"source\"");
    am_plan_source* src = nullptr;
    for (int64_t i = 0; i < nsrc; i++) if (sources[i] && sources[i]->name == name) src = sources[i];
    if (!src) throw invalid("plan: unknown source \"" + name + "\"");
    Frame f;
    f.rows = src->rows;
    const json::Value* cols = node.get("columns");
    if (cols && cols->kind == json::Value::Array) {
      for (const json::Value& c : cols->arr) {
        const std::string cn = str_of(&c, "scan column");
        size_t k = 0;
        while (k < src->names.size() && src->names[k] != cn) k++;
        if (k == src->names.size()) throw invalid("plan: source \"" + name + "\" has no column \"" + cn + "\"");
        f.names.push_back(cn);
        f.cols.push_back(src->cols[k]);
        retain(src->cols[k]);
      }
    } else {
      for (size_t k = 0; k < src->names.size(); k++) {
        f.names.push_back(src->names[k]);
        f.cols.push_back(src->cols[k]);
        retain(src->cols[k]);
      }
    }
    if (explain) *explain << pad << "scan " << name << " [" << f.cols.size() << " columns, " << f.rows << " rows]\n";
    return f;
  }
  const json::Value* in = node.get("input");
  if (!in) throw invalid("plan: \"" + op + "\" needs an \"input\"");
  if (op == "select" || op == "with_columns") {
    const json::Value* exprs = node.get("exprs");
    if (!exprs || exprs->kind != json::Value::Array) throw invalid("plan: " + op + ".exprs entries are [name, sexpr] pairs");
    if (explain) *explain << pad << op << " " << exprs->arr.size() << " column(s)\n";
    Frame f = eval(*in, sources, nsrc, explain, depth + 1);
    Frame g;
    g.rows = f.rows;
    g.perm = f.perm;
    if (g.perm) retain(g.perm);
    if (op == "with_columns") {
      for (size_t i = 0; i < f.cols.size(); i++) {
        g.names.push_back(f.names[i]);
        g.cols.push_back(f.cols[i]);
        retain(f.cols[i]);
      }
    }
    for (const json::Value& e : exprs->arr) {
      if (e.kind != json::Value::Array || e.arr.size() != 2 || e.arr[0].kind != json::Value::String ||
          e.arr[1].kind != json::Value::String)
        throw invalid("plan: " + op + ".exprs entries are [name, sexpr] pairs");
      const std::string ref = column_ref(e.arr[1].str);
      const int k = f.find(ref);
      if (k < 0) throw invalid("plan: unknown column \"" + ref + "\"");
      am_array* c = f.cols[size_t(k)];
      retain(c);
      const int existing = g.find(e.arr[0].str);
      if (existing >= 0) {
        am::release(g.cols[size_t(existing)]);
        g.cols[size_t(existing)] = c;
      } else {
        g.names.push_back(e.arr[0].str);
        g.cols.push_back(c);
      }
    }
    return g;
  }
  if (op == "sort") {
    std::vector<KeySpec> keys = sort_keys(node);
    if (explain) {
      *explain << pad << "sort by";
      for (auto& k : keys)
        *explain << " " << k.col << (k.desc ? " desc" : " asc") << (k.nulls_first ? " nulls_first" : "")
                 << (k.float_order == 1 ? " total" : k.float_order == 2 ? " nan_largest" : "");
      *explain << " (GPU radix argsort, one fused take)\n";
    }
    Frame f = eval(*in, sources, nsrc, explain, depth + 1);
    return sort_frame(std::move(f), keys);
  }
  if (op == "limit") {
    const json::Value* c = node.get("count");
    if (!c || c->kind != json::Value::Number || c->num < 0) throw invalid("plan: limit needs a non-negative \"count\"");
    const json::Value* o = node.get("offset");
    const int64_t off = (o && o->kind == json::Value::Number) ? int64_t(o->num) : 0;
    if (off < 0) throw invalid("plan: limit \"offset\" must be non-negative");
    if (explain) *explain << pad << "limit " << int64_t(c->num) << " offset " << off << "\n";
    // LIMIT over a one-key sort of an unpermuted frame (ORDER BY ... LIMIT): the sort's first
    // offset + count rows by radix selection, identical to the full sort's prefix; only those rows
    // are gathered.
    if (!explain && in->kind == json::Value::Object && in->get("op") && in->get("op")->kind == json::Value::String &&
        in->get("op")->str == "sort" && in->get("input")) {
      std::vector<KeySpec> keys = sort_keys(*in);
      if (keys.size() == 1) {
        Frame f = eval(*in->get("input"), sources, nsrc, nullptr, depth + 2);
        const int ki = f.find(keys[0].col);
        if (ki < 0) throw invalid("plan: unknown sort column \"" + keys[0].col + "\"");
        const int64_t want = std::min<int64_t>(off + int64_t(c->num), f.rows);
        if (!f.perm && f.rows > 0 && want < f.rows) {
          SortKey key{f.cols[size_t(ki)], keys[0].desc, keys[0].nulls_first, keys[0].float_order};
          if (key.float_order < 0 || key.float_order > 2) throw invalid("unknown float_order " + std::to_string(key.float_order));
          check_index_rows(f.rows, "sort");
          cudaStream_t st = stream();
          use_on(key.col, st);
          if (am_array* top = radix_top_k(key, want, st)) {
            const int64_t start = std::min(off, want);
            am_array* cut = nullptr;
            const int rc = am_slice(top, start, want - start, &cut);
            am::release(top);
            if (rc != 0) throw Error(am_last_error());
            f.perm = cut;
            f.rows = want - start;
            return f;
          }
        }
        // Otherwise the full sort, then the slice.
        f = sort_frame(std::move(f), keys);
        return limit_frame(std::move(f), off, int64_t(c->num));
      }
    }
    Frame f = eval(*in, sources, nsrc, explain, depth + 1);
    return limit_frame(std::move(f), off, int64_t(c->num));
  }
  throw invalid("plan: op \"" + op + "\" is not supported by this build (scan, select, with_columns, sort and limit are)");
}

template <class F>
int guard(F&& f) {
  try {
    return f();
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 1;
  }
}

}  // namespace

extern "C" {

int am_plan_source_create(const char* name, am_array** columns, const char** names, int64_t n_columns,
                          am_plan_source** out) {
  if (!name || !out || n_columns < 0 || (n_columns > 0 && (!columns || !names))) return 2;
  for (int64_t i = 0; i < n_columns; i++) if (!columns[i] || !names[i]) return 2;
  return guard([&] {
    auto* s = new am_plan_source_t();
    s->name = name;
    for (int64_t i = 0; i < n_columns; i++) {
      if (i > 0 && columns[i]->length != columns[0]->length) {
        int64_t a = columns[0]->length, b = columns[i]->length;
        delete s;
        throw length_mismatch(a, b);
      }
      retain(columns[i]);
      s->cols.push_back(columns[i]);
      s->names.push_back(names[i]);
    }
    s->rows = n_columns ? columns[0]->length : 0;
    *out = s;
    return 0;
  });
}

void am_plan_source_release(am_plan_source* s) { delete s; }

int am_plan_run(const char* plan_json, am_plan_source** sources, int64_t n_sources, int optimize, am_plan_result** out) {
  (void)optimize;
  if (!plan_json || !out || n_sources < 0 || (n_sources > 0 && !sources)) return 2;
  return guard([&] {
    json::Value root = json::parse(plan_json);
    Frame f = eval(root, sources, n_sources, nullptr, 0);
    std::vector<int> all;
    for (size_t i = 0; i < f.cols.size(); i++) all.push_back(int(i));
    auto* r = new am_plan_result_t();
    try {
      r->cols = materialize(f, all);
    } catch (...) {
      delete r;
      throw;
    }
    r->names = f.names;
    r->rows = f.rows;
    *out = r;
    return 0;
  });
}

const char* am_plan_explain(const char* plan_json, am_plan_source** sources, int64_t n_sources, int optimize) {
  (void)optimize;
  if (!plan_json) return nullptr;
  std::ostringstream os;
  int rc = guard([&] {
    json::Value root = json::parse(plan_json);
    // Explaining evaluates nothing on the device: validate the tree and describe it.
    std::function<void(const json::Value&, int)> walk = [&](const json::Value& n, int d) {
      if (n.kind != json::Value::Object) throw invalid("plan: a node must be an object");
      const std::string op = str_of(n.get("op"), "\"op\"");
      const std::string pad(size_t(d) * 2, ' ');
      if (op == "scan") {
        const std::string name = str_of(n.get("source"), "scan \"source\"");
        bool found = false;
        for (int64_t i = 0; i < n_sources; i++) if (sources && sources[i] && sources[i]->name == name) found = true;
        if (!found) throw invalid("plan: unknown source \"" + name + "\"");
        os << pad << "scan " << name << "\n";
        return;
      }
      if (op == "sort") {
        auto keys = sort_keys(n);
        os << pad << "sort by";
        for (auto& k : keys) os << " " << k.col << (k.desc ? " desc" : " asc");
        os << " -> gpu radix argsort + fused take\n";
      } else if (op == "limit" || op == "select" || op == "with_columns") {
        os << pad << op << "\n";
      } else {
        throw invalid("plan: op \"" + op + "\" is not supported by this build (scan, select, with_columns, sort and limit are)");
      }
      const json::Value* in = n.get("input");
      if (!in) throw invalid("plan: \"" + op + "\" needs an \"input\"");
      walk(*in, d + 1);
    };
    walk(root, 0);
    return 0;
  });
  if (rc != 0) return nullptr;
  tls().scratch_text = os.str();
  return tls().scratch_text.c_str();
}

int64_t am_plan_column_count(am_plan_result* r) { return r ? int64_t(r->cols.size()) : -1; }
int64_t am_plan_row_count(am_plan_result* r) { return r ? r->rows : -1; }
const char* am_plan_column_name(am_plan_result* r, int64_t i) {
  if (!r || i < 0 || i >= int64_t(r->names.size())) return nullptr;
  return r->names[size_t(i)].c_str();
}
int am_plan_column(am_plan_result* r, int64_t i, am_array** out) {
  if (!r || !out) return 2;
  if (i < 0 || i >= int64_t(r->cols.size())) {
    set_last_error("Invalid ArrowArray: plan column index out of range");
    return 1;
  }
  retain(r->cols[size_t(i)]);
  *out = r->cols[size_t(i)];
  return 0;
}
void am_plan_result_release(am_plan_result* r) { delete r; }

}  // extern "C"
