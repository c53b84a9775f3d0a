// A small JSON reader for the plan engine: objects, arrays, strings (with escapes), numbers, true,
// false and null. Throws am::Error with the byte offset of the first problem. Objects and arrays nest
// at most kMaxDepth deep: the reader (and the plan walk after it) recurses once a level, and a deeper
// input would overflow the calling thread's stack instead of failing.
#pragma once

#include <cstdlib>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "am_internal.h"

namespace am {
namespace json {

struct Value {
  enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
  bool b = false;
  double num = 0;
  std::string str;
  std::vector<Value> arr;
  std::vector<std::pair<std::string, Value>> obj;

  const Value* get(const std::string& k) const {
    if (kind != Object) return nullptr;
    for (auto& kv : obj) if (kv.first == k) return &kv.second;
    return nullptr;
  }
  bool is_null() const { return kind == Null; }
};

constexpr int kMaxDepth = 512;

class Parser {
 public:
  explicit Parser(const std::string& s) : s_(s) {}
  Value parse() {
    Value v = value();
    ws();
    if (i_ != s_.size()) fail("trailing characters");
    return v;
  }

 private:
  const std::string& s_;
  size_t i_ = 0;
  int depth_ = 0;
  struct Level {
    Parser& p;
    explicit Level(Parser& q) : p(q) {
      if (++p.depth_ > kMaxDepth) p.fail("nested more than " + std::to_string(kMaxDepth) + " levels deep");
    }
    ~Level() { p.depth_--; }
  };
  [[noreturn]] void fail(const std::string& m) {
    throw invalid("plan: JSON " + m + " at byte " + std::to_string(i_));
  }
  void ws() {
    while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\n' || s_[i_] == '\t' || s_[i_] == '\r')) i_++;
  }
  bool lit(const char* w) {
    size_t n = std::char_traits<char>::length(w);
    if (s_.compare(i_, n, w) == 0) { i_ += n; return true; }
    return false;
  }
  Value value() {
    ws();
    if (i_ >= s_.size()) fail("unexpected end");
    Value v;
    char c = s_[i_];
    if (c == '{') {
      const Level level(*this);
      v.kind = Value::Object;
      i_++;
      ws();
      if (i_ < s_.size() && s_[i_] == '}') { i_++; return v; }
      for (;;) {
        ws();
        if (i_ >= s_.size() || s_[i_] != '"') fail("expected a key");
        std::string k = string();
        ws();
        if (i_ >= s_.size() || s_[i_] != ':') fail("expected ':'");
        i_++;
        v.obj.emplace_back(k, value());
        ws();
        if (i_ < s_.size() && s_[i_] == ',') { i_++; continue; }
        if (i_ < s_.size() && s_[i_] == '}') { i_++; return v; }
        fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      const Level level(*this);
      v.kind = Value::Array;
      i_++;
      ws();
      if (i_ < s_.size() && s_[i_] == ']') { i_++; return v; }
      for (;;) {
        v.arr.push_back(value());
        ws();
        if (i_ < s_.size() && s_[i_] == ',') { i_++; continue; }
        if (i_ < s_.size() && s_[i_] == ']') { i_++; return v; }
        fail("expected ',' or ']'");
      }
    }
    if (c == '"') { v.kind = Value::String; v.str = string(); return v; }
    if (lit("true")) { v.kind = Value::Bool; v.b = true; return v; }
    if (lit("false")) { v.kind = Value::Bool; v.b = false; return v; }
    if (lit("null")) return v;
    if (c == '-' || (c >= '0' && c <= '9')) {
      const char* start = s_.c_str() + i_;
      char* end = nullptr;
      v.kind = Value::Number;
      v.num = std::strtod(start, &end);
      if (end == start) fail("bad number");
      i_ += size_t(end - start);
      return v;
    }
    fail("unexpected character");
  }
  static void utf8(std::string& out, unsigned cp) {
    if (cp < 0x80) out += char(cp);
    else if (cp < 0x800) { out += char(0xC0 | (cp >> 6)); out += char(0x80 | (cp & 0x3F)); }
    else if (cp < 0x10000) { out += char(0xE0 | (cp >> 12)); out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F)); }
    else { out += char(0xF0 | (cp >> 18)); out += char(0x80 | ((cp >> 12) & 0x3F)); out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F)); }
  }
  unsigned hex4() {
    if (i_ + 4 > s_.size()) fail("short \\u escape");
    unsigned v = 0;
    for (int k = 0; k < 4; k++) {
      char h = s_[i_++];
      v <<= 4;
      if (h >= '0' && h <= '9') v |= unsigned(h - '0');
      else if (h >= 'a' && h <= 'f') v |= unsigned(h - 'a' + 10);
      else if (h >= 'A' && h <= 'F') v |= unsigned(h - 'A' + 10);
      else fail("bad \\u escape");
    }
    return v;
  }
  std::string string() {
    i_++;  // opening quote
    std::string out;
    while (i_ < s_.size()) {
      char c = s_[i_++];
      if (c == '"') return out;
      if (c != '\\') { out += c; continue; }
      if (i_ >= s_.size()) break;
      char e = s_[i_++];
      switch (e) {
        case '"': out += '"'; break;
        case '\\': out += '\\'; break;
        case '/': out += '/'; break;
        case 'b': out += '\b'; break;
        case 'f': out += '\f'; break;
        case 'n': out += '\n'; break;
        case 'r': out += '\r'; break;
        case 't': out += '\t'; break;
        case 'u': {
          unsigned cp = hex4();
          if (cp >= 0xD800 && cp < 0xDC00 && i_ + 6 <= s_.size() && s_[i_] == '\\' && s_[i_ + 1] == 'u') {
            i_ += 2;
            unsigned lo = hex4();
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          }
          utf8(out, cp);
          break;
        }
        default: fail("bad escape");
      }
    }
    fail("unterminated string");
  }
};

inline Value parse(const std::string& s) { return Parser(s).parse(); }

}  // namespace json
}  // namespace am
