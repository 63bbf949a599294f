// json_min.hpp - a small JSON reader for scene files (RFC 8259 values:
// objects, arrays, strings with escapes, numbers, true/false/null).
// Parse errors throw std::runtime_error with the byte offset.
#pragma once
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace rgjson {

struct Value {
  enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
  bool b = false;
  double num = 0.0;
  std::string str;
  std::vector<Value> arr;
  std::map<std::string, Value> obj;

  bool is_object() const { return kind == Object; }
  bool is_array() const { return kind == Array; }
  bool is_number() const { return kind == Number; }
  bool has(const std::string& k) const { return kind == Object && obj.count(k) != 0; }
  const Value& operator[](const std::string& k) const {
    static const Value none;
    if (kind != Object) return none;
    auto it = obj.find(k);
    return it == obj.end() ? none : it->second;
  }
  double number(double def) const {
    if (kind == Number) return num;
    if (kind == Bool) return b ? 1.0 : 0.0;
    return def;
  }
  bool boolean(bool def) const {
    if (kind == Bool) return b;
    if (kind == Number) return num != 0.0;
    return def;
  }
  std::string string(const std::string& def) const { return kind == String ? str : def; }
};

class Parser {
 public:
  explicit Parser(const std::string& text) : s_(text) {}
  Value parse() {
    Value v = value();
    ws();
    if (p_ != s_.size()) fail("trailing characters");
    return v;
  }

 private:
  const std::string& s_;
  size_t p_ = 0;

  [[noreturn]] void fail(const char* what) const {
    throw std::runtime_error(std::string("JSON: ") + what + " at byte " + std::to_string(p_));
  }
  void ws() {
    while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\t' || s_[p_] == '\n' || s_[p_] == '\r')) ++p_;
  }
  bool lit(const char* w) {
    size_t n = std::char_traits<char>::length(w);
    if (s_.compare(p_, n, w) == 0) {
      p_ += n;
      return true;
    }
    return false;
  }
  Value value() {
    ws();
    if (p_ >= s_.size()) fail("unexpected end");
    Value v;
    char c = s_[p_];
    if (c == '{') {
      v.kind = Value::Object;
      ++p_;
      ws();
      if (p_ < s_.size() && s_[p_] == '}') { ++p_; return v; }
      for (;;) {
        ws();
        if (p_ >= s_.size() || s_[p_] != '"') fail("expected key");
        std::string k = string_lit();
        ws();
        if (p_ >= s_.size() || s_[p_] != ':') fail("expected ':'");
        ++p_;
        v.obj[k] = value();
        ws();
        if (p_ < s_.size() && s_[p_] == ',') { ++p_; continue; }
        if (p_ < s_.size() && s_[p_] == '}') { ++p_; return v; }
        fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.kind = Value::Array;
      ++p_;
      ws();
      if (p_ < s_.size() && s_[p_] == ']') { ++p_; return v; }
      for (;;) {
        v.arr.push_back(value());
        ws();
        if (p_ < s_.size() && s_[p_] == ',') { ++p_; continue; }
        if (p_ < s_.size() && s_[p_] == ']') { ++p_; return v; }
        fail("expected ',' or ']'");
      }
    }
    if (c == '"') {
      v.kind = Value::String;
      v.str = string_lit();
      return v;
    }
    if (lit("true")) { v.kind = Value::Bool; v.b = true; return v; }
    if (lit("false")) { v.kind = Value::Bool; v.b = false; return v; }
    if (lit("null")) return v;
    const char* begin = s_.c_str() + p_;
    char* end = nullptr;
    double d = std::strtod(begin, &end);
    if (end == begin) fail("bad value");
    p_ += (size_t)(end - begin);
    v.kind = Value::Number;
    v.num = d;
    return v;
  }
  static void put_utf8(std::string& o, unsigned cp) {
    if (cp < 0x80) {
      o += (char)cp;
    } else if (cp < 0x800) {
      o += (char)(0xC0 | (cp >> 6)); o += (char)(0x80 | (cp & 0x3F));
    } else if (cp < 0x10000) {
      o += (char)(0xE0 | (cp >> 12)); o += (char)(0x80 | ((cp >> 6) & 0x3F)); o += (char)(0x80 | (cp & 0x3F));
    } else {
      o += (char)(0xF0 | (cp >> 18)); o += (char)(0x80 | ((cp >> 12) & 0x3F));
      o += (char)(0x80 | ((cp >> 6) & 0x3F)); o += (char)(0x80 | (cp & 0x3F));
    }
  }
  unsigned hex4() {
    if (p_ + 4 > s_.size()) fail("bad \\u escape");
    unsigned v = 0;
    for (int k = 0; k < 4; ++k) {
      char h = s_[p_++];
      v <<= 4;
      if (h >= '0' && h <= '9') v |= (unsigned)(h - '0');
      else if (h >= 'a' && h <= 'f') v |= (unsigned)(h - 'a' + 10);
      else if (h >= 'A' && h <= 'F') v |= (unsigned)(h - 'A' + 10);
      else fail("bad \\u escape");
    }
    return v;
  }
  std::string string_lit() {
    ++p_;  // opening quote
    std::string o;
    while (p_ < s_.size()) {
      char c = s_[p_++];
      if (c == '"') return o;
      if (c != '\\') { o += c; continue; }
      if (p_ >= s_.size()) break;
      char e = s_[p_++];
      switch (e) {
        case '"': o += '"'; break;
        case '\\': o += '\\'; break;
        case '/': o += '/'; break;
        case 'b': o += '\b'; break;
        case 'f': o += '\f'; break;
        case 'n': o += '\n'; break;
        case 'r': o += '\r'; break;
        case 't': o += '\t'; break;
        case 'u': {
          unsigned cp = hex4();
          if (cp >= 0xD800 && cp < 0xDC00 && p_ + 6 <= s_.size() && s_[p_] == '\\' && s_[p_ + 1] == 'u') {
            p_ += 2;
            unsigned lo = hex4();
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          }
          put_utf8(o, cp);
          break;
        }
        default: fail("bad escape");
      }
    }
    fail("unterminated string");
  }
};

inline Value parse(const std::string& text) { return Parser(text).parse(); }

}  // namespace rgjson
