// Minimal JSON reader for SuperConga simulation configurations.
//
// The reference reads its configuration with jsoncpp (src/simulation.cu:68-85);
// this reader covers the subset those configs use: objects, arrays, numbers,
// strings, booleans and null.  Lookups of absent keys yield a null value whose
// accessors return the caller's default, mirroring jsoncpp's behaviour for
// missing members (asDouble() of null is 0, asBool() false, asString() "").
#pragma once

#include <cctype>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace scb {

class JsonValue {
public:
  enum Kind { Null, Bool, Number, String, Array, Object };

  JsonValue() = default;

  Kind kind() const { return kind_; }
  bool is_null() const { return kind_ == Null; }
  bool is_object() const { return kind_ == Object; }
  bool is_array() const { return kind_ == Array; }

  bool has(const std::string &key) const {
    return kind_ == Object && obj_.count(key) != 0;
  }
  const JsonValue &operator[](const std::string &key) const {
    if (kind_ != Object) return null_value();
    auto it = obj_.find(key);
    return it == obj_.end() ? null_value() : it->second;
  }
  const JsonValue &operator[](size_t i) const {
    if (kind_ != Array || i >= arr_.size()) return null_value();
    return arr_[i];
  }
  size_t size() const {
    return kind_ == Array ? arr_.size() : kind_ == Object ? obj_.size() : 0;
  }
  std::vector<std::string> keys() const {
    std::vector<std::string> k;
    for (auto &kv : order_) k.push_back(kv);
    return k;
  }
  double as_double(double def = 0.0) const {
    if (kind_ == Number) return num_;
    if (kind_ == Bool) return b_ ? 1.0 : 0.0;
    return def;
  }
  int as_int(int def = 0) const {
    if (kind_ == Number) return (int)num_;
    if (kind_ == Bool) return b_ ? 1 : 0;
    return def;
  }
  bool as_bool(bool def = false) const {
    if (kind_ == Bool) return b_;
    if (kind_ == Number) return num_ != 0.0;
    return def;
  }
  std::string as_string(const std::string &def = "") const {
    return kind_ == String ? str_ : def;
  }

  static JsonValue parse(const std::string &text) {
    size_t pos = 0;
    JsonValue v = parse_value(text, pos);
    skip_ws(text, pos);
    if (pos != text.size()) throw std::runtime_error("json: trailing characters");
    return v;
  }

private:
  static const JsonValue &null_value() {
    static const JsonValue n;
    return n;
  }
  static void skip_ws(const std::string &s, size_t &p) {
    while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
  }
  static JsonValue parse_value(const std::string &s, size_t &p) {
    skip_ws(s, p);
    if (p >= s.size()) throw std::runtime_error("json: unexpected end");
    const char c = s[p];
    JsonValue v;
    if (c == '{') {
      v.kind_ = Object;
      ++p;
      skip_ws(s, p);
      if (p < s.size() && s[p] == '}') {
        ++p;
        return v;
      }
      while (true) {
        skip_ws(s, p);
        JsonValue key = parse_value(s, p);
        if (key.kind_ != String) throw std::runtime_error("json: object key must be a string");
        skip_ws(s, p);
        if (p >= s.size() || s[p] != ':') throw std::runtime_error("json: expected ':'");
        ++p;
        JsonValue val = parse_value(s, p);
        if (!v.obj_.count(key.str_)) v.order_.push_back(key.str_);
        v.obj_[key.str_] = std::move(val);
        skip_ws(s, p);
        if (p < s.size() && s[p] == ',') {
          ++p;
          continue;
        }
        if (p < s.size() && s[p] == '}') {
          ++p;
          break;
        }
        throw std::runtime_error("json: expected ',' or '}'");
      }
      return v;
    }
    if (c == '[') {
      v.kind_ = Array;
      ++p;
      skip_ws(s, p);
      if (p < s.size() && s[p] == ']') {
        ++p;
        return v;
      }
      while (true) {
        v.arr_.push_back(parse_value(s, p));
        skip_ws(s, p);
        if (p < s.size() && s[p] == ',') {
          ++p;
          continue;
        }
        if (p < s.size() && s[p] == ']') {
          ++p;
          break;
        }
        throw std::runtime_error("json: expected ',' or ']'");
      }
      return v;
    }
    if (c == '"') {
      v.kind_ = String;
      ++p;
      while (p < s.size() && s[p] != '"') {
        if (s[p] == '\\' && p + 1 < s.size()) {
          const char e = s[p + 1];
          v.str_ += (e == 'n') ? '\n' : (e == 't') ? '\t' : e;
          p += 2;
        } else {
          v.str_ += s[p++];
        }
      }
      if (p >= s.size()) throw std::runtime_error("json: unterminated string");
      ++p;
      return v;
    }
    if (s.compare(p, 4, "true") == 0) {
      v.kind_ = Bool;
      v.b_ = true;
      p += 4;
      return v;
    }
    if (s.compare(p, 5, "false") == 0) {
      v.kind_ = Bool;
      v.b_ = false;
      p += 5;
      return v;
    }
    if (s.compare(p, 4, "null") == 0) {
      p += 4;
      return v;
    }
    const char *begin = s.c_str() + p;
    char *end = nullptr;
    const double d = std::strtod(begin, &end);
    if (end == begin) throw std::runtime_error("json: invalid value");
    v.kind_ = Number;
    v.num_ = d;
    p += (size_t)(end - begin);
    return v;
  }

  Kind kind_ = Null;
  bool b_ = false;
  double num_ = 0.0;
  std::string str_;
  std::vector<JsonValue> arr_;
  std::map<std::string, JsonValue> obj_;
  std::vector<std::string> order_;
};

}  // namespace scb
