#include "json.h"

#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace ssb::json {

const Value* Value::find(const std::string& key) const {
  if (type_ != Type::Object) return nullptr;
  for (const auto& kv : members_)
    if (kv.first == key) return &kv.second;
  return nullptr;
}

Value& Value::set(const std::string& key, Value v) {
  if (type_ != Type::Object) { type_ = Type::Object; members_.clear(); }
  for (auto& kv : members_)
    if (kv.first == key) { kv.second = std::move(v); return kv.second; }
  members_.emplace_back(key, std::move(v));
  return members_.back().second;
}

// ----------------------------------------------------------------------------- reader

class Parser {
 public:
  Parser(const std::string& text, const std::string& where) : s_(text), where_(where) {}

  Value document() {
    Value v = value(0);
    ws();
    if (p_ != s_.size()) fail("trailing characters");
    return v;
  }

 private:
  const std::string& s_;
  const std::string& where_;
  std::size_t p_ = 0;

  [[noreturn]] void fail(const std::string& what) const {
    std::size_t line = 1;
    for (std::size_t i = 0; i < p_ && i < s_.size(); ++i) line += s_[i] == '\n';
    throw std::runtime_error(where_ + ": JSON parse error at line " + std::to_string(line) + ": " + what);
  }
  void ws() {
    while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\n' || s_[p_] == '\r' || s_[p_] == '\t')) ++p_;
  }
  bool eat(char c) {
    ws();
    if (p_ < s_.size() && s_[p_] == c) { ++p_; return true; }
    return false;
  }
  void expect(char c) {
    if (!eat(c)) fail(std::string("expected '") + c + "'");
  }
  bool word(const char* w) {
    std::size_t n = 0;
    while (w[n]) ++n;
    if (s_.compare(p_, n, w) == 0) { p_ += n; return true; }
    return false;
  }

  static void utf8(std::string& out, unsigned cp) {
    if (cp < 0x80) out += static_cast<char>(cp);
    else if (cp < 0x800) { out += static_cast<char>(0xC0 | (cp >> 6)); out += static_cast<char>(0x80 | (cp & 0x3F)); }
    else if (cp < 0x10000) {
      out += static_cast<char>(0xE0 | (cp >> 12)); out += static_cast<char>(0x80 | ((cp >> 6) & 0x3F)); out += static_cast<char>(0x80 | (cp & 0x3F));
    } else {
      out += static_cast<char>(0xF0 | (cp >> 18)); out += static_cast<char>(0x80 | ((cp >> 12) & 0x3F));
      out += static_cast<char>(0x80 | ((cp >> 6) & 0x3F)); out += static_cast<char>(0x80 | (cp & 0x3F));
    }
  }
  unsigned hex4() {
    if (p_ + 4 > s_.size()) fail("truncated \\u escape");
    unsigned v = 0;
    for (int i = 0; i < 4; ++i) {
      const char c = s_[p_++];
      v <<= 4;
      if (c >= '0' && c <= '9') v |= static_cast<unsigned>(c - '0');
      else if (c >= 'a' && c <= 'f') v |= static_cast<unsigned>(c - 'a' + 10);
      else if (c >= 'A' && c <= 'F') v |= static_cast<unsigned>(c - 'A' + 10);
      else fail("bad \\u escape");
    }
    return v;
  }
  std::string str() {
    // the opening quote is consumed
    std::string out;
    for (;;) {
      if (p_ >= s_.size()) fail("unterminated string");
      const char c = s_[p_++];
      if (c == '"') return out;
      if (c != '\\') { out += c; continue; }
      if (p_ >= s_.size()) fail("unterminated escape");
      const char e = s_[p_++];
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
          if (cp >= 0xD800 && cp < 0xDC00 && p_ + 1 < s_.size() && s_[p_] == '\\' && s_[p_ + 1] == 'u') {
            p_ += 2;
            const unsigned lo = hex4();
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          }
          utf8(out, cp);
          break;
        }
        default: fail("bad escape");
      }
    }
  }
  Value num() {
    const std::size_t b = p_;
    bool isInt = true;
    if (p_ < s_.size() && s_[p_] == '-') ++p_;
    while (p_ < s_.size()) {
      const char c = s_[p_];
      if (c >= '0' && c <= '9') { ++p_; continue; }
      if (c == '.' || c == 'e' || c == 'E' || c == '+' || c == '-') { isInt = false; ++p_; continue; }
      break;
    }
    const std::string lit = s_.substr(b, p_ - b);
    if (lit.empty() || lit == "-") fail("bad number");
    char* end = nullptr;
    if (isInt && lit.size() < 18) {
      const long long i = std::strtoll(lit.c_str(), &end, 10);
      if (*end) fail("bad number " + lit);
      Value v = Value::integer(i);
      return v;
    }
    const double d = std::strtod(lit.c_str(), &end);
    if (*end) fail("bad number " + lit);
    return Value::number(d);
  }
  Value value(int depth) {
    if (depth > 256) fail("nesting too deep");
    ws();
    if (p_ >= s_.size()) fail("unexpected end");
    const char c = s_[p_];
    if (c == '{') {
      ++p_;
      Value v = Value::object();
      if (eat('}')) return v;
      do {
        ws();
        if (p_ >= s_.size() || s_[p_] != '"') fail("expected a member name");
        ++p_;
        std::string key = str();
        expect(':');
        v.members_.emplace_back(std::move(key), value(depth + 1));
      } while (eat(','));
      expect('}');
      return v;
    }
    if (c == '[') {
      ++p_;
      Value v = Value::array();
      if (eat(']')) return v;
      do v.items_.push_back(value(depth + 1));
      while (eat(','));
      expect(']');
      return v;
    }
    if (c == '"') { ++p_; return Value::string(str()); }
    if (word("true")) return Value::boolean(true);
    if (word("false")) return Value::boolean(false);
    if (word("null")) return Value::null();
    return num();
  }
};

Value parse(const std::string& text, const std::string& where) { return Parser(text, where).document(); }

Value read_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw std::runtime_error("cannot open " + path);
  std::ostringstream ss;
  ss << in.rdbuf();
  return parse(ss.str(), path);
}

// ----------------------------------------------------------------------------- writer

std::string format_number(double d) {
  if (!std::isfinite(d)) return "null";
  if (d == 0) d = 0.0;
  char buf[64];
  const auto r = std::to_chars(buf, buf + sizeof buf, d);
  return std::string(buf, r.ptr);
}

namespace {

void quote(const std::string& s, std::string& out) {
  out += '"';
  for (const unsigned char c : s) {
    switch (c) {
      case '"': out += "\\\""; break;
      case '\\': out += "\\\\"; break;
      case '\b': out += "\\b"; break;
      case '\f': out += "\\f"; break;
      case '\n': out += "\\n"; break;
      case '\r': out += "\\r"; break;
      case '\t': out += "\\t"; break;
      default:
        if (c < 0x20) {
          char buf[8];
          std::snprintf(buf, sizeof buf, "\\u%04x", c);
          out += buf;
        } else {
          out += static_cast<char>(c);
        }
    }
  }
  out += '"';
}

}  // namespace

void dump_to(const Value& v, std::string& out, int indent, int level) {
  switch (v.type_) {
    case Value::Type::Null: out += "null"; break;
    case Value::Type::Bool: out += v.b_ ? "true" : "false"; break;
    case Value::Type::Int: out += std::to_string(v.i_); break;
    case Value::Type::Number: out += format_number(v.d_); break;
    case Value::Type::String: quote(v.s_, out); break;
    case Value::Type::Array: {
      out += '[';
      bool first = true;
      for (const Value& x : v.items_) {
        if (!first) out += ',';
        first = false;
        dump_to(x, out, -1, level + 1);
      }
      out += ']';
      break;
    }
    case Value::Type::Object: {
      if (v.members_.empty()) { out += "{}"; break; }
      out += '{';
      const std::string pad = indent >= 0 ? "\n" + std::string(static_cast<std::size_t>((level + 1) * indent), ' ') : "";
      const std::string close = indent >= 0 ? "\n" + std::string(static_cast<std::size_t>(level * indent), ' ') : "";
      bool first = true;
      for (const auto& kv : v.members_) {
        if (!first) out += ',';
        first = false;
        out += pad;
        quote(kv.first, out);
        out += indent >= 0 ? ": " : ":";
        dump_to(kv.second, out, indent, level + 1);
      }
      out += close;
      out += '}';
      break;
    }
  }
}

std::string dump(const Value& v, int indent) {
  std::string out;
  dump_to(v, out, indent, 0);
  return out;
}

void write_file(const std::string& path, const Value& v, int indent) {
  std::ofstream out(path, std::ios::binary);
  if (!out) throw std::runtime_error("cannot write " + path);
  out << dump(v, indent) << '\n';
  if (!out) throw std::runtime_error("write failed: " + path);
}

// ----------------------------------------------------------------------------- typed access

const Value& member(const Value& obj, const char* key, const std::string& where) {
  if (!obj.is_object()) throw std::runtime_error(where + ": expected an object holding \"" + key + "\"");
  const Value* v = obj.find(key);
  if (!v) throw std::runtime_error(where + ": missing member \"" + key + "\"");
  return *v;
}

double number(const Value& obj, const char* key, const std::string& where) {
  const Value& v = member(obj, key, where);
  if (!v.is_number()) throw std::runtime_error(where + ": member \"" + key + "\" is not a number");
  return v.as_double();
}

long long integer(const Value& obj, const char* key, const std::string& where) {
  const double d = number(obj, key, where);
  if (d != std::floor(d)) throw std::runtime_error(where + ": member \"" + key + "\" is not an integer");
  return static_cast<long long>(d);
}

bool boolean(const Value& obj, const char* key, const std::string& where) {
  const Value& v = member(obj, key, where);
  if (!v.is_bool()) throw std::runtime_error(where + ": member \"" + key + "\" is not a boolean");
  return v.as_bool();
}

std::string string(const Value& obj, const char* key, const std::string& where) {
  const Value& v = member(obj, key, where);
  if (!v.is_string()) throw std::runtime_error(where + ": member \"" + key + "\" is not a string");
  return v.as_string();
}

std::string string_or(const Value& obj, const char* key, const std::string& fallback) {
  const Value* v = obj.find(key);
  return (v && v->is_string()) ? v->as_string() : fallback;
}

double number_or(const Value& obj, const char* key, double fallback) {
  const Value* v = obj.find(key);
  return (v && v->is_number()) ? v->as_double() : fallback;
}

}  // namespace ssb::json
