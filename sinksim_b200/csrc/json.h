// A small JSON value model, reader and writer for the engine's data files.
//
// Reading: numbers are converted with strtod, which rounds correctly, so every double written as its shortest
// round-trip decimal comes back bit for bit. Objects keep their member order.
// Writing follows the layout of the reference's files (engine/src/json.cpp:13-62): objects one member per line,
// arrays on one line, doubles as the shortest decimal that round-trips (std::to_chars), -0 as 0, non-finite as
// null, integers as integers.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace ssb::json {

class Value {
 public:
  enum class Type { Null, Bool, Int, Number, String, Array, Object };

  Value() = default;
  static Value null() { return Value(); }
  static Value boolean(bool b) { Value v; v.type_ = Type::Bool; v.b_ = b; return v; }
  static Value integer(long long i) { Value v; v.type_ = Type::Int; v.i_ = i; v.d_ = static_cast<double>(i); return v; }
  static Value number(double d) { Value v; v.type_ = Type::Number; v.d_ = d; return v; }
  static Value string(std::string s) { Value v; v.type_ = Type::String; v.s_ = std::move(s); return v; }
  static Value array() { Value v; v.type_ = Type::Array; return v; }
  static Value object() { Value v; v.type_ = Type::Object; return v; }
  template <class T>
  static Value numbers(const std::vector<T>& xs) {
    Value v = array();
    v.items_.reserve(xs.size());
    for (const T& x : xs) v.items_.push_back(number(static_cast<double>(x)));
    return v;
  }
  template <class T>
  static Value integers(const std::vector<T>& xs) {
    Value v = array();
    v.items_.reserve(xs.size());
    for (const T& x : xs) v.items_.push_back(integer(static_cast<long long>(x)));
    return v;
  }

  Type type() const { return type_; }
  bool is_null() const { return type_ == Type::Null; }
  bool is_bool() const { return type_ == Type::Bool; }
  bool is_number() const { return type_ == Type::Int || type_ == Type::Number; }
  bool is_string() const { return type_ == Type::String; }
  bool is_array() const { return type_ == Type::Array; }
  bool is_object() const { return type_ == Type::Object; }

  bool as_bool() const { return b_; }
  double as_double() const { return d_; }
  const std::string& as_string() const { return s_; }
  const std::vector<Value>& items() const { return items_; }
  std::vector<Value>& items() { return items_; }
  const std::vector<std::pair<std::string, Value>>& members() const { return members_; }
  std::size_t size() const { return type_ == Type::Object ? members_.size() : items_.size(); }

  // Object access: nullptr when absent (or when this is not an object).
  const Value* find(const std::string& key) const;
  bool contains(const std::string& key) const { return find(key) != nullptr; }
  // Object insertion keeping order; replaces an existing member of the same name.
  Value& set(const std::string& key, Value v);
  void push(Value v) { items_.push_back(std::move(v)); }

 private:
  friend class Parser;
  Type type_ = Type::Null;
  bool b_ = false;
  long long i_ = 0;
  double d_ = 0;
  std::string s_;
  std::vector<Value> items_;
  std::vector<std::pair<std::string, Value>> members_;
  friend std::string dump(const Value&, int);
  friend void dump_to(const Value&, std::string&, int, int);
};

Value parse(const std::string& text, const std::string& where);
Value read_file(const std::string& path);
void write_file(const std::string& path, const Value& v, int indent = 2);
std::string dump(const Value& v, int indent = -1);
std::string format_number(double d);

// Typed member access that throws std::runtime_error naming `where`.
const Value& member(const Value& obj, const char* key, const std::string& where);
double number(const Value& obj, const char* key, const std::string& where);
long long integer(const Value& obj, const char* key, const std::string& where);
bool boolean(const Value& obj, const char* key, const std::string& where);
std::string string(const Value& obj, const char* key, const std::string& where);
std::string string_or(const Value& obj, const char* key, const std::string& fallback);
double number_or(const Value& obj, const char* key, double fallback);

}  // namespace ssb::json
