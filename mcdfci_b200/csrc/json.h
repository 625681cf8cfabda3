// Minimal JSON value and parser for the solver's input decks (the reference
// reads them with nlohmann::json, src/input.h:31-46).  Supports objects,
// arrays, strings (with \" \\ \/ \b \f \n \r \t \uXXXX escapes), numbers,
// true/false/null, and RFC 7386 merge-patch, which the reference uses to lay
// an input deck over its defaults (src/run_wrapper.h:84-87).
#pragma once

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace mcd {

class Json {
 public:
  enum Kind { Null, Bool, Number, String, Array, Object };

  Json() = default;
  static Json boolean(bool b) { Json j; j.kind_ = Bool; j.b_ = b; return j; }
  static Json number(double d) { Json j; j.kind_ = Number; j.d_ = d; return j; }
  static Json string(std::string s) { Json j; j.kind_ = String; j.s_ = std::move(s); return j; }
  static Json array() { Json j; j.kind_ = Array; return j; }
  static Json object() { Json j; j.kind_ = Object; return j; }

  Kind kind() const { return kind_; }
  bool is_null() const { return kind_ == Null; }
  bool is_object() const { return kind_ == Object; }
  bool is_number() const { return kind_ == Number; }
  bool is_string() const { return kind_ == String; }
  bool is_bool() const { return kind_ == Bool; }
  bool is_array() const { return kind_ == Array; }

  double as_number(const std::string& what) const;
  bool as_bool(const std::string& what) const;
  const std::string& as_string(const std::string& what) const;
  const std::vector<Json>& items() const { return a_; }
  std::vector<Json>& items() { return a_; }
  const std::map<std::string, Json>& members() const { return o_; }

  bool has(const std::string& key) const { return kind_ == Object && o_.count(key) > 0; }
  const Json& at(const std::string& key) const;
  Json& operator[](const std::string& key);  // creates (and turns null into an object)

  void merge_patch(const Json& patch);
  std::string dump(int indent = 4) const;

  static Json parse(const std::string& text);
  static Json parse_file(const std::string& path);

 private:
  void dump_to(std::string& out, int indent, int level) const;
  Kind kind_ = Null;
  bool b_ = false;
  double d_ = 0.0;
  std::string s_;
  std::vector<Json> a_;
  std::map<std::string, Json> o_;
};

}  // namespace mcd
