// json.hpp -- a small JSON reader for the pipeline's configuration file.
//
// The reference reads its configuration with nlohmann::json
// (source/stages/argument_parser.cpp:10-60), which holds numbers as double or
// 64-bit integers and converts on get<>(). value::as_float does the same
// (parse to double, then narrow), so a step size such as "0.01" becomes the
// same float in both.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace dpa_host {
namespace json {

struct error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

class value {
 public:
  enum class kind { null, boolean, number, string, array, object };

  value() = default;
  kind type() const { return kind_; }
  bool is_null() const { return kind_ == kind::null; }

  bool as_bool() const;
  double as_double() const;
  float as_float() const { return static_cast<float>(as_double()); }
  const std::string& as_string() const;
  const std::vector<value>& as_array() const;
  const std::map<std::string, value>& as_object() const;

  bool contains(const std::string& key) const;
  const value& operator[](const std::string& key) const;  // throws when missing
  const value& operator[](size_t index) const;

  static value parse(const std::string& text);
  static value parse_file(const std::string& path);

 private:
  friend class parser;
  kind kind_ = kind::null;
  bool boolean_ = false;
  double number_ = 0.0;
  std::string string_;
  std::vector<value> array_;
  std::map<std::string, value> object_;
};

}  // namespace json
}  // namespace dpa_host
