// json.cpp -- see json.hpp (RFC 8259 subset: no duplicate-key semantics).
#include "json.hpp"

#include <cstdlib>
#include <fstream>
#include <sstream>

namespace dpa_host {
namespace json {

class parser {
 public:
  explicit parser(const std::string& text) : s_(text) {}

  value document() {
    value v = parse_value(0);
    skip_space();
    if (p_ != s_.size()) fail("trailing characters");
    return v;
  }

 private:
  [[noreturn]] void fail(const std::string& what) const {
    throw error("JSON: " + what + " at offset " + std::to_string(p_));
  }
  void skip_space() {
    while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\t' || s_[p_] == '\n' || s_[p_] == '\r'))
      ++p_;
  }
  bool consume(const char* word) {
    size_t n = 0;
    while (word[n]) ++n;
    if (s_.compare(p_, n, word) == 0) {
      p_ += n;
      return true;
    }
    return false;
  }

  value parse_value(int depth) {
    if (depth > 256) fail("nesting too deep");
    skip_space();
    if (p_ >= s_.size()) fail("unexpected end");
    value v;
    const char c = s_[p_];
    if (c == '{') {
      v.kind_ = value::kind::object;
      ++p_;
      skip_space();
      if (p_ < s_.size() && s_[p_] == '}') {
        ++p_;
        return v;
      }
      while (true) {
        skip_space();
        if (p_ >= s_.size() || s_[p_] != '"') fail("expected a key");
        std::string key = parse_string();
        skip_space();
        if (p_ >= s_.size() || s_[p_] != ':') fail("expected ':'");
        ++p_;
        v.object_[key] = parse_value(depth + 1);
        skip_space();
        if (p_ < s_.size() && s_[p_] == ',') {
          ++p_;
          continue;
        }
        if (p_ < s_.size() && s_[p_] == '}') {
          ++p_;
          return v;
        }
        fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.kind_ = value::kind::array;
      ++p_;
      skip_space();
      if (p_ < s_.size() && s_[p_] == ']') {
        ++p_;
        return v;
      }
      while (true) {
        v.array_.push_back(parse_value(depth + 1));
        skip_space();
        if (p_ < s_.size() && s_[p_] == ',') {
          ++p_;
          continue;
        }
        if (p_ < s_.size() && s_[p_] == ']') {
          ++p_;
          return v;
        }
        fail("expected ',' or ']'");
      }
    }
    if (c == '"') {
      v.kind_ = value::kind::string;
      v.string_ = parse_string();
      return v;
    }
    if (consume("true")) {
      v.kind_ = value::kind::boolean;
      v.boolean_ = true;
      return v;
    }
    if (consume("false")) {
      v.kind_ = value::kind::boolean;
      return v;
    }
    if (consume("null")) return v;
    if (c == '-' || (c >= '0' && c <= '9')) {
      const size_t start = p_;
      if (s_[p_] == '-') ++p_;
      while (p_ < s_.size() && ((s_[p_] >= '0' && s_[p_] <= '9') || s_[p_] == '.' ||
                                s_[p_] == 'e' || s_[p_] == 'E' || s_[p_] == '+' || s_[p_] == '-'))
        ++p_;
      const std::string token = s_.substr(start, p_ - start);
      char* end = nullptr;
      v.kind_ = value::kind::number;
      v.number_ = std::strtod(token.c_str(), &end);
      if (!end || *end != '\0') fail("bad number '" + token + "'");
      return v;
    }
    fail(std::string("unexpected character '") + c + "'");
  }

  static void append_utf8(std::string& out, uint32_t cp) {
    if (cp < 0x80) {
      out += char(cp);
    } else if (cp < 0x800) {
      out += char(0xc0 | (cp >> 6));
      out += char(0x80 | (cp & 0x3f));
    } else if (cp < 0x10000) {
      out += char(0xe0 | (cp >> 12));
      out += char(0x80 | ((cp >> 6) & 0x3f));
      out += char(0x80 | (cp & 0x3f));
    } else {
      out += char(0xf0 | (cp >> 18));
      out += char(0x80 | ((cp >> 12) & 0x3f));
      out += char(0x80 | ((cp >> 6) & 0x3f));
      out += char(0x80 | (cp & 0x3f));
    }
  }

  uint32_t hex4() {
    if (p_ + 4 > s_.size()) fail("bad \\u escape");
    uint32_t v = 0;
    for (int i = 0; i < 4; ++i) {
      const char h = s_[p_++];
      v <<= 4;
      if (h >= '0' && h <= '9') v |= uint32_t(h - '0');
      else if (h >= 'a' && h <= 'f') v |= uint32_t(h - 'a' + 10);
      else if (h >= 'A' && h <= 'F') v |= uint32_t(h - 'A' + 10);
      else fail("bad \\u escape");
    }
    return v;
  }

  std::string parse_string() {
    ++p_;  // opening quote
    std::string out;
    while (true) {
      if (p_ >= s_.size()) fail("unterminated string");
      const char c = s_[p_++];
      if (c == '"') return out;
      if (c != '\\') {
        out += c;
        continue;
      }
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
          uint32_t cp = hex4();
          if (cp >= 0xd800 && cp < 0xdc00 && p_ + 1 < s_.size() && s_[p_] == '\\' &&
              s_[p_ + 1] == 'u') {
            p_ += 2;
            const uint32_t lo = hex4();
            cp = 0x10000 + ((cp - 0xd800) << 10) + (lo - 0xdc00);
          }
          append_utf8(out, cp);
          break;
        }
        default: fail("bad escape");
      }
    }
  }

  const std::string& s_;
  size_t p_ = 0;
};

bool value::as_bool() const {
  if (kind_ != kind::boolean) throw error("JSON: value is not a boolean");
  return boolean_;
}
double value::as_double() const {
  if (kind_ != kind::number) throw error("JSON: value is not a number");
  return number_;
}
const std::string& value::as_string() const {
  if (kind_ != kind::string) throw error("JSON: value is not a string");
  return string_;
}
const std::vector<value>& value::as_array() const {
  if (kind_ != kind::array) throw error("JSON: value is not an array");
  return array_;
}
const std::map<std::string, value>& value::as_object() const {
  if (kind_ != kind::object) throw error("JSON: value is not an object");
  return object_;
}
bool value::contains(const std::string& key) const {
  return kind_ == kind::object && object_.count(key) != 0;
}
const value& value::operator[](const std::string& key) const {
  const auto& o = as_object();
  const auto it = o.find(key);
  if (it == o.end()) throw error("JSON: missing key '" + key + "'");
  return it->second;
}
const value& value::operator[](size_t index) const {
  const auto& a = as_array();
  if (index >= a.size()) throw error("JSON: array index out of range");
  return a[index];
}

value value::parse(const std::string& text) { return parser(text).document(); }

value value::parse_file(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw error("JSON: cannot open " + path);
  std::stringstream ss;
  ss << in.rdbuf();
  return parse(ss.str());
}

}  // namespace json
}  // namespace dpa_host
