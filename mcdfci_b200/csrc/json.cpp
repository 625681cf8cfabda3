#include "json.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

namespace mcd {
namespace {

struct Parser {
  const std::string& t;
  size_t i = 0;
  explicit Parser(const std::string& text) : t(text) {}

  [[noreturn]] void fail(const std::string& msg) {
    throw std::invalid_argument("JSON parse error at offset " + std::to_string(i) + ": " + msg);
  }
  void ws() {
    while (i < t.size() && (t[i] == ' ' || t[i] == '\t' || t[i] == '\n' || t[i] == '\r')) ++i;
  }
  bool lit(const char* s) {
    size_t n = 0;
    while (s[n]) ++n;
    if (t.compare(i, n, s) == 0) {
      i += n;
      return true;
    }
    return false;
  }
  static void put_utf8(std::string& out, unsigned cp) {
    if (cp < 0x80) {
      out += static_cast<char>(cp);
    } else if (cp < 0x800) {
      out += static_cast<char>(0xC0 | (cp >> 6));
      out += static_cast<char>(0x80 | (cp & 0x3F));
    } else {
      out += static_cast<char>(0xE0 | (cp >> 12));
      out += static_cast<char>(0x80 | ((cp >> 6) & 0x3F));
      out += static_cast<char>(0x80 | (cp & 0x3F));
    }
  }
  std::string str() {
    if (t[i] != '"') fail("expected string");
    ++i;
    std::string out;
    while (i < t.size() && t[i] != '"') {
      char c = t[i++];
      if (c == '\\') {
        if (i >= t.size()) fail("bad escape");
        char e = t[i++];
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
            if (i + 4 > t.size()) fail("bad \\u escape");
            put_utf8(out, static_cast<unsigned>(std::strtoul(t.substr(i, 4).c_str(), nullptr, 16)));
            i += 4;
            break;
          }
          default: fail("bad escape");
        }
      } else {
        out += c;
      }
    }
    if (i >= t.size()) fail("unterminated string");
    ++i;
    return out;
  }
  Json value() {
    ws();
    if (i >= t.size()) fail("unexpected end");
    const char c = t[i];
    if (c == '{') {
      ++i;
      Json o = Json::object();
      ws();
      if (i < t.size() && t[i] == '}') {
        ++i;
        return o;
      }
      while (true) {
        ws();
        std::string k = str();
        ws();
        if (i >= t.size() || t[i] != ':') fail("expected ':'");
        ++i;
        o[k] = value();
        ws();
        if (i < t.size() && t[i] == ',') {
          ++i;
          continue;
        }
        if (i < t.size() && t[i] == '}') {
          ++i;
          return o;
        }
        fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      ++i;
      Json a = Json::array();
      ws();
      if (i < t.size() && t[i] == ']') {
        ++i;
        return a;
      }
      while (true) {
        a.items().push_back(value());
        ws();
        if (i < t.size() && t[i] == ',') {
          ++i;
          continue;
        }
        if (i < t.size() && t[i] == ']') {
          ++i;
          return a;
        }
        fail("expected ',' or ']'");
      }
    }
    if (c == '"') return Json::string(str());
    if (lit("true")) return Json::boolean(true);
    if (lit("false")) return Json::boolean(false);
    if (lit("null")) return Json();
    const char* b = t.c_str() + i;
    char* e = nullptr;
    const double d = std::strtod(b, &e);
    if (e == b) fail("unexpected character");
    i += static_cast<size_t>(e - b);
    return Json::number(d);
  }
};

void esc(std::string& out, const std::string& s) {
  out += '"';
  for (char c : s) {
    switch (c) {
      case '"': out += "\\\""; break;
      case '\\': out += "\\\\"; break;
      case '\n': out += "\\n"; break;
      case '\t': out += "\\t"; break;
      case '\r': out += "\\r"; break;
      default: out += c;
    }
  }
  out += '"';
}

}  // namespace

double Json::as_number(const std::string& what) const {
  if (kind_ == Number) return d_;
  if (kind_ == Bool) return b_ ? 1.0 : 0.0;
  throw std::invalid_argument(what + " must be a number.");
}

bool Json::as_bool(const std::string& what) const {
  if (kind_ == Bool) return b_;
  if (kind_ == Number) return d_ != 0.0;
  throw std::invalid_argument(what + " must be a boolean.");
}

const std::string& Json::as_string(const std::string& what) const {
  if (kind_ != String) throw std::invalid_argument(what + " must be a string.");
  return s_;
}

const Json& Json::at(const std::string& key) const {
  static const Json null;
  if (kind_ != Object) return null;
  auto it = o_.find(key);
  return it == o_.end() ? null : it->second;
}

Json& Json::operator[](const std::string& key) {
  if (kind_ == Null) kind_ = Object;
  if (kind_ != Object) throw std::invalid_argument("not a JSON object: " + key);
  return o_[key];
}

void Json::merge_patch(const Json& patch) {
  if (!patch.is_object()) {
    *this = patch;
    return;
  }
  if (!is_object()) *this = Json::object();
  for (const auto& kv : patch.o_) {
    if (kv.second.is_null())
      o_.erase(kv.first);
    else
      o_[kv.first].merge_patch(kv.second);
  }
}

void Json::dump_to(std::string& out, int indent, int level) const {
  const std::string pad(static_cast<size_t>(indent) * (level + 1), ' ');
  const std::string pad0(static_cast<size_t>(indent) * level, ' ');
  switch (kind_) {
    case Null: out += "null"; break;
    case Bool: out += b_ ? "true" : "false"; break;
    case Number: {
      char buf[64];
      if (std::floor(d_) == d_ && std::fabs(d_) < 1e15)
        std::snprintf(buf, sizeof buf, "%.0f", d_);
      else
        std::snprintf(buf, sizeof buf, "%.17g", d_);
      out += buf;
      break;
    }
    case String: esc(out, s_); break;
    case Array: {
      out += "[";
      for (size_t k = 0; k < a_.size(); ++k) {
        out += k ? ", " : "";
        a_[k].dump_to(out, indent, level + 1);
      }
      out += "]";
      break;
    }
    case Object: {
      out += "{\n";
      size_t k = 0;
      for (const auto& kv : o_) {
        out += pad;
        esc(out, kv.first);
        out += ": ";
        kv.second.dump_to(out, indent, level + 1);
        out += (++k < o_.size()) ? ",\n" : "\n";
      }
      out += pad0 + "}";
      break;
    }
  }
}

std::string Json::dump(int indent) const {
  std::string out;
  dump_to(out, indent, 0);
  return out;
}

Json Json::parse(const std::string& text) {
  Parser p(text);
  Json v = p.value();
  p.ws();
  if (p.i != text.size()) p.fail("trailing characters");
  return v;
}

Json Json::parse_file(const std::string& path) {
  std::ifstream f(path);
  if (f.fail()) throw std::invalid_argument("Can not read the input file " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  try {
    return parse(ss.str());
  } catch (const std::exception&) {
    throw std::invalid_argument("Can not read the input file " + path);
  }
}

}  // namespace mcd
