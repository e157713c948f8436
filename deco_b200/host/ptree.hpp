// ptree.hpp — the subset of boost::property_tree the reference's configuration
// code uses (IO/ptree.hpp:27-119, every `param.get<T>("a.b")` call site), so the
// reference's param_*.json files read unchanged.
//
//   ptree::get<T>(path), get<T>(path, default), get_child(path), put(path, v),
//   get_value<T>(), empty(), iteration over (key, child) pairs;
//   read_json(istream&, ptree&) and json_parser_error;
//   remove_json_comments(text): strips // and /* */ comments and blank lines
//   the way IO/ptree.hpp:27-84 does before parsing.
//
// Values are kept as strings, as in boost: numbers are converted on get<T>()
// with stream extraction that must consume the whole string.
#pragma once
#include <cctype>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace deco {

struct ptree_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct json_parser_error : ptree_error {
  using ptree_error::ptree_error;
};

class ptree {
 public:
  using value_type = std::pair<const std::string, ptree>;

  ptree() = default;
  explicit ptree(std::string v) : data_(std::move(v)) {}

  bool empty() const { return kids_.empty(); }
  const std::string& data() const { return data_; }
  std::vector<std::pair<std::string, ptree>>::const_iterator begin() const { return kids_.begin(); }
  std::vector<std::pair<std::string, ptree>>::const_iterator end() const { return kids_.end(); }
  size_t size() const { return kids_.size(); }

  template <typename T>
  T get_value() const {
    return convert<T>(data_, "<value>");
  }

  const ptree* find(const std::string& path) const {
    const ptree* node = this;
    size_t pos = 0;
    while (node) {
      size_t dot = path.find('.', pos);
      std::string key = path.substr(pos, dot == std::string::npos ? std::string::npos : dot - pos);
      const ptree* next = nullptr;
      for (auto& kv : node->kids_)
        if (kv.first == key) { next = &kv.second; break; }
      node = next;
      if (dot == std::string::npos) break;
      pos = dot + 1;
    }
    return node;
  }

  const ptree& get_child(const std::string& path) const {
    const ptree* p = find(path);
    if (!p) throw ptree_error("No such node (" + path + ")");
    return *p;
  }
  ptree& get_child(const std::string& path) { return const_cast<ptree&>(static_cast<const ptree*>(this)->get_child(path)); }

  template <typename T>
  T get(const std::string& path) const {
    return convert<T>(get_child(path).data_, path);
  }
  template <typename T>
  T get(const std::string& path, const T& dflt) const {
    const ptree* p = find(path);
    if (!p) return dflt;
    try {
      return convert<T>(p->data_, path);
    } catch (const ptree_error&) {
      return dflt;
    }
  }

  template <typename T>
  ptree& put(const std::string& path, const T& value) {
    ptree* node = this;
    size_t pos = 0;
    for (;;) {
      size_t dot = path.find('.', pos);
      std::string key = path.substr(pos, dot == std::string::npos ? std::string::npos : dot - pos);
      ptree* next = nullptr;
      for (auto& kv : node->kids_)
        if (kv.first == key) { next = &kv.second; break; }
      if (!next) {
        node->kids_.emplace_back(key, ptree());
        next = &node->kids_.back().second;
      }
      node = next;
      if (dot == std::string::npos) break;
      pos = dot + 1;
    }
    std::ostringstream os;
    os.precision(17);
    os << value;
    node->data_ = os.str();
    return *node;
  }

  ptree& add_child(const std::string& key, ptree child) {
    kids_.emplace_back(key, std::move(child));
    return kids_.back().second;
  }

 private:
  template <typename T>
  static T convert(const std::string& s, const std::string& path) {
    if constexpr (std::is_same<T, std::string>::value) {
      return s;
    } else {
      std::istringstream is(s);
      is.imbue(std::locale::classic());
      T v{};
      is >> v;
      if (!is.eof()) is >> std::ws;
      if (is.fail() || is.bad() || is.get() != std::char_traits<char>::eof())
        throw ptree_error("conversion of data to type failed (" + path + " = \"" + s + "\")");
      return v;
    }
  }

  std::string data_;
  std::vector<std::pair<std::string, ptree>> kids_;
  friend class json_reader;
};

// Comment stripping with the same rules as IO/ptree.hpp:27-84: a `//` ends the
// line, `/* ... */` may span lines, lines left empty are dropped.
inline std::string remove_json_comments(const std::string& input) {
  std::istringstream in(input);
  std::ostringstream out;
  std::string line;
  bool in_block = false;
  while (std::getline(in, line)) {
    std::string kept;
    size_t pos = 0;
    while (pos < line.size()) {
      if (in_block) {
        size_t e = line.find("*/", pos);
        if (e == std::string::npos) break;
        in_block = false;
        pos = e + 2;
        continue;
      }
      size_t sl = line.find("//", pos), ml = line.find("/*", pos);
      if (sl != std::string::npos && (ml == std::string::npos || sl < ml)) {
        kept += line.substr(pos, sl - pos);
        break;
      }
      if (ml != std::string::npos) {
        kept += line.substr(pos, ml - pos);
        size_t e = line.find("*/", ml + 2);
        if (e == std::string::npos) { in_block = true; break; }
        pos = e + 2;
        continue;
      }
      kept += line.substr(pos);
      break;
    }
    if (!kept.empty() && kept.find_first_not_of(" \t\r\n") != std::string::npos) out << kept << '\n';
  }
  return out.str();
}

class json_reader {
 public:
  explicit json_reader(const std::string& s) : s_(s) {}
  void parse(ptree& root) {
    ws();
    value(root);
    ws();
    if (i_ != s_.size()) fail("trailing characters");
  }

 private:
  [[noreturn]] void fail(const std::string& what) {
    size_t line = 1;
    for (size_t k = 0; k < i_ && k < s_.size(); ++k) line += s_[k] == '\n';
    throw json_parser_error("<json>(" + std::to_string(line) + "): " + what);
  }
  void ws() {
    while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_;
  }
  char peek() { return i_ < s_.size() ? s_[i_] : '\0'; }
  void expect(char c) {
    ws();
    if (peek() != c) fail(std::string("expected '") + c + "'");
    ++i_;
  }
  std::string str() {
    expect('"');
    std::string out;
    while (i_ < s_.size() && s_[i_] != '"') {
      char c = s_[i_++];
      if (c == '\\' && i_ < s_.size()) {
        char e = s_[i_++];
        switch (e) {
          case 'n': out += '\n'; break;
          case 't': out += '\t'; break;
          case 'r': out += '\r'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'u': out += '?'; i_ += 4; break;
          default: out += e;
        }
      } else {
        out += c;
      }
    }
    if (peek() != '"') fail("unterminated string");
    ++i_;
    return out;
  }
  void value(ptree& node) {
    ws();
    char c = peek();
    if (c == '{') {
      ++i_;
      ws();
      if (peek() == '}') { ++i_; return; }
      for (;;) {
        std::string key = str();
        expect(':');
        ptree child;
        value(child);
        node.kids_.emplace_back(key, std::move(child));
        ws();
        if (peek() == ',') { ++i_; continue; }
        if (peek() == '}') { ++i_; return; }
        fail("expected ',' or '}'");
      }
    } else if (c == '[') {
      ++i_;
      ws();
      if (peek() == ']') { ++i_; return; }
      for (;;) {
        ptree child;
        value(child);
        node.kids_.emplace_back("", std::move(child));
        ws();
        if (peek() == ',') { ++i_; continue; }
        if (peek() == ']') { ++i_; return; }
        fail("expected ',' or ']'");
      }
    } else if (c == '"') {
      node.data_ = str();
    } else {
      size_t b = i_;
      while (i_ < s_.size() && !std::isspace((unsigned char)s_[i_]) && s_[i_] != ',' && s_[i_] != '}' &&
             s_[i_] != ']')
        ++i_;
      if (b == i_) fail("unexpected character");
      node.data_ = s_.substr(b, i_ - b);
    }
  }
  const std::string& s_;
  size_t i_ = 0;
};

inline void read_json(std::istream& is, ptree& pt) {
  std::string text((std::istreambuf_iterator<char>(is)), std::istreambuf_iterator<char>());
  ptree tmp;
  json_reader(text).parse(tmp);
  pt = std::move(tmp);
}

inline ptree read_json_string(const std::string& text) {
  ptree pt;
  json_reader(remove_json_comments(text)).parse(pt);
  return pt;
}

inline ptree read_json_file(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw ptree_error("Could not open file " + path);
  std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  return read_json_string(text);
}

}  // namespace deco
