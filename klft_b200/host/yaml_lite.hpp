// yaml_lite.hpp -- a block-style YAML subset reader for klft input files.
//
// klft parses its input with yaml-cpp (InputParser.hpp:33-125); yaml-cpp is not
// available here, so this reader covers the subset klft's inputs use: nested
// block mappings by indentation, block sequences ("- item"), flow sequences
// ("[a, b]"), scalars (plain, single- or double-quoted), comments and blank
// lines.  Lookups mirror yaml-cpp: node["key"] (missing keys give an empty
// node), node.as<T>(default), iteration over sequence items.
#pragma once

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace klft {
namespace yaml {

struct Node {
  enum Kind { Null, Scalar, Seq, Map } kind = Null;
  std::string value;
  std::vector<Node> items;
  std::vector<std::pair<std::string, Node>> entries;

  explicit operator bool() const { return kind != Null; }
  const Node &operator[](const std::string &key) const {
    static const Node none;
    for (const auto &e : entries)
      if (e.first == key) return e.second;
    return none;
  }
  const Node &operator[](size_t i) const {
    static const Node none;
    return i < items.size() ? items[i] : none;
  }
  size_t size() const { return kind == Seq ? items.size() : entries.size(); }
  std::vector<Node>::const_iterator begin() const { return items.begin(); }
  std::vector<Node>::const_iterator end() const { return items.end(); }

  template <class T> T as(const T &fallback) const;
  template <class T> T as() const {
    if (kind != Scalar) throw std::runtime_error("yaml: not a scalar");
    return as<T>(T());
  }
};

inline std::string trim(const std::string &s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

inline std::string strip_comment(const std::string &s) {
  char q = 0;
  for (size_t i = 0; i < s.size(); ++i) {
    const char c = s[i];
    if (q) {
      if (c == q) q = 0;
    } else if (c == '"' || c == '\'') {
      q = c;
    } else if (c == '#' && (i == 0 || std::isspace((unsigned char)s[i - 1]))) {
      return s.substr(0, i);
    }
  }
  return s;
}

inline std::string unquote(const std::string &s) {
  if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') || (s.front() == '\'' && s.back() == '\'')))
    return s.substr(1, s.size() - 2);
  return s;
}

inline Node scalar_or_flow(const std::string &text) {
  Node n;
  const std::string t = trim(text);
  if (t.empty()) return n;
  if (t.front() == '[') {
    if (t.back() != ']') throw std::runtime_error("yaml: unterminated flow sequence: " + t);
    n.kind = Node::Seq;
    std::string inner = t.substr(1, t.size() - 2);
    int depth = 0;
    std::string cur;
    for (char c : inner) {
      if (c == '[') ++depth;
      if (c == ']') --depth;
      if (c == ',' && depth == 0) {
        n.items.push_back(scalar_or_flow(cur));
        cur.clear();
      } else {
        cur += c;
      }
    }
    if (!trim(cur).empty()) n.items.push_back(scalar_or_flow(cur));
    return n;
  }
  n.kind = Node::Scalar;
  n.value = unquote(t);
  return n;
}

struct Line {
  int indent;
  std::string text;
};

// Parses lines[i..] at indentation > parent_indent into a block node.
inline Node parse_block(const std::vector<Line> &lines, size_t &i, int parent_indent) {
  Node node;
  if (i >= lines.size() || lines[i].indent <= parent_indent) return node;
  const int ind = lines[i].indent;
  const bool is_seq = lines[i].text.rfind("- ", 0) == 0 || lines[i].text == "-";
  node.kind = is_seq ? Node::Seq : Node::Map;
  while (i < lines.size() && lines[i].indent == ind) {
    const std::string &t = lines[i].text;
    if (is_seq) {
      if (!(t.rfind("- ", 0) == 0 || t == "-")) throw std::runtime_error("yaml: mixed sequence/mapping: " + t);
      const std::string rest = t.size() > 1 ? trim(t.substr(2)) : std::string();
      ++i;
      if (rest.empty()) node.items.push_back(parse_block(lines, i, ind));
      else node.items.push_back(scalar_or_flow(rest));
    } else {
      const size_t colon = [&] {
        char q = 0;
        for (size_t k = 0; k < t.size(); ++k) {
          if (q) { if (t[k] == q) q = 0; continue; }
          if (t[k] == '"' || t[k] == '\'') { q = t[k]; continue; }
          if (t[k] == ':' && (k + 1 == t.size() || t[k + 1] == ' ')) return k;
        }
        return std::string::npos;
      }();
      if (colon == std::string::npos) throw std::runtime_error("yaml: expected 'key: value': " + t);
      const std::string key = unquote(trim(t.substr(0, colon)));
      const std::string rest = trim(t.substr(colon + 1));
      ++i;
      if (rest.empty()) node.entries.emplace_back(key, parse_block(lines, i, ind));
      else node.entries.emplace_back(key, scalar_or_flow(rest));
    }
  }
  if (i < lines.size() && lines[i].indent > ind) throw std::runtime_error("yaml: bad indentation: " + lines[i].text);
  return node;
}

inline Node Load(const std::string &text) {
  std::vector<Line> lines;
  std::istringstream in(text);
  std::string raw;
  while (std::getline(in, raw)) {
    if (!raw.empty() && raw.back() == '\r') raw.pop_back();
    const std::string s = strip_comment(raw);
    if (trim(s).empty() || trim(s) == "---") continue;
    int indent = 0;
    while (indent < (int)s.size() && s[indent] == ' ') ++indent;
    if (indent < (int)s.size() && s[indent] == '\t') throw std::runtime_error("yaml: tabs are not allowed");
    lines.push_back({indent, trim(s)});
  }
  size_t i = 0;
  Node root = parse_block(lines, i, -1);
  if (i != lines.size()) throw std::runtime_error("yaml: trailing content");
  return root;
}

inline Node LoadFile(const std::string &path) {
  std::ifstream f(path);
  if (!f.is_open()) throw std::runtime_error("bad file: " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return Load(ss.str());
}

template <> inline std::string Node::as<std::string>(const std::string &fb) const {
  return kind == Scalar ? value : fb;
}
template <> inline bool Node::as<bool>(const bool &fb) const {
  if (kind != Scalar) return fb;
  std::string v;
  for (char c : value) v += (char)std::tolower((unsigned char)c);
  if (v == "true" || v == "yes" || v == "on" || v == "y") return true;
  if (v == "false" || v == "no" || v == "off" || v == "n") return false;
  throw std::runtime_error("yaml: not a boolean: " + value);
}
template <> inline int Node::as<int>(const int &fb) const {
  if (kind != Scalar) return fb;
  char *e = nullptr;
  const long v = std::strtol(value.c_str(), &e, 0);
  if (!e || *e) throw std::runtime_error("yaml: not an integer: " + value);
  return (int)v;
}
template <> inline size_t Node::as<size_t>(const size_t &fb) const {
  if (kind != Scalar) return fb;
  char *e = nullptr;
  const unsigned long long v = std::strtoull(value.c_str(), &e, 0);
  if (!e || *e || value[0] == '-') throw std::runtime_error("yaml: not an unsigned integer: " + value);
  return (size_t)v;
}
template <> inline double Node::as<double>(const double &fb) const {
  if (kind != Scalar) return fb;
  char *e = nullptr;
  const double v = std::strtod(value.c_str(), &e);
  if (!e || *e) throw std::runtime_error("yaml: not a number: " + value);
  return v;
}

}  // namespace yaml
}  // namespace klft
