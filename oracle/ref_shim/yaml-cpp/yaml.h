/*
 * Minimal stand-in for the part of yaml-cpp's interface that the reference's
 * config.hpp touches (Node, operator[], as<T>, IsMap, map iteration, Load,
 * LoadFile, stream output, Emitter, NodeType::Map).  It parses block
 * mappings of scalars, which is all the reference's configuration files and
 * config_defaults.hpp contain.  It lets the reference's host integrator be
 * compiled as the CPU checker in oracle/_ref/.  TEST INFRASTRUCTURE ONLY.
 */
#ifndef MISO_REF_SHIM_YAML_H
#define MISO_REF_SHIM_YAML_H

#include <cstdlib>
#include <fstream>
#include <memory>
#include <ostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace YAML {

struct NodeType {
  enum value { Undefined, Null, Scalar, Sequence, Map };
};

struct NodeData {
  NodeType::value type = NodeType::Null;
  std::string scalar;
  std::vector<std::pair<std::string, std::shared_ptr<NodeData>>> map;
};

class Node {
public:
  Node() : p_(std::make_shared<NodeData>()) {}
  explicit Node(NodeType::value t) : p_(std::make_shared<NodeData>()) { p_->type = t; }
  Node(const Node &) = default;
  explicit Node(std::shared_ptr<NodeData> p) : p_(std::move(p)) {}

  Node &operator=(const Node &rhs) {
    if (p_ == rhs.p_) return *this;
    NodeData copy = *rhs.p_;
    *p_ = std::move(copy);
    return *this;
  }
  Node &operator=(const std::string &s) {
    p_->type = NodeType::Scalar;
    p_->scalar = s;
    p_->map.clear();
    return *this;
  }
  Node &operator=(const char *s) { return *this = std::string(s); }

  explicit operator bool() const { return p_->type != NodeType::Undefined; }
  bool operator!() const { return p_->type == NodeType::Undefined; }
  bool IsMap() const { return p_->type == NodeType::Map; }
  bool IsScalar() const { return p_->type == NodeType::Scalar; }
  bool IsNull() const { return p_->type == NodeType::Null; }

  Node operator[](const std::string &key) {
    if (p_->type != NodeType::Map) {
      p_->type = NodeType::Map;
      p_->scalar.clear();
    }
    for (auto &kv : p_->map)
      if (kv.first == key) return Node(kv.second);
    auto child = std::make_shared<NodeData>();
    child->type = NodeType::Undefined;
    p_->map.emplace_back(key, child);
    return Node(child);
  }
  const Node operator[](const std::string &key) const {
    if (p_->type == NodeType::Map)
      for (auto &kv : p_->map)
        if (kv.first == key) return Node(kv.second);
    return Node(NodeType::Undefined);
  }

  template <typename T> T as() const {
    if (p_->type != NodeType::Scalar)
      throw std::runtime_error("yaml stand-in: node is not a scalar");
    const std::string &s = p_->scalar;
    if constexpr (std::is_same_v<T, std::string>) {
      return s;
    } else if constexpr (std::is_same_v<T, bool>) {
      if (s == "true" || s == "True" || s == "TRUE" || s == "yes") return true;
      if (s == "false" || s == "False" || s == "FALSE" || s == "no") return false;
      throw std::runtime_error("yaml stand-in: bad bool " + s);
    } else if constexpr (std::is_integral_v<T>) {
      return static_cast<T>(std::strtol(s.c_str(), nullptr, 10));
    } else {
      return static_cast<T>(std::strtod(s.c_str(), nullptr));
    }
  }

  class const_iterator;
  const_iterator begin() const;
  const_iterator end() const;

  const std::shared_ptr<NodeData> &data() const { return p_; }

private:
  std::shared_ptr<NodeData> p_;
};

struct NodeEntry {
  Node first, second;
};

class Node::const_iterator {
public:
  const_iterator(const NodeData *d, size_t i) : d_(d), i_(i) { skip(); }
  NodeEntry operator*() const {
    Node k;
    k = d_->map[i_].first;
    return NodeEntry{k, Node(d_->map[i_].second)};
  }
  const_iterator &operator++() {
    ++i_;
    skip();
    return *this;
  }
  bool operator!=(const const_iterator &o) const { return i_ != o.i_ || d_ != o.d_; }

private:
  void skip() {
    while (d_ && i_ < d_->map.size() && d_->map[i_].second->type == NodeType::Undefined) ++i_;
  }
  const NodeData *d_;
  size_t i_;
};

inline Node::const_iterator Node::begin() const {
  return const_iterator(p_->type == NodeType::Map ? p_.get() : nullptr, 0);
}
inline Node::const_iterator Node::end() const {
  const NodeData *d = p_->type == NodeType::Map ? p_.get() : nullptr;
  return const_iterator(d, d ? d->map.size() : 0);
}

namespace detail {
inline std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r");
  return s.substr(a, b - a + 1);
}
inline std::string strip_comment(const std::string &s) {
  bool sq = false, dq = false;
  for (size_t i = 0; i < s.size(); ++i) {
    char c = s[i];
    if (c == '\'' && !dq) sq = !sq;
    else if (c == '"' && !sq) dq = !dq;
    else if (c == '#' && !sq && !dq && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t'))
      return s.substr(0, i);
  }
  return s;
}
inline std::string unquote(const std::string &v) {
  if (v.size() >= 2 && ((v.front() == '"' && v.back() == '"') ||
                        (v.front() == '\'' && v.back() == '\'')))
    return v.substr(1, v.size() - 2);
  return v;
}
inline void emit(std::ostream &os, const NodeData &d, int indent) {
  for (auto &kv : d.map) {
    const NodeData &c = *kv.second;
    if (c.type == NodeType::Undefined) continue;
    os << std::string(indent, ' ') << kv.first << ":";
    if (c.type == NodeType::Map) {
      os << "\n";
      emit(os, c, indent + 2);
    } else if (c.type == NodeType::Scalar) {
      os << " " << c.scalar << "\n";
    } else {
      os << " ~\n";
    }
  }
}
} // namespace detail

inline Node Load(const std::string &text) {
  Node root(NodeType::Map);
  std::vector<std::pair<int, std::shared_ptr<NodeData>>> stack;
  stack.emplace_back(-1, root.data());
  std::istringstream in(text);
  std::string raw;
  while (std::getline(in, raw)) {
    std::string line = detail::strip_comment(raw);
    if (detail::trim(line).empty()) continue;
    int indent = (int)line.find_first_not_of(' ');
    std::string body = detail::trim(line);
    size_t colon = body.find(':');
    if (colon == std::string::npos) throw std::runtime_error("yaml stand-in: expected key: " + body);
    std::string key = detail::unquote(detail::trim(body.substr(0, colon)));
    std::string val = detail::trim(body.substr(colon + 1));
    while (stack.size() > 1 && stack.back().first >= indent) stack.pop_back();
    auto parent = stack.back().second;
    if (parent->type != NodeType::Map) {
      parent->type = NodeType::Map;
      parent->scalar.clear();
    }
    auto child = std::make_shared<NodeData>();
    if (val.empty()) {
      child->type = NodeType::Null;
    } else {
      child->type = NodeType::Scalar;
      child->scalar = detail::unquote(val);
    }
    bool replaced = false;
    for (auto &kv : parent->map)
      if (kv.first == key) {
        kv.second = child;
        replaced = true;
      }
    if (!replaced) parent->map.emplace_back(key, child);
    stack.emplace_back(indent, child);
  }
  return root;
}

inline Node LoadFile(const std::string &path) {
  std::ifstream f(path);
  if (!f) throw std::runtime_error("yaml stand-in: cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return Load(ss.str());
}

inline std::ostream &operator<<(std::ostream &os, const Node &n) {
  detail::emit(os, *n.data(), 0);
  return os;
}

class Emitter {
public:
  Emitter &operator<<(const Node &n) {
    std::ostringstream os;
    os << n;
    s_ += os.str();
    return *this;
  }
  const char *c_str() const { return s_.c_str(); }

private:
  std::string s_;
};

} // namespace YAML

#endif
