// Flat "key : value" YAML reader for the drop-in operators: the subset of yaml-cpp the
// reference's driver.cpp (lines 17-22) and Spatial::init (Spatial_euler3d_cons_expl_cart_
// fv_Agrid.h:197-272) use -- LoadFile, operator[], operator!, as<T>() for int, double,
// bool and std::string. As in yaml-cpp, as<T>() on a missing key throws.
#pragma once

#include <cctype>
#include <fstream>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>

namespace YAML {

class Node {
  std::shared_ptr<std::map<std::string, std::string>> kv_;
  std::string val_;
  bool defined_ = false;

 public:
  Node() {}
  explicit Node(std::shared_ptr<std::map<std::string, std::string>> m) : kv_(m), defined_(true) {}
  Node(std::string v, bool d) : val_(std::move(v)), defined_(d) {}

  bool operator!() const { return !defined_; }
  explicit operator bool() const { return defined_; }

  Node operator[](const std::string &key) const {
    if (!kv_) return Node("", false);
    auto it = kv_->find(key);
    return it == kv_->end() ? Node("", false) : Node(it->second, true);
  }

  template <class T> T as() const;
};

namespace detail {
inline std::string trim(const std::string &s) {
  const size_t b = s.find_first_not_of(" \t\r\n");
  if (b == std::string::npos) return "";
  const size_t e = s.find_last_not_of(" \t\r\n");
  return s.substr(b, e - b + 1);
}
inline void need(bool defined) {
  if (!defined) throw std::runtime_error("yaml: bad conversion (missing key)");
}
}  // namespace detail

template <> inline std::string Node::as<std::string>() const { detail::need(defined_); return val_; }
template <> inline double Node::as<double>() const { detail::need(defined_); return std::stod(val_); }
template <> inline float Node::as<float>() const { detail::need(defined_); return std::stof(val_); }
template <> inline int Node::as<int>() const { detail::need(defined_); return std::stoi(val_); }
template <> inline bool Node::as<bool>() const {
  detail::need(defined_);
  std::string v = val_;
  for (auto &c : v) c = (char)std::tolower((unsigned char)c);
  if (v == "true" || v == "yes" || v == "on" || v == "y") return true;
  if (v == "false" || v == "no" || v == "off" || v == "n") return false;
  throw std::runtime_error("yaml: bad bool conversion");
}

inline Node LoadFile(const std::string &fname) {
  std::ifstream f(fname);
  if (!f) throw std::runtime_error("yaml: cannot open " + fname);
  auto m = std::make_shared<std::map<std::string, std::string>>();
  std::string line;
  while (std::getline(f, line)) {
    const size_t h = line.find('#');
    if (h != std::string::npos) line = line.substr(0, h);
    line = detail::trim(line);
    if (line.empty() || line == "---") continue;
    const size_t c = line.find(':');
    if (c == std::string::npos) continue;
    (*m)[detail::trim(line.substr(0, c))] = detail::trim(line.substr(c + 1));
  }
  return Node(m);
}

}  // namespace YAML
