// Project-written stand-in for the subset of yaml-cpp that the reference calls
// (driver.cpp:17-22, Spatial_euler3d_cons_expl_cart_fv_Agrid.h:197-272): a flat
// "key : value" document, LoadFile, operator[], operator!, as<T>() for int, double,
// bool and std::string. Test infrastructure only (the oracle build).
//
// Like yaml-cpp, as<T>() on a missing key throws (the reference reads "perturb"
// without checking that it exists).
#pragma once

#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <memory>

namespace YAML {

  class Node {
    std::shared_ptr<std::map<std::string, std::string>> kv;
    std::string val;
    bool defined = false;
  public:
    Node() {}
    explicit Node(std::shared_ptr<std::map<std::string, std::string>> m) : kv(m), defined(true) {}
    Node(std::string v, bool d) : val(v), defined(d) {}

    bool operator!() const { return !defined; }
    explicit operator bool() const { return defined; }

    Node operator[](std::string const &key) const {
      if (!kv) return Node("", false);
      auto it = kv->find(key);
      if (it == kv->end()) return Node("", false);
      return Node(it->second, true);
    }

    template <class T> T as() const;
  };

  namespace detail {
    inline std::string trim(std::string const &s) {
      size_t b = s.find_first_not_of(" \t\r\n");
      if (b == std::string::npos) return "";
      size_t e = s.find_last_not_of(" \t\r\n");
      return s.substr(b, e - b + 1);
    }
  }

  template <> inline std::string Node::as<std::string>() const {
    if (!defined) throw std::runtime_error("yaml: bad conversion (missing key)");
    return val;
  }
  template <> inline double Node::as<double>() const {
    if (!defined) throw std::runtime_error("yaml: bad conversion (missing key)");
    size_t pos = 0;
    double d = std::stod(val, &pos);
    return d;
  }
  template <> inline int Node::as<int>() const {
    if (!defined) throw std::runtime_error("yaml: bad conversion (missing key)");
    return std::stoi(val);
  }
  template <> inline bool Node::as<bool>() const {
    if (!defined) throw std::runtime_error("yaml: bad conversion (missing key)");
    std::string v = val;
    for (auto &c : v) c = (char)std::tolower((unsigned char)c);
    if (v == "true" || v == "yes" || v == "on" || v == "y") return true;
    if (v == "false" || v == "no" || v == "off" || v == "n") return false;
    throw std::runtime_error("yaml: bad bool conversion");
  }

  inline Node LoadFile(std::string const &fname) {
    std::ifstream f(fname);
    if (!f) throw std::runtime_error("yaml: cannot open " + fname);
    auto m = std::make_shared<std::map<std::string, std::string>>();
    std::string line;
    while (std::getline(f, line)) {
      size_t h = line.find('#');
      if (h != std::string::npos) line = line.substr(0, h);
      line = detail::trim(line);
      if (line.empty() || line == "---") continue;
      size_t c = line.find(':');
      if (c == std::string::npos) continue;
      (*m)[detail::trim(line.substr(0, c))] = detail::trim(line.substr(c + 1));
    }
    return Node(m);
  }
}
