// Project-written stand-in for YAKL's SimpleNetCDF writer, which the reference uses only
// for output (Spatial_euler3d_cons_expl_cart_fv_Agrid.h:1714-1790). It writes no file:
// it records every array and scalar the reference hands it, by variable name (the last
// write of a name wins), so that the test harness (ref_harness.cpp) can read back the
// fields the reference's own output() computed. No arithmetic. Test infrastructure only.
#pragma once

#include <map>
#include <string>
#include <type_traits>
#include <vector>

namespace yakl {
  int constexpr NETCDF_MODE_WRITE = 1;
  int constexpr NETCDF_MODE_READ  = 0;

  inline std::map<std::string, std::vector<double>> &netcdf_record() {
    static std::map<std::string, std::vector<double>> rec;
    return rec;
  }

  class SimpleNetCDF {
    template <class T> static void put(T const &a, std::string const &name) {
      std::vector<double> v;
      if constexpr (std::is_arithmetic<T>::value) {
        v.push_back((double)a);
      } else {
        v.resize(a.totElems());
        for (size_t i = 0; i < v.size(); i++) v[i] = (double)a.data()[i];
      }
      netcdf_record()[name] = v;
    }
  public:
    void create(std::string const &) {}
    void open(std::string const &, int = 0) {}
    void close() {}
    int getDimSize(std::string const &) { return 0; }
    template <class T> void write(T const &a, std::string const &name, std::vector<std::string> const &) { put(a, name); }
    template <class T> void write1(T const &a, std::string const &name, int, std::string const &) { put(a, name); }
    template <class T> void write1(T const &a, std::string const &name, std::vector<std::string> const &, int,
                                   std::string const &) { put(a, name); }
  };
}
