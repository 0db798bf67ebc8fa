// Project-written no-op stand-in for YAKL's SimpleNetCDF writer, which the reference
// uses only for output (Spatial_euler3d_cons_expl_cart_fv_Agrid.h:1714-1790).
// netCDF output is not part of the timed hot path; the oracle build discards it.
// Test infrastructure only.
#pragma once

#include <string>
#include <vector>

namespace yakl {
  int constexpr NETCDF_MODE_WRITE = 1;
  int constexpr NETCDF_MODE_READ  = 0;

  class SimpleNetCDF {
  public:
    void create(std::string const &) {}
    void open(std::string const &, int = 0) {}
    void close() {}
    int getDimSize(std::string const &) { return 0; }
    template <class T> void write(T const &, std::string const &, std::vector<std::string> const &) {}
    template <class T> void write1(T const &, std::string const &, int, std::string const &) {}
    template <class T> void write1(T const &, std::string const &, std::vector<std::string> const &, int, std::string const &) {}
  };
}
