// netCDF (classic data model, 64-bit-offset format) writer of the output file
// (awfl_netcdf.cu). Host code only.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace awfl {
namespace nc {

struct Layout {
  std::vector<unsigned char> header;  // with numrecs = 0
  uint64_t fixed_begin[6];
  uint64_t rec_begin;
  uint64_t rec_size;
  uint64_t cells;
  int nrec;  // record fields after t: the six diagnostics + one per tracer
};
Layout layout(int nx, int ny, int nz, const std::vector<std::string> &tracers = {});

// fields: [6 + ntracers][nz][ny][nx] (dens_pert, u, v, w, pot_temp_pert, pressure_pert,
// then tracer_<name> for each name in tracers); hy_*: the halo-inclusive cell profiles
// (nz + 2hs). Returns 0, or -1 with *err set.
int write(const char *path, int nx, int ny, int nz, double dx, double dy, double dz, int hs,
          const double *hy_dens, const double *hy_pres, const double *hy_theta, const double *fields, double etime,
          std::string *err, const std::vector<std::string> &tracers = {});

}  // namespace nc
}  // namespace awfl
