// Output file of Spatial::output (Spatial:1705-1791) without the netCDF library: a
// project-written writer of the netCDF classic data model, 64-bit-offset format ("CDF"
// version 2: big-endian header of dimensions, attributes and variables with their file
// offsets, then the fixed-size variables, then one record per output time holding every
// record variable's slice), as the published netCDF classic format specification defines.
//
// The file holds what the reference's SimpleNetCDF calls write (Spatial:1715-1778):
// dimensions x, y, z and the unlimited t; fixed variables x(x), y(y), z(z), hyDens(z),
// hyPressure(z), hyTheta(z); record variables t(t) and dens_pert, u, v, w, pot_temp_pert,
// pressure_pert and one tracer_<name> per tracer (t, z, y, x), all double. etime == 0 creates the file with record 0;
// any other etime appends a record (the reference reads the current length of t).
// Host code only.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "awfl_netcdf.h"

namespace awfl {
namespace nc {
namespace {

constexpr uint32_t kDimTag = 0x0A, kVarTag = 0x0B, kDouble = 6;
const char *const kFixed[6] = {"x", "y", "z", "hyDens", "hyPressure", "hyTheta"};
const char *const kRecord[7] = {"t", "dens_pert", "u", "v", "w", "pot_temp_pert", "pressure_pert"};

void put32(std::vector<unsigned char> &b, uint32_t v) {
  for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
}
void put64(std::vector<unsigned char> &b, uint64_t v) {
  for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
}
void put_name(std::vector<unsigned char> &b, const char *name) {
  const size_t n = std::strlen(name);
  put32(b, (uint32_t)n);
  b.insert(b.end(), name, name + n);
  while (b.size() % 4) b.push_back(0);
}
void set64(std::vector<unsigned char> &b, size_t at, uint64_t v) {
  for (int i = 0; i < 8; i++) b[at + i] = (unsigned char)(v >> (56 - 8 * i));
}
// big-endian doubles
void put_doubles(std::vector<unsigned char> &b, const double *x, size_t n) {
  for (size_t i = 0; i < n; i++) {
    uint64_t u;
    std::memcpy(&u, &x[i], 8);
    put64(b, u);
  }
}

}  // namespace

Layout layout(int nx, int ny, int nz, const std::vector<std::string> &tracers) {
  const int nrec = 6 + (int)tracers.size();  // record fields after t
  Layout L;
  std::vector<unsigned char> &h = L.header;
  const char magic[4] = {'C', 'D', 'F', 2};
  h.insert(h.end(), magic, magic + 4);
  put32(h, 0);  // numrecs, set when records are written
  // dimensions: x, y, z, t (unlimited: length 0)
  put32(h, kDimTag);
  put32(h, 4);
  const char *dn[4] = {"x", "y", "z", "t"};
  const uint32_t dl[4] = {(uint32_t)nx, (uint32_t)ny, (uint32_t)nz, 0};
  for (int d = 0; d < 4; d++) {
    put_name(h, dn[d]);
    put32(h, dl[d]);
  }
  put64(h, 0);  // no global attributes (ABSENT: two zero words)
  put32(h, kVarTag);
  put32(h, (uint32_t)(7 + nrec));
  std::vector<size_t> begin_at;
  auto var = [&](const char *name, std::initializer_list<uint32_t> dims, uint64_t vsize) {
    put_name(h, name);
    put32(h, (uint32_t)dims.size());
    for (uint32_t d : dims) put32(h, d);
    put64(h, 0);  // no variable attributes
    put32(h, kDouble);
    put32(h, (uint32_t)vsize);
    begin_at.push_back(h.size());
    put64(h, 0);  // begin, set below
  };
  const uint64_t cells = (uint64_t)nx * ny * nz;
  var(kFixed[0], {0}, 8ull * nx);
  var(kFixed[1], {1}, 8ull * ny);
  for (int f = 2; f < 6; f++) var(kFixed[f], {2}, 8ull * nz);
  var(kRecord[0], {3}, 8);
  for (int f = 1; f < 7; f++) var(kRecord[f], {3, 2, 1, 0}, 8 * cells);
  for (const std::string &t : tracers) var(("tracer_" + t).c_str(), {3, 2, 1, 0}, 8 * cells);
  // file offsets: fixed variables back to back after the header, then the records
  uint64_t off = h.size();
  const uint64_t fixed_len[6] = {8ull * nx, 8ull * ny, 8ull * nz, 8ull * nz, 8ull * nz, 8ull * nz};
  for (int f = 0; f < 6; f++) {
    set64(h, begin_at[f], off);
    L.fixed_begin[f] = off;
    off += fixed_len[f];
  }
  L.rec_begin = off;
  set64(h, begin_at[6], off);
  off += 8;
  for (int f = 1; f <= nrec; f++) {
    set64(h, begin_at[6 + f], off);
    off += 8 * cells;
  }
  L.rec_size = 8 + (uint64_t)nrec * 8 * cells;
  L.nrec = nrec;
  L.cells = cells;
  return L;
}

int write(const char *path, int nx, int ny, int nz, double dx, double dy, double dz, int hs,
          const double *hy_dens, const double *hy_pres, const double *hy_theta, const double *fields, double etime,
          std::string *err, const std::vector<std::string> &tracers) {
  const Layout L = layout(nx, ny, nz, tracers);
  FILE *f = nullptr;
  uint32_t rec = 0;
  if (etime == 0.) {
    f = std::fopen(path, "wb");
    if (!f) { *err = std::string("cannot create ") + path; return -1; }
    std::vector<unsigned char> b(L.header);
    const int n[3] = {nx, ny, nz};
    const double d[3] = {dx, dy, dz};
    for (int a = 0; a < 3; a++)
      for (int i = 0; i < n[a]; i++) {
        const double v = (i + 0.5) * d[a];  // Spatial:1718-1728
        put_doubles(b, &v, 1);
      }
    put_doubles(b, hy_dens + hs, nz);
    put_doubles(b, hy_pres + hs, nz);
    put_doubles(b, hy_theta + hs, nz);
    if (b.size() != L.rec_begin || std::fwrite(b.data(), 1, b.size(), f) != b.size()) {
      std::fclose(f);
      *err = std::string("write error on ") + path;
      return -1;
    }
  } else {
    f = std::fopen(path, "r+b");
    if (!f) { *err = std::string("cannot open ") + path + " (etime != 0 appends to an existing file)"; return -1; }
    std::vector<unsigned char> h(L.header.size());
    if (std::fread(h.data(), 1, h.size(), f) != h.size() ||
        std::memcmp(h.data(), L.header.data(), 4) != 0 ||
        std::memcmp(h.data() + 8, L.header.data() + 8, h.size() - 8) != 0) {
      std::fclose(f);
      *err = std::string(path) + " is not an output file of this grid";
      return -1;
    }
    rec = ((uint32_t)h[4] << 24) | ((uint32_t)h[5] << 16) | ((uint32_t)h[6] << 8) | h[7];
  }
  // record rec: t, then the six fields
  std::vector<unsigned char> b;
  b.reserve((size_t)L.rec_size);
  put_doubles(b, &etime, 1);
  put_doubles(b, fields, (size_t)L.nrec * L.cells);
  const uint64_t at = L.rec_begin + (uint64_t)rec * L.rec_size;
  bool ok = std::fseek(f, (long)at, SEEK_SET) == 0 && std::fwrite(b.data(), 1, b.size(), f) == b.size();
  std::vector<unsigned char> nr;
  put32(nr, rec + 1);
  ok = ok && std::fseek(f, 4, SEEK_SET) == 0 && std::fwrite(nr.data(), 1, 4, f) == 4;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) { *err = std::string("write error on ") + path; return -1; }
  return 0;
}

}  // namespace nc
}  // namespace awfl
