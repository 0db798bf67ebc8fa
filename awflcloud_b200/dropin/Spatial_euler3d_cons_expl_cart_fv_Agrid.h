// Drop-in spatial operator: the interface of the reference's
// Spatial_euler3d_cons_expl_cart_fv_Agrid.h (mrnorman/awflCloud; "Spatial" below) with the
// work done on the GPU by libawfl.so through its C ABI (include/awfl.h).
//
// Same class template, typedefs, constants, members and methods that driver.cpp and
// Temporal_ader.h use (Spatial:14-155, 159-187, 192-340, 345-560, 565-594, 1705-1797),
// plus the README's get()/applyTendencies() extras (README.md:59-112) as thin host-side
// wrappers. The state lives in device memory owned by the array objects; every operator
// call is a C-ABI call on the legacy default stream.
//
// Differences from the reference, each deliberate:
//  * output(): an outFile ending in ".nc" gets the reference's netCDF file (Spatial:1705-1791)
//    from awfl_write_netcdf, the library's own writer of the netCDF classic data model
//    (64-bit offset format; no netCDF library). An outFile ending in ".bin" gets the state
//    (5 variables, halos included, FP64) raw at every output time, overwriting the previous
//    one; any other name: output() does nothing.
//  * Tracers: the reference compiles their transport out (NO_TRACERS, Spatial:10) but still
//    runs initTracers (Spatial:505-560) and writes tracer_<name> fields in output
//    (Spatial:1778-1783); both are here on the device (awfl_init_tracers,
//    awfl_write_netcdf_tracers; tracers are FP64 for either precision, halos zero). Their
//    tendencies are zero, so they stay constant (the reference adds an uninitialised
//    tendency array to them, Temporal_ader.h:67-69) -- unless the extra YAML key
//    tracer_transport is true (either precision): the reference's compiled-out tracer code
//    then runs (awfl_split_tracers per split; addTracer's posDef flags select the limited
//    tracers).
//  * Optional extra YAML keys (absent = reference behaviour): tracer_transport (bool),
//    precision (fp64 | fp32),
//    device, bubble (cosine | linear) with bubble_x0/y0/z0, bubble_radius (or
//    bubble_xrad/yrad/zrad), bubble_amp, bubble_pwr; noise_amp, noise_seed, noise_dist
//    (uniform | normal; noise_amp is then the standard deviation).
#pragma once

#include <cstring>
#include <fstream>
#include <initializer_list>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "const.h"

namespace awfl_dropin {

inline void check(int rc, const awfl_ctx *c, const std::string &what) {
  if (rc != AWFL_OK) endrun(what + ": " + awfl_last_error(c));
}

// Device array allocated through the C ABI. Copies share the allocation, like the
// reference's YAKL arrays. C-order, last dimension fastest.
class DeviceArray {
 public:
  DeviceArray() {}
  DeviceArray(const char *label, size_t elem_bytes, std::initializer_list<long> dims)
      : dims_(dims), esz_(elem_bytes), label_(label) {
    void *p = nullptr;
    const long bytes = (long)(totElems() * esz_);
    check(awfl_device_alloc(&p, bytes), nullptr, std::string("allocation of ") + label);
    check(awfl_memset_device(p, 0, bytes, nullptr), nullptr, std::string("zero fill of ") + label);
    ptr_ = std::shared_ptr<void>(p, [](void *q) { awfl_device_free(q); });
  }
  void *data() const { return ptr_.get(); }
  bool initialized() const { return (bool)ptr_; }
  size_t totElems() const {
    size_t n = dims_.empty() ? 0 : 1;
    for (long d : dims_) n *= (size_t)d;
    return n;
  }
  int extent(int i) const { return (int)dims_.at(i); }
  size_t elemBytes() const { return esz_; }
  const std::string &label() const { return label_; }
  // All elements, converted to double.
  std::vector<double> createHostCopy() const {
    std::vector<double> out(totElems());
    if (esz_ == sizeof(double)) {
      check(awfl_copy_d2h(out.data(), data(), (long)(out.size() * esz_), nullptr), nullptr, "copy to host");
    } else {
      std::vector<float> f(totElems());
      check(awfl_copy_d2h(f.data(), data(), (long)(f.size() * esz_), nullptr), nullptr, "copy to host");
      for (size_t i = 0; i < f.size(); i++) out[i] = f[i];
    }
    check(awfl_stream_synchronize(nullptr), nullptr, "synchronize");
    return out;
  }
  // Replace the first n elements from host doubles (converted to the element type).
  void copyFromHost(const double *src, size_t n) {
    if (esz_ == sizeof(double)) {
      check(awfl_copy_h2d(data(), src, (long)(n * esz_), nullptr), nullptr, "copy to device");
    } else {
      std::vector<float> f(src, src + n);
      check(awfl_copy_h2d(data(), f.data(), (long)(n * esz_), nullptr), nullptr, "copy to device");
    }
    check(awfl_stream_synchronize(nullptr), nullptr, "synchronize");
  }

 private:
  std::shared_ptr<void> ptr_;
  std::vector<long> dims_;
  size_t esz_ = sizeof(double);
  std::string label_;
};

}  // namespace awfl_dropin

template <int nTimeDerivs, bool timeAvg, int nAder> class Spatial_euler3d_cons_expl_cart_fv_Agrid {
 public:
  static_assert(nTimeDerivs == 1, "ERROR: This Spatial class isn't setup to use nTimeDerivs > 1");
  static_assert(timeAvg, "the B200 library time-averages the ADER edge states (Temporal_ader)");
  static_assert(nAder == ngll, "the B200 library uses nAder = ngll (Temporal_ader.h:8)");

  Spatial_euler3d_cons_expl_cart_fv_Agrid() { numTracers = 0; }
  ~Spatial_euler3d_cons_expl_cart_fv_Agrid() {
    if (ctx) awfl_destroy(ctx);
  }
  Spatial_euler3d_cons_expl_cart_fv_Agrid(const Spatial_euler3d_cons_expl_cart_fv_Agrid &) = delete;
  Spatial_euler3d_cons_expl_cart_fv_Agrid &operator=(const Spatial_euler3d_cons_expl_cart_fv_Agrid &) = delete;

  int static constexpr hs = (ord - 1) / 2;
  int static constexpr numState = 5;

  struct Location {
    int l;
    int k;
    int j;
    int i;
  };

  typedef awfl_dropin::DeviceArray StateArr;
  typedef awfl_dropin::DeviceArray TracerArr;
  typedef awfl_dropin::DeviceArray StateTendArr;
  typedef awfl_dropin::DeviceArray TracerTendArr;

  int static constexpr idR = 0;
  int static constexpr idU = 1;
  int static constexpr idV = 2;
  int static constexpr idW = 3;
  int static constexpr idT = 4;

  int static constexpr BC_PERIODIC = 0;
  int static constexpr BC_WALL = 1;

  int static constexpr DATA_SPEC_THERMAL = 1;
  int static constexpr DATA_SPEC_COLLISION = 2;
  int static constexpr DATA_SPEC_STRAKA = 3;
  int static constexpr DATA_SPEC_IGW = 4;

  bool sim2d = false;
  bool perturb = false;
  real dx = 0, dy = 0, dz = 0;
  real dtInit = 0;
  bool dimSwitch = true;

  int numTracers;
  std::vector<std::string> tracerName;
  std::vector<std::string> tracerDesc;
  std::vector<bool> tracerPosVect;

  int nx = 0, ny = 0, nz = 0;
  real xlen = 0, ylen = 0, zlen = 0;
  int bc_x = 0, bc_y = 0, bc_z = 0;
  bool weno_scalars = true, weno_winds = true;
  std::string outFile;
  int dataSpec = DATA_SPEC_THERMAL;

  // B200 library context and the optional extensions read from the YAML file
  awfl_ctx *ctx = nullptr;
  int precision = AWFL_FP64;
  bool tracerTransport = false;  // YAML tracer_transport: run the tracer code
  int device = 0;
  awfl_init_spec initSpec{};

  static_assert(ord % 2 == 1, "ERROR: ord must be an odd integer");

  void addTracer(std::string name, bool posDef = true, std::string desc = "") {
    tracerName.push_back(name);
    tracerDesc.push_back(desc);
    tracerPosVect.push_back(posDef);
  }

  // FP32 states carry a second plane, the Kahan compensation of the stage updates.
  StateArr createStateArr() {
    const int planes = precision == AWFL_FP32 ? 2 : 1;
    return StateArr("stateArr", elemBytes(), {planes * numState, nz + 2 * hs, ny + 2 * hs, nx + 2 * hs});
  }
  TracerArr createTracerArr() {
    return TracerArr("tracerArr", sizeof(real), {numTracers, nz + 2 * hs, ny + 2 * hs, nx + 2 * hs});
  }
  StateTendArr createStateTendArr() { return StateTendArr("stateTendArr", elemBytes(), {numState, nz, ny, nx}); }
  TracerTendArr createTracerTendArr() {
    return TracerTendArr("tracerTendArr", sizeof(real), {numTracers, nz, ny, nx});
  }

  int numSplit() { return 3; }

  // Spatial:159-187: the acoustic CFL step, computed once and cached.
  real computeTimeStep(real cfl, StateArr const &state) {
    if (dtInit <= 0) {
      double dt = 0;
      awfl_dropin::check(awfl_cfl(ctx, state.data(), cfl, &dt, nullptr), ctx, "computeTimeStep");
      dtInit = dt;
    }
    return dtInit;
  }

  // Spatial:192-340
  void init(std::string inFile) {
    dtInit = 0;
    dimSwitch = true;
    YAML::Node config = YAML::LoadFile(inFile);
    if (!config) { endrun("ERROR: Invalid YAML input file"); }
    if (!config["nx"]) { endrun("ERROR: No nx in input file"); }
    if (!config["ny"]) { endrun("ERROR: No ny in input file"); }
    if (!config["nz"]) { endrun("ERROR: No nz in input file"); }
    if (!config["xlen"]) { endrun("ERROR: No xlen in input file"); }
    if (!config["ylen"]) { endrun("ERROR: No ylen in input file"); }
    if (!config["zlen"]) { endrun("ERROR: No zlen in input file"); }
    if (!config["bc_x"]) { endrun("ERROR: No bc_x in input file"); }
    if (!config["bc_y"]) { endrun("ERROR: No bc_y in input file"); }
    if (!config["bc_z"]) { endrun("ERROR: No bc_z in input file"); }
    if (!config["weno_scalars"]) { endrun("ERROR: No weno_scalars in input file"); }
    if (!config["weno_winds"]) { endrun("ERROR: No weno_winds in input file"); }
    if (!config["initData"]) { endrun("ERROR: No initData in input file"); }
    if (!config["outFile"]) { endrun("ERROR: No outFile in input file"); }
    nx = config["nx"].as<int>();
    ny = config["ny"].as<int>();
    nz = config["nz"].as<int>();
    sim2d = ny == 1;
    xlen = config["xlen"].as<real>();
    ylen = config["ylen"].as<real>();
    zlen = config["zlen"].as<real>();
    weno_scalars = config["weno_scalars"].as<bool>();
    weno_winds = config["weno_winds"].as<bool>();
    const std::string dataStr = config["initData"].as<std::string>();
    if (dataStr == "thermal") dataSpec = DATA_SPEC_THERMAL;
    else if (dataStr == "collision") dataSpec = DATA_SPEC_COLLISION;
    else if (dataStr == "straka") dataSpec = DATA_SPEC_STRAKA;
    else if (dataStr == "igw") dataSpec = DATA_SPEC_IGW;
    else endrun("ERROR: Invalid dataSpec");
    bc_x = parseBC(config["bc_x"].as<std::string>(), "Invalid bc_x");
    bc_y = parseBC(config["bc_y"].as<std::string>(), "Invalid bc_y");
    bc_z = parseBC(config["bc_z"].as<std::string>(), "Invalid bc_z");
    outFile = config["outFile"].as<std::string>();
    dx = xlen / nx;
    dy = ylen / ny;
    dz = zlen / nz;
    perturb = config["perturb"].as<bool>();  // like the reference: required, throws if absent

    // extensions
    if (config["precision"]) {
      const std::string p = config["precision"].as<std::string>();
      if (p == "fp64") precision = AWFL_FP64;
      else if (p == "fp32") precision = AWFL_FP32;
      else endrun("ERROR: precision must be fp64 or fp32");
    }
    if (config["device"]) device = config["device"].as<int>();
    if (config["tracer_transport"]) tracerTransport = config["tracer_transport"].as<bool>();
    initSpec = awfl_init_spec{};
    initSpec.kind = AWFL_INIT_REFERENCE;
    if (config["bubble"]) {
      const std::string b = config["bubble"].as<std::string>();
      initSpec.kind = AWFL_INIT_BUBBLE;
      initSpec.shape = b == "linear" ? 0 : 1;
      auto get = [&](const char *k, double d) { return config[k] ? config[k].as<double>() : d; };
      const double rad = get("bubble_radius", 2000.0);
      initSpec.x0 = get("bubble_x0", xlen / 2);
      initSpec.y0 = get("bubble_y0", ylen / 2);
      initSpec.z0 = get("bubble_z0", 2000.0);
      initSpec.xrad = get("bubble_xrad", rad);
      initSpec.yrad = get("bubble_yrad", rad);
      initSpec.zrad = get("bubble_zrad", rad);
      initSpec.amp = get("bubble_amp", 3.0);
      initSpec.pwr = get("bubble_pwr", 1.0);
    }
    if (config["noise_amp"]) initSpec.noise_amp = config["noise_amp"].as<double>();
    initSpec.noise_seed = config["noise_seed"] ? (unsigned long long)config["noise_seed"].as<double>() : 20261203ULL;
    if (config["noise_dist"]) {
      const std::string d = config["noise_dist"].as<std::string>();
      if (d != "uniform" && d != "normal") endrun("ERROR: noise_dist must be uniform or normal");
      initSpec.noise_kind = d == "normal" ? AWFL_NOISE_NORMAL : AWFL_NOISE_UNIFORM;
    }

    numTracers = (int)tracerName.size();

    awfl_config cfg{};
    cfg.nx = nx; cfg.ny = ny; cfg.nz = nz;
    cfg.xlen = xlen; cfg.ylen = ylen; cfg.zlen = zlen;
    cfg.bc_x = bc_x; cfg.bc_y = bc_y; cfg.bc_z = bc_z;
    cfg.weno_scalars = weno_scalars; cfg.weno_winds = weno_winds;
    cfg.data_spec = dataSpec;
    cfg.ord = ord;
    cfg.precision = precision;
    if (ctx) awfl_destroy(ctx);
    ctx = nullptr;
    awfl_dropin::check(awfl_create(&cfg, device, &ctx), nullptr, "init");
  }

  // Spatial:345-500: hydrostatic background (built by the library) and initial data.
  void initState(StateArr &state) {
    awfl_dropin::check(awfl_init_state(ctx, state.data(), &initSpec, nullptr), ctx, "initState");
    if (perturb) {  // Spatial:488-499, same host loop and rand() sequence
      std::vector<double> h = state.createHostCopy();
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nx; i++) {
            const real rval = (real)rand() / (real)RAND_MAX;
            h[idx(idT, hs + k, hs + j, hs + i)] *= 1. + rval * 1.e-7;
          }
      state.copyFromHost(h.data(), (size_t)numState * (nz + 2 * hs) * (ny + 2 * hs) * (nx + 2 * hs));
    }
  }

  void initTracers(TracerArr &tracers) {
    if (!tracers.initialized() || tracers.totElems() == 0) return;
    awfl_dropin::check(awfl_memset_device(tracers.data(), 0, (long)(tracers.totElems() * tracers.elemBytes()), nullptr),
                       ctx, "initTracers");
    awfl_dropin::check(awfl_init_tracers(ctx, static_cast<double *>(tracers.data()), numTracers, nullptr), ctx,
                       "initTracers");
  }

  // Spatial:565-594: X,Y,Z then Z,Y,X; the dir-halos of the state are filled in place.
  void computeTendencies(StateArr &state, StateTendArr &stateTend, TracerArr &tracers, TracerTendArr &tracerTend,
                         real &dt, int splitIndex) {
    (void)tracers;
    const int dir = dirOf(splitIndex);
    awfl_dropin::check(awfl_compute_tendencies(ctx, state.data(), stateTend.data(), dt, dir, nullptr), ctx,
                       "computeTendencies");
    if (tracerTend.initialized() && tracerTend.totElems() > 0)
      awfl_dropin::check(
          awfl_memset_device(tracerTend.data(), 0, (long)(tracerTend.totElems() * tracerTend.elemBytes()), nullptr),
          ctx, "tracer tendency");
    if (splitIndex == numSplit() - 1) dimSwitch = !dimSwitch;
  }

  // computeTendencies(split) followed by the apply (Temporal_ader.h:63-65) as one fused
  // kernel; the same results, without a tendency array.
  void computeAndApplyTendencies(StateArr &state, real dt, int splitIndex) {
    const int dir = dirOf(splitIndex);
    awfl_dropin::check(awfl_split(ctx, state.data(), dt, dir, nullptr), ctx, "computeAndApplyTendencies");
    if (splitIndex == numSplit() - 1) dimSwitch = !dimSwitch;
  }

  // The same split with the tracers advanced too (tracer_transport: true): one
  // awfl_split_tracers call (the state as awfl_split advances it).
  void computeAndApplyTendencies(StateArr &state, TracerArr &tracers, real dt, int splitIndex) {
    const int dir = dirOf(splitIndex);
    if (tracerTransport && numTracers > 0 && tracers.initialized() && tracers.totElems() > 0) {
      std::vector<int> pos(numTracers);
      for (int t = 0; t < numTracers; t++) pos[t] = tracerPosVect[t] ? 1 : 0;
      awfl_dropin::check(awfl_split_tracers(ctx, state.data(), static_cast<double *>(tracers.data()), numTracers,
                                            pos.data(), dt, dir, nullptr),
                         ctx, "tracer transport");
    } else {
      awfl_dropin::check(awfl_split(ctx, state.data(), dt, dir, nullptr), ctx, "computeAndApplyTendencies");
    }
    if (splitIndex == numSplit() - 1) dimSwitch = !dimSwitch;
  }

  // README extras ------------------------------------------------------------------------
  // state(l,hs+k,hs+j,hs+i) += dt * tend(l,k,j,i) for this split stage.
  void applyTendencies(StateArr &state, StateTendArr const &tend, real dt, int splitIndex) {
    (void)splitIndex;
    awfl_dropin::check(awfl_apply_tendencies(ctx, state.data(), tend.data(), dt, nullptr), ctx, "applyTendencies");
  }
  // One value, read back from the device (the interior cell of loc; halos are not indexed).
  real get(StateArr const &state, Location const &loc, int splitIndex) const {
    (void)splitIndex;
    return readOne(state, idx(loc.l, hs + loc.k, hs + loc.j, hs + loc.i));
  }
  real get(StateTendArr const &tend, Location const &loc, int timeDeriv, int splitIndex) const {
    (void)splitIndex;
    if (timeDeriv != 0) endrun("ERROR: only the time-averaged tendency (timeDeriv 0) is stored");
    return readOne(tend, (((size_t)loc.l * nz + loc.k) * ny + loc.j) * nx + loc.i);
  }
  const char *getSpatialName() { return getName(); }

  const char *getName() { return "1-D Uniform Transport with upwind FV on A-grid"; }

  void output(StateArr const &state, TracerArr const &tracers, real etime) {
    if (outFile.size() >= 3 && outFile.compare(outFile.size() - 3, 3, ".nc") == 0) {
      const bool tr = numTracers > 0 && tracers.initialized() && tracers.totElems() > 0;
      std::vector<const char *> names;
      for (int t = 0; tr && t < numTracers; t++) names.push_back(tracerName[t].c_str());
      awfl_dropin::check(awfl_write_netcdf_tracers(ctx, outFile.c_str(), state.data(),
                                                   tr ? static_cast<const double *>(tracers.data()) : nullptr,
                                                   tr ? numTracers : 0, names.data(), etime, nullptr),
                         ctx, "output");
      return;
    }
    if (outFile.size() < 4 || outFile.compare(outFile.size() - 4, 4, ".bin") != 0) return;
    std::vector<double> h = state.createHostCopy();
    const size_t n = (size_t)numState * (nz + 2 * hs) * (ny + 2 * hs) * (nx + 2 * hs);
    std::ofstream f(outFile, std::ios::binary | std::ios::trunc);
    f.write(reinterpret_cast<const char *>(h.data()), (std::streamsize)(n * sizeof(double)));
  }

  void finalize(StateArr const &state, TracerArr const &tracers) {
    (void)state;
    (void)tracers;
  }

 private:
  size_t elemBytes() const { return precision == AWFL_FP32 ? sizeof(float) : sizeof(double); }
  int dirOf(int splitIndex) const {
    const int d = dimSwitch ? splitIndex : 2 - splitIndex;
    awfl_dropin::check(awfl_set_dimswitch(ctx, dimSwitch ? 1 : 0), ctx, "dimSwitch");
    return d;
  }
  size_t idx(int l, int k, int j, int i) const {
    return (((size_t)l * (nz + 2 * hs) + k) * (ny + 2 * hs) + j) * (nx + 2 * hs) + i;
  }
  static int parseBC(const std::string &s, const char *msg) {
    if (s == "periodic") return BC_PERIODIC;
    if (s == "wall") return BC_WALL;
    endrun(msg);
    return BC_PERIODIC;
  }
  real readOne(awfl_dropin::DeviceArray const &a, size_t i) const {
    if (a.elemBytes() == sizeof(double)) {
      double v = 0;
      awfl_dropin::check(awfl_copy_d2h(&v, (const char *)a.data() + i * sizeof(double), sizeof(double), nullptr), ctx,
                         "get");
      awfl_dropin::check(awfl_stream_synchronize(nullptr), ctx, "get");
      return v;
    }
    float v = 0;
    awfl_dropin::check(awfl_copy_d2h(&v, (const char *)a.data() + i * sizeof(float), sizeof(float), nullptr), ctx, "get");
    awfl_dropin::check(awfl_stream_synchronize(nullptr), ctx, "get");
    return v;
  }
};
