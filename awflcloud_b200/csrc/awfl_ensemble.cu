// Ensemble (batching) form: host side of awfl_ensemble_* (include/awfl.h).
//
// An ensemble owns one awfl_ctx per member (each with its own grid size, background and
// time step) and advances all members together: per split stage one persistent kernel
// (awfl_ens.cuh) walks a tile list covering every member, and a pair of time steps (the
// X,Y,Z / Z,Y,X alternation) is replayed from a CUDA graph. The autotuner times every
// candidate tile shape of each direction on scratch copies of the members' states and
// keeps the fastest. An FP64 member's result is bit-identical to stepping its context
// alone with awfl_step (same per-tile arithmetic, any shape); FP32 members agree to FP32
// rounding.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/awfl.h"
#include "awfl_ens.cuh"
#include "awfl_fp32_args.h"
#include "awfl_internal.h"

namespace awfl {
namespace host {
const awfl_config &ctx_cfg(const awfl_ctx *c);
int ctx_hs(const awfl_ctx *c);
int ctx_sim2d(const awfl_ctx *c);
int ctx_nsm(const awfl_ctx *c);
int ctx_device(const awfl_ctx *c);
int ctx_set_device(awfl_ctx *c);
long ctx_state_elems(const awfl_ctx *c);
SweepArgs ctx_sweep_args64(awfl_ctx *c, void *state, double dt, int dir);
SweepArgs32 ctx_sweep_args32(awfl_ctx *c, void *state, double dt, int dir);
}  // namespace host
}  // namespace awfl

using namespace awfl;
using namespace awfl::host;

struct awfl_ensemble {
  int device = 0, nsm = 148, prec = AWFL_FP64, ord = 5;
  std::vector<awfl_ctx *> mem;
  std::vector<void *> state;
  std::vector<double> dt;
  int dimswitch = 1;
  int shape[3] = {0, 0, 0};
  int grid[3] = {0, 0, 0};
  // device work lists (one allocation) and their host descriptors
  void *d_lists = nullptr;
  EnsList<SweepArgs> l64[3] = {};
  EnsList<SweepArgs32> l32[3] = {};
  bool lists_ok = false;
  // CUDA graphs of two steps starting with dimSwitch 1 and 0
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  cudaStream_t cap = nullptr;
  // autotuner record: per direction, per candidate shape, ms per launch (<0: not run)
  std::vector<float> tune_ms[3];
  std::string err;
};

namespace {

thread_local std::string g_ens_error;

int efail(awfl_ensemble *e, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (e) e->err = buf;
  else g_ens_error = buf;
  return code;
}

int ecuda(awfl_ensemble *e, cudaError_t c, const char *what) {
  return efail(e, AWFL_ERR_CUDA, "%s: %s", what, cudaGetErrorString(c));
}

int eset_device(awfl_ensemble *e) {
  int cur = -1;
  cudaError_t c = cudaGetDevice(&cur);
  if (c != cudaSuccess) return ecuda(e, c, "cudaGetDevice");
  if (cur != e->device) {
    c = cudaSetDevice(e->device);
    if (c != cudaSuccess) return ecuda(e, c, "cudaSetDevice");
  }
  return AWFL_OK;
}

void drop_graphs(awfl_ensemble *e) {
  for (auto &g : e->exec) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

int line_len(const awfl_config &c, int dir) { return dir == 0 ? c.nx : (dir == 1 ? c.ny : c.nz); }

// Tile grid of one member in one direction (the single-grid sweep's CTA grid).
void tiles(const awfl_config &c, int dir, int W, int *nbx, int *nby) {
  if (dir == 0) { *nbx = (c.ny + W - 1) / W; *nby = c.nz; }
  else if (dir == 1) { *nbx = (c.nx + W - 1) / W; *nby = c.nz; }
  else { *nbx = (c.nx + W - 1) / W; *nby = c.ny; }
}

// Builds the three work lists for the current shapes and the given states (the bound
// ones, or the tuner's scratch copies) into one device allocation.
int build_lists(awfl_ensemble *e, const std::vector<void *> &states, void **d_out, EnsList<SweepArgs> (&l64)[3],
                EnsList<SweepArgs32> (&l32)[3]) {
  const int n = (int)e->mem.size();
  const size_t asz = e->prec == AWFL_FP32 ? sizeof(SweepArgs32) : sizeof(SweepArgs);
  // layout per direction: args[n] | prefix[n+1] | nbx[n], 64-byte aligned pieces (the
  // FP32 arguments hold a 64-byte-aligned tensor map field)
  auto up64 = [](size_t x) { return (x + 63) & ~size_t(63); };
  const size_t per = up64(asz * n) + up64(sizeof(long) * (n + 1)) + up64(sizeof(int) * n);
  std::vector<unsigned char> host(per * 3, 0);
  for (int dir = 0; dir < 3; dir++) {
    int C, W;
    ens_shape(e->ord, dir, e->shape[dir], &C, &W);
    std::vector<int> order;
    for (int m = 0; m < n; m++)
      if (!(dir == 1 && ctx_sim2d(e->mem[m]))) order.push_back(m);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      return line_len(ctx_cfg(e->mem[a]), dir) > line_len(ctx_cfg(e->mem[b]), dir);
    });
    unsigned char *base = host.data() + per * dir;
    unsigned char *pa = base;
    long *pp = (long *)(base + up64(asz * n));
    int *pn = (int *)(base + up64(asz * n) + up64(sizeof(long) * (n + 1)));
    long total = 0;
    for (size_t q = 0; q < order.size(); q++) {
      const int m = order[q];
      awfl_ctx *c = e->mem[m];
      if (e->prec == AWFL_FP32) {
        SweepArgs32 A = ctx_sweep_args32(c, states[m], e->dt[m], dir);
        prepare_sweep_map32(A, e->ord, dir, C, W);  // the member's tensor map for this shape
        std::memcpy(pa + q * asz, &A, asz);
      } else {
        SweepArgs A = ctx_sweep_args64(c, states[m], e->dt[m], dir);
        std::memcpy(pa + q * asz, &A, asz);
      }
      int nbx, nby;
      tiles(ctx_cfg(c), dir, W, &nbx, &nby);
      pp[q] = total;
      pn[q] = nbx;
      total += (long)nbx * nby;
    }
    pp[order.size()] = total;
    l64[dir].n = l32[dir].n = (int)order.size();
    l64[dir].total = l32[dir].total = total;
  }
  void *d = nullptr;
  cudaError_t c = cudaMalloc(&d, host.size());
  if (c != cudaSuccess) return efail(e, AWFL_ERR_NOMEM, "cudaMalloc ensemble work lists: %s", cudaGetErrorString(c));
  c = cudaMemcpy(d, host.data(), host.size(), cudaMemcpyHostToDevice);
  if (c != cudaSuccess) {
    cudaFree(d);
    return ecuda(e, c, "upload of ensemble work lists");
  }
  for (int dir = 0; dir < 3; dir++) {
    unsigned char *base = (unsigned char *)d + per * dir;
    l64[dir].args = (const SweepArgs *)base;
    l32[dir].args = (const SweepArgs32 *)base;
    l64[dir].prefix = l32[dir].prefix = (const long *)(base + up64(asz * n));
    l64[dir].nbx = l32[dir].nbx = (const int *)(base + up64(asz * n) + up64(sizeof(long) * (n + 1)));
  }
  *d_out = d;
  return AWFL_OK;
}

int grid_for(awfl_ensemble *e, int dir, int shape, long total, int *grid) {
  int occ = 0;
  cudaError_t c = e->prec == AWFL_FP32 ? ens_run_fp32(e->ord, dir, shape, nullptr, 0, &occ, nullptr)
                                       : ens_run_fp64(e->ord, dir, shape, nullptr, 0, &occ, nullptr);
  if (c != cudaSuccess) return ecuda(e, c, "occupancy query");
  long g = (long)std::max(occ, 1) * e->nsm;
  if (g > total) g = total;
  *grid = (int)std::max(g, 1L);
  return AWFL_OK;
}

cudaError_t launch_dir(awfl_ensemble *e, int dir, int shape, int grid, const EnsList<SweepArgs> &l64,
                       const EnsList<SweepArgs32> &l32, cudaStream_t st) {
  if (l64.total == 0) return cudaSuccess;
  return e->prec == AWFL_FP32 ? ens_run_fp32(e->ord, dir, shape, &l32, grid, nullptr, st)
                              : ens_run_fp64(e->ord, dir, shape, &l64, grid, nullptr, st);
}

int ensure_lists(awfl_ensemble *e) {
  if (e->lists_ok) return AWFL_OK;
  for (size_t m = 0; m < e->mem.size(); m++)
    if (!e->state[m]) return efail(e, AWFL_ERR_STATE, "member %zu has no bound state (awfl_ensemble_bind)", m);
  drop_graphs(e);
  if (e->d_lists) {  // work already queued may still read the old lists
    cudaError_t c = cudaDeviceSynchronize();
    if (c != cudaSuccess) return ecuda(e, c, "synchronize before rebuilding the work lists");
    cudaFree(e->d_lists);
    e->d_lists = nullptr;
  }
  int rc = build_lists(e, e->state, &e->d_lists, e->l64, e->l32);
  if (rc) return rc;
  for (int dir = 0; dir < 3; dir++) {
    rc = grid_for(e, dir, e->shape[dir], e->l64[dir].total, &e->grid[dir]);
    if (rc) return rc;
  }
  e->lists_ok = true;
  return AWFL_OK;
}

// One step's three stage launches (dimSwitch ds) on stream st.
cudaError_t launch_step(awfl_ensemble *e, int ds, cudaStream_t st) {
  for (int spl = 0; spl < 3; spl++) {
    const int dir = ds ? spl : 2 - spl;
    cudaError_t c = launch_dir(e, dir, e->shape[dir], e->grid[dir], e->l64[dir], e->l32[dir], st);
    if (c != cudaSuccess) return c;
  }
  return cudaSuccess;
}

int ensure_graph(awfl_ensemble *e, int ds) {
  if (e->exec[ds]) return AWFL_OK;
  if (!e->cap) {
    cudaError_t c = cudaStreamCreateWithFlags(&e->cap, cudaStreamNonBlocking);
    if (c != cudaSuccess) return ecuda(e, c, "cudaStreamCreate");
  }
  cudaError_t c = cudaStreamBeginCapture(e->cap, cudaStreamCaptureModeThreadLocal);
  if (c != cudaSuccess) return ecuda(e, c, "cudaStreamBeginCapture");
  cudaError_t l = launch_step(e, ds, e->cap);
  if (l == cudaSuccess) l = launch_step(e, !ds, e->cap);
  cudaGraph_t g = nullptr;
  c = cudaStreamEndCapture(e->cap, &g);
  if (l != cudaSuccess || c != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return ecuda(e, l != cudaSuccess ? l : c, "capture of the ensemble step graph");
  }
  c = cudaGraphInstantiate(&e->exec[ds], g, 0);
  cudaGraphDestroy(g);
  if (c != cudaSuccess) {
    e->exec[ds] = nullptr;
    return ecuda(e, c, "cudaGraphInstantiate");
  }
  return AWFL_OK;
}

}  // namespace

extern "C" {

int awfl_ensemble_create(const awfl_config *cfgs, int nmembers, int device, awfl_ensemble **out) {
  if (!out) return efail(nullptr, AWFL_ERR_ARG, "ens is NULL");
  *out = nullptr;
  if (!cfgs || nmembers < 1) return efail(nullptr, AWFL_ERR_ARG, "need at least one member configuration");
  if (device < 0) return efail(nullptr, AWFL_ERR_ARG, "an ensemble needs a device");
  for (int m = 1; m < nmembers; m++)
    if (cfgs[m].precision != cfgs[0].precision || cfgs[m].ord != cfgs[0].ord)
      return efail(nullptr, AWFL_ERR_ARG, "member %d: every member must have the same precision and ord", m);
  awfl_ensemble *e = new (std::nothrow) awfl_ensemble();
  if (!e) return efail(nullptr, AWFL_ERR_NOMEM, "out of host memory");
  e->device = device;
  e->prec = cfgs[0].precision;
  e->ord = cfgs[0].ord;
  for (int m = 0; m < nmembers; m++) {
    awfl_ctx *c = nullptr;
    const int rc = awfl_create(&cfgs[m], device, &c);
    if (rc) {
      efail(nullptr, rc, "member %d: %s", m, awfl_last_error(nullptr));
      awfl_ensemble_destroy(e);
      return rc;
    }
    e->mem.push_back(c);
  }
  e->state.assign(nmembers, nullptr);
  e->dt.assign(nmembers, 0.0);
  e->nsm = ctx_nsm(e->mem[0]);
  for (int dir = 0; dir < 3; dir++) e->tune_ms[dir].assign(ens_num_shapes(e->ord, dir), -1.f);
  *out = e;
  return AWFL_OK;
}

int awfl_ensemble_destroy(awfl_ensemble *e) {
  if (!e) return AWFL_OK;
  if (!e->mem.empty()) eset_device(e);
  drop_graphs(e);
  if (e->cap) cudaStreamDestroy(e->cap);
  if (e->d_lists) cudaFree(e->d_lists);
  for (awfl_ctx *c : e->mem) awfl_destroy(c);
  delete e;
  return AWFL_OK;
}

const char *awfl_ensemble_last_error(const awfl_ensemble *e) { return e ? e->err.c_str() : g_ens_error.c_str(); }

int awfl_ensemble_size(const awfl_ensemble *e, int *n) {
  if (!e || !n) return AWFL_ERR_ARG;
  *n = (int)e->mem.size();
  return AWFL_OK;
}

int awfl_ensemble_member(awfl_ensemble *e, int i, awfl_ctx **ctx) {
  if (!e || !ctx) return AWFL_ERR_ARG;
  if (i < 0 || i >= (int)e->mem.size()) return efail(e, AWFL_ERR_ARG, "member index %d out of range", i);
  *ctx = e->mem[i];
  return AWFL_OK;
}

int awfl_ensemble_bind(awfl_ensemble *e, int i, void *d_state, double dt) {
  if (!e) return AWFL_ERR_ARG;
  if (i < 0 || i >= (int)e->mem.size()) return efail(e, AWFL_ERR_ARG, "member index %d out of range", i);
  if (!d_state || (reinterpret_cast<uintptr_t>(d_state) & 7)) return efail(e, AWFL_ERR_ARG, "state pointer is NULL or misaligned");
  if (!(dt > 0.0) || !std::isfinite(dt)) return efail(e, AWFL_ERR_ARG, "dt must be positive and finite");
  e->state[i] = d_state;
  e->dt[i] = dt;
  e->lists_ok = false;
  return AWFL_OK;
}

int awfl_ensemble_step(awfl_ensemble *e, int nsteps, void *stream) {
  if (!e) return AWFL_ERR_ARG;
  if (nsteps < 0) return efail(e, AWFL_ERR_ARG, "nsteps must be >= 0");
  int rc = eset_device(e);
  if (rc) return rc;
  rc = ensure_lists(e);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int ds = e->dimswitch;
  if (nsteps >= 2) {
    rc = ensure_graph(e, ds);
    if (rc) return rc;
    for (int n = 0; n + 1 < nsteps; n += 2) {
      cudaError_t c = cudaGraphLaunch(e->exec[ds], st);
      if (c != cudaSuccess) return ecuda(e, c, "cudaGraphLaunch");
    }
  }
  if (nsteps & 1) {
    cudaError_t c = launch_step(e, ds, st);
    if (c != cudaSuccess) return ecuda(e, c, "ensemble step");
    e->dimswitch = !ds;
  }
  return AWFL_OK;
}

int awfl_ensemble_tune(awfl_ensemble *e, int reps, void *stream) {
  if (!e) return AWFL_ERR_ARG;
  if (reps < 1) return efail(e, AWFL_ERR_ARG, "reps must be >= 1");
  int rc = eset_device(e);
  if (rc) return rc;
  rc = ensure_lists(e);  // validates the bindings
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // scratch copies of every member's state: tuning launches advance them, not the bound states
  const int n = (int)e->mem.size();
  std::vector<size_t> off(n + 1, 0);
  const size_t esz = e->prec == AWFL_FP32 ? sizeof(float) : sizeof(double);
  for (int m = 0; m < n; m++) off[m + 1] = off[m] + (((size_t)ctx_state_elems(e->mem[m]) * esz + 255) & ~size_t(255));
  unsigned char *scratch = nullptr;
  cudaError_t c = cudaMalloc(&scratch, off[n]);
  if (c != cudaSuccess) return efail(e, AWFL_ERR_NOMEM, "cudaMalloc tuning scratch (%zu bytes): %s", off[n], cudaGetErrorString(c));
  std::vector<void *> sst(n);
  for (int m = 0; m < n && c == cudaSuccess; m++) {
    sst[m] = scratch + off[m];
    c = cudaMemcpyAsync(sst[m], e->state[m], (size_t)ctx_state_elems(e->mem[m]) * esz, cudaMemcpyDeviceToDevice, st);
  }
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if (c == cudaSuccess) c = cudaEventCreate(&ev[0]);
  if (c == cudaSuccess) c = cudaEventCreate(&ev[1]);
  void *d_tmp = nullptr;
  const int saved[3] = {e->shape[0], e->shape[1], e->shape[2]};
  for (int dir = 0; dir < 3 && c == cudaSuccess && rc == AWFL_OK; dir++) {
    int best = 0;
    float best_ms = 0.f;
    for (int s = 0; s < ens_num_shapes(e->ord, dir) && c == cudaSuccess && rc == AWFL_OK; s++) {
      e->shape[dir] = s;
      EnsList<SweepArgs> l64[3];
      EnsList<SweepArgs32> l32[3];
      rc = build_lists(e, sst, &d_tmp, l64, l32);
      if (rc) break;
      int grid = 1;
      rc = grid_for(e, dir, s, l64[dir].total, &grid);
      if (rc == AWFL_OK && l64[dir].total > 0) {
        c = launch_dir(e, dir, s, grid, l64[dir], l32[dir], st);  // warm-up
        if (c == cudaSuccess) c = cudaEventRecord(ev[0], st);
        for (int r = 0; r < reps && c == cudaSuccess; r++) c = launch_dir(e, dir, s, grid, l64[dir], l32[dir], st);
        if (c == cudaSuccess) c = cudaEventRecord(ev[1], st);
        if (c == cudaSuccess) c = cudaEventSynchronize(ev[1]);
        float ms = 0.f;
        if (c == cudaSuccess) c = cudaEventElapsedTime(&ms, ev[0], ev[1]);
        ms /= reps;
        e->tune_ms[dir][s] = ms;
        if (s == 0 || ms < best_ms) {
          best = s;
          best_ms = ms;
        }
      }
      cudaStreamSynchronize(st);
      cudaFree(d_tmp);
      d_tmp = nullptr;
    }
    e->shape[dir] = best;
  }
  if (ev[0]) cudaEventDestroy(ev[0]);
  if (ev[1]) cudaEventDestroy(ev[1]);
  cudaStreamSynchronize(st);
  cudaFree(scratch);
  if (c != cudaSuccess || rc != AWFL_OK) {
    for (int d = 0; d < 3; d++) e->shape[d] = saved[d];
    e->lists_ok = false;
    return rc ? rc : ecuda(e, c, "ensemble autotuning");
  }
  e->lists_ok = false;  // rebuild the lists (and graphs) with the chosen shapes
  return ensure_lists(e);
}

int awfl_ensemble_get_shape(const awfl_ensemble *e, int dir, int *shape, int *chunk, int *lines, int *grid) {
  if (!e || dir < 0 || dir > 2) return AWFL_ERR_ARG;
  int C, W;
  ens_shape(e->ord, dir, e->shape[dir], &C, &W);
  if (shape) *shape = e->shape[dir];
  if (chunk) *chunk = C;
  if (lines) *lines = W;
  if (grid) *grid = e->grid[dir];
  return AWFL_OK;
}

int awfl_ensemble_tuning(const awfl_ensemble *e, int dir, int i, int *chunk, int *lines, float *ms) {
  if (!e || dir < 0 || dir > 2) return AWFL_ERR_ARG;
  if (i < 0 || i >= ens_num_shapes(e->ord, dir)) return AWFL_ERR_ARG;
  int C, W;
  ens_shape(e->ord, dir, i, &C, &W);
  if (chunk) *chunk = C;
  if (lines) *lines = W;
  if (ms) *ms = e->tune_ms[dir][i];
  return AWFL_OK;
}

int awfl_ensemble_num_shapes(const awfl_ensemble *e, int dir, int *n) {
  if (!e || dir < 0 || dir > 2 || !n) return AWFL_ERR_ARG;
  *n = ens_num_shapes(e->ord, dir);
  return AWFL_OK;
}

int awfl_ensemble_set_shape(awfl_ensemble *e, int dir, int shape) {
  if (!e || dir < 0 || dir > 2) return AWFL_ERR_ARG;
  if (shape < 0 || shape >= ens_num_shapes(e->ord, dir)) return efail(e, AWFL_ERR_ARG, "shape index %d out of range", shape);
  e->shape[dir] = shape;
  e->lists_ok = false;
  return AWFL_OK;
}

int awfl_ensemble_get_dimswitch(const awfl_ensemble *e, int *value) {
  if (!e || !value) return AWFL_ERR_ARG;
  *value = e->dimswitch;
  return AWFL_OK;
}

int awfl_ensemble_set_dimswitch(awfl_ensemble *e, int value) {
  if (!e) return AWFL_ERR_ARG;
  e->dimswitch = value != 0;
  return AWFL_OK;
}

}  // extern "C"
