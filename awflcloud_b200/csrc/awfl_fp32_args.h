// Kernel arguments of the FP32 form (shared by awfl_fp32.cu and the host code).
#pragma once

namespace awfl {

// Background constants of the FP32 form (FP32 copies of FP64 host values).
struct Bg32 {
  const float *rho_c, *rt_c, *irt_c, *p_c;  // cell rows, (nz+2hs): rho_h, (rho theta)_h, 1/(rho theta)_h, C0*(rho theta)_h^gamma
  const float *rho_g, *rt_g, *irt_g, *p_g;  // GLL points, nz*ngll (z); point ngll-1 of cell k == point 0 of cell k+1
  const float *rho_f, *rt_f, *irt_f, *p_f;  // z faces 0..nz: bottom point of cell k, top of cell nz-1 for face nz
};

// A TMA tensor map (the 128-byte CUtensorMap of the CUDA driver API, opaque here),
// 64-byte aligned as TMA requires.
struct alignas(64) TmaMap {
  unsigned long long w[16];
};

struct SweepArgs32 {
  TmaMap tmap;   // single-grid sweeps with tma != 0: the state as a 3-D tensor
                 // {nx+2hs, ny+2hs, 5*(nz+2hs)} floats, box = one chunk of one variable
  float *state;  // plane 0 of the FP32 state
  float *comp;   // plane 1: Kahan compensation
  float *tend;
  int nx, ny, nz;
  int bc, weno_s, weno_w, sim2d, mode;
  float inv_dxd;
  float dt;
  Bg32 bg;
  int tma;             // interior chunks' stencil rows arrive by TMA through tmap
  unsigned int *err;   // set to nonzero if a bounded wait of the sweep gave up
  // x sweeps of a slab: the neighbouring slabs' halo columns (values), as SweepArgs::xh
  const float *xh[2];
};

// Encodes *m as the tiled tensor map of an FP32 state with halo-inclusive extents
// xe x ye x ze per variable (dims {xe, ye, 5*ze}) and the given box (x, y, z extents).
// Returns false (m untouched) where TMA cannot address the layout: a state base not
// 16-byte aligned, a row pitch not a multiple of 16 bytes, or an encoder error.
bool encode_state_map32(TmaMap *m, const float *state, int xe, int ye, int ze, const unsigned (&box)[3]);
// Sets A.tmap/A.tma for a sweep of direction dir with chunk C and W lines per CTA (the box
// of awfl_sweep.cuh's TMA path); A.tma = 0 where TMA cannot address the layout.
bool prepare_sweep_map32(SweepArgs32 &A, int ord, int dir, int C, int W);
// Looks the encoder up now (context creation), not inside a caller's stream capture.
void warm_tma_encoder();

}  // namespace awfl
