// Kernel arguments of the FP32 form (shared by awfl_fp32.cu and the host code).
#pragma once

namespace awfl {

// Background constants of the FP32 form (FP32 copies of FP64 host values).
struct Bg32 {
  const float *rho_c, *rt_c, *irt_c, *p_c;  // cell rows, (nz+2hs): rho_h, (rho theta)_h, 1/(rho theta)_h, C0*(rho theta)_h^gamma
  const float *rho_g, *rt_g, *irt_g, *p_g;  // GLL points, nz*ngll (z); point ngll-1 of cell k == point 0 of cell k+1
  const float *rho_f, *rt_f, *irt_f, *p_f;  // z faces 0..nz: bottom point of cell k, top of cell nz-1 for face nz
};

struct SweepArgs32 {
  float *state;  // plane 0 of the FP32 state
  float *comp;   // plane 1: Kahan compensation
  float *tend;
  int nx, ny, nz;
  int bc, weno_s, weno_w, sim2d, mode;
  float inv_dxd;
  float dt;
  Bg32 bg;
};

}  // namespace awfl
