// Exact discrete adjoint kernels (efwi_exact.cu).
#pragma once
#include "efwi_common.cuh"
#include "efwi_tma.cuh"

namespace efwi {

struct ExactArgs {
  Geo g;
  Fields f;        // forward state S_k (read)
  Psi ps;          // forward memory variables of S_k (read)
  Fields a;        // adjoint fields (updated in place)
  Psi lin, lout;   // adjoint memory variables: read from lin, written to lout
  const float *lam, *mu, *buoy;
  float *g0, *g1;  // images: stress stage (lambda, mu); velocity stage (buoyancy, unused)
};

// Transpose of the stress stage of step k (+ lambda/mu images), then of the
// velocity stage of step k-1 (+ buoyancy image); the grid is
// (ceil(ny/32), ceil(nx/bx), ceil(nz/zchunk)) with 32 x bx threads, bx 4 or 8.
void launch_adj_stress_exact(int bx, dim3 grid, cudaStream_t st, const ExactArgs &A, int zchunk,
                             int nzc);
void launch_adj_velocity_exact(int bx, dim3 grid, cudaStream_t st, const ExactArgs &A, int zchunk,
                               int nzc);
// The same with every plane's operands staged by bulk tensor copies (bitwise
// the same results).  Stress stage maps (halo boxes): adjoint szz sxx syy sxz
// sxy syz, lambda, mu, forward vz vx vy.  Velocity stage maps: adjoint vz vx
// vy, buoyancy, forward sxz sxx sxy syz syy szz.
void launch_adj_stress_tma(int bx, dim3 grid, cudaStream_t st, const Maps<11> &maps,
                           const ExactArgs &A, int zchunk, int *status);
void launch_adj_velocity_tma(int bx, dim3 grid, cudaStream_t st, const Maps<10> &maps,
                             const ExactArgs &A, int zchunk, int *status);

__global__ void k_buoy_to_rho(const float *gB, const float *buoy, float *grho, int nz, int nx,
                              int ny, int py);
__global__ void k_stf_gradient(Fields a, const long long *src_cell, const float *w2, float *out,
                               int k, float scale);
__global__ void k_state_convert(Geo g, float *full, Fields f, Psi ps, int to_engine);
__global__ void k_illumination(Geo g, Fields f, Psi ps, int S, const float *buoy, int do_stress,
                               float *hl, float *hm, float *hb);
__global__ void k_buoy_to_rho_sq(float *hb, const float *buoy, int nz, int nx, int ny, int py);

}  // namespace efwi
