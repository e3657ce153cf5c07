// Shared device-side definitions of the B200 elastic propagation engine.
//
// Layout (HBM): every volume is [nz][nx][py] float32, y fastest -- the
// torch-native C order of the caller's tensors (the reference transposes to
// z-fastest on the host, libCUFD.cu:72-80), with the y pitch py = ny rounded
// up to a multiple of 4 so that every row starts on a 16-byte boundary (the
// alignment of bulk tensor copies).  Shots of one batch are stacked with
// stride N = nz*nx*py.
//
// C-PML memory variables live only in their slabs (the reference keeps 18
// full-grid arrays, libCUFD.cu:173-191):
//   z slab  [2*np][nx][ny]   cells with z < np or z > nz-np-1
//   x slab  [nz][2*np][ny]   cells with x < np or x > nx-np-1
//   y slab  [nz][nx][2*np]   cells with y < np or y > ny-np-1
// Each axis buffer holds 6 variables (PSI_* below).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace efwi {

// 4th-order staggered coefficients (stress.cu:33-34).
#define EFWI_C1 1.125f
#define EFWI_C2 (1.0f / 24.0f)

// Per-axis memory-variable slots.  For axis a:
//   0: d(v_a)/da            (integer points)   -- stress kernel
//   1,2: d(v_b)/da, b != a  (half points)      -- stress kernel
//   3: d(s_aa)/da           (half points)      -- velocity kernel
//   4,5: d(s_ab)/da         (integer points)   -- velocity kernel
// z: 0 vz_z 1 vx_z 2 vy_z 3 szz_z 4 sxz_z 5 syz_z
// x: 0 vx_x 1 vz_x 2 vy_x 3 sxx_x 4 sxz_x 5 sxy_x
// y: 0 vy_y 1 vz_y 2 vx_y 3 syy_y 4 syz_y 5 sxy_y
enum { PSI_VA = 0, PSI_VB1 = 1, PSI_VB2 = 2, PSI_SAA = 3, PSI_SAB1 = 4, PSI_SAB2 = 5 };

// Coefficient rows of one axis profile [6][n]: 1/K, a, b, 1/K_half, a_half,
// b_half (utilities.cu:204-320).  The reference divides by K; the kernels
// multiply by the stored reciprocal (a rounding difference of at most one
// unit in the last place).
enum { CK = 0, CA = 1, CB = 2, CKH = 3, CAH = 4, CBH = 5 };

struct Geo {
  int nz, nx, ny, np;
  long long N;      // cells per volume (with the y pitch)
  long long sz;     // z stride = nx*py
  int sx;           // x stride = py, the y pitch
  float dt, idz, idx, idy;
  long long slab_z, slab_x, slab_y;  // elements per variable of each slab
  const float *cz, *cx, *cy;         // [6][n] coefficient rows
};

struct Fields {
  float *vz, *vx, *vy, *szz, *sxx, *syy, *sxz, *sxy, *syz;
};

struct Psi {
  float *z, *x, *y;  // [6][slab] per axis
};

__device__ __forceinline__ long long cell(const Geo &g, int z, int x, int y) {
  return ((long long)z * g.nx + x) * g.sx + y;
}

__device__ __forceinline__ float dminus(float m2, float m1, float p0, float p1) {
  // c1 (f[i] - f[i-1]) - c2 (f[i+1] - f[i-2])
  return EFWI_C1 * (p0 - m1) - EFWI_C2 * (p1 - m2);
}
__device__ __forceinline__ float dplus(float m1, float p0, float p1, float p2) {
  // c1 (f[i+1] - f[i]) - c2 (f[i+2] - f[i-1])
  return EFWI_C1 * (p1 - p0) - EFWI_C2 * (p2 - m1);
}

__device__ __forceinline__ bool slab_s(int i, int n, int np) { return i < np || i > n - np - 1; }
// Velocity-kernel x/y slab test of the reference (quirk Q2, velocity.cu:46):
// the high side starts one cell later.
__device__ __forceinline__ bool slab_v(int i, int n, int np) { return i < np || i > n - np; }

__device__ __forceinline__ int slab_c(int i, int n, int np) { return i < np ? i : i - (n - 2 * np); }

// Offsets within one slab variable; 32-bit, as a slab holds fewer cells
// than a volume (fewer than 2^31, checked by efwi_create).
__device__ __forceinline__ int psi_z_idx(const Geo &g, int z, int x, int y) {
  return (slab_c(z, g.nz, g.np) * g.nx + x) * g.ny + y;
}
__device__ __forceinline__ int psi_x_idx(const Geo &g, int z, int x, int y) {
  return (z * (2 * g.np) + slab_c(x, g.nx, g.np)) * g.ny + y;
}
__device__ __forceinline__ int psi_y_idx(const Geo &g, int z, int x, int y) {
  return (z * g.nx + x) * (2 * g.np) + slab_c(y, g.ny, g.np);
}

// Reads of adjoint memory variables at neighbours: zero outside the slab
// (the reference's full-grid arrays are never written there).
__device__ __forceinline__ float psi_z_get(const Geo &g, const float *p, int z, int x, int y) {
  return slab_s(z, g.nz, g.np) ? p[psi_z_idx(g, z, x, y)] : 0.0f;
}
__device__ __forceinline__ float psi_x_get(const Geo &g, const float *p, int z, int x, int y) {
  return slab_s(x, g.nx, g.np) ? p[psi_x_idx(g, z, x, y)] : 0.0f;
}
__device__ __forceinline__ float psi_y_get(const Geo &g, const float *p, int z, int x, int y) {
  return slab_s(y, g.ny, g.np) ? p[psi_y_idx(g, z, x, y)] : 0.0f;
}

}  // namespace efwi
