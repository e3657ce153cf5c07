// Exact discrete adjoint of the forward time step, with fused imaging.
//
// The forward step (stress.cu:36-97 then velocity.cu:35-96, restated in
// efwi_fwd.cu) is linear in the state (9 fields + 18 C-PML memory
// variables) for a fixed model.  These kernels apply its transpose, stage by
// stage, in gather form: each thread owns one cell of the adjoint state and
// collects what the forward stencils at its neighbours read from it.  This
// has no reference counterpart; the reference's adjoint kernels
// (stress_adj.cu, velocity_adj.cu) keep the material coefficients outside
// the transposed differences and are not this transpose.
//
// Notation for one C-PML-modified derivative of the forward step at cell n:
//   d = D f / h,  psi' = b psi + a d,  d' = d / K + psi'   (slab cells)
//   d' = d                                                (other cells)
// The stage adds c * d' to an output field.  With G = c * (adjoint of the
// output) and L the adjoint of psi' carried back from the later steps, the
// adjoint of d is
//   Q = G / K + a (L + G)    (slab),    Q = G    (other cells),
// and the adjoint of psi before the stage is b (L + G).  The adjoint of the
// input field f then gathers -D-transposed Q / h: the transpose of D- is
// -D+, of D+ is -D-, and of the quirk-Q1 difference (velocity.cu:79)
// c1 Q[j] - (c1 + c2) Q[j+1] + c2 Q[j+2].  Q is zero outside [2, n-3]^3,
// the cells the forward step updates.
//
// K_EV  transpose of the velocity stage (reads the adjoint velocities at
//       neighbours, updates the adjoint stresses), + buoyancy image
//       gB += a_v . (dt * modified stress divergence of the forward state)
// K_ES  transpose of the stress stage (reads the adjoint stresses, lambda
//       and mu at neighbours, updates the adjoint velocities), + lambda and
//       mu images from the forward velocities.
// The adjoint memory variables are read from `lin` and written to `lout`
// (two buffers used in turn): neighbours read them while the owner updates.
//
// Tiling: a CTA owns a 32 (y) x BX (x) column tile and marches a chunk of z
// planes.  The Q of the x- and y-axis terms and the forward fields of the
// images are staged in shared memory per plane (tile plus a 2-cell halo),
// the z-axis terms in register queues; every global load of a plane is
// issued before the plane's one barrier.
#include "efwi_common.cuh"
#include "efwi_exact.h"
#include "efwi_tma.cuh"

namespace efwi {
namespace {

// 32-bit offsets: a volume holds fewer than 2^31 cells (checked by efwi_create).
__device__ __forceinline__ int cell32(const Geo &g, int z, int x, int y) {
  return (z * g.nx + x) * g.sx + y;
}
__device__ __forceinline__ int psi32_z(const Geo &g, int z, int x, int y) {
  return (slab_c(z, g.nz, g.np) * g.nx + x) * g.ny + y;
}
__device__ __forceinline__ int psi32_x(const Geo &g, int z, int x, int y) {
  return (z * (2 * g.np) + slab_c(x, g.nx, g.np)) * g.ny + y;
}
__device__ __forceinline__ int psi32_y(const Geo &g, int z, int x, int y) {
  return (z * g.nx + x) * (2 * g.np) + slab_c(y, g.ny, g.np);
}

__device__ __forceinline__ float qpml(float G, bool slab, float L, float kinv, float a) {
  return slab ? G * kinv + a * (L + G) : G;
}

// 4th-order difference operators over four gathered values.
//   dminus(q[j-2], q[j-1], q[j], q[j+1]),  dplus(q[j-1], q[j], q[j+1], q[j+2])
// (efwi_common.cuh) and the transpose of the quirk-Q1 difference.
__device__ __forceinline__ float dq_t(float p0, float p1, float p2) {
  return EFWI_C1 * p0 - (EFWI_C1 + EFWI_C2) * p1 + EFWI_C2 * p2;
}

// ------------------------------------------------------------ stress stage
// Adjoint "G" values of the stress stage at cell n.
struct GS {
  float ez, ex, ey, xz, xy, yz;
};

__device__ __forceinline__ GS gs_from(float l, float u, float azz, float axx, float ayy, float axz,
                                      float axy, float ayz, float dt) {
  const float l2u = l + 2.0f * u;
  GS r;
  r.ez = (l2u * azz + l * (axx + ayy)) * dt;
  r.ex = (l2u * axx + l * (azz + ayy)) * dt;
  r.ey = (l2u * ayy + l * (azz + axx)) * dt;
  r.xz = u * axz * dt;
  r.xy = u * axy * dt;
  r.yz = u * ayz * dt;
  return r;
}

__device__ __forceinline__ GS gs_at(const ExactArgs &A, int n) {
  return gs_from(A.lam[n], A.mu[n], A.a.szz[n], A.a.sxx[n], A.a.syy[n], A.a.sxz[n], A.a.sxy[n],
                 A.a.syz[n], A.g.dt);
}

// Q of the z-axis terms of the stress stage at (zn, x, y):
// ez (slot 0, integer points), vx_z (slot 1, half), vy_z (slot 2, half).
__device__ __forceinline__ void qs_z(const ExactArgs &A, int zn, int x, int y, float &qez,
                                     float &qvx, float &qvy) {
  const Geo &g = A.g;
  if (zn < 2 || zn > g.nz - 3) { qez = qvx = qvy = 0.f; return; }
  const int n = cell32(g, zn, x, y);
  const GS G = gs_at(A, n);
  if (slab_s(zn, g.nz, g.np)) {
    const int k = psi32_z(g, zn, x, y);
    const float *c = g.cz;
    const int nz = g.nz;
    qez = qpml(G.ez, true, A.lin.z[PSI_VA * (int)g.slab_z + k], c[CK * nz + zn], c[CA * nz + zn]);
    qvx = qpml(G.xz, true, A.lin.z[PSI_VB1 * (int)g.slab_z + k], c[CKH * nz + zn], c[CAH * nz + zn]);
    qvy = qpml(G.yz, true, A.lin.z[PSI_VB2 * (int)g.slab_z + k], c[CKH * nz + zn], c[CAH * nz + zn]);
  } else {
    qez = G.ez; qvx = G.xz; qvy = G.yz;
  }
}

// x-axis terms: ex (slot 0, integer), vz_x (slot 1, half), vy_x (slot 2, half).
__device__ __forceinline__ void qs_x(const ExactArgs &A, int z, int xn, int y, float &qex,
                                     float &qvz, float &qvy) {
  const Geo &g = A.g;
  if (xn < 2 || xn > g.nx - 3) { qex = qvz = qvy = 0.f; return; }
  const int n = cell32(g, z, xn, y);
  const GS G = gs_at(A, n);
  if (slab_s(xn, g.nx, g.np)) {
    const int k = psi32_x(g, z, xn, y);
    const float *c = g.cx;
    const int nx = g.nx;
    qex = qpml(G.ex, true, A.lin.x[PSI_VA * (int)g.slab_x + k], c[CK * nx + xn], c[CA * nx + xn]);
    qvz = qpml(G.xz, true, A.lin.x[PSI_VB1 * (int)g.slab_x + k], c[CKH * nx + xn], c[CAH * nx + xn]);
    qvy = qpml(G.xy, true, A.lin.x[PSI_VB2 * (int)g.slab_x + k], c[CKH * nx + xn], c[CAH * nx + xn]);
  } else {
    qex = G.ex; qvz = G.xz; qvy = G.xy;
  }
}

// y-axis terms: ey (slot 0, integer), vz_y (slot 1, half), vx_y (slot 2, half).
__device__ __forceinline__ void qs_y(const ExactArgs &A, int z, int x, int yn, float &qey,
                                     float &qvz, float &qvx) {
  const Geo &g = A.g;
  if (yn < 2 || yn > g.ny - 3) { qey = qvz = qvx = 0.f; return; }
  const int n = cell32(g, z, x, yn);
  const GS G = gs_at(A, n);
  if (slab_s(yn, g.ny, g.np)) {
    const int k = psi32_y(g, z, x, yn);
    const float *c = g.cy;
    const int ny = g.ny;
    qey = qpml(G.ey, true, A.lin.y[PSI_VA * (int)g.slab_y + k], c[CK * ny + yn], c[CA * ny + yn]);
    qvz = qpml(G.yz, true, A.lin.y[PSI_VB1 * (int)g.slab_y + k], c[CKH * ny + yn], c[CAH * ny + yn]);
    qvx = qpml(G.xy, true, A.lin.y[PSI_VB2 * (int)g.slab_y + k], c[CKH * ny + yn], c[CAH * ny + yn]);
  } else {
    qey = G.ey; qvz = G.yz; qvx = G.xy;
  }
}

// Own cell of the stress stage: G and the Q of its x- and y-axis terms.
__device__ __forceinline__ GS qs_own(const ExactArgs &A, int z, int x, int y, float qx[3],
                                     float qy[3]) {
  const Geo &g = A.g;
  const GS G = gs_at(A, cell32(g, z, x, y));
  if (slab_s(x, g.nx, g.np)) {
    const int k = psi32_x(g, z, x, y);
    const float *c = g.cx;
    const int nx = g.nx;
    qx[0] = qpml(G.ex, true, A.lin.x[PSI_VA * (int)g.slab_x + k], c[CK * nx + x], c[CA * nx + x]);
    qx[1] = qpml(G.xz, true, A.lin.x[PSI_VB1 * (int)g.slab_x + k], c[CKH * nx + x], c[CAH * nx + x]);
    qx[2] = qpml(G.xy, true, A.lin.x[PSI_VB2 * (int)g.slab_x + k], c[CKH * nx + x], c[CAH * nx + x]);
  } else {
    qx[0] = G.ex; qx[1] = G.xz; qx[2] = G.xy;
  }
  if (slab_s(y, g.ny, g.np)) {
    const int k = psi32_y(g, z, x, y);
    const float *c = g.cy;
    const int ny = g.ny;
    qy[0] = qpml(G.ey, true, A.lin.y[PSI_VA * (int)g.slab_y + k], c[CK * ny + y], c[CA * ny + y]);
    qy[1] = qpml(G.yz, true, A.lin.y[PSI_VB1 * (int)g.slab_y + k], c[CKH * ny + y], c[CAH * ny + y]);
    qy[2] = qpml(G.xy, true, A.lin.y[PSI_VB2 * (int)g.slab_y + k], c[CKH * ny + y], c[CAH * ny + y]);
  } else {
    qy[0] = G.ey; qy[1] = G.yz; qy[2] = G.xy;
  }
  return G;
}

// Per z plane, the CTA evaluates the Q of the x-axis terms on its tile plus
// two rows on each side, and of the y-axis terms plus two columns on each
// side, into shared memory (one evaluation per point); the z-axis terms of
// the thread's own column run in a register queue of planes z-2 .. z+2.
// The shared buffers alternate by plane parity, so one barrier per plane
// separates the writes of a plane from the reads of the plane before.
template <int BX>
__global__ void __launch_bounds__(32 * BX) k_adj_stress_exact(ExactArgs A, int zchunk, int nzc) {
  __shared__ float sqx[2][3][BX + 4][32];
  __shared__ float sqy[2][3][BX][36];
  // forward velocities of the images (vz, vx, vy) along x and along y
  __shared__ float sfx[2][3][BX + 4][32];
  __shared__ float sfy[2][3][BX][36];
  const Geo &g = A.g;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int y = blockIdx.x * 32 + tx;
  const int x = blockIdx.y * BX + ty;
  const int z0 = max((int)blockIdx.z * zchunk, 2);
  const int z1 = min((int)blockIdx.z * zchunk + zchunk, g.nz - 2);
  (void)nzc;
  if (z0 >= z1) return;  // uniform over the CTA
  const int np = g.np, nz = g.nz, nx = g.nx, ny = g.ny;
  const int sz = (int)g.sz;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;
  const bool xin = x >= 2 && x <= nx - 3, yin = y >= 2 && y <= ny - 3;
  const bool act = xin && yin;
  const bool xs = slab_s(x, nx, np), ys = slab_s(y, ny, np);
  // halo roles: rows 0, 1, BX+2, BX+3 of sqx (threads ty < 4) and columns
  // 0, 1, 34, 35 of sqy (threads tx < 4)
  const int hr = ty < 2 ? ty : BX + ty;
  const int hxn = (int)blockIdx.y * BX - 2 + hr;
  const int hc = tx < 2 ? tx : 32 + tx;
  const int hyn = (int)blockIdx.x * 32 - 2 + hc;

  float qez[5], qvx[5], qvy[5];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    qez[k] = qvx[k] = qvy[k] = 0.f;
    if (act) qs_z(A, z0 - 2 + k, x, y, qez[k], qvx[k], qvy[k]);
  }
  // z queues of the forward velocities: vz at z-2 .. z+1, vx and vy at z-1 .. z+2
  const float *fvz = A.f.vz, *fvx = A.f.vx, *fvy = A.f.vy;
  float zvz[4] = {0.f, 0.f, 0.f, 0.f}, zvx[4] = {0.f, 0.f, 0.f, 0.f}, zvy[4] = {0.f, 0.f, 0.f, 0.f};
  if (act) {
    const int i0 = cell32(g, z0, x, y);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      zvz[k] = fvz[i0 + (k - 2) * sz];
      zvx[k] = fvx[i0 + (k - 1) * sz];
      zvy[k] = fvy[i0 + (k - 1) * sz];
    }
  }
  const bool hxin = hxn >= 0 && hxn < nx, hyin = hyn >= 0 && hyn < ny;

  int buf = 0;
  for (int z = z0; z < z1; ++z, buf ^= 1) {
    qez[4] = qvx[4] = qvy[4] = 0.f;
    if (act) qs_z(A, z + 2, x, y, qez[4], qvx[4], qvy[4]);
    float ox[3] = {0.f, 0.f, 0.f}, oy[3] = {0.f, 0.f, 0.f};
    GS G{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (act) G = qs_own(A, z, x, y, ox, oy);
    float fo[3] = {0.f, 0.f, 0.f};  // own vz vx vy
    if (act) {
      const int i = cell32(g, z, x, y);
      fo[0] = fvz[i]; fo[1] = fvx[i]; fo[2] = fvy[i];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      sqx[buf][k][ty + 2][tx] = ox[k]; sqy[buf][k][ty][tx + 2] = oy[k];
      sfx[buf][k][ty + 2][tx] = fo[k]; sfy[buf][k][ty][tx + 2] = fo[k];
    }
    if (ty < 4) {
      float h0 = 0.f, h1 = 0.f, h2 = 0.f, f0 = 0.f, f1 = 0.f, f2 = 0.f;
      if (yin) qs_x(A, z, hxn, y, h0, h1, h2);
      if (yin && hxin) {
        const int j = cell32(g, z, hxn, y);
        f0 = fvz[j]; f1 = fvx[j]; f2 = fvy[j];
      }
      sqx[buf][0][hr][tx] = h0; sqx[buf][1][hr][tx] = h1; sqx[buf][2][hr][tx] = h2;
      sfx[buf][0][hr][tx] = f0; sfx[buf][1][hr][tx] = f1; sfx[buf][2][hr][tx] = f2;
    }
    if (tx < 4) {
      float h0 = 0.f, h1 = 0.f, h2 = 0.f, f0 = 0.f, f1 = 0.f, f2 = 0.f;
      if (xin) qs_y(A, z, x, hyn, h0, h1, h2);
      if (xin && hyin) {
        const int j = cell32(g, z, x, hyn);
        f0 = fvz[j]; f1 = fvx[j]; f2 = fvy[j];
      }
      sqy[buf][0][ty][hc] = h0; sqy[buf][1][ty][hc] = h1; sqy[buf][2][ty][hc] = h2;
      sfy[buf][0][ty][hc] = f0; sfy[buf][1][ty][hc] = f1; sfy[buf][2][ty][hc] = f2;
    }
    __syncthreads();

    if (act) {
      const int i = cell32(g, z, x, y);
      const float(*QX)[BX + 4][32] = sqx[buf];
      const float(*QY)[BX][36] = sqy[buf];
      // ---- adjoint velocities
      const float dvz = -dplus(qez[1], qez[2], qez[3], qez[4]) * idz -
                        dminus(QX[1][ty][tx], QX[1][ty + 1][tx], QX[1][ty + 2][tx], QX[1][ty + 3][tx]) * idx -
                        dminus(QY[1][ty][tx], QY[1][ty][tx + 1], QY[1][ty][tx + 2], QY[1][ty][tx + 3]) * idy;
      const float dvx = -dplus(QX[0][ty + 1][tx], QX[0][ty + 2][tx], QX[0][ty + 3][tx], QX[0][ty + 4][tx]) * idx -
                        dminus(qvx[0], qvx[1], qvx[2], qvx[3]) * idz -
                        dminus(QY[2][ty][tx], QY[2][ty][tx + 1], QY[2][ty][tx + 2], QY[2][ty][tx + 3]) * idy;
      const float dvy = -dplus(QY[0][ty][tx + 1], QY[0][ty][tx + 2], QY[0][ty][tx + 3], QY[0][ty][tx + 4]) * idy -
                        dminus(QX[2][ty][tx], QX[2][ty + 1][tx], QX[2][ty + 2][tx], QX[2][ty + 3][tx]) * idx -
                        dminus(qvy[0], qvy[1], qvy[2], qvy[3]) * idz;

      // ---- images from the forward velocities of the same step
      const float(*FX)[BX + 4][32] = sfx[buf];
      const float(*FY)[BX][36] = sfy[buf];
      float ezz = dminus(zvz[0], zvz[1], zvz[2], zvz[3]) * idz;
      float exx = dminus(FX[1][ty][tx], FX[1][ty + 1][tx], FX[1][ty + 2][tx], FX[1][ty + 3][tx]) * idx;
      float eyy = dminus(FY[2][ty][tx], FY[2][ty][tx + 1], FY[2][ty][tx + 2], FY[2][ty][tx + 3]) * idy;
      float dvx_dz = dplus(zvx[0], zvx[1], zvx[2], zvx[3]) * idz;
      float dvy_dz = dplus(zvy[0], zvy[1], zvy[2], zvy[3]) * idz;
      float dvx_dy = dplus(FY[1][ty][tx + 1], FY[1][ty][tx + 2], FY[1][ty][tx + 3], FY[1][ty][tx + 4]) * idy;
      float dvz_dx = dplus(FX[0][ty + 1][tx], FX[0][ty + 2][tx], FX[0][ty + 3][tx], FX[0][ty + 4][tx]) * idx;
      float dvz_dy = dplus(FY[0][ty][tx + 1], FY[0][ty][tx + 2], FY[0][ty][tx + 3], FY[0][ty][tx + 4]) * idy;
      float dvy_dx = dplus(FX[2][ty + 1][tx], FX[2][ty + 2][tx], FX[2][ty + 3][tx], FX[2][ty + 4][tx]) * idx;
      if (slab_s(z, nz, np)) {
        const float *c = g.cz;
        const float Kz = c[CK * nz + z], az = c[CA * nz + z], bz = c[CB * nz + z];
        const float Kzh = c[CKH * nz + z], azh = c[CAH * nz + z], bzh = c[CBH * nz + z];
        const int k = psi32_z(g, z, x, y);
        const float *p = A.ps.z;
        ezz = ezz * Kz + (bz * p[PSI_VA * (int)g.slab_z + k] + az * ezz);
        dvx_dz = dvx_dz * Kzh + (bzh * p[PSI_VB1 * (int)g.slab_z + k] + azh * dvx_dz);
        dvy_dz = dvy_dz * Kzh + (bzh * p[PSI_VB2 * (int)g.slab_z + k] + azh * dvy_dz);
        A.lout.z[PSI_VA * (int)g.slab_z + k] = bz * (A.lin.z[PSI_VA * (int)g.slab_z + k] + G.ez);
        A.lout.z[PSI_VB1 * (int)g.slab_z + k] = bzh * (A.lin.z[PSI_VB1 * (int)g.slab_z + k] + G.xz);
        A.lout.z[PSI_VB2 * (int)g.slab_z + k] = bzh * (A.lin.z[PSI_VB2 * (int)g.slab_z + k] + G.yz);
      }
      if (xs) {
        const float *c = g.cx;
        const float Kx = c[CK * nx + x], ax = c[CA * nx + x], bx = c[CB * nx + x];
        const float Kxh = c[CKH * nx + x], axh = c[CAH * nx + x], bxh = c[CBH * nx + x];
        const int k = psi32_x(g, z, x, y);
        const float *p = A.ps.x;
        exx = exx * Kx + (bx * p[PSI_VA * (int)g.slab_x + k] + ax * exx);
        dvz_dx = dvz_dx * Kxh + (bxh * p[PSI_VB1 * (int)g.slab_x + k] + axh * dvz_dx);
        dvy_dx = dvy_dx * Kxh + (bxh * p[PSI_VB2 * (int)g.slab_x + k] + axh * dvy_dx);
        A.lout.x[PSI_VA * (int)g.slab_x + k] = bx * (A.lin.x[PSI_VA * (int)g.slab_x + k] + G.ex);
        A.lout.x[PSI_VB1 * (int)g.slab_x + k] = bxh * (A.lin.x[PSI_VB1 * (int)g.slab_x + k] + G.xz);
        A.lout.x[PSI_VB2 * (int)g.slab_x + k] = bxh * (A.lin.x[PSI_VB2 * (int)g.slab_x + k] + G.xy);
      }
      if (ys) {
        const float *c = g.cy;
        const float Ky = c[CK * ny + y], ay = c[CA * ny + y], by = c[CB * ny + y];
        const float Kyh = c[CKH * ny + y], ayh = c[CAH * ny + y], byh = c[CBH * ny + y];
        const int k = psi32_y(g, z, x, y);
        const float *p = A.ps.y;
        eyy = eyy * Ky + (by * p[PSI_VA * (int)g.slab_y + k] + ay * eyy);
        dvz_dy = dvz_dy * Kyh + (byh * p[PSI_VB1 * (int)g.slab_y + k] + ayh * dvz_dy);
        dvx_dy = dvx_dy * Kyh + (byh * p[PSI_VB2 * (int)g.slab_y + k] + ayh * dvx_dy);
        A.lout.y[PSI_VA * (int)g.slab_y + k] = by * (A.lin.y[PSI_VA * (int)g.slab_y + k] + G.ey);
        A.lout.y[PSI_VB1 * (int)g.slab_y + k] = byh * (A.lin.y[PSI_VB1 * (int)g.slab_y + k] + G.yz);
        A.lout.y[PSI_VB2 * (int)g.slab_y + k] = byh * (A.lin.y[PSI_VB2 * (int)g.slab_y + k] + G.xy);
      }
      if (A.g0) {
        const float azz = A.a.szz[i], axx = A.a.sxx[i], ayy = A.a.syy[i];
        const float axz = A.a.sxz[i], axy = A.a.sxy[i], ayz = A.a.syz[i];
        A.g0[i] += (azz + axx + ayy) * (ezz + exx + eyy) * dt;
        A.g1[i] += (2.0f * (azz * ezz + axx * exx + ayy * eyy) + axz * (dvx_dz + dvz_dx) +
                    axy * (dvx_dy + dvy_dx) + ayz * (dvy_dz + dvz_dy)) * dt;
      }
      A.a.vz[i] += dvz;
      A.a.vx[i] += dvx;
      A.a.vy[i] += dvy;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) { qez[k] = qez[k + 1]; qvx[k] = qvx[k + 1]; qvy[k] = qvy[k + 1]; }
#pragma unroll
    for (int k = 0; k < 3; ++k) { zvz[k] = zvz[k + 1]; zvx[k] = zvx[k + 1]; zvy[k] = zvy[k + 1]; }
    if (act && z + 1 < z1) {
      const int i = cell32(g, z, x, y);
      zvz[3] = fvz[i + 2 * sz];
      zvx[3] = fvx[i + 3 * sz];
      zvy[3] = fvy[i + 3 * sz];
    }
  }
}

// ---------------------------------------------------------- velocity stage
// G of the velocity stage at cell n: adjoint velocity * buoyancy * dt.
__device__ __forceinline__ void gv_at(const ExactArgs &A, int n, float &gz, float &gx,
                                      float &gy) {
  const float s = A.buoy[n] * A.g.dt;
  gz = A.a.vz[n] * s;
  gx = A.a.vx[n] * s;
  gy = A.a.vy[n] * s;
}

// z-axis terms of the velocity stage at (zn, x, y):
// vz <- szz (slot 3, half), vx <- sxz (slot 4, integer), vy <- syz (slot 5, integer).
__device__ __forceinline__ void qv_z(const ExactArgs &A, int zn, int x, int y, float &qzz,
                                     float &qxz, float &qyz) {
  const Geo &g = A.g;
  if (zn < 2 || zn > g.nz - 3) { qzz = qxz = qyz = 0.f; return; }
  float gz, gx, gy;
  gv_at(A, cell32(g, zn, x, y), gz, gx, gy);
  if (slab_s(zn, g.nz, g.np)) {
    const int k = psi32_z(g, zn, x, y);
    const float *c = g.cz;
    const int nz = g.nz;
    qzz = qpml(gz, true, A.lin.z[PSI_SAA * (int)g.slab_z + k], c[CKH * nz + zn], c[CAH * nz + zn]);
    qxz = qpml(gx, true, A.lin.z[PSI_SAB1 * (int)g.slab_z + k], c[CK * nz + zn], c[CA * nz + zn]);
    qyz = qpml(gy, true, A.lin.z[PSI_SAB2 * (int)g.slab_z + k], c[CK * nz + zn], c[CA * nz + zn]);
  } else {
    qzz = gz; qxz = gx; qyz = gy;
  }
}

// x-axis terms (quirk-Q2 slabs): vz <- sxz (slot 4, integer), vx <- sxx
// (slot 3, half), vy <- sxy (slot 5, integer).
__device__ __forceinline__ void qv_x(const ExactArgs &A, int z, int xn, int y, float &qxz,
                                     float &qxx, float &qxy) {
  const Geo &g = A.g;
  if (xn < 2 || xn > g.nx - 3) { qxz = qxx = qxy = 0.f; return; }
  float gz, gx, gy;
  gv_at(A, cell32(g, z, xn, y), gz, gx, gy);
  if (slab_v(xn, g.nx, g.np)) {
    const int k = psi32_x(g, z, xn, y);
    const float *c = g.cx;
    const int nx = g.nx;
    qxz = qpml(gz, true, A.lin.x[PSI_SAB1 * (int)g.slab_x + k], c[CK * nx + xn], c[CA * nx + xn]);
    qxx = qpml(gx, true, A.lin.x[PSI_SAA * (int)g.slab_x + k], c[CKH * nx + xn], c[CAH * nx + xn]);
    qxy = qpml(gy, true, A.lin.x[PSI_SAB2 * (int)g.slab_x + k], c[CK * nx + xn], c[CA * nx + xn]);
  } else {
    qxz = gz; qxx = gx; qxy = gy;
  }
}

// y-axis terms (quirk-Q2 slabs): vz <- syz (slot 4, integer), vx <- sxy
// (slot 5, integer), vy <- syy (slot 3, half).
__device__ __forceinline__ void qv_y(const ExactArgs &A, int z, int x, int yn, float &qyz,
                                     float &qxy, float &qyy) {
  const Geo &g = A.g;
  if (yn < 2 || yn > g.ny - 3) { qyz = qxy = qyy = 0.f; return; }
  float gz, gx, gy;
  gv_at(A, cell32(g, z, x, yn), gz, gx, gy);
  if (slab_v(yn, g.ny, g.np)) {
    const int k = psi32_y(g, z, x, yn);
    const float *c = g.cy;
    const int ny = g.ny;
    qyz = qpml(gz, true, A.lin.y[PSI_SAB1 * (int)g.slab_y + k], c[CK * ny + yn], c[CA * ny + yn]);
    qxy = qpml(gx, true, A.lin.y[PSI_SAB2 * (int)g.slab_y + k], c[CK * ny + yn], c[CA * ny + yn]);
    qyy = qpml(gy, true, A.lin.y[PSI_SAA * (int)g.slab_y + k], c[CKH * ny + yn], c[CAH * ny + yn]);
  } else {
    qyz = gz; qxy = gx; qyy = gy;
  }
}

// Own cell of the velocity stage: G and the Q of its x- and y-axis terms
// (qx: vz <- sxz, vx <- sxx, vy <- sxy; qy: vz <- syz, vx <- sxy, vy <- syy).
__device__ __forceinline__ void qv_own(const ExactArgs &A, int z, int x, int y, float &gz,
                                       float &gx, float &gy, float qx[3], float qy[3]) {
  const Geo &g = A.g;
  gv_at(A, cell32(g, z, x, y), gz, gx, gy);
  if (slab_v(x, g.nx, g.np)) {
    const int k = psi32_x(g, z, x, y);
    const float *c = g.cx;
    const int nx = g.nx;
    qx[0] = qpml(gz, true, A.lin.x[PSI_SAB1 * (int)g.slab_x + k], c[CK * nx + x], c[CA * nx + x]);
    qx[1] = qpml(gx, true, A.lin.x[PSI_SAA * (int)g.slab_x + k], c[CKH * nx + x], c[CAH * nx + x]);
    qx[2] = qpml(gy, true, A.lin.x[PSI_SAB2 * (int)g.slab_x + k], c[CK * nx + x], c[CA * nx + x]);
  } else {
    qx[0] = gz; qx[1] = gx; qx[2] = gy;
  }
  if (slab_v(y, g.ny, g.np)) {
    const int k = psi32_y(g, z, x, y);
    const float *c = g.cy;
    const int ny = g.ny;
    qy[0] = qpml(gz, true, A.lin.y[PSI_SAB1 * (int)g.slab_y + k], c[CK * ny + y], c[CA * ny + y]);
    qy[1] = qpml(gx, true, A.lin.y[PSI_SAB2 * (int)g.slab_y + k], c[CK * ny + y], c[CA * ny + y]);
    qy[2] = qpml(gy, true, A.lin.y[PSI_SAA * (int)g.slab_y + k], c[CKH * ny + y], c[CAH * ny + y]);
  } else {
    qy[0] = gz; qy[1] = gx; qy[2] = gy;
  }
}

// Same staging as k_adj_stress_exact.
template <int BX>
__global__ void __launch_bounds__(32 * BX) k_adj_velocity_exact(ExactArgs A, int zchunk, int nzc) {
  __shared__ float sqx[2][3][BX + 4][32];
  __shared__ float sqy[2][3][BX][36];
  // forward stresses of the image: sxz, sxx, sxy along x; syz, sxy, syy along y
  __shared__ float sfx[2][3][BX + 4][32];
  __shared__ float sfy[2][3][BX][36];
  const Geo &g = A.g;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int y = blockIdx.x * 32 + tx;
  const int x = blockIdx.y * BX + ty;
  const int z0 = max((int)blockIdx.z * zchunk, 2);
  const int z1 = min((int)blockIdx.z * zchunk + zchunk, g.nz - 2);
  (void)nzc;
  if (z0 >= z1) return;  // uniform over the CTA
  const int np = g.np, nz = g.nz, nx = g.nx, ny = g.ny;
  const int sz = (int)g.sz;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;
  const bool xin = x >= 2 && x <= nx - 3, yin = y >= 2 && y <= ny - 3;
  const bool act = xin && yin;
  const bool xs = slab_v(x, nx, np), ys = slab_v(y, ny, np);
  const int hr = ty < 2 ? ty : BX + ty;
  const int hxn = (int)blockIdx.y * BX - 2 + hr;
  const int hc = tx < 2 ? tx : 32 + tx;
  const int hyn = (int)blockIdx.x * 32 - 2 + hc;

  float qzz[5], qxz[5], qyz[5];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    qzz[k] = qxz[k] = qyz[k] = 0.f;
    if (act) qv_z(A, z0 - 2 + k, x, y, qzz[k], qxz[k], qyz[k]);
  }
  // z queues of the forward stresses: szz at z-1 .. z+2, sxz and syz at z-2 .. z+1
  const float *fszz = A.f.szz, *fsxx = A.f.sxx, *fsyy = A.f.syy;
  const float *fsxz = A.f.sxz, *fsxy = A.f.sxy, *fsyz = A.f.syz;
  float zszz[4] = {0.f, 0.f, 0.f, 0.f}, zsxz[4] = {0.f, 0.f, 0.f, 0.f}, zsyz[4] = {0.f, 0.f, 0.f, 0.f};
  if (act) {
    const int i0 = cell32(g, z0, x, y);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      zszz[k] = fszz[i0 + (k - 1) * sz];
      zsxz[k] = fsxz[i0 + (k - 2) * sz];
      zsyz[k] = fsyz[i0 + (k - 2) * sz];
    }
  }
  const bool hxin = hxn >= 0 && hxn < nx, hyin = hyn >= 0 && hyn < ny;

  int buf = 0;
  for (int z = z0; z < z1; ++z, buf ^= 1) {
    qzz[4] = qxz[4] = qyz[4] = 0.f;
    if (act) qv_z(A, z + 2, x, y, qzz[4], qxz[4], qyz[4]);
    float ox[3] = {0.f, 0.f, 0.f}, oy[3] = {0.f, 0.f, 0.f};
    float gz = 0.f, gx = 0.f, gy = 0.f;
    if (act) qv_own(A, z, x, y, gz, gx, gy, ox, oy);
    float fo[5] = {0.f, 0.f, 0.f, 0.f, 0.f};  // own sxz sxx sxy syz syy
    if (act) {
      const int i = cell32(g, z, x, y);
      fo[0] = fsxz[i]; fo[1] = fsxx[i]; fo[2] = fsxy[i]; fo[3] = fsyz[i]; fo[4] = fsyy[i];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) { sqx[buf][k][ty + 2][tx] = ox[k]; sqy[buf][k][ty][tx + 2] = oy[k]; }
    sfx[buf][0][ty + 2][tx] = fo[0]; sfx[buf][1][ty + 2][tx] = fo[1]; sfx[buf][2][ty + 2][tx] = fo[2];
    sfy[buf][0][ty][tx + 2] = fo[3]; sfy[buf][1][ty][tx + 2] = fo[2]; sfy[buf][2][ty][tx + 2] = fo[4];
    if (ty < 4) {
      float h0 = 0.f, h1 = 0.f, h2 = 0.f, f0 = 0.f, f1 = 0.f, f2 = 0.f;
      if (yin) qv_x(A, z, hxn, y, h0, h1, h2);
      if (yin && hxin) {
        const int j = cell32(g, z, hxn, y);
        f0 = fsxz[j]; f1 = fsxx[j]; f2 = fsxy[j];
      }
      sqx[buf][0][hr][tx] = h0; sqx[buf][1][hr][tx] = h1; sqx[buf][2][hr][tx] = h2;
      sfx[buf][0][hr][tx] = f0; sfx[buf][1][hr][tx] = f1; sfx[buf][2][hr][tx] = f2;
    }
    if (tx < 4) {
      float h0 = 0.f, h1 = 0.f, h2 = 0.f, f0 = 0.f, f1 = 0.f, f2 = 0.f;
      if (xin) qv_y(A, z, x, hyn, h0, h1, h2);
      if (xin && hyin) {
        const int j = cell32(g, z, x, hyn);
        f0 = fsyz[j]; f1 = fsxy[j]; f2 = fsyy[j];
      }
      sqy[buf][0][ty][hc] = h0; sqy[buf][1][ty][hc] = h1; sqy[buf][2][ty][hc] = h2;
      sfy[buf][0][ty][hc] = f0; sfy[buf][1][ty][hc] = f1; sfy[buf][2][ty][hc] = f2;
    }
    __syncthreads();

    if (act) {
      const int i = cell32(g, z, x, y);
      const float(*QX)[BX + 4][32] = sqx[buf];
      const float(*QY)[BX][36] = sqy[buf];
      // ---- adjoint stresses (x: 0 vz<-sxz, 1 vx<-sxx, 2 vy<-sxy;
      //                        y: 0 vz<-syz, 1 vx<-sxy, 2 vy<-syy)
      const float dszz = -dminus(qzz[0], qzz[1], qzz[2], qzz[3]) * idz;
      const float dsxx = -dminus(QX[1][ty][tx], QX[1][ty + 1][tx], QX[1][ty + 2][tx], QX[1][ty + 3][tx]) * idx;
      const float dsyy = -dminus(QY[2][ty][tx], QY[2][ty][tx + 1], QY[2][ty][tx + 2], QY[2][ty][tx + 3]) * idy;
      const float dsxz = -dplus(QX[0][ty + 1][tx], QX[0][ty + 2][tx], QX[0][ty + 3][tx], QX[0][ty + 4][tx]) * idx -
                         dplus(qxz[1], qxz[2], qxz[3], qxz[4]) * idz;
      const float dsyz = -dplus(QY[0][ty][tx + 1], QY[0][ty][tx + 2], QY[0][ty][tx + 3], QY[0][ty][tx + 4]) * idy -
                         dplus(qyz[1], qyz[2], qyz[3], qyz[4]) * idz;
      const float dsxy = -dplus(QY[1][ty][tx + 1], QY[1][ty][tx + 2], QY[1][ty][tx + 3], QY[1][ty][tx + 4]) * idy +
                         dq_t(QX[2][ty + 2][tx], QX[2][ty + 3][tx], QX[2][ty + 4][tx]) * idx;

      // ---- buoyancy image from the forward stresses of the same step
      const float(*FX)[BX + 4][32] = sfx[buf];
      const float(*FY)[BX][36] = sfy[buf];
      float dszz_dz = dplus(zszz[0], zszz[1], zszz[2], zszz[3]) * idz;
      float dsxz_dx = dminus(FX[0][ty][tx], FX[0][ty + 1][tx], FX[0][ty + 2][tx], FX[0][ty + 3][tx]) * idx;
      float dsyz_dy = dminus(FY[0][ty][tx], FY[0][ty][tx + 1], FY[0][ty][tx + 2], FY[0][ty][tx + 3]) * idy;
      float dsxz_dz = dminus(zsxz[0], zsxz[1], zsxz[2], zsxz[3]) * idz;
      float dsxx_dx = dplus(FX[1][ty + 1][tx], FX[1][ty + 2][tx], FX[1][ty + 3][tx], FX[1][ty + 4][tx]) * idx;
      float dsxy_dy = dminus(FY[1][ty][tx], FY[1][ty][tx + 1], FY[1][ty][tx + 2], FY[1][ty][tx + 3]) * idy;
      float dsyz_dz = dminus(zsyz[0], zsyz[1], zsyz[2], zsyz[3]) * idz;
      const float sxy0 = FX[2][ty + 2][tx], sxym1 = FX[2][ty + 1][tx], sxym2 = FX[2][ty][tx];
      float dsxy_dx = (EFWI_C1 * (sxy0 - sxym1) - EFWI_C2 * (sxym1 - sxym2)) * idx;
      float dsyy_dy = dplus(FY[2][ty][tx + 1], FY[2][ty][tx + 2], FY[2][ty][tx + 3], FY[2][ty][tx + 4]) * idy;
      if (slab_s(z, nz, np)) {
        const float *c = g.cz;
        const float Kz = c[CK * nz + z], bz = c[CB * nz + z], Kzh = c[CKH * nz + z], bzh = c[CBH * nz + z];
        const int k = psi32_z(g, z, x, y);
        const float *p = A.ps.z;
        dszz_dz = dszz_dz * Kzh + p[PSI_SAA * (int)g.slab_z + k];
        dsxz_dz = dsxz_dz * Kz + p[PSI_SAB1 * (int)g.slab_z + k];
        dsyz_dz = dsyz_dz * Kz + p[PSI_SAB2 * (int)g.slab_z + k];
        A.lout.z[PSI_SAA * (int)g.slab_z + k] = bzh * (A.lin.z[PSI_SAA * (int)g.slab_z + k] + gz);
        A.lout.z[PSI_SAB1 * (int)g.slab_z + k] = bz * (A.lin.z[PSI_SAB1 * (int)g.slab_z + k] + gx);
        A.lout.z[PSI_SAB2 * (int)g.slab_z + k] = bz * (A.lin.z[PSI_SAB2 * (int)g.slab_z + k] + gy);
      }
      if (xs) {
        const float *c = g.cx;
        const float Kx = c[CK * nx + x], bx = c[CB * nx + x], Kxh = c[CKH * nx + x], bxh = c[CBH * nx + x];
        const int k = psi32_x(g, z, x, y);
        const float *p = A.ps.x;
        dsxz_dx = dsxz_dx * Kx + p[PSI_SAB1 * (int)g.slab_x + k];
        dsxx_dx = dsxx_dx * Kxh + p[PSI_SAA * (int)g.slab_x + k];
        dsxy_dx = dsxy_dx * Kx + p[PSI_SAB2 * (int)g.slab_x + k];
        A.lout.x[PSI_SAB1 * (int)g.slab_x + k] = bx * (A.lin.x[PSI_SAB1 * (int)g.slab_x + k] + gz);
        A.lout.x[PSI_SAA * (int)g.slab_x + k] = bxh * (A.lin.x[PSI_SAA * (int)g.slab_x + k] + gx);
        A.lout.x[PSI_SAB2 * (int)g.slab_x + k] = bx * (A.lin.x[PSI_SAB2 * (int)g.slab_x + k] + gy);
      }
      if (ys) {
        const float *c = g.cy;
        const float Ky = c[CK * ny + y], by = c[CB * ny + y], Kyh = c[CKH * ny + y], byh = c[CBH * ny + y];
        const int k = psi32_y(g, z, x, y);
        const float *p = A.ps.y;
        dsyz_dy = dsyz_dy * Ky + p[PSI_SAB1 * (int)g.slab_y + k];
        dsxy_dy = dsxy_dy * Ky + p[PSI_SAB2 * (int)g.slab_y + k];
        dsyy_dy = dsyy_dy * Kyh + p[PSI_SAA * (int)g.slab_y + k];
        A.lout.y[PSI_SAB1 * (int)g.slab_y + k] = by * (A.lin.y[PSI_SAB1 * (int)g.slab_y + k] + gz);
        A.lout.y[PSI_SAB2 * (int)g.slab_y + k] = by * (A.lin.y[PSI_SAB2 * (int)g.slab_y + k] + gx);
        A.lout.y[PSI_SAA * (int)g.slab_y + k] = byh * (A.lin.y[PSI_SAA * (int)g.slab_y + k] + gy);
      }
      if (A.g0) {
        A.g0[i] += (A.a.vz[i] * (dszz_dz + dsxz_dx + dsyz_dy) + A.a.vx[i] * (dsxz_dz + dsxx_dx + dsxy_dy) +
                    A.a.vy[i] * (dsyz_dz + dsxy_dx + dsyy_dy)) * dt;
      }
      A.a.szz[i] += dszz;
      A.a.sxx[i] += dsxx;
      A.a.syy[i] += dsyy;
      A.a.sxz[i] += dsxz;
      A.a.syz[i] += dsyz;
      A.a.sxy[i] += dsxy;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) { qzz[k] = qzz[k + 1]; qxz[k] = qxz[k + 1]; qyz[k] = qyz[k + 1]; }
#pragma unroll
    for (int k = 0; k < 3; ++k) { zszz[k] = zszz[k + 1]; zsxz[k] = zsxz[k + 1]; zsyz[k] = zsyz[k + 1]; }
    if (act && z + 1 < z1) {
      const int i = cell32(g, z, x, y);
      zszz[3] = fszz[i + 3 * sz];
      zsxz[3] = fsxz[i + 2 * sz];
      zsyz[3] = fsyz[i + 2 * sz];
    }
  }
}


// ------------------------------------------------ bulk-copy staged variants
// The same transposes with every plane's operands staged by bulk tensor
// copies (efwi_tma.cuh) into a ring of R plane slots of halo boxes,
// 40 (y) x (TX + 4) (x): the inputs of G and the forward fields of the
// images.  The CTA's ring runs over planes z0-2 .. z1+1; computing plane z
// reads the slot of z (x/y neighbours, own cell) and the centres of z+1 and
// z+2 (the z-stencil queue heads), so three slots stay resident and R-3
// are in flight.  The Q of the tile and its halo are formed from the slot
// (the kernels above form the halo's from global loads), the operands of the
// read-modify-writes are loaded before the ring wait, and the per-cell
// arithmetic is the same expression as above, so results are bitwise equal.

// Slot fields of the stress-stage transpose.
enum { ES_ZZ = 0, ES_XX, ES_YY, ES_XZ, ES_XY, ES_YZ, ES_L, ES_M, ES_VZ, ES_VX, ES_VY, ES_N };
// Slot fields of the velocity-stage transpose.
enum { EV_VZ = 0, EV_VX, EV_VY, EV_B, EV_SXZ, EV_SXX, EV_SXY, EV_SYZ, EV_SYY, EV_SZZ, EV_N };

template <class Ring>
__device__ __forceinline__ GS gs_slot(const Ring &ring, int j, int o, float dt) {
  return gs_from(ring.halo(j, ES_L)[o], ring.halo(j, ES_M)[o], ring.halo(j, ES_ZZ)[o],
                 ring.halo(j, ES_XX)[o], ring.halo(j, ES_YY)[o], ring.halo(j, ES_XZ)[o],
                 ring.halo(j, ES_XY)[o], ring.halo(j, ES_YZ)[o], dt);
}

// Q of the z-axis terms of the stress stage at plane zn from G (qs_z).
__device__ __forceinline__ void qs_z_of(const ExactArgs &A, const GS &G, int zn, int x, int y,
                                        float &qez, float &qvx, float &qvy) {
  const Geo &g = A.g;
  if (zn < 2 || zn > g.nz - 3) { qez = qvx = qvy = 0.f; return; }
  if (slab_s(zn, g.nz, g.np)) {
    const int k = psi32_z(g, zn, x, y);
    const float *c = g.cz;
    const int nz = g.nz;
    qez = qpml(G.ez, true, A.lin.z[PSI_VA * (int)g.slab_z + k], c[CK * nz + zn], c[CA * nz + zn]);
    qvx = qpml(G.xz, true, A.lin.z[PSI_VB1 * (int)g.slab_z + k], c[CKH * nz + zn], c[CAH * nz + zn]);
    qvy = qpml(G.yz, true, A.lin.z[PSI_VB2 * (int)g.slab_z + k], c[CKH * nz + zn], c[CAH * nz + zn]);
  } else {
    qez = G.ez; qvx = G.xz; qvy = G.yz;
  }
}

// x-axis terms at row xn from G (qs_x).
__device__ __forceinline__ void qs_x_of(const ExactArgs &A, const GS &G, int z, int xn, int y,
                                        float &qex, float &qvz, float &qvy) {
  const Geo &g = A.g;
  if (xn < 2 || xn > g.nx - 3) { qex = qvz = qvy = 0.f; return; }
  if (slab_s(xn, g.nx, g.np)) {
    const int k = psi32_x(g, z, xn, y);
    const float *c = g.cx;
    const int nx = g.nx;
    qex = qpml(G.ex, true, A.lin.x[PSI_VA * (int)g.slab_x + k], c[CK * nx + xn], c[CA * nx + xn]);
    qvz = qpml(G.xz, true, A.lin.x[PSI_VB1 * (int)g.slab_x + k], c[CKH * nx + xn], c[CAH * nx + xn]);
    qvy = qpml(G.xy, true, A.lin.x[PSI_VB2 * (int)g.slab_x + k], c[CKH * nx + xn], c[CAH * nx + xn]);
  } else {
    qex = G.ex; qvz = G.xz; qvy = G.xy;
  }
}

// y-axis terms at column yn from G (qs_y).
__device__ __forceinline__ void qs_y_of(const ExactArgs &A, const GS &G, int z, int x, int yn,
                                        float &qey, float &qvz, float &qvx) {
  const Geo &g = A.g;
  if (yn < 2 || yn > g.ny - 3) { qey = qvz = qvx = 0.f; return; }
  if (slab_s(yn, g.ny, g.np)) {
    const int k = psi32_y(g, z, x, yn);
    const float *c = g.cy;
    const int ny = g.ny;
    qey = qpml(G.ey, true, A.lin.y[PSI_VA * (int)g.slab_y + k], c[CK * ny + yn], c[CA * ny + yn]);
    qvz = qpml(G.yz, true, A.lin.y[PSI_VB1 * (int)g.slab_y + k], c[CKH * ny + yn], c[CAH * ny + yn]);
    qvx = qpml(G.xy, true, A.lin.y[PSI_VB2 * (int)g.slab_y + k], c[CKH * ny + yn], c[CAH * ny + yn]);
  } else {
    qey = G.ey; qvz = G.yz; qvx = G.xy;
  }
}

template <int TX, int R, int MINB>
__global__ void __launch_bounds__(32 * TX, MINB)
k_adj_stress_tma(const __grid_constant__ Maps<ES_N> maps, ExactArgs A, int zchunk, int *status) {
  using Ring = PlaneRing<ES_N, 0, 0, TX, R>;
  __shared__ float sqx[3][TX + 4][32];
  __shared__ float sqy[3][TX][36];
  extern __shared__ __align__(128) unsigned char smem[];
  Ring ring;
  ring.bind(smem);
  const Geo &g = A.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int y0 = blockIdx.x * 32, x0 = blockIdx.y * TX;
  const int y = y0 + tx, x = x0 + ty;
  const int z0 = max((int)blockIdx.z * zchunk, 2);
  const int z1 = min((int)blockIdx.z * zchunk + zchunk, g.nz - 2);
  if (z0 >= z1) return;  // uniform over the CTA, before any barrier
  const int nq = z1 - z0, nj = nq + 4;  // ring planes z0-2 .. z1+1
  if (tid == 0) ring.init();
  __syncthreads();
  if (tid == 0)
    for (int j = 0; j < nj && j < R; ++j) ring.issue(maps, j, y0, x0, z0 - 2 + j, z0 - 2 + j);

  const int np = g.np, nz = g.nz, nx = g.nx, ny = g.ny;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;
  const bool xin = x >= 2 && x <= nx - 3, yin = y >= 2 && y <= ny - 3;
  const bool act = xin && yin;
  const bool xs = slab_s(x, nx, np), ys = slab_s(y, ny, np);
  // halo roles: rows 0, 1, TX+2, TX+3 of sqx (threads ty < 4) and columns
  // 0, 1, 34, 35 of sqy (threads tx < 4)
  const int hr = ty < 2 ? ty : TX + ty;
  const int hxn = x0 - 2 + hr;
  const int hc = tx < 2 ? tx : 32 + tx;
  const int hyn = y0 - 2 + hc;
  const int own = (ty + TMA_HX) * TMA_BOXY + tx + TMA_HY;  // own cell in a box
  const int hro = hr * TMA_BOXY + tx + TMA_HY;             // halo row cell
  const int hco = (ty + TMA_HX) * TMA_BOXY + hc + 2;       // halo column cell

  bool ok = true;
  for (int j = 0; j < 4; ++j) ok = ring.wait(j) && ok;
  // queues: Q_z of planes z-2 .. z+2 (head z+2 per plane); forward vz at
  // z-2 .. z+1, vx and vy at z-1 .. z+2 (heads z+1 and z+2 per plane)
  float qez[5] = {}, qvx[5] = {}, qvy[5] = {};
  float zvz[4] = {}, zvx[4] = {}, zvy[4] = {};
  if (ok && act) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
      qs_z_of(A, gs_slot(ring, k, own, dt), z0 - 2 + k, x, y, qez[k], qvx[k], qvy[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      zvz[k] = ring.halo(k, ES_VZ)[own];
      zvx[k] = ring.halo(k + 1, ES_VX)[own];
      zvy[k] = ring.halo(k + 1, ES_VY)[own];
    }
  }
  if (__syncthreads_or(!ok)) {
    ring_abort(ring, 0, min(nj, R), R, tid, status);
    return;
  }
  // slots 0 and 1 (planes z0-2, z0-1) are free after the queue fill
  if (tid == 0)
    for (int j = R; j < R + 2 && j < nj; ++j) {
      fence_proxy_async_smem();
      ring.issue(maps, j, y0, x0, z0 - 2 + j, z0 - 2 + j);
    }

  for (int q = 0; q < nq; ++q) {
    const int z = z0 + q, jc = q + 2;
    const int i = act ? cell32(g, z, x, y) : 0;
    float av0 = 0.f, av1 = 0.f, av2 = 0.f, gi0 = 0.f, gi1 = 0.f;
    if (act) {  // read-modify-write operands, before the wait
      av0 = A.a.vz[i]; av1 = A.a.vx[i]; av2 = A.a.vy[i];
      if (A.g0) { gi0 = A.g0[i]; gi1 = A.g1[i]; }
    }
    const bool got = ring.wait(q + 4);
    GS G{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (got) {
      qez[4] = qvx[4] = qvy[4] = 0.f;
      if (act) qs_z_of(A, gs_slot(ring, q + 4, own, dt), z + 2, x, y, qez[4], qvx[4], qvy[4]);
      zvz[3] = ring.halo(q + 3, ES_VZ)[own];
      zvx[3] = ring.halo(q + 4, ES_VX)[own];
      zvy[3] = ring.halo(q + 4, ES_VY)[own];
      float ox[3] = {0.f, 0.f, 0.f}, oy[3] = {0.f, 0.f, 0.f};
      if (act) {  // qs_own
        G = gs_slot(ring, jc, own, dt);
        qs_x_of(A, G, z, x, y, ox[0], ox[1], ox[2]);
        qs_y_of(A, G, z, x, y, oy[0], oy[1], oy[2]);
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) { sqx[k][ty + 2][tx] = ox[k]; sqy[k][ty][tx + 2] = oy[k]; }
      if (ty < 4) {
        float h0 = 0.f, h1 = 0.f, h2 = 0.f;
        if (yin) qs_x_of(A, gs_slot(ring, jc, hro, dt), z, hxn, y, h0, h1, h2);
        sqx[0][hr][tx] = h0; sqx[1][hr][tx] = h1; sqx[2][hr][tx] = h2;
      }
      if (tx < 4) {
        float h0 = 0.f, h1 = 0.f, h2 = 0.f;
        if (xin) qs_y_of(A, gs_slot(ring, jc, hco, dt), z, x, hyn, h0, h1, h2);
        sqy[0][ty][hc] = h0; sqy[1][ty][hc] = h1; sqy[2][ty][hc] = h2;
      }
    }
    __syncthreads();
    if (got && act) {
      const float(*QX)[TX + 4][32] = sqx;
      const float(*QY)[TX][36] = sqy;
      // ---- adjoint velocities
      const float dvz = -dplus(qez[1], qez[2], qez[3], qez[4]) * idz -
                        dminus(QX[1][ty][tx], QX[1][ty + 1][tx], QX[1][ty + 2][tx], QX[1][ty + 3][tx]) * idx -
                        dminus(QY[1][ty][tx], QY[1][ty][tx + 1], QY[1][ty][tx + 2], QY[1][ty][tx + 3]) * idy;
      const float dvx = -dplus(QX[0][ty + 1][tx], QX[0][ty + 2][tx], QX[0][ty + 3][tx], QX[0][ty + 4][tx]) * idx -
                        dminus(qvx[0], qvx[1], qvx[2], qvx[3]) * idz -
                        dminus(QY[2][ty][tx], QY[2][ty][tx + 1], QY[2][ty][tx + 2], QY[2][ty][tx + 3]) * idy;
      const float dvy = -dplus(QY[0][ty][tx + 1], QY[0][ty][tx + 2], QY[0][ty][tx + 3], QY[0][ty][tx + 4]) * idy -
                        dminus(QX[2][ty][tx], QX[2][ty + 1][tx], QX[2][ty + 2][tx], QX[2][ty + 3][tx]) * idx -
                        dminus(qvy[0], qvy[1], qvy[2], qvy[3]) * idz;

      // ---- images from the forward velocities of the same step; box row r
      // is x = x0 - 2 + r, box column c is y = y0 - 4 + c
      const BoxView fz{ring.halo(jc, ES_VZ) + own}, fx{ring.halo(jc, ES_VX) + own},
          fy{ring.halo(jc, ES_VY) + own};
      float ezz = dminus(zvz[0], zvz[1], zvz[2], zvz[3]) * idz;
      float exx = dminus(fx.x(-2), fx.x(-1), fx.c(), fx.x(1)) * idx;
      float eyy = dminus(fy.y(-2), fy.y(-1), fy.c(), fy.y(1)) * idy;
      float dvx_dz = dplus(zvx[0], zvx[1], zvx[2], zvx[3]) * idz;
      float dvy_dz = dplus(zvy[0], zvy[1], zvy[2], zvy[3]) * idz;
      float dvx_dy = dplus(fx.y(-1), fx.c(), fx.y(1), fx.y(2)) * idy;
      float dvz_dx = dplus(fz.x(-1), fz.c(), fz.x(1), fz.x(2)) * idx;
      float dvz_dy = dplus(fz.y(-1), fz.c(), fz.y(1), fz.y(2)) * idy;
      float dvy_dx = dplus(fy.x(-1), fy.c(), fy.x(1), fy.x(2)) * idx;
      if (slab_s(z, nz, np)) {
        const float *c = g.cz;
        const float Kz = c[CK * nz + z], az = c[CA * nz + z], bz = c[CB * nz + z];
        const float Kzh = c[CKH * nz + z], azh = c[CAH * nz + z], bzh = c[CBH * nz + z];
        const int k = psi32_z(g, z, x, y);
        const float *p = A.ps.z;
        ezz = ezz * Kz + (bz * p[PSI_VA * (int)g.slab_z + k] + az * ezz);
        dvx_dz = dvx_dz * Kzh + (bzh * p[PSI_VB1 * (int)g.slab_z + k] + azh * dvx_dz);
        dvy_dz = dvy_dz * Kzh + (bzh * p[PSI_VB2 * (int)g.slab_z + k] + azh * dvy_dz);
        A.lout.z[PSI_VA * (int)g.slab_z + k] = bz * (A.lin.z[PSI_VA * (int)g.slab_z + k] + G.ez);
        A.lout.z[PSI_VB1 * (int)g.slab_z + k] = bzh * (A.lin.z[PSI_VB1 * (int)g.slab_z + k] + G.xz);
        A.lout.z[PSI_VB2 * (int)g.slab_z + k] = bzh * (A.lin.z[PSI_VB2 * (int)g.slab_z + k] + G.yz);
      }
      if (xs) {
        const float *c = g.cx;
        const float Kx = c[CK * nx + x], ax = c[CA * nx + x], bx = c[CB * nx + x];
        const float Kxh = c[CKH * nx + x], axh = c[CAH * nx + x], bxh = c[CBH * nx + x];
        const int k = psi32_x(g, z, x, y);
        const float *p = A.ps.x;
        exx = exx * Kx + (bx * p[PSI_VA * (int)g.slab_x + k] + ax * exx);
        dvz_dx = dvz_dx * Kxh + (bxh * p[PSI_VB1 * (int)g.slab_x + k] + axh * dvz_dx);
        dvy_dx = dvy_dx * Kxh + (bxh * p[PSI_VB2 * (int)g.slab_x + k] + axh * dvy_dx);
        A.lout.x[PSI_VA * (int)g.slab_x + k] = bx * (A.lin.x[PSI_VA * (int)g.slab_x + k] + G.ex);
        A.lout.x[PSI_VB1 * (int)g.slab_x + k] = bxh * (A.lin.x[PSI_VB1 * (int)g.slab_x + k] + G.xz);
        A.lout.x[PSI_VB2 * (int)g.slab_x + k] = bxh * (A.lin.x[PSI_VB2 * (int)g.slab_x + k] + G.xy);
      }
      if (ys) {
        const float *c = g.cy;
        const float Ky = c[CK * ny + y], ay = c[CA * ny + y], by = c[CB * ny + y];
        const float Kyh = c[CKH * ny + y], ayh = c[CAH * ny + y], byh = c[CBH * ny + y];
        const int k = psi32_y(g, z, x, y);
        const float *p = A.ps.y;
        eyy = eyy * Ky + (by * p[PSI_VA * (int)g.slab_y + k] + ay * eyy);
        dvz_dy = dvz_dy * Kyh + (byh * p[PSI_VB1 * (int)g.slab_y + k] + ayh * dvz_dy);
        dvx_dy = dvx_dy * Kyh + (byh * p[PSI_VB2 * (int)g.slab_y + k] + ayh * dvx_dy);
        A.lout.y[PSI_VA * (int)g.slab_y + k] = by * (A.lin.y[PSI_VA * (int)g.slab_y + k] + G.ey);
        A.lout.y[PSI_VB1 * (int)g.slab_y + k] = byh * (A.lin.y[PSI_VB1 * (int)g.slab_y + k] + G.yz);
        A.lout.y[PSI_VB2 * (int)g.slab_y + k] = byh * (A.lin.y[PSI_VB2 * (int)g.slab_y + k] + G.xy);
      }
      if (A.g0) {
        const float azz = ring.halo(jc, ES_ZZ)[own], axx = ring.halo(jc, ES_XX)[own],
                    ayy = ring.halo(jc, ES_YY)[own];
        const float axz = ring.halo(jc, ES_XZ)[own], axy = ring.halo(jc, ES_XY)[own],
                    ayz = ring.halo(jc, ES_YZ)[own];
        A.g0[i] = gi0 + (azz + axx + ayy) * (ezz + exx + eyy) * dt;
        A.g1[i] = gi1 + (2.0f * (azz * ezz + axx * exx + ayy * eyy) + axz * (dvx_dz + dvz_dx) +
                         axy * (dvx_dy + dvy_dx) + ayz * (dvy_dz + dvz_dy)) * dt;
      }
      A.a.vz[i] = av0 + dvz;
      A.a.vx[i] = av1 + dvx;
      A.a.vy[i] = av2 + dvy;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) { qez[k] = qez[k + 1]; qvx[k] = qvx[k + 1]; qvy[k] = qvy[k + 1]; }
#pragma unroll
    for (int k = 0; k < 3; ++k) { zvz[k] = zvz[k + 1]; zvx[k] = zvx[k + 1]; zvy[k] = zvy[k + 1]; }
    if (__syncthreads_or(!got)) {
      ring_abort(ring, q + 4, min(nj, q + 2 + R), R, tid, status);
      return;
    }
    const int jn = jc + R;  // the slot of plane z is free: refill it
    if (tid == 0 && jn < nj) {
      fence_proxy_async_smem();
      ring.issue(maps, jn, y0, x0, z0 - 2 + jn, z0 - 2 + jn);
    }
  }
}

// G of the velocity stage from slot values (gv_at).
template <class Ring>
__device__ __forceinline__ void gv_slot(const Ring &ring, int j, int o, float dt, float &gz,
                                        float &gx, float &gy) {
  const float s = ring.halo(j, EV_B)[o] * dt;
  gz = ring.halo(j, EV_VZ)[o] * s;
  gx = ring.halo(j, EV_VX)[o] * s;
  gy = ring.halo(j, EV_VY)[o] * s;
}

// z-, x- and y-axis terms of the velocity stage from G (qv_z, qv_x, qv_y).
__device__ __forceinline__ void qv_z_of(const ExactArgs &A, float gz, float gx, float gy, int zn,
                                        int x, int y, float &qzz, float &qxz, float &qyz) {
  const Geo &g = A.g;
  if (zn < 2 || zn > g.nz - 3) { qzz = qxz = qyz = 0.f; return; }
  if (slab_s(zn, g.nz, g.np)) {
    const int k = psi32_z(g, zn, x, y);
    const float *c = g.cz;
    const int nz = g.nz;
    qzz = qpml(gz, true, A.lin.z[PSI_SAA * (int)g.slab_z + k], c[CKH * nz + zn], c[CAH * nz + zn]);
    qxz = qpml(gx, true, A.lin.z[PSI_SAB1 * (int)g.slab_z + k], c[CK * nz + zn], c[CA * nz + zn]);
    qyz = qpml(gy, true, A.lin.z[PSI_SAB2 * (int)g.slab_z + k], c[CK * nz + zn], c[CA * nz + zn]);
  } else {
    qzz = gz; qxz = gx; qyz = gy;
  }
}

__device__ __forceinline__ void qv_x_of(const ExactArgs &A, float gz, float gx, float gy, int z,
                                        int xn, int y, float &qxz, float &qxx, float &qxy) {
  const Geo &g = A.g;
  if (xn < 2 || xn > g.nx - 3) { qxz = qxx = qxy = 0.f; return; }
  if (slab_v(xn, g.nx, g.np)) {
    const int k = psi32_x(g, z, xn, y);
    const float *c = g.cx;
    const int nx = g.nx;
    qxz = qpml(gz, true, A.lin.x[PSI_SAB1 * (int)g.slab_x + k], c[CK * nx + xn], c[CA * nx + xn]);
    qxx = qpml(gx, true, A.lin.x[PSI_SAA * (int)g.slab_x + k], c[CKH * nx + xn], c[CAH * nx + xn]);
    qxy = qpml(gy, true, A.lin.x[PSI_SAB2 * (int)g.slab_x + k], c[CK * nx + xn], c[CA * nx + xn]);
  } else {
    qxz = gz; qxx = gx; qxy = gy;
  }
}

__device__ __forceinline__ void qv_y_of(const ExactArgs &A, float gz, float gx, float gy, int z,
                                        int x, int yn, float &qyz, float &qxy, float &qyy) {
  const Geo &g = A.g;
  if (yn < 2 || yn > g.ny - 3) { qyz = qxy = qyy = 0.f; return; }
  if (slab_v(yn, g.ny, g.np)) {
    const int k = psi32_y(g, z, x, yn);
    const float *c = g.cy;
    const int ny = g.ny;
    qyz = qpml(gz, true, A.lin.y[PSI_SAB1 * (int)g.slab_y + k], c[CK * ny + yn], c[CA * ny + yn]);
    qxy = qpml(gx, true, A.lin.y[PSI_SAB2 * (int)g.slab_y + k], c[CK * ny + yn], c[CA * ny + yn]);
    qyy = qpml(gy, true, A.lin.y[PSI_SAA * (int)g.slab_y + k], c[CKH * ny + yn], c[CAH * ny + yn]);
  } else {
    qyz = gz; qxy = gx; qyy = gy;
  }
}

template <int TX, int R, int MINB>
__global__ void __launch_bounds__(32 * TX, MINB)
k_adj_velocity_tma(const __grid_constant__ Maps<EV_N> maps, ExactArgs A, int zchunk, int *status) {
  using Ring = PlaneRing<EV_N, 0, 0, TX, R>;
  __shared__ float sqx[3][TX + 4][32];
  __shared__ float sqy[3][TX][36];
  extern __shared__ __align__(128) unsigned char smem[];
  Ring ring;
  ring.bind(smem);
  const Geo &g = A.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int y0 = blockIdx.x * 32, x0 = blockIdx.y * TX;
  const int y = y0 + tx, x = x0 + ty;
  const int z0 = max((int)blockIdx.z * zchunk, 2);
  const int z1 = min((int)blockIdx.z * zchunk + zchunk, g.nz - 2);
  if (z0 >= z1) return;
  const int nq = z1 - z0, nj = nq + 4;
  if (tid == 0) ring.init();
  __syncthreads();
  if (tid == 0)
    for (int j = 0; j < nj && j < R; ++j) ring.issue(maps, j, y0, x0, z0 - 2 + j, z0 - 2 + j);

  const int np = g.np, nz = g.nz, nx = g.nx, ny = g.ny;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;
  const bool xin = x >= 2 && x <= nx - 3, yin = y >= 2 && y <= ny - 3;
  const bool act = xin && yin;
  const bool xs = slab_v(x, nx, np), ys = slab_v(y, ny, np);
  const int hr = ty < 2 ? ty : TX + ty;
  const int hxn = x0 - 2 + hr;
  const int hc = tx < 2 ? tx : 32 + tx;
  const int hyn = y0 - 2 + hc;
  const int own = (ty + TMA_HX) * TMA_BOXY + tx + TMA_HY;
  const int hro = hr * TMA_BOXY + tx + TMA_HY;
  const int hco = (ty + TMA_HX) * TMA_BOXY + hc + 2;

  bool ok = true;
  for (int j = 0; j < 4; ++j) ok = ring.wait(j) && ok;
  // queues: Q_z of planes z-2 .. z+2; forward szz at z-1 .. z+2, sxz and
  // syz at z-2 .. z+1
  float qzz[5] = {}, qxz[5] = {}, qyz[5] = {};
  float zszz[4] = {}, zsxz[4] = {}, zsyz[4] = {};
  if (ok && act) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      float gz, gx, gy;
      gv_slot(ring, k, own, dt, gz, gx, gy);
      qv_z_of(A, gz, gx, gy, z0 - 2 + k, x, y, qzz[k], qxz[k], qyz[k]);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      zszz[k] = ring.halo(k + 1, EV_SZZ)[own];
      zsxz[k] = ring.halo(k, EV_SXZ)[own];
      zsyz[k] = ring.halo(k, EV_SYZ)[own];
    }
  }
  if (__syncthreads_or(!ok)) {
    ring_abort(ring, 0, min(nj, R), R, tid, status);
    return;
  }
  if (tid == 0)
    for (int j = R; j < R + 2 && j < nj; ++j) {
      fence_proxy_async_smem();
      ring.issue(maps, j, y0, x0, z0 - 2 + j, z0 - 2 + j);
    }

  for (int q = 0; q < nq; ++q) {
    const int z = z0 + q, jc = q + 2;
    const int i = act ? cell32(g, z, x, y) : 0;
    float as0 = 0.f, as1 = 0.f, as2 = 0.f, as3 = 0.f, as4 = 0.f, as5 = 0.f, gi0 = 0.f;
    if (act) {  // read-modify-write operands, before the wait
      as0 = A.a.szz[i]; as1 = A.a.sxx[i]; as2 = A.a.syy[i];
      as3 = A.a.sxz[i]; as4 = A.a.syz[i]; as5 = A.a.sxy[i];
      if (A.g0) gi0 = A.g0[i];
    }
    const bool got = ring.wait(q + 4);
    float gz = 0.f, gx = 0.f, gy = 0.f;
    if (got) {
      qzz[4] = qxz[4] = qyz[4] = 0.f;
      if (act) {
        float hz, hx, hy;
        gv_slot(ring, q + 4, own, dt, hz, hx, hy);
        qv_z_of(A, hz, hx, hy, z + 2, x, y, qzz[4], qxz[4], qyz[4]);
      }
      zszz[3] = ring.halo(q + 4, EV_SZZ)[own];
      zsxz[3] = ring.halo(q + 3, EV_SXZ)[own];
      zsyz[3] = ring.halo(q + 3, EV_SYZ)[own];
      float ox[3] = {0.f, 0.f, 0.f}, oy[3] = {0.f, 0.f, 0.f};
      if (act) {  // qv_own
        gv_slot(ring, jc, own, dt, gz, gx, gy);
        qv_x_of(A, gz, gx, gy, z, x, y, ox[0], ox[1], ox[2]);
        qv_y_of(A, gz, gx, gy, z, x, y, oy[0], oy[1], oy[2]);
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) { sqx[k][ty + 2][tx] = ox[k]; sqy[k][ty][tx + 2] = oy[k]; }
      if (ty < 4) {
        float h0 = 0.f, h1 = 0.f, h2 = 0.f;
        if (yin) {
          float hz, hx, hy;
          gv_slot(ring, jc, hro, dt, hz, hx, hy);
          qv_x_of(A, hz, hx, hy, z, hxn, y, h0, h1, h2);
        }
        sqx[0][hr][tx] = h0; sqx[1][hr][tx] = h1; sqx[2][hr][tx] = h2;
      }
      if (tx < 4) {
        float h0 = 0.f, h1 = 0.f, h2 = 0.f;
        if (xin) {
          float hz, hx, hy;
          gv_slot(ring, jc, hco, dt, hz, hx, hy);
          qv_y_of(A, hz, hx, hy, z, x, hyn, h0, h1, h2);
        }
        sqy[0][ty][hc] = h0; sqy[1][ty][hc] = h1; sqy[2][ty][hc] = h2;
      }
    }
    __syncthreads();
    if (got && act) {
      const float(*QX)[TX + 4][32] = sqx;
      const float(*QY)[TX][36] = sqy;
      // ---- adjoint stresses (x: 0 vz<-sxz, 1 vx<-sxx, 2 vy<-sxy;
      //                        y: 0 vz<-syz, 1 vx<-sxy, 2 vy<-syy)
      const float dszz = -dminus(qzz[0], qzz[1], qzz[2], qzz[3]) * idz;
      const float dsxx = -dminus(QX[1][ty][tx], QX[1][ty + 1][tx], QX[1][ty + 2][tx], QX[1][ty + 3][tx]) * idx;
      const float dsyy = -dminus(QY[2][ty][tx], QY[2][ty][tx + 1], QY[2][ty][tx + 2], QY[2][ty][tx + 3]) * idy;
      const float dsxz = -dplus(QX[0][ty + 1][tx], QX[0][ty + 2][tx], QX[0][ty + 3][tx], QX[0][ty + 4][tx]) * idx -
                         dplus(qxz[1], qxz[2], qxz[3], qxz[4]) * idz;
      const float dsyz = -dplus(QY[0][ty][tx + 1], QY[0][ty][tx + 2], QY[0][ty][tx + 3], QY[0][ty][tx + 4]) * idy -
                         dplus(qyz[1], qyz[2], qyz[3], qyz[4]) * idz;
      const float dsxy = -dplus(QY[1][ty][tx + 1], QY[1][ty][tx + 2], QY[1][ty][tx + 3], QY[1][ty][tx + 4]) * idy +
                         dq_t(QX[2][ty + 2][tx], QX[2][ty + 3][tx], QX[2][ty + 4][tx]) * idx;

      // ---- buoyancy image from the forward stresses of the same step
      const BoxView fxz{ring.halo(jc, EV_SXZ) + own}, fxx{ring.halo(jc, EV_SXX) + own},
          fxy{ring.halo(jc, EV_SXY) + own}, fyz{ring.halo(jc, EV_SYZ) + own},
          fyy{ring.halo(jc, EV_SYY) + own};
      float dszz_dz = dplus(zszz[0], zszz[1], zszz[2], zszz[3]) * idz;
      float dsxz_dx = dminus(fxz.x(-2), fxz.x(-1), fxz.c(), fxz.x(1)) * idx;
      float dsyz_dy = dminus(fyz.y(-2), fyz.y(-1), fyz.c(), fyz.y(1)) * idy;
      float dsxz_dz = dminus(zsxz[0], zsxz[1], zsxz[2], zsxz[3]) * idz;
      float dsxx_dx = dplus(fxx.x(-1), fxx.c(), fxx.x(1), fxx.x(2)) * idx;
      float dsxy_dy = dminus(fxy.y(-2), fxy.y(-1), fxy.c(), fxy.y(1)) * idy;
      float dsyz_dz = dminus(zsyz[0], zsyz[1], zsyz[2], zsyz[3]) * idz;
      const float sxy0 = fxy.c(), sxym1 = fxy.x(-1), sxym2 = fxy.x(-2);
      float dsxy_dx = (EFWI_C1 * (sxy0 - sxym1) - EFWI_C2 * (sxym1 - sxym2)) * idx;
      float dsyy_dy = dplus(fyy.y(-1), fyy.c(), fyy.y(1), fyy.y(2)) * idy;
      if (slab_s(z, nz, np)) {
        const float *c = g.cz;
        const float Kz = c[CK * nz + z], bz = c[CB * nz + z], Kzh = c[CKH * nz + z], bzh = c[CBH * nz + z];
        const int k = psi32_z(g, z, x, y);
        const float *p = A.ps.z;
        dszz_dz = dszz_dz * Kzh + p[PSI_SAA * (int)g.slab_z + k];
        dsxz_dz = dsxz_dz * Kz + p[PSI_SAB1 * (int)g.slab_z + k];
        dsyz_dz = dsyz_dz * Kz + p[PSI_SAB2 * (int)g.slab_z + k];
        A.lout.z[PSI_SAA * (int)g.slab_z + k] = bzh * (A.lin.z[PSI_SAA * (int)g.slab_z + k] + gz);
        A.lout.z[PSI_SAB1 * (int)g.slab_z + k] = bz * (A.lin.z[PSI_SAB1 * (int)g.slab_z + k] + gx);
        A.lout.z[PSI_SAB2 * (int)g.slab_z + k] = bz * (A.lin.z[PSI_SAB2 * (int)g.slab_z + k] + gy);
      }
      if (xs) {
        const float *c = g.cx;
        const float Kx = c[CK * nx + x], bx = c[CB * nx + x], Kxh = c[CKH * nx + x], bxh = c[CBH * nx + x];
        const int k = psi32_x(g, z, x, y);
        const float *p = A.ps.x;
        dsxz_dx = dsxz_dx * Kx + p[PSI_SAB1 * (int)g.slab_x + k];
        dsxx_dx = dsxx_dx * Kxh + p[PSI_SAA * (int)g.slab_x + k];
        dsxy_dx = dsxy_dx * Kx + p[PSI_SAB2 * (int)g.slab_x + k];
        A.lout.x[PSI_SAB1 * (int)g.slab_x + k] = bx * (A.lin.x[PSI_SAB1 * (int)g.slab_x + k] + gz);
        A.lout.x[PSI_SAA * (int)g.slab_x + k] = bxh * (A.lin.x[PSI_SAA * (int)g.slab_x + k] + gx);
        A.lout.x[PSI_SAB2 * (int)g.slab_x + k] = bx * (A.lin.x[PSI_SAB2 * (int)g.slab_x + k] + gy);
      }
      if (ys) {
        const float *c = g.cy;
        const float Ky = c[CK * ny + y], by = c[CB * ny + y], Kyh = c[CKH * ny + y], byh = c[CBH * ny + y];
        const int k = psi32_y(g, z, x, y);
        const float *p = A.ps.y;
        dsyz_dy = dsyz_dy * Ky + p[PSI_SAB1 * (int)g.slab_y + k];
        dsxy_dy = dsxy_dy * Ky + p[PSI_SAB2 * (int)g.slab_y + k];
        dsyy_dy = dsyy_dy * Kyh + p[PSI_SAA * (int)g.slab_y + k];
        A.lout.y[PSI_SAB1 * (int)g.slab_y + k] = by * (A.lin.y[PSI_SAB1 * (int)g.slab_y + k] + gz);
        A.lout.y[PSI_SAB2 * (int)g.slab_y + k] = by * (A.lin.y[PSI_SAB2 * (int)g.slab_y + k] + gx);
        A.lout.y[PSI_SAA * (int)g.slab_y + k] = byh * (A.lin.y[PSI_SAA * (int)g.slab_y + k] + gy);
      }
      if (A.g0) {
        const float avz = ring.halo(jc, EV_VZ)[own], avx = ring.halo(jc, EV_VX)[own],
                    avy = ring.halo(jc, EV_VY)[own];
        A.g0[i] = gi0 + (avz * (dszz_dz + dsxz_dx + dsyz_dy) + avx * (dsxz_dz + dsxx_dx + dsxy_dy) +
                         avy * (dsyz_dz + dsxy_dx + dsyy_dy)) * dt;
      }
      A.a.szz[i] = as0 + dszz;
      A.a.sxx[i] = as1 + dsxx;
      A.a.syy[i] = as2 + dsyy;
      A.a.sxz[i] = as3 + dsxz;
      A.a.syz[i] = as4 + dsyz;
      A.a.sxy[i] = as5 + dsxy;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) { qzz[k] = qzz[k + 1]; qxz[k] = qxz[k + 1]; qyz[k] = qyz[k + 1]; }
#pragma unroll
    for (int k = 0; k < 3; ++k) { zszz[k] = zszz[k + 1]; zsxz[k] = zsxz[k + 1]; zsyz[k] = zsyz[k + 1]; }
    if (__syncthreads_or(!got)) {
      ring_abort(ring, q + 4, min(nj, q + 2 + R), R, tid, status);
      return;
    }
    const int jn = jc + R;
    if (tid == 0 && jn < nj) {
      fence_proxy_async_smem();
      ring.issue(maps, jn, y0, x0, z0 - 2 + jn, z0 - 2 + jn);
    }
  }
}

}  // namespace

void launch_adj_stress_exact(int bx, dim3 grid, cudaStream_t st, const ExactArgs &A, int zchunk,
                             int nzc) {
  if (bx == 8)
    k_adj_stress_exact<8><<<grid, dim3(32, 8), 0, st>>>(A, zchunk, nzc);
  else
    k_adj_stress_exact<4><<<grid, dim3(32, 4), 0, st>>>(A, zchunk, nzc);
}

void launch_adj_velocity_exact(int bx, dim3 grid, cudaStream_t st, const ExactArgs &A, int zchunk,
                               int nzc) {
  if (bx == 8)
    k_adj_velocity_exact<8><<<grid, dim3(32, 8), 0, st>>>(A, zchunk, nzc);
  else
    k_adj_velocity_exact<4><<<grid, dim3(32, 4), 0, st>>>(A, zchunk, nzc);
}

// Bulk-copy staged exact kernels: tile 32 x TX, ring of R planes.
template <int TX, int R, int MINB>
static void adj_stress_tma_launch(dim3 grid, cudaStream_t st, const Maps<11> &maps,
                                  const ExactArgs &A, int zchunk, int *status) {
  constexpr int B = PlaneRing<ES_N, 0, 0, TX, R>::BYTES;
  static std::atomic<unsigned long long> smem_set{0};
  set_smem_once(k_adj_stress_tma<TX, R, MINB>, B, smem_set);
  k_adj_stress_tma<TX, R, MINB><<<grid, dim3(32, TX), B, st>>>(maps, A, zchunk, status);
}

template <int TX, int R, int MINB>
static void adj_velocity_tma_launch(dim3 grid, cudaStream_t st, const Maps<10> &maps,
                                    const ExactArgs &A, int zchunk, int *status) {
  constexpr int B = PlaneRing<EV_N, 0, 0, TX, R>::BYTES;
  static std::atomic<unsigned long long> smem_set{0};
  set_smem_once(k_adj_velocity_tma<TX, R, MINB>, B, smem_set);
  k_adj_velocity_tma<TX, R, MINB><<<grid, dim3(32, TX), B, st>>>(maps, A, zchunk, status);
}

void launch_adj_stress_tma(int bx, dim3 grid, cudaStream_t st, const Maps<11> &maps,
                           const ExactArgs &A, int zchunk, int *status) {
  if (bx == 8) adj_stress_tma_launch<8, 5, 2>(grid, st, maps, A, zchunk, status);
  else adj_stress_tma_launch<4, 5, 3>(grid, st, maps, A, zchunk, status);
}

void launch_adj_velocity_tma(int bx, dim3 grid, cudaStream_t st, const Maps<10> &maps,
                             const ExactArgs &A, int zchunk, int *status) {
  if (bx == 8) adj_velocity_tma_launch<8, 5, 2>(grid, st, maps, A, zchunk, status);
  else adj_velocity_tma_launch<4, 5, 3>(grid, st, maps, A, zchunk, status);
}

// dJ/dstf of step k: the source adds 1500^2 * dt * w^2(k) * stf(k) to szz,
// sxx and syy at the source cell after the stress stage of step k
// (utilities.cu:442-479, taper Src_Rec.cu:146), so its derivative is that
// factor times the adjoint of the three stresses there at that point.
__global__ void k_stf_gradient(Fields a, const long long *src_cell, const float *w2, float *out,
                               int k, float scale) {
  if (threadIdx.x != 0) return;
  const long long i = src_cell[0];
  if (i < 0) return;
  out[k] = scale * w2[k] * (a.szz[i] + a.sxx[i] + a.syy[i]);
}

// rho image from the buoyancy image: B = 1/rho on [2, n-3]^3
// (Model.cu:65-76), so dJ/drho = -dJ/dB * B^2 there and 0 elsewhere.
__global__ void k_buoy_to_rho(const float *gB, const float *buoy, float *grho, int nz, int nx,
                              int ny, int py) {
  const long long n = (long long)nz * nx * py;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % py);
    const long long zx = i / py;
    const int x = (int)(zx % nx), z = (int)(zx / nx);
    const bool in = z >= 2 && z <= nz - 3 && x >= 2 && x <= nx - 3 && y >= 2 && y <= ny - 3;
    const float b = buoy[i];
    grho[i] = in ? -gB[i] * b * b : 0.0f;
  }
}

// Source illumination (diagonal pseudo-Hessian of Shin et al. 2001): for the
// state S_k after forward step k-1, adds at every cell of [2, n-3]^3, summed
// over the S shots of the batch,
//   hl += 3 (dt div)^2                       (d sigma_ii / d lambda = dt div)
//   hm += dt^2 (4 sum_i e_ii^2 + sum_i<j (e_ij + e_ji)^2)
//   hb += dt^2 |modified stress divergence|^2 (d v / d B)
// from the C-PML-modified derivatives of the forward step: the stress-stage
// terms of step k (velocities and stress memory variables of S_k, when
// do_stress) and the velocity-stage terms of step k-1 (stresses and updated
// velocity memory variables of S_k).  Grid (ceil(ny/32), ceil(nx/4),
// ceil((nz-4)/8)), 32 x 4 threads; each thread sums its shots in order.
__global__ void __launch_bounds__(128)
k_illumination(Geo g, Fields f, Psi ps, int S, const float *buoy, int do_stress, float *hl,
               float *hm, float *hb) {
  const int y = blockIdx.x * 32 + threadIdx.x;
  const int x = blockIdx.y * 4 + threadIdx.y;
  const int np = g.np, nz = g.nz, nx = g.nx, ny = g.ny;
  if (x < 2 || x > nx - 3 || y < 2 || y > ny - 3) return;
  const int z0 = 2 + (int)blockIdx.z * 8, z1 = min(z0 + 8, nz - 2);
  const int sz = (int)g.sz, sx = g.sx;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy, dt2 = dt * dt;
  const bool xs = slab_s(x, nx, np), ys = slab_s(y, ny, np);
  const bool xv = slab_v(x, nx, np), yv = slab_v(y, ny, np);
  for (int z = z0; z < z1; ++z) {
    const int i = cell32(g, z, x, y);
    const bool zs = slab_s(z, nz, np);
    float al = 0.f, am = 0.f, ab = 0.f;
    for (int s = 0; s < S; ++s) {
      const long long so = (long long)s * g.N;
      const float *pz = ps.z + (long long)s * 6 * g.slab_z;
      const float *px = ps.x + (long long)s * 6 * g.slab_x;
      const float *py = ps.y + (long long)s * 6 * g.slab_y;
      if (do_stress) {
        const float *vz = f.vz + so, *vx = f.vx + so, *vy = f.vy + so;
        float ezz = dminus(vz[i - 2 * sz], vz[i - sz], vz[i], vz[i + sz]) * idz;
        float exx = dminus(vx[i - 2 * sx], vx[i - sx], vx[i], vx[i + sx]) * idx;
        float eyy = dminus(vy[i - 2], vy[i - 1], vy[i], vy[i + 1]) * idy;
        float dvx_dz = dplus(vx[i - sz], vx[i], vx[i + sz], vx[i + 2 * sz]) * idz;
        float dvy_dz = dplus(vy[i - sz], vy[i], vy[i + sz], vy[i + 2 * sz]) * idz;
        float dvx_dy = dplus(vx[i - 1], vx[i], vx[i + 1], vx[i + 2]) * idy;
        float dvz_dx = dplus(vz[i - sx], vz[i], vz[i + sx], vz[i + 2 * sx]) * idx;
        float dvz_dy = dplus(vz[i - 1], vz[i], vz[i + 1], vz[i + 2]) * idy;
        float dvy_dx = dplus(vy[i - sx], vy[i], vy[i + sx], vy[i + 2 * sx]) * idx;
        if (zs) {
          const float *c = g.cz;
          const int k = psi32_z(g, z, x, y), sl = (int)g.slab_z;
          ezz = ezz * c[CK * nz + z] + (c[CB * nz + z] * pz[PSI_VA * sl + k] + c[CA * nz + z] * ezz);
          dvx_dz = dvx_dz * c[CKH * nz + z] + (c[CBH * nz + z] * pz[PSI_VB1 * sl + k] + c[CAH * nz + z] * dvx_dz);
          dvy_dz = dvy_dz * c[CKH * nz + z] + (c[CBH * nz + z] * pz[PSI_VB2 * sl + k] + c[CAH * nz + z] * dvy_dz);
        }
        if (xs) {
          const float *c = g.cx;
          const int k = psi32_x(g, z, x, y), sl = (int)g.slab_x;
          exx = exx * c[CK * nx + x] + (c[CB * nx + x] * px[PSI_VA * sl + k] + c[CA * nx + x] * exx);
          dvz_dx = dvz_dx * c[CKH * nx + x] + (c[CBH * nx + x] * px[PSI_VB1 * sl + k] + c[CAH * nx + x] * dvz_dx);
          dvy_dx = dvy_dx * c[CKH * nx + x] + (c[CBH * nx + x] * px[PSI_VB2 * sl + k] + c[CAH * nx + x] * dvy_dx);
        }
        if (ys) {
          const float *c = g.cy;
          const int k = psi32_y(g, z, x, y), sl = (int)g.slab_y;
          eyy = eyy * c[CK * ny + y] + (c[CB * ny + y] * py[PSI_VA * sl + k] + c[CA * ny + y] * eyy);
          dvz_dy = dvz_dy * c[CKH * ny + y] + (c[CBH * ny + y] * py[PSI_VB1 * sl + k] + c[CAH * ny + y] * dvz_dy);
          dvx_dy = dvx_dy * c[CKH * ny + y] + (c[CBH * ny + y] * py[PSI_VB2 * sl + k] + c[CAH * ny + y] * dvx_dy);
        }
        const float div = ezz + exx + eyy;
        const float exz = dvx_dz + dvz_dx, exy = dvx_dy + dvy_dx, eyz = dvy_dz + dvz_dy;
        al += 3.0f * div * div * dt2;
        am += (4.0f * (ezz * ezz + exx * exx + eyy * eyy) + exz * exz + exy * exy + eyz * eyz) * dt2;
      }
      const float *szz = f.szz + so, *sxx = f.sxx + so, *syy = f.syy + so;
      const float *sxz = f.sxz + so, *sxy = f.sxy + so, *syz = f.syz + so;
      float dszz_dz = dplus(szz[i - sz], szz[i], szz[i + sz], szz[i + 2 * sz]) * idz;
      float dsxz_dx = dminus(sxz[i - 2 * sx], sxz[i - sx], sxz[i], sxz[i + sx]) * idx;
      float dsyz_dy = dminus(syz[i - 2], syz[i - 1], syz[i], syz[i + 1]) * idy;
      float dsxz_dz = dminus(sxz[i - 2 * sz], sxz[i - sz], sxz[i], sxz[i + sz]) * idz;
      float dsxx_dx = dplus(sxx[i - sx], sxx[i], sxx[i + sx], sxx[i + 2 * sx]) * idx;
      float dsxy_dy = dminus(sxy[i - 2], sxy[i - 1], sxy[i], sxy[i + 1]) * idy;
      float dsyz_dz = dminus(syz[i - 2 * sz], syz[i - sz], syz[i], syz[i + sz]) * idz;
      float dsxy_dx = (EFWI_C1 * (sxy[i] - sxy[i - sx]) - EFWI_C2 * (sxy[i - sx] - sxy[i - 2 * sx])) * idx;
      float dsyy_dy = dplus(syy[i - 1], syy[i], syy[i + 1], syy[i + 2]) * idy;
      if (zs) {
        const float *c = g.cz;
        const int k = psi32_z(g, z, x, y), sl = (int)g.slab_z;
        dszz_dz = dszz_dz * c[CKH * nz + z] + pz[PSI_SAA * sl + k];
        dsxz_dz = dsxz_dz * c[CK * nz + z] + pz[PSI_SAB1 * sl + k];
        dsyz_dz = dsyz_dz * c[CK * nz + z] + pz[PSI_SAB2 * sl + k];
      }
      if (xv) {
        const float *c = g.cx;
        const int k = psi32_x(g, z, x, y), sl = (int)g.slab_x;
        dsxz_dx = dsxz_dx * c[CK * nx + x] + px[PSI_SAB1 * sl + k];
        dsxx_dx = dsxx_dx * c[CKH * nx + x] + px[PSI_SAA * sl + k];
        dsxy_dx = dsxy_dx * c[CK * nx + x] + px[PSI_SAB2 * sl + k];
      }
      if (yv) {
        const float *c = g.cy;
        const int k = psi32_y(g, z, x, y), sl = (int)g.slab_y;
        dsyz_dy = dsyz_dy * c[CK * ny + y] + py[PSI_SAB1 * sl + k];
        dsxy_dy = dsxy_dy * c[CK * ny + y] + py[PSI_SAB2 * sl + k];
        dsyy_dy = dsyy_dy * c[CKH * ny + y] + py[PSI_SAA * sl + k];
      }
      const float qz = dszz_dz + dsxz_dx + dsyz_dy, qx = dsxz_dz + dsxx_dx + dsxy_dy,
                  qy = dsyz_dz + dsxy_dx + dsyy_dy;
      ab += (qz * qz + qx * qx + qy * qy) * dt2;
    }
    hl[i] += al;
    hm[i] += am;
    hb[i] += ab;
  }
  (void)buoy;
}

// Illumination of rho from that of the buoyancy: (dB/drho)^2 = B^4 on
// [2, n-3]^3 (Model.cu:65-76), 0 elsewhere; in place.
__global__ void k_buoy_to_rho_sq(float *hb, const float *buoy, int nz, int nx, int ny, int py) {
  const long long n = (long long)nz * nx * py;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % py);
    const long long zx = i / py;
    const int x = (int)(zx % nx), z = (int)(zx / nx);
    const bool in = z >= 2 && z <= nz - 3 && x >= 2 && x <= nx - 3 && y >= 2 && y <= ny - 3;
    const float b2 = buoy[i] * buoy[i];
    hb[i] = in ? hb[i] * b2 * b2 : 0.0f;
  }
}

// State of the oracle's layout, [27][nz][nx][ny] (9 fields, then the 18
// memory variables in the order m_vz_z m_vz_x m_vz_y m_vx_z m_vx_x m_vx_y
// m_vy_z m_vy_x m_vy_y m_szz_z m_sxx_x m_syy_y m_sxz_z m_sxz_x m_sxy_x
// m_sxy_y m_syz_y m_syz_z), to or from the engine's pitched fields and
// slab memory variables.  Memory variables outside their slab are not
// stored; `to_engine` = 0 leaves them unchanged in the full-grid array.
__constant__ signed char c_psi_axis[18] = {0, 1, 2, 0, 1, 2, 0, 1, 2, 0, 1, 2, 0, 1, 1, 2, 2, 0};
__constant__ signed char c_psi_slot[18] = {0, 1, 1, 1, 0, 2, 2, 2, 0, 3, 3, 3, 4, 4, 5, 5, 4, 5};

__global__ void k_state_convert(Geo g, float *full, Fields f, Psi ps, int to_engine) {
  const long long nc = (long long)g.nz * g.nx * g.ny;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 27 * nc;
       t += (long long)gridDim.x * blockDim.x) {
    const int comp = (int)(t / nc);
    const long long r = t - comp * nc;
    const int y = (int)(r % g.ny);
    const long long zx = r / g.ny;
    const int x = (int)(zx % g.nx), z = (int)(zx / g.nx);
    float *dst = nullptr;
    if (comp < 9) {
      float *fl[9] = {f.vz, f.vx, f.vy, f.szz, f.sxx, f.syy, f.sxz, f.sxy, f.syz};
      dst = fl[comp] + cell(g, z, x, y);
    } else {
      const int ax = c_psi_axis[comp - 9], slot = c_psi_slot[comp - 9];
      if (ax == 0 && slab_s(z, g.nz, g.np)) dst = ps.z + slot * g.slab_z + psi_z_idx(g, z, x, y);
      if (ax == 1 && slab_s(x, g.nx, g.np)) dst = ps.x + slot * g.slab_x + psi_x_idx(g, z, x, y);
      if (ax == 2 && slab_s(y, g.ny, g.np)) dst = ps.y + slot * g.slab_y + psi_y_idx(g, z, x, y);
    }
    if (!dst) continue;
    if (to_engine) *dst = full[t];
    else full[t] = *dst;
  }
}

}  // namespace efwi
