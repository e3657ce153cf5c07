// Reverse sweep of the reference gradient (mode "reference").
//
// One reverse time step of the reference (libCUFD.cu:532-612) is
//   velocity(rev) -> restore v shell -> add_source(sub) -> stress(rev)
//   -> restore sigma shell -> velocity_adj -> res_injection -> stress_adj.
// Here it runs as two fused kernels plus the shell restores:
//   K1 = velocity(rev) [interior, rho imaging]   + velocity_adj [2, n-3]
//   K2 = add_source(sub) + stress(rev) [interior, lambda/mu imaging]
//        + stress_adj [2, n-3]
// The reorderings are exact: velocity_adj reads only adjoint stresses and
// stress-type adjoint memory variables, which stress(rev) does not touch;
// the rho image reads the adjoint velocity before velocity_adj updates it,
// and the lambda/mu image reads the adjoint stress before stress_adj
// updates it, as in the reference's sequential order.
//
// Restated kernels: velocity.cu:102-131, stress.cu:103-135,
// velocity_adj.cu:59-144, stress_adj.cu:52-142.  The adjoint memory
// variables reuse the forward slab buffers (the reference re-zeroes and
// reuses its 18 full-grid arrays, libCUFD.cu:481-498).
#include "efwi_common.cuh"
#include "efwi_kernels.h"

namespace efwi {

namespace {

// -D+ / -D- of slab memory variables at neighbours, zero outside the slab.
__device__ __forceinline__ float nxp(const Geo &g, const float *p, int z, int x, int y) {
  return -dplus(psi_x_get(g, p, z, x - 1, y), psi_x_get(g, p, z, x, y),
                psi_x_get(g, p, z, x + 1, y), psi_x_get(g, p, z, x + 2, y));
}
__device__ __forceinline__ float nxm(const Geo &g, const float *p, int z, int x, int y) {
  return -dminus(psi_x_get(g, p, z, x - 2, y), psi_x_get(g, p, z, x - 1, y),
                 psi_x_get(g, p, z, x, y), psi_x_get(g, p, z, x + 1, y));
}
__device__ __forceinline__ float nyp(const Geo &g, const float *p, int z, int x, int y) {
  return -dplus(psi_y_get(g, p, z, x, y - 1), psi_y_get(g, p, z, x, y),
                psi_y_get(g, p, z, x, y + 1), psi_y_get(g, p, z, x, y + 2));
}
__device__ __forceinline__ float nym(const Geo &g, const float *p, int z, int x, int y) {
  return -dminus(psi_y_get(g, p, z, x, y - 2), psi_y_get(g, p, z, x, y - 1),
                 psi_y_get(g, p, z, x, y), psi_y_get(g, p, z, x, y + 1));
}
__device__ __forceinline__ float nzp(const Geo &g, const float *p, int z, int x, int y) {
  return -dplus(psi_z_get(g, p, z - 1, x, y), psi_z_get(g, p, z, x, y),
                psi_z_get(g, p, z + 1, x, y), psi_z_get(g, p, z + 2, x, y));
}
__device__ __forceinline__ float nzm(const Geo &g, const float *p, int z, int x, int y) {
  return -dminus(psi_z_get(g, p, z - 2, x, y), psi_z_get(g, p, z - 1, x, y),
                 psi_z_get(g, p, z, x, y), psi_z_get(g, p, z + 1, x, y));
}

struct Coef {
  float K, a, b, Kh, ah, bh;
};
__device__ __forceinline__ Coef coef(const float *c, int n, int i) {
  Coef r;
  r.K = c[CK * n + i]; r.a = c[CA * n + i]; r.b = c[CB * n + i];
  r.Kh = c[CKH * n + i]; r.ah = c[CAH * n + i]; r.bh = c[CBH * n + i];
  return r;
}

}  // namespace

template <int BX>
__global__ void __launch_bounds__(32 * BX)
k_rev_velocity(Geo g, Fields f, Fields a, Psi ps, const float *__restrict__ lam,
               const float *__restrict__ mu, const float *__restrict__ buoy, float *grho,
               int zchunk, int nzc, int do_rev, int do_adj) {
  const int y = blockIdx.x * 32 + threadIdx.x;
  const int x = blockIdx.y * BX + threadIdx.y;
  const int zc = blockIdx.z % nzc;
  const int z0 = max(zc * zchunk, 2);
  const int z1 = min(zc * zchunk + zchunk, g.nz - 2);
  if (x < 2 || x > g.nx - 3 || y < 2 || y > g.ny - 3 || z0 >= z1) return;

  const int np = g.np, nz = g.nz, nx = g.nx, ny = g.ny;
  const long long sz = g.sz;
  const int sx = g.sx;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;
  const bool xin = x >= np && x <= nx - 1 - np, yin = y >= np && y <= ny - 1 - np;
  const bool xs = slab_s(x, nx, np), ys = slab_s(y, ny, np);
  const Coef cx = coef(g.cx, nx, x), cy = coef(g.cy, ny, y);

  const float *__restrict__ szz = f.szz;
  const float *__restrict__ sxx = f.sxx;
  const float *__restrict__ syy = f.syy;
  const float *__restrict__ sxz = f.sxz;
  const float *__restrict__ sxy = f.sxy;
  const float *__restrict__ syz = f.syz;
  const float *__restrict__ aszz = a.szz;
  const float *__restrict__ asxx = a.sxx;
  const float *__restrict__ asyy = a.syy;
  const float *__restrict__ asxz = a.sxz;
  const float *__restrict__ asxy = a.sxy;
  const float *__restrict__ asyz = a.syz;
  const float *psz = ps.z, *psx = ps.x, *psy = ps.y;
  float *pz = ps.z, *px = ps.x, *py = ps.y;

  for (int z = z0; z < z1; ++z) {
    const long long i = ((long long)z * nx + x) * sx + y;
    const float b = buoy[i];
    const float avz0 = a.vz[i], avx0 = a.vx[i], avy0 = a.vy[i];
    if (do_rev && xin && yin && z >= np && z <= nz - 1 - np) {
      const float dz_ = dplus(szz[i - sz], szz[i], szz[i + sz], szz[i + 2 * sz]) * idz +
                        dminus(sxz[i - 2 * sx], sxz[i - sx], sxz[i], sxz[i + sx]) * idx +
                        dminus(syz[i - 2], syz[i - 1], syz[i], syz[i + 1]) * idy;
      const float dx_ = dminus(sxz[i - 2 * sz], sxz[i - sz], sxz[i], sxz[i + sz]) * idz +
                        dplus(sxx[i - sx], sxx[i], sxx[i + sx], sxx[i + 2 * sx]) * idx +
                        dminus(sxy[i - 2], sxy[i - 1], sxy[i], sxy[i + 1]) * idy;
      const float dy_ = dminus(syz[i - 2 * sz], syz[i - sz], syz[i], syz[i + sz]) * idz +
                        (EFWI_C1 * (sxy[i] - sxy[i - sx]) - EFWI_C2 * (sxy[i - sx] - sxy[i - 2 * sx])) * idx +
                        dplus(syy[i - 1], syy[i], syy[i + 1], syy[i + 2]) * idy;
      f.vz[i] = f.vz[i] - dz_ * b * dt;
      f.vx[i] = f.vx[i] - dx_ * b * dt;
      f.vy[i] = f.vy[i] - dy_ * b * dt;
      const float nb2 = -(b * b);
      grho[i] = grho[i] - (avz0 * dz_ * dt * nb2 + avx0 * dx_ * dt * nb2 + avy0 * dy_ * dt * nb2);
    }
    if (!do_adj) continue;
    const bool zs = slab_s(z, nz, np);
    const Coef cz = coef(g.cz, nz, z);
    const float l = lam[i], u = mu[i], l2u = l + 2.0f * u;
    // ---- adjoint vx
    {
      const float dszz_dx = -dplus(aszz[i - sx], aszz[i], aszz[i + sx], aszz[i + 2 * sx]) * idx;
      const float dsxx_dx = -dplus(asxx[i - sx], asxx[i], asxx[i + sx], asxx[i + 2 * sx]) * idx;
      const float dsyy_dx = -dplus(asyy[i - sx], asyy[i], asyy[i + sx], asyy[i + 2 * sx]) * idx;
      const float dsxz_dz = -dminus(asxz[i - 2 * sz], asxz[i - sz], asxz[i], asxz[i + sz]) * idz;
      const float dsxy_dy = -dminus(asxy[i - 2], asxy[i - 1], asxy[i], asxy[i + 1]) * idy;
      float acc = l2u * dsxx_dx * cx.K * dt + l * dszz_dx * cx.K * dt + l * dsyy_dx * cx.K * dt +
                  u * cz.Kh * dsxz_dz * dt + u * cy.Kh * dsxy_dy * dt;
      if (xs) acc += cx.a * (nxp(g, psx + PSI_VA * g.slab_x, z, x, y) * idx);
      if (zs) acc += cz.ah * (nzm(g, psz + PSI_VB1 * g.slab_z, z, x, y) * idz);
      if (ys) acc += cy.ah * (nym(g, psy + PSI_VB2 * g.slab_y, z, x, y) * idy);
      const float v = avx0 + acc;
      a.vx[i] = v;
      if (xs) { const long long k = PSI_SAA * g.slab_x + psi_x_idx(g, z, x, y); px[k] = cx.bh * px[k] + b * v * dt; }
      if (zs) { const long long k = PSI_SAB1 * g.slab_z + psi_z_idx(g, z, x, y); pz[k] = cz.b * pz[k] + b * v * dt; }
      if (ys) { const long long k = PSI_SAB2 * g.slab_y + psi_y_idx(g, z, x, y); py[k] = cy.b * py[k] + b * v * dt; }
    }
    // ---- adjoint vz
    {
      const float dszz_dz = -dplus(aszz[i - sz], aszz[i], aszz[i + sz], aszz[i + 2 * sz]) * idz;
      const float dsxx_dz = -dplus(asxx[i - sz], asxx[i], asxx[i + sz], asxx[i + 2 * sz]) * idz;
      const float dsyy_dz = -dplus(asyy[i - sz], asyy[i], asyy[i + sz], asyy[i + 2 * sz]) * idz;
      const float dsxz_dx = -dminus(asxz[i - 2 * sx], asxz[i - sx], asxz[i], asxz[i + sx]) * idx;
      const float dsyz_dy = -dminus(asyz[i - 2], asyz[i - 1], asyz[i], asyz[i + 1]) * idy;
      float acc = l2u * dszz_dz * cz.K * dt + l * dsxx_dz * cz.K * dt + l * dsyy_dz * cz.K * dt +
                  u * cy.Kh * dsyz_dy * dt + u * cx.Kh * dsxz_dx * dt;
      if (zs) acc += cz.a * (nzp(g, psz + PSI_VA * g.slab_z, z, x, y) * idz);
      if (ys) acc += cy.ah * (nym(g, psy + PSI_VB1 * g.slab_y, z, x, y) * idy);
      if (xs) acc += cx.ah * (nxm(g, psx + PSI_VB1 * g.slab_x, z, x, y) * idx);
      const float v = avz0 + acc;
      a.vz[i] = v;
      if (xs) { const long long k = PSI_SAB1 * g.slab_x + psi_x_idx(g, z, x, y); px[k] = cx.b * px[k] + b * v * dt; }
      if (zs) { const long long k = PSI_SAA * g.slab_z + psi_z_idx(g, z, x, y); pz[k] = cz.bh * pz[k] + b * v * dt; }
      if (ys) { const long long k = PSI_SAB1 * g.slab_y + psi_y_idx(g, z, x, y); py[k] = cy.b * py[k] + b * v * dt; }
    }
    // ---- adjoint vy
    {
      const float dsyy_dy = -dplus(asyy[i - 1], asyy[i], asyy[i + 1], asyy[i + 2]) * idy;
      const float dsxx_dy = -dplus(asxx[i - 1], asxx[i], asxx[i + 1], asxx[i + 2]) * idy;
      const float dszz_dy = -dplus(aszz[i - 1], aszz[i], aszz[i + 1], aszz[i + 2]) * idy;
      const float dsxy_dx = -dminus(asxy[i - 2 * sx], asxy[i - sx], asxy[i], asxy[i + sx]) * idx;
      const float dsyz_dz = -dminus(asyz[i - 2 * sz], asyz[i - sz], asyz[i], asyz[i + sz]) * idz;
      float acc = l2u * dsyy_dy * cy.K * dt + l * dsxx_dy * cy.K * dt + l * dszz_dy * cy.K * dt +
                  u * cx.Kh * dsxy_dx * dt + u * cz.Kh * dsyz_dz * dt;
      if (ys) acc += cy.a * (nyp(g, psy + PSI_VA * g.slab_y, z, x, y) * idy);
      if (xs) acc += cx.ah * (nxm(g, psx + PSI_VB2 * g.slab_x, z, x, y) * idx);
      if (zs) acc += cz.ah * (nzm(g, psz + PSI_VB2 * g.slab_z, z, x, y) * idz);
      const float v = avy0 + acc;
      a.vy[i] = v;
      if (xs) { const long long k = PSI_SAB2 * g.slab_x + psi_x_idx(g, z, x, y); px[k] = cx.b * px[k] + b * v * dt; }
      if (zs) { const long long k = PSI_SAB2 * g.slab_z + psi_z_idx(g, z, x, y); pz[k] = cz.bh * pz[k] + b * v * dt; }
      if (ys) { const long long k = PSI_SAA * g.slab_y + psi_y_idx(g, z, x, y); py[k] = cy.b * py[k] + b * v * dt; }
    }
  }
}

template <int BX>
__global__ void __launch_bounds__(32 * BX)
k_rev_stress(Geo g, Fields f, Fields a, Psi ps, const float *__restrict__ lam,
             const float *__restrict__ mu, const float *__restrict__ buoy, float *glam,
             float *gmu, int zchunk, int nzc, int do_rev, int do_adj, SrcArgs src) {
  const int y = blockIdx.x * 32 + threadIdx.x;
  const int x = blockIdx.y * BX + threadIdx.y;
  const int zc = blockIdx.z % nzc;
  const int z0 = max(zc * zchunk, 2);
  const int z1 = min(zc * zchunk + zchunk, g.nz - 2);
  if (x < 2 || x > g.nx - 3 || y < 2 || y > g.ny - 3 || z0 >= z1) return;

  const int np = g.np, nz = g.nz, nx = g.nx, ny = g.ny;
  const long long sz = g.sz;
  const int sx = g.sx;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;
  const bool xin = x >= np && x <= nx - 1 - np, yin = y >= np && y <= ny - 1 - np;
  const bool xs = slab_s(x, nx, np), ys = slab_s(y, ny, np);
  const Coef cx = coef(g.cx, nx, x), cy = coef(g.cy, ny, y);
  const long long src_cell = (do_rev && src.cell) ? src.cell[0] : -1;
  const float src_amp = (do_rev && src.stf) ? src.stf[src.it] : 0.f;

  const float *__restrict__ vz = f.vz;
  const float *__restrict__ vx = f.vx;
  const float *__restrict__ vy = f.vy;
  const float *__restrict__ avz = a.vz;
  const float *__restrict__ avx = a.vx;
  const float *__restrict__ avy = a.vy;
  const float *psz = ps.z, *psx = ps.x, *psy = ps.y;
  float *pz = ps.z, *px = ps.x, *py = ps.y;

  for (int z = z0; z < z1; ++z) {
    const long long i = ((long long)z * nx + x) * sx + y;
    const float l = lam[i], u = mu[i], l2u = l + 2.0f * u;
    const float azz0 = a.szz[i], axx0 = a.sxx[i], ayy0 = a.syy[i];
    const float axz0 = a.sxz[i], axy0 = a.sxy[i], ayz0 = a.syz[i];
    if (do_rev) {
      float szz = f.szz[i], sxx = f.sxx[i], syy = f.syy[i];
      if (i == src_cell) {
        const double am = 2250000.0 * (double)src_amp * (double)dt;
        szz = (float)((double)szz - am);
        sxx = (float)((double)sxx - am);
        syy = (float)((double)syy - am);
      }
      if (xin && yin && z >= np && z <= nz - 1 - np) {
        const float ezz = dminus(vz[i - 2 * sz], vz[i - sz], vz[i], vz[i + sz]) * idz;
        const float exx = dminus(vx[i - 2 * sx], vx[i - sx], vx[i], vx[i + sx]) * idx;
        const float eyy = dminus(vy[i - 2], vy[i - 1], vy[i], vy[i + 1]) * idy;
        szz = szz - (l2u * ezz + l * exx + l * eyy) * dt;
        sxx = sxx - (l * ezz + l2u * exx + l * eyy) * dt;
        syy = syy - (l * ezz + l * exx + l2u * eyy) * dt;
        const float dvx_dz = dplus(vx[i - sz], vx[i], vx[i + sz], vx[i + 2 * sz]) * idz;
        const float dvx_dy = dplus(vx[i - 1], vx[i], vx[i + 1], vx[i + 2]) * idy;
        const float dvz_dx = dplus(vz[i - sx], vz[i], vz[i + sx], vz[i + 2 * sx]) * idx;
        const float dvz_dy = dplus(vz[i - 1], vz[i], vz[i + 1], vz[i + 2]) * idy;
        const float dvy_dx = dplus(vy[i - sx], vy[i], vy[i + sx], vy[i + 2 * sx]) * idx;
        const float dvy_dz = dplus(vy[i - sz], vy[i], vy[i + sz], vy[i + 2 * sz]) * idz;
        f.sxz[i] = f.sxz[i] - u * (dvx_dz + dvz_dx) * dt;
        f.sxy[i] = f.sxy[i] - u * (dvx_dy + dvy_dx) * dt;
        f.syz[i] = f.syz[i] - u * (dvy_dz + dvz_dy) * dt;
        glam[i] = glam[i] - (azz0 + axx0 + ayy0) * (ezz + exx + eyy) * dt;
        gmu[i] = gmu[i] - (2.0f * azz0 * ezz + 2.0f * axx0 * exx + 2.0f * ayy0 * eyy +
                           axz0 * (dvx_dz + dvz_dx) + ayz0 * (dvy_dz + dvz_dy) +
                           axy0 * (dvy_dx + dvx_dy)) * dt;
      }
      f.szz[i] = szz; f.sxx[i] = sxx; f.syy[i] = syy;
    }
    if (!do_adj) continue;
    const bool zs = slab_s(z, nz, np);
    const Coef cz = coef(g.cz, nz, z);
    const float b = buoy[i];
    // ---- sxz
    {
      const float dvz_dx = -dplus(avz[i - sx], avz[i], avz[i + sx], avz[i + 2 * sx]) * idx;
      const float dvx_dz = -dplus(avx[i - sz], avx[i], avx[i + sz], avx[i + 2 * sz]) * idz;
      float acc = dvz_dx * cx.K * b * dt + dvx_dz * cz.K * b * dt;
      if (xs) acc += cx.a * (nxp(g, psx + PSI_SAB1 * g.slab_x, z, x, y) * idx);
      if (zs) acc += cz.a * (nzp(g, psz + PSI_SAB1 * g.slab_z, z, x, y) * idz);
      const float s = axz0 + acc;
      a.sxz[i] = s;
      if (xs) { const long long k = PSI_VB1 * g.slab_x + psi_x_idx(g, z, x, y); px[k] = cx.bh * px[k] + s * u * dt; }
      if (zs) { const long long k = PSI_VB1 * g.slab_z + psi_z_idx(g, z, x, y); pz[k] = cz.bh * pz[k] + s * u * dt; }
    }
    // ---- sxy
    {
      const float dvy_dx = -dplus(avy[i - sx], avy[i], avy[i + sx], avy[i + 2 * sx]) * idx;
      const float dvx_dy = -dplus(avx[i - 1], avx[i], avx[i + 1], avx[i + 2]) * idy;
      float acc = dvy_dx * cx.K * b * dt + dvx_dy * cy.K * b * dt;
      if (xs) acc += cx.a * (nxp(g, psx + PSI_SAB2 * g.slab_x, z, x, y) * idx);
      if (ys) acc += cy.a * (nyp(g, psy + PSI_SAB2 * g.slab_y, z, x, y) * idy);
      const float s = axy0 + acc;
      a.sxy[i] = s;
      if (ys) { const long long k = PSI_VB2 * g.slab_y + psi_y_idx(g, z, x, y); py[k] = cy.bh * py[k] + s * u * dt; }
      if (xs) { const long long k = PSI_VB2 * g.slab_x + psi_x_idx(g, z, x, y); px[k] = cx.bh * px[k] + s * u * dt; }
    }
    // ---- syz
    {
      const float dvz_dy = -dplus(avz[i - 1], avz[i], avz[i + 1], avz[i + 2]) * idy;
      const float dvy_dz = -dplus(avy[i - sz], avy[i], avy[i + sz], avy[i + 2 * sz]) * idz;
      float acc = dvz_dy * cy.K * b * dt + dvy_dz * cz.K * b * dt;
      if (ys) acc += cy.a * (nyp(g, psy + PSI_SAB1 * g.slab_y, z, x, y) * idy);
      if (zs) acc += cz.a * (nzp(g, psz + PSI_SAB2 * g.slab_z, z, x, y) * idz);
      const float s = ayz0 + acc;
      a.syz[i] = s;
      if (ys) { const long long k = PSI_VB1 * g.slab_y + psi_y_idx(g, z, x, y); py[k] = cy.bh * py[k] + s * u * dt; }
      if (zs) { const long long k = PSI_VB2 * g.slab_z + psi_z_idx(g, z, x, y); pz[k] = cz.bh * pz[k] + s * u * dt; }
    }
    // ---- normal stresses
    {
      const float dvx_dx = -dminus(avx[i - 2 * sx], avx[i - sx], avx[i], avx[i + sx]) * idx;
      const float dvz_dz = -dminus(avz[i - 2 * sz], avz[i - sz], avz[i], avz[i + sz]) * idz;
      const float dvy_dy = -dminus(avy[i - 2], avy[i - 1], avy[i], avy[i + 1]) * idy;
      float sxx = axx0 + b * dvx_dx * cx.Kh * dt;
      float szz = azz0 + b * dvz_dz * cz.Kh * dt;
      float syy = ayy0 + b * dvy_dy * cy.Kh * dt;
      if (xs) sxx += cx.ah * (nxm(g, psx + PSI_SAA * g.slab_x, z, x, y) * idx);
      if (zs) szz += cz.ah * (nzm(g, psz + PSI_SAA * g.slab_z, z, x, y) * idz);
      if (ys) syy += cy.ah * (nym(g, psy + PSI_SAA * g.slab_y, z, x, y) * idy);
      a.sxx[i] = sxx; a.szz[i] = szz; a.syy[i] = syy;
      if (xs) { const long long k = PSI_VA * g.slab_x + psi_x_idx(g, z, x, y); px[k] = cx.b * px[k] + l * szz * dt + l2u * sxx * dt + l * syy * dt; }
      if (zs) { const long long k = PSI_VA * g.slab_z + psi_z_idx(g, z, x, y); pz[k] = cz.b * pz[k] + l2u * szz * dt + l * sxx * dt + l * syy * dt; }
      if (ys) { const long long k = PSI_VA * g.slab_y + psi_y_idx(g, z, x, y); py[k] = cy.b * py[k] + l * szz * dt + l * sxx * dt + l2u * syy * dt; }
    }
  }
}

void launch_rev_velocity(int bx, dim3 grid, cudaStream_t st, const Geo &g, const Fields &f,
                         const Fields &a, const Psi &ps, const float *lam, const float *mu,
                         const float *buoy, float *grho, int zchunk, int nzc, int do_rev,
                         int do_adj) {
  if (bx == 8)
    k_rev_velocity<8><<<grid, dim3(32, 8), 0, st>>>(g, f, a, ps, lam, mu, buoy, grho, zchunk,
                                                   nzc, do_rev, do_adj);
  else
    k_rev_velocity<4><<<grid, dim3(32, 4), 0, st>>>(g, f, a, ps, lam, mu, buoy, grho, zchunk,
                                                   nzc, do_rev, do_adj);
}

void launch_rev_stress(int bx, dim3 grid, cudaStream_t st, const Geo &g, const Fields &f,
                       const Fields &a, const Psi &ps, const float *lam, const float *mu,
                       const float *buoy, float *glam, float *gmu, int zchunk, int nzc,
                       int do_rev, int do_adj, const SrcArgs &src) {
  if (bx == 8)
    k_rev_stress<8><<<grid, dim3(32, 8), 0, st>>>(g, f, a, ps, lam, mu, buoy, glam, gmu, zchunk,
                                                 nzc, do_rev, do_adj, src);
  else
    k_rev_stress<4><<<grid, dim3(32, 4), 0, st>>>(g, f, a, ps, lam, mu, buoy, glam, gmu, zchunk,
                                                 nzc, do_rev, do_adj, src);
}

}  // namespace efwi
