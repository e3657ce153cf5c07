// Forward half-steps of the staggered-grid velocity-stress scheme.
//
// K_S  stress update + C-PML (slabs only) + point-source injection
//      (restates stress.cu:36-97 and add_source, utilities.cu:442-479)
// K_V  velocity update + C-PML (slabs only)
//      (restates velocity.cu:35-96, quirks Q1 and Q2 kept)
//
// Tiling: a CTA owns a 32 (y) x BX (x) column tile and marches a chunk of z.
// The z-stencil operands stay in per-thread register queues; the y and x
// neighbours are read through the read-only path and served by L1 (the y
// neighbours are in the same 128-byte lines as the warp's own loads, the x
// neighbours are the rows of the other warps of the CTA).  Each interior
// value therefore crosses HBM once per half-step.
#include "efwi_common.cuh"
#include "efwi_kernels.h"

namespace efwi {

// One thread's column (y, x) of z chunk zc of shot `shot`; the kernels
// below map their launch onto these columns.
__device__ __forceinline__ void stress_fwd_column(const Geo &g, const Fields &f, const Psi &ps,
                                                  const float *__restrict__ lam,
                                                  const float *__restrict__ mu, int y, int x,
                                                  int shot, int zc, int zchunk,
                                                  const SrcArgs &src) {
  const int z0 = max(zc * zchunk, 2);
  const int z1 = min(zc * zchunk + zchunk, g.nz - 2);
  if (x < 2 || x > g.nx - 3 || y < 2 || y > g.ny - 3 || z0 >= z1) return;

  const long long so = (long long)shot * g.N;
  const float *__restrict__ vz = f.vz + so;
  const float *__restrict__ vx = f.vx + so;
  const float *__restrict__ vy = f.vy + so;
  float *szz = f.szz + so, *sxx = f.sxx + so, *syy = f.syy + so;
  float *sxz = f.sxz + so, *sxy = f.sxy + so, *syz = f.syz + so;
  float *pzb = ps.z + (long long)shot * 6 * g.slab_z;
  float *pxb = ps.x + (long long)shot * 6 * g.slab_x;
  float *pyb = ps.y + (long long)shot * 6 * g.slab_y;

  const int np = g.np, nz = g.nz, nx = g.nx, ny = g.ny;
  const long long sz = g.sz;
  const int sx = g.sx;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;

  const bool xs = slab_s(x, nx, np), ys = slab_s(y, ny, np);
  float Kx = 1.f, ax = 0.f, bx = 0.f, Kxh = 1.f, axh = 0.f, bxh = 0.f;
  float Ky = 1.f, ay = 0.f, by = 0.f, Kyh = 1.f, ayh = 0.f, byh = 0.f;
  if (xs) {
    Kx = g.cx[CK * nx + x]; ax = g.cx[CA * nx + x]; bx = g.cx[CB * nx + x];
    Kxh = g.cx[CKH * nx + x]; axh = g.cx[CAH * nx + x]; bxh = g.cx[CBH * nx + x];
  }
  if (ys) {
    Ky = g.cy[CK * ny + y]; ay = g.cy[CA * ny + y]; by = g.cy[CB * ny + y];
    Kyh = g.cy[CKH * ny + y]; ayh = g.cy[CAH * ny + y]; byh = g.cy[CBH * ny + y];
  }
  const long long src_cell = src.cell ? src.cell[shot] : -1;
  const float src_amp = src.stf ? src.stf[(long long)shot * src.nt + src.it] : 0.f;

  long long i = ((long long)z0 * nx + x) * sx + y;
  // z queues: vz needs z-2..z+1 (D-), vx and vy need z-1..z+2 (D+).
  float qz0 = vz[i - 2 * sz], qz1 = vz[i - sz], qz2 = vz[i], qz3 = vz[i + sz];
  float qx0 = vx[i - sz], qx1 = vx[i], qx2 = vx[i + sz], qx3 = vx[i + 2 * sz];
  float qy0 = vy[i - sz], qy1 = vy[i], qy2 = vy[i + sz], qy3 = vy[i + 2 * sz];

  for (int z = z0; z < z1; ++z, i += sz) {
    const bool zs = slab_s(z, nz, np);
    float ezz = dminus(qz0, qz1, qz2, qz3) * idz;
    float exx = dminus(vx[i - 2 * sx], vx[i - sx], qx1, vx[i + sx]) * idx;
    float eyy = dminus(vy[i - 2], vy[i - 1], qy1, vy[i + 1]) * idy;
    float dvx_dz = dplus(qx0, qx1, qx2, qx3) * idz;
    float dvy_dz = dplus(qy0, qy1, qy2, qy3) * idz;
    float dvx_dy = dplus(vx[i - 1], qx1, vx[i + 1], vx[i + 2]) * idy;
    float dvz_dx = dplus(vz[i - sx], qz2, vz[i + sx], vz[i + 2 * sx]) * idx;
    float dvz_dy = dplus(vz[i - 1], qz2, vz[i + 1], vz[i + 2]) * idy;
    float dvy_dx = dplus(vy[i - sx], qy1, vy[i + sx], vy[i + 2 * sx]) * idx;

    if (zs) {
      const float Kz = g.cz[CK * nz + z], az = g.cz[CA * nz + z], bz = g.cz[CB * nz + z];
      const float Kzh = g.cz[CKH * nz + z], azh = g.cz[CAH * nz + z], bzh = g.cz[CBH * nz + z];
      const long long k = psi_z_idx(g, z, x, y);
      float m;
      m = bz * pzb[PSI_VA * g.slab_z + k] + az * ezz;
      pzb[PSI_VA * g.slab_z + k] = m; ezz = ezz * Kz + m;
      m = bzh * pzb[PSI_VB1 * g.slab_z + k] + azh * dvx_dz;
      pzb[PSI_VB1 * g.slab_z + k] = m; dvx_dz = dvx_dz * Kzh + m;
      m = bzh * pzb[PSI_VB2 * g.slab_z + k] + azh * dvy_dz;
      pzb[PSI_VB2 * g.slab_z + k] = m; dvy_dz = dvy_dz * Kzh + m;
    }
    if (xs) {
      const long long k = psi_x_idx(g, z, x, y);
      float m;
      m = bx * pxb[PSI_VA * g.slab_x + k] + ax * exx;
      pxb[PSI_VA * g.slab_x + k] = m; exx = exx * Kx + m;
      m = bxh * pxb[PSI_VB1 * g.slab_x + k] + axh * dvz_dx;
      pxb[PSI_VB1 * g.slab_x + k] = m; dvz_dx = dvz_dx * Kxh + m;
      m = bxh * pxb[PSI_VB2 * g.slab_x + k] + axh * dvy_dx;
      pxb[PSI_VB2 * g.slab_x + k] = m; dvy_dx = dvy_dx * Kxh + m;
    }
    if (ys) {
      const long long k = psi_y_idx(g, z, x, y);
      float m;
      m = by * pyb[PSI_VA * g.slab_y + k] + ay * eyy;
      pyb[PSI_VA * g.slab_y + k] = m; eyy = eyy * Ky + m;
      m = byh * pyb[PSI_VB1 * g.slab_y + k] + ayh * dvz_dy;
      pyb[PSI_VB1 * g.slab_y + k] = m; dvz_dy = dvz_dy * Kyh + m;
      m = byh * pyb[PSI_VB2 * g.slab_y + k] + ayh * dvx_dy;
      pyb[PSI_VB2 * g.slab_y + k] = m; dvx_dy = dvx_dy * Kyh + m;
    }

    const float l = lam[i], u = mu[i], l2u = l + 2.0f * u;
    float nzz = szz[i] + (l2u * ezz + l * exx + l * eyy) * dt;
    float nxx = sxx[i] + (l * ezz + l2u * exx + l * eyy) * dt;
    float nyy = syy[i] + (l * ezz + l * exx + l2u * eyy) * dt;
    if (i == src_cell) {
      // add_source runs after the stress kernel; its amplitude is formed in
      // double from pow(1500, 2) (utilities.cu:450-461).
      const double a = 2250000.0 * (double)src_amp * (double)dt;
      nzz = (float)((double)nzz + a);
      nxx = (float)((double)nxx + a);
      nyy = (float)((double)nyy + a);
    }
    szz[i] = nzz; sxx[i] = nxx; syy[i] = nyy;
    sxz[i] = sxz[i] + u * (dvx_dz + dvz_dx) * dt;
    sxy[i] = sxy[i] + u * (dvx_dy + dvy_dx) * dt;
    syz[i] = syz[i] + u * (dvy_dz + dvz_dy) * dt;

    qz0 = qz1; qz1 = qz2; qz2 = qz3;
    qx0 = qx1; qx1 = qx2; qx2 = qx3;
    qy0 = qy1; qy1 = qy2; qy2 = qy3;
    if (z + 1 < z1) {
      qz3 = vz[i + 2 * sz];
      qx3 = vx[i + 3 * sz];
      qy3 = vy[i + 3 * sz];
    }
  }
}

__device__ __forceinline__ void velocity_fwd_column(const Geo &g, const Fields &f, const Psi &ps,
                                                    const float *__restrict__ buoy, int y, int x,
                                                    int shot, int zc, int zchunk) {
  const int z0 = max(zc * zchunk, 2);
  const int z1 = min(zc * zchunk + zchunk, g.nz - 2);
  if (x < 2 || x > g.nx - 3 || y < 2 || y > g.ny - 3 || z0 >= z1) return;

  const long long so = (long long)shot * g.N;
  float *vz = f.vz + so, *vx = f.vx + so, *vy = f.vy + so;
  const float *__restrict__ szz = f.szz + so;
  const float *__restrict__ sxx = f.sxx + so;
  const float *__restrict__ syy = f.syy + so;
  const float *__restrict__ sxz = f.sxz + so;
  const float *__restrict__ sxy = f.sxy + so;
  const float *__restrict__ syz = f.syz + so;
  float *pzb = ps.z + (long long)shot * 6 * g.slab_z;
  float *pxb = ps.x + (long long)shot * 6 * g.slab_x;
  float *pyb = ps.y + (long long)shot * 6 * g.slab_y;

  const int np = g.np, nz = g.nz, nx = g.nx, ny = g.ny;
  const long long sz = g.sz;
  const int sx = g.sx;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;

  const bool xs = slab_v(x, nx, np), ys = slab_v(y, ny, np);
  float Kx = 1.f, ax = 0.f, bx = 0.f, Kxh = 1.f, axh = 0.f, bxh = 0.f;
  float Ky = 1.f, ay = 0.f, by = 0.f, Kyh = 1.f, ayh = 0.f, byh = 0.f;
  if (xs) {
    Kx = g.cx[CK * nx + x]; ax = g.cx[CA * nx + x]; bx = g.cx[CB * nx + x];
    Kxh = g.cx[CKH * nx + x]; axh = g.cx[CAH * nx + x]; bxh = g.cx[CBH * nx + x];
  }
  if (ys) {
    Ky = g.cy[CK * ny + y]; ay = g.cy[CA * ny + y]; by = g.cy[CB * ny + y];
    Kyh = g.cy[CKH * ny + y]; ayh = g.cy[CAH * ny + y]; byh = g.cy[CBH * ny + y];
  }

  long long i = ((long long)z0 * nx + x) * sx + y;
  // z queues: szz needs z-1..z+2 (D+), sxz and syz need z-2..z+1 (D-).
  float qa0 = szz[i - sz], qa1 = szz[i], qa2 = szz[i + sz], qa3 = szz[i + 2 * sz];
  float qb0 = sxz[i - 2 * sz], qb1 = sxz[i - sz], qb2 = sxz[i], qb3 = sxz[i + sz];
  float qc0 = syz[i - 2 * sz], qc1 = syz[i - sz], qc2 = syz[i], qc3 = syz[i + sz];

  for (int z = z0; z < z1; ++z, i += sz) {
    const bool zs = slab_s(z, nz, np);
    const float b = buoy[i];
    float dszz_dz = dplus(qa0, qa1, qa2, qa3) * idz;
    float dsxz_dx = dminus(sxz[i - 2 * sx], sxz[i - sx], qb2, sxz[i + sx]) * idx;
    float dsyz_dy = dminus(syz[i - 2], syz[i - 1], qc2, syz[i + 1]) * idy;
    float dsxz_dz = dminus(qb0, qb1, qb2, qb3) * idz;
    float dsxx_dx = dplus(sxx[i - sx], sxx[i], sxx[i + sx], sxx[i + 2 * sx]) * idx;
    const float sxy_m1 = sxy[i - 1], sxy_0 = sxy[i];
    float dsxy_dy = dminus(sxy[i - 2], sxy_m1, sxy_0, sxy[i + 1]) * idy;
    float dsyz_dz = dminus(qc0, qc1, qc2, qc3) * idz;
    // Quirk Q1 (velocity.cu:79): c2 * (sxy[i-1] - sxy[i-2]) along x.
    const float sxy_xm1 = sxy[i - sx], sxy_xm2 = sxy[i - 2 * sx];
    float dsxy_dx = (EFWI_C1 * (sxy_0 - sxy_xm1) - EFWI_C2 * (sxy_xm1 - sxy_xm2)) * idx;
    float dsyy_dy = dplus(syy[i - 1], syy[i], syy[i + 1], syy[i + 2]) * idy;

    if (zs) {
      const float Kz = g.cz[CK * nz + z], az = g.cz[CA * nz + z], bz = g.cz[CB * nz + z];
      const float Kzh = g.cz[CKH * nz + z], azh = g.cz[CAH * nz + z], bzh = g.cz[CBH * nz + z];
      const long long k = psi_z_idx(g, z, x, y);
      float m;
      m = bzh * pzb[PSI_SAA * g.slab_z + k] + azh * dszz_dz;
      pzb[PSI_SAA * g.slab_z + k] = m; dszz_dz = dszz_dz * Kzh + m;
      m = bz * pzb[PSI_SAB1 * g.slab_z + k] + az * dsxz_dz;
      pzb[PSI_SAB1 * g.slab_z + k] = m; dsxz_dz = dsxz_dz * Kz + m;
      m = bz * pzb[PSI_SAB2 * g.slab_z + k] + az * dsyz_dz;
      pzb[PSI_SAB2 * g.slab_z + k] = m; dsyz_dz = dsyz_dz * Kz + m;
    }
    if (xs) {
      const long long k = psi_x_idx(g, z, x, y);
      float m;
      m = bx * pxb[PSI_SAB1 * g.slab_x + k] + ax * dsxz_dx;
      pxb[PSI_SAB1 * g.slab_x + k] = m; dsxz_dx = dsxz_dx * Kx + m;
      m = bxh * pxb[PSI_SAA * g.slab_x + k] + axh * dsxx_dx;
      pxb[PSI_SAA * g.slab_x + k] = m; dsxx_dx = dsxx_dx * Kxh + m;
      m = bx * pxb[PSI_SAB2 * g.slab_x + k] + ax * dsxy_dx;
      pxb[PSI_SAB2 * g.slab_x + k] = m; dsxy_dx = dsxy_dx * Kx + m;
    }
    if (ys) {
      const long long k = psi_y_idx(g, z, x, y);
      float m;
      m = by * pyb[PSI_SAB1 * g.slab_y + k] + ay * dsyz_dy;
      pyb[PSI_SAB1 * g.slab_y + k] = m; dsyz_dy = dsyz_dy * Ky + m;
      m = by * pyb[PSI_SAB2 * g.slab_y + k] + ay * dsxy_dy;
      pyb[PSI_SAB2 * g.slab_y + k] = m; dsxy_dy = dsxy_dy * Ky + m;
      m = byh * pyb[PSI_SAA * g.slab_y + k] + ayh * dsyy_dy;
      pyb[PSI_SAA * g.slab_y + k] = m; dsyy_dy = dsyy_dy * Kyh + m;
    }

    vz[i] = vz[i] + (dszz_dz + dsxz_dx + dsyz_dy) * b * dt;
    vx[i] = vx[i] + (dsxz_dz + dsxx_dx + dsxy_dy) * b * dt;
    vy[i] = vy[i] + (dsyz_dz + dsxy_dx + dsyy_dy) * b * dt;

    qa0 = qa1; qa1 = qa2; qa2 = qa3;
    qb0 = qb1; qb1 = qb2; qb2 = qb3;
    qc0 = qc1; qc1 = qc2; qc2 = qc3;
    if (z + 1 < z1) {
      qa3 = szz[i + 3 * sz];
      qb3 = sxz[i + 2 * sz];
      qc3 = syz[i + 2 * sz];
    }
  }
}

template <int BX>
__global__ void __launch_bounds__(32 * BX)
k_stress_fwd(Geo g, Fields f, Psi ps, const float *__restrict__ lam,
             const float *__restrict__ mu, int zchunk, int nzc, SrcArgs src) {
  const int shot = blockIdx.z / nzc;
  stress_fwd_column(g, f, ps, lam, mu, blockIdx.x * 32 + threadIdx.x, blockIdx.y * BX + threadIdx.y,
                    shot, blockIdx.z - shot * nzc, zchunk, src);
}

template <int BX>
__global__ void __launch_bounds__(32 * BX)
k_velocity_fwd(Geo g, Fields f, Psi ps, const float *__restrict__ buoy, int zchunk, int nzc) {
  const int shot = blockIdx.z / nzc;
  velocity_fwd_column(g, f, ps, buoy, blockIdx.x * 32 + threadIdx.x, blockIdx.y * BX + threadIdx.y,
                      shot, blockIdx.z - shot * nzc, zchunk);
}

// Several domains of different sizes (shot windows) in one persistent
// launch: CTA b takes tiles b, b + gridDim.x, ... of the concatenated tile
// lists; tile t of domain d is (z chunk, x tile, y tile) in that order.
__device__ __forceinline__ int find_domain(const Domain *dom, int ndom, int t) {
  int lo = 0, hi = ndom - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (dom[mid].tile0 <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int BX>
__global__ void __launch_bounds__(32 * BX)
k_stress_fwd_multi(const Domain *__restrict__ dom, int ndom, int ntiles, int zchunk, int it) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Domain &d = dom[find_domain(dom, ndom, t)];
    const int lt = t - d.tile0;
    const int by = lt % d.tiles_y, r = lt / d.tiles_y;
    const int bx = r % d.tiles_x, zc = r / d.tiles_x;
    SrcArgs src{&d.src_cell, d.stf, d.nt, it};
    stress_fwd_column(d.g, d.f, d.ps, d.lam, d.mu, by * 32 + threadIdx.x, bx * BX + threadIdx.y, 0,
                      zc, zchunk, src);
  }
}

template <int BX>
__global__ void __launch_bounds__(32 * BX)
k_velocity_fwd_multi(const Domain *__restrict__ dom, int ndom, int ntiles, int zchunk) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const Domain &d = dom[find_domain(dom, ndom, t)];
    const int lt = t - d.tile0;
    const int by = lt % d.tiles_y, r = lt / d.tiles_y;
    const int bx = r % d.tiles_x, zc = r / d.tiles_x;
    velocity_fwd_column(d.g, d.f, d.ps, d.buoy, by * 32 + threadIdx.x, bx * BX + threadIdx.y, 0, zc,
                        zchunk);
  }
}

// Receivers of all domains (recording, utilities.cu:481-495): receiver u
// sits at cell rec_cell[u] of domain rec_dom[u] and is receiver rec_r[u] of
// that domain's shot, whose time-major traces [nt][3][nrec] start at
// trace_off.  Receivers outside their window are not listed (their traces
// stay zero).
__global__ void k_record_multi(const Domain *__restrict__ dom, const int *__restrict__ rec_dom,
                               const int *__restrict__ rec_cell, const int *__restrict__ rec_r,
                               int nrec, float *traces_tm, int it, const int *it_dev) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nrec) return;
  if (it_dev) it = *it_dev + 1;
  const Domain &d = dom[rec_dom[u]];
  const int i = rec_cell[u], r = rec_r[u];
  float *t = traces_tm + d.trace_off + (long long)it * 3 * d.nrec;
  t[r] = d.f.vx[i];
  t[d.nrec + r] = d.f.vy[i];
  t[2 * d.nrec + r] = d.f.vz[i];
}

int multi_blocks(int bx) {
  static int cached[2] = {0, 0};
  const int k = bx == 8 ? 1 : 0;
  if (!cached[k]) {
    int dev = 0, sms = 148, a = 1, b = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (bx == 8) {
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_stress_fwd_multi<8>, 256, 0);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_velocity_fwd_multi<8>, 256, 0);
    } else {
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, k_stress_fwd_multi<4>, 128, 0);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_velocity_fwd_multi<4>, 128, 0);
    }
    cached[k] = sms * max(1, min(a, b));
  }
  return cached[k];
}

void launch_fwd_multi(int bx, int blocks, cudaStream_t st, const Domain *dom, int ndom, int ntiles,
                      int zchunk, int it) {
  if (bx == 8) {
    k_stress_fwd_multi<8><<<blocks, dim3(32, 8), 0, st>>>(dom, ndom, ntiles, zchunk, it);
    k_velocity_fwd_multi<8><<<blocks, dim3(32, 8), 0, st>>>(dom, ndom, ntiles, zchunk);
  } else {
    k_stress_fwd_multi<4><<<blocks, dim3(32, 4), 0, st>>>(dom, ndom, ntiles, zchunk, it);
    k_velocity_fwd_multi<4><<<blocks, dim3(32, 4), 0, st>>>(dom, ndom, ntiles, zchunk);
  }
}

void launch_stress_fwd(int bx, dim3 grid, cudaStream_t st, const Geo &g, const Fields &f,
                       const Psi &ps, const float *lam, const float *mu, int zchunk, int nzc,
                       const SrcArgs &src) {
  if (bx == 8)
    k_stress_fwd<8><<<grid, dim3(32, 8), 0, st>>>(g, f, ps, lam, mu, zchunk, nzc, src);
  else
    k_stress_fwd<4><<<grid, dim3(32, 4), 0, st>>>(g, f, ps, lam, mu, zchunk, nzc, src);
}

void launch_velocity_fwd(int bx, dim3 grid, cudaStream_t st, const Geo &g, const Fields &f,
                         const Psi &ps, const float *buoy, int zchunk, int nzc) {
  if (bx == 8)
    k_velocity_fwd<8><<<grid, dim3(32, 8), 0, st>>>(g, f, ps, buoy, zchunk, nzc);
  else
    k_velocity_fwd<4><<<grid, dim3(32, 4), 0, st>>>(g, f, ps, buoy, zchunk, nzc);
}

}  // namespace efwi
