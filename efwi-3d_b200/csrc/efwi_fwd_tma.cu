// Forward half-steps with TMA-staged planes (same arithmetic as efwi_fwd.cu).
//
// K_S: halo boxes vz, vx, vy (x/y neighbours from shared memory), point
//      boxes lambda, mu and the six stresses; the z neighbours of vz, vx, vy
//      stay in register queues fed by plain loads one plane ahead.
// K_V: halo boxes sxz, syz, sxx, sxy, syy, point boxes vz, vx, vy and the
//      buoyancy; z queues of szz, sxz, syz.
// Results are stored straight from registers (one 128-byte row per warp).
// Restated reference kernels: stress.cu:36-97, add_source
// (utilities.cu:442-479), velocity.cu:35-96 (quirks Q1 and Q2 kept).
//
// Fused epilogues (efwi_fuse.cuh): K_S stores the step's starting state at
// the boundary-shell points (gradient sweeps, from_bnd); K_V records the
// receivers (recording).
#include "efwi_common.cuh"
#include "efwi_fuse.cuh"
#include "efwi_kernels.h"
#include "efwi_tma.cuh"

namespace efwi {

template <int TX, int R, int MINB>
__global__ void __launch_bounds__(32 * TX, MINB)
k_stress_fwd_tma(const __grid_constant__ Maps<11> maps, Geo g, Fields f, Psi ps, int zchunk,
                 int nzc, SrcArgs src, ShellMap shell, int *status) {
  using Ring = PlaneRing<3, 8, 2, TX, R>;  // vz vx vy | szz sxx syy sxz sxy syz | lam mu
  extern __shared__ __align__(128) unsigned char smem[];
  Ring ring;
  ring.bind(smem);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int y0 = blockIdx.x * 32, x0 = blockIdx.y * TX;
  const int shot = blockIdx.z / nzc;
  const int zc = blockIdx.z - shot * nzc;
  const int z0 = max(zc * zchunk, 2);
  const int z1 = min(zc * zchunk + zchunk, g.nz - 2);
  if (z0 >= z1) return;  // uniform over the CTA, before any barrier
  const int nq = z1 - z0;
  const int y = y0 + tx, x = x0 + ty;
  const int np = g.np, nz = g.nz, nx = g.nx, ny = g.ny;
  const bool act = x >= 2 && x <= nx - 3 && y >= 2 && y <= ny - 3;

  if (tid == 0) ring.init();
  __syncthreads();
  if (tid == 0)
    for (int q = 0; q < nq && q < R; ++q) ring.issue(maps, q, y0, x0, shot * nz + z0 + q, z0 + q);

  const long long so = (long long)shot * g.N;
  const float *__restrict__ vz = f.vz + so;
  const float *__restrict__ vx = f.vx + so;
  const float *__restrict__ vy = f.vy + so;
  float *szz = f.szz + so, *sxx = f.sxx + so, *syy = f.syy + so;
  float *sxz = f.sxz + so, *sxy = f.sxy + so, *syz = f.syz + so;
  float *pzb = ps.z + (long long)shot * 6 * g.slab_z;
  float *pxb = ps.x + (long long)shot * 6 * g.slab_x;
  float *pyb = ps.y + (long long)shot * 6 * g.slab_y;
  const int sz = (int)g.sz;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;

  const bool xs = slab_s(x, nx, np), ys = slab_s(y, ny, np);
  float Kx = 1.f, ax = 0.f, bx = 0.f, Kxh = 1.f, axh = 0.f, bxh = 0.f;
  float Ky = 1.f, ay = 0.f, by = 0.f, Kyh = 1.f, ayh = 0.f, byh = 0.f;
  if (act && xs) {
    Kx = g.cx[CK * nx + x]; ax = g.cx[CA * nx + x]; bx = g.cx[CB * nx + x];
    Kxh = g.cx[CKH * nx + x]; axh = g.cx[CAH * nx + x]; bxh = g.cx[CBH * nx + x];
  }
  if (act && ys) {
    Ky = g.cy[CK * ny + y]; ay = g.cy[CA * ny + y]; by = g.cy[CB * ny + y];
    Kyh = g.cy[CKH * ny + y]; ayh = g.cy[CAH * ny + y]; byh = g.cy[CBH * ny + y];
  }
  const long long src_cell = src.cell ? src.cell[shot] : -1;
  const int sit = src.it_dev ? *src.it_dev : src.it;
  const float src_amp = src.stf ? src.stf[(long long)shot * src.nt + sit] : 0.f;

  int i = act ? (int)cell(g, z0, x, y) : 0;
  float qz0 = 0.f, qz1 = 0.f, qz2 = 0.f, qz3 = 0.f, qx0 = 0.f, qx1 = 0.f, qx2 = 0.f, qx3 = 0.f;
  float qy0 = 0.f, qy1 = 0.f, qy2 = 0.f, qy3 = 0.f;
  if (act) {
    qz0 = vz[i - 2 * sz]; qz1 = vz[i - sz]; qz2 = vz[i]; qz3 = vz[i + sz];
    qx0 = vx[i - sz]; qx1 = vx[i]; qx2 = vx[i + sz]; qx3 = vx[i + 2 * sz];
    qy0 = vy[i - sz]; qy1 = vy[i]; qy2 = vy[i + sz]; qy3 = vy[i + 2 * sz];
  }
  const int off = (ty + TMA_HX) * TMA_BOXY + tx + TMA_HY;
  const int pt = ty * 32 + tx;

  for (int q = 0; q < nq; ++q, i += sz) {
    const int z = z0 + q;
    float hz = 0.f, hx = 0.f, hy = 0.f;
    if (act && q + 1 < nq) {
      hz = vz[i + 2 * sz]; hx = vx[i + 3 * sz]; hy = vy[i + 3 * sz];
      if (q + 2 < nq) {  // heads of the plane after next (z + 4 <= nz - 1)
        prefetch_l2(vz + i + 3 * sz); prefetch_l2(vx + i + 4 * sz); prefetch_l2(vy + i + 4 * sz);
      }
    }
    // shell row of this plane, loaded before the wait so that its latency
    // overlaps it
    const int srow = (shell.rows && act) ? shell.rows[z * nx + x] : -1;
    const bool got = ring.wait(q);
    if (act && got) {
      const BoxView bz{ring.halo(q, 0) + off}, bxv{ring.halo(q, 1) + off},
          byv{ring.halo(q, 2) + off};
      const bool zs = slab_s(z, nz, np);
      float ezz = dminus(qz0, qz1, qz2, qz3) * idz;
      float exx = dminus(bxv.x(-2), bxv.x(-1), qx1, bxv.x(1)) * idx;
      float eyy = dminus(byv.y(-2), byv.y(-1), qy1, byv.y(1)) * idy;
      float dvx_dz = dplus(qx0, qx1, qx2, qx3) * idz;
      float dvy_dz = dplus(qy0, qy1, qy2, qy3) * idz;
      float dvx_dy = dplus(bxv.y(-1), qx1, bxv.y(1), bxv.y(2)) * idy;
      float dvz_dx = dplus(bz.x(-1), qz2, bz.x(1), bz.x(2)) * idx;
      float dvz_dy = dplus(bz.y(-1), qz2, bz.y(1), bz.y(2)) * idy;
      float dvy_dx = dplus(byv.x(-1), qy1, byv.x(1), byv.x(2)) * idx;
      if (zs) {
        const float Kz = g.cz[CK * nz + z], az = g.cz[CA * nz + z], bzc = g.cz[CB * nz + z];
        const float Kzh = g.cz[CKH * nz + z], azh = g.cz[CAH * nz + z], bzh = g.cz[CBH * nz + z];
        const long long k = psi_z_idx(g, z, x, y);
        float m;
        m = bzc * pzb[PSI_VA * g.slab_z + k] + az * ezz;
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
      const float l = ring.point(q, 6)[pt], u = ring.point(q, 7)[pt], l2u = l + 2.0f * u;
      {  // from_bnd: the state at the start of the step
        const int sk = shell_index(shell, srow, y);
        if (sk >= 0) {
          float *st = shell.store + sk;
          const int n = shell.npts;
          st[0] = ring.point(q, 0)[pt]; st[n] = ring.point(q, 3)[pt];
          st[2 * n] = ring.point(q, 1)[pt]; st[3 * n] = ring.point(q, 2)[pt];
          st[4 * n] = ring.point(q, 4)[pt]; st[5 * n] = ring.point(q, 5)[pt];
          st[6 * n] = qz2; st[7 * n] = qx1; st[8 * n] = qy1;
        }
      }
      float nzz = ring.point(q, 0)[pt] + (l2u * ezz + l * exx + l * eyy) * dt;
      float nxx = ring.point(q, 1)[pt] + (l * ezz + l2u * exx + l * eyy) * dt;
      float nyy = ring.point(q, 2)[pt] + (l * ezz + l * exx + l2u * eyy) * dt;
      if ((long long)i == src_cell) {
        // add_source follows the stress kernel; amplitude formed in double
        // from pow(1500, 2) (utilities.cu:450-461).
        const double a = 2250000.0 * (double)src_amp * (double)dt;
        nzz = (float)((double)nzz + a);
        nxx = (float)((double)nxx + a);
        nyy = (float)((double)nyy + a);
      }
      szz[i] = nzz; sxx[i] = nxx; syy[i] = nyy;
      sxz[i] = ring.point(q, 3)[pt] + u * (dvx_dz + dvz_dx) * dt;
      sxy[i] = ring.point(q, 4)[pt] + u * (dvx_dy + dvy_dx) * dt;
      syz[i] = ring.point(q, 5)[pt] + u * (dvy_dz + dvz_dy) * dt;
    }
    qz0 = qz1; qz1 = qz2; qz2 = qz3; qz3 = hz;
    qx0 = qx1; qx1 = qx2; qx2 = qx3; qx3 = hx;
    qy0 = qy1; qy1 = qy2; qy2 = qy3; qy3 = hy;
    if (__syncthreads_or(!got)) {
      ring_abort(ring, q, nq, R, tid, status);
      return;
    }
    if (tid == 0 && q + R < nq) {
      fence_proxy_async_smem();
      ring.issue(maps, q + R, y0, x0, shot * nz + z0 + q + R, z0 + q + R);
    }
  }
}

template <int TX, int R, int MINB>
__global__ void __launch_bounds__(32 * TX, MINB)
k_velocity_fwd_tma(const __grid_constant__ Maps<9> maps, Geo g, Fields f, Psi ps, int zchunk,
                   int nzc, RecFuse rec, int *status) {
  using Ring = PlaneRing<5, 4, 1, TX, R>;  // sxz syz sxx sxy syy | vz vx vy | buoy
  extern __shared__ __align__(128) unsigned char smem[];
  Ring ring;
  ring.bind(smem);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int y0 = blockIdx.x * 32, x0 = blockIdx.y * TX;
  const int shot = blockIdx.z / nzc;
  const int zc = blockIdx.z - shot * nzc;
  const int z0 = max(zc * zchunk, 2);
  const int z1 = min(zc * zchunk + zchunk, g.nz - 2);
  if (z0 >= z1) return;
  const int nq = z1 - z0;
  const int y = y0 + tx, x = x0 + ty;
  const int np = g.np, nz = g.nz, nx = g.nx, ny = g.ny;
  const bool act = x >= 2 && x <= nx - 3 && y >= 2 && y <= ny - 3;

  if (tid == 0) ring.init();
  __syncthreads();
  if (tid == 0)
    for (int q = 0; q < nq && q < R; ++q) ring.issue(maps, q, y0, x0, shot * nz + z0 + q, z0 + q);

  const long long so = (long long)shot * g.N;
  float *vz = f.vz + so, *vx = f.vx + so, *vy = f.vy + so;
  const float *__restrict__ szz = f.szz + so;
  const float *__restrict__ sxz = f.sxz + so;
  const float *__restrict__ syz = f.syz + so;
  float *pzb = ps.z + (long long)shot * 6 * g.slab_z;
  float *pxb = ps.x + (long long)shot * 6 * g.slab_x;
  float *pyb = ps.y + (long long)shot * 6 * g.slab_y;
  const int sz = (int)g.sz;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;

  const bool xs = slab_v(x, nx, np), ys = slab_v(y, ny, np);
  float Kx = 1.f, ax = 0.f, bx = 0.f, Kxh = 1.f, axh = 0.f, bxh = 0.f;
  float Ky = 1.f, ay = 0.f, by = 0.f, Kyh = 1.f, ayh = 0.f, byh = 0.f;
  if (act && xs) {
    Kx = g.cx[CK * nx + x]; ax = g.cx[CA * nx + x]; bx = g.cx[CB * nx + x];
    Kxh = g.cx[CKH * nx + x]; axh = g.cx[CAH * nx + x]; bxh = g.cx[CBH * nx + x];
  }
  if (act && ys) {
    Ky = g.cy[CK * ny + y]; ay = g.cy[CA * ny + y]; by = g.cy[CB * ny + y];
    Kyh = g.cy[CKH * ny + y]; ayh = g.cy[CAH * ny + y]; byh = g.cy[CBH * ny + y];
  }

  int i = act ? (int)cell(g, z0, x, y) : 0;
  float qa0 = 0.f, qa1 = 0.f, qa2 = 0.f, qa3 = 0.f, qb0 = 0.f, qb1 = 0.f, qb2 = 0.f, qb3 = 0.f;
  float qc0 = 0.f, qc1 = 0.f, qc2 = 0.f, qc3 = 0.f;
  if (act) {
    qa0 = szz[i - sz]; qa1 = szz[i]; qa2 = szz[i + sz]; qa3 = szz[i + 2 * sz];
    qb0 = sxz[i - 2 * sz]; qb1 = sxz[i - sz]; qb2 = sxz[i]; qb3 = sxz[i + sz];
    qc0 = syz[i - 2 * sz]; qc1 = syz[i - sz]; qc2 = syz[i]; qc3 = syz[i + sz];
  }
  const int off = (ty + TMA_HX) * TMA_BOXY + tx + TMA_HY;
  const int pt = ty * 32 + tx;

  for (int q = 0; q < nq; ++q, i += sz) {
    const int z = z0 + q;
    float ha = 0.f, hb = 0.f, hc = 0.f;
    if (act && q + 1 < nq) {
      ha = szz[i + 3 * sz]; hb = sxz[i + 2 * sz]; hc = syz[i + 2 * sz];
      if (q + 2 < nq) {
        prefetch_l2(szz + i + 4 * sz); prefetch_l2(sxz + i + 3 * sz); prefetch_l2(syz + i + 3 * sz);
      }
    }
    // receiver map of this plane (-1: none), loaded before the wait
    const int rmap = rec.a.plane ? rec.a.plane[shot * nz + z] : -1;
    const bool got = ring.wait(q);
    if (act && got) {
      const BoxView bxz{ring.halo(q, 0) + off}, byz{ring.halo(q, 1) + off};
      const BoxView bxx{ring.halo(q, 2) + off}, bxy{ring.halo(q, 3) + off},
          byy{ring.halo(q, 4) + off};
      const bool zs = slab_s(z, nz, np);
      const float b = ring.point(q, 3)[pt];
      float dszz_dz = dplus(qa0, qa1, qa2, qa3) * idz;
      float dsxz_dx = dminus(bxz.x(-2), bxz.x(-1), qb2, bxz.x(1)) * idx;
      float dsyz_dy = dminus(byz.y(-2), byz.y(-1), qc2, byz.y(1)) * idy;
      float dsxz_dz = dminus(qb0, qb1, qb2, qb3) * idz;
      float dsxx_dx = dplus(bxx.x(-1), bxx.c(), bxx.x(1), bxx.x(2)) * idx;
      const float sxy_m1 = bxy.y(-1), sxy_0 = bxy.c();
      float dsxy_dy = dminus(bxy.y(-2), sxy_m1, sxy_0, bxy.y(1)) * idy;
      float dsyz_dz = dminus(qc0, qc1, qc2, qc3) * idz;
      // Quirk Q1 (velocity.cu:79): c2 * (sxy[i-1] - sxy[i-2]) along x.
      const float sxy_xm1 = bxy.x(-1), sxy_xm2 = bxy.x(-2);
      float dsxy_dx = (EFWI_C1 * (sxy_0 - sxy_xm1) - EFWI_C2 * (sxy_xm1 - sxy_xm2)) * idx;
      float dsyy_dy = dplus(byy.y(-1), byy.c(), byy.y(1), byy.y(2)) * idy;
      if (zs) {
        const float Kz = g.cz[CK * nz + z], az = g.cz[CA * nz + z], bzc = g.cz[CB * nz + z];
        const float Kzh = g.cz[CKH * nz + z], azh = g.cz[CAH * nz + z], bzh = g.cz[CBH * nz + z];
        const long long k = psi_z_idx(g, z, x, y);
        float m;
        m = bzh * pzb[PSI_SAA * g.slab_z + k] + azh * dszz_dz;
        pzb[PSI_SAA * g.slab_z + k] = m; dszz_dz = dszz_dz * Kzh + m;
        m = bzc * pzb[PSI_SAB1 * g.slab_z + k] + az * dsxz_dz;
        pzb[PSI_SAB1 * g.slab_z + k] = m; dsxz_dz = dsxz_dz * Kz + m;
        m = bzc * pzb[PSI_SAB2 * g.slab_z + k] + az * dsyz_dz;
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
      const float nvz = ring.point(q, 0)[pt] + (dszz_dz + dsxz_dx + dsyz_dy) * b * dt;
      const float nvx = ring.point(q, 1)[pt] + (dsxz_dz + dsxx_dx + dsxy_dy) * b * dt;
      const float nvy = ring.point(q, 2)[pt] + (dsyz_dz + dsxy_dx + dsyy_dy) * b * dt;
      vz[i] = nvz; vx[i] = nvx; vy[i] = nvy;
      if (rmap >= 0) {
        const int u = rec.a.map[(long long)rmap * rec.a.nxpy + x * g.sx + y];
        if (u >= 0) record_cell(rec.a, rec.tm, rec.it, u, nvz, nvx, nvy);
      }
    }
    qa0 = qa1; qa1 = qa2; qa2 = qa3; qa3 = ha;
    qb0 = qb1; qb1 = qb2; qb2 = qb3; qb3 = hb;
    qc0 = qc1; qc1 = qc2; qc2 = qc3; qc3 = hc;
    if (__syncthreads_or(!got)) {
      ring_abort(ring, q, nq, R, tid, status);
      return;
    }
    if (tid == 0 && q + R < nq) {
      fence_proxy_async_smem();
      ring.issue(maps, q + R, y0, x0, shot * nz + z0 + q + R, z0 + q + R);
    }
  }
}


// Launch configurations of the forward TMA kernels: (TX, ring depth,
// minimum resident CTAs per SM).  cfg 0-2 use 32 x 4 tiles, cfg 3 32 x 8.
template <int TX, int R, int MINB>
static void stress_launch(dim3 grid, cudaStream_t st, const Maps<11> &maps, const Geo &g,
                          const Fields &f, const Psi &ps, int zchunk, int nzc, const SrcArgs &src,
                          const ShellMap &shell, int *status) {
  constexpr int B = PlaneRing<3, 8, 2, TX, R>::BYTES;
  static std::atomic<unsigned long long> smem_set{0};
  set_smem_once(k_stress_fwd_tma<TX, R, MINB>, B, smem_set);
  k_stress_fwd_tma<TX, R, MINB><<<grid, dim3(32, TX), B, st>>>(maps, g, f, ps, zchunk, nzc, src,
                                                              shell, status);
}

template <int TX, int R, int MINB>
static void velocity_launch(dim3 grid, cudaStream_t st, const Maps<9> &maps, const Geo &g,
                            const Fields &f, const Psi &ps, int zchunk, int nzc,
                            const RecFuse &rec, int *status) {
  constexpr int B = PlaneRing<5, 4, 1, TX, R>::BYTES;
  static std::atomic<unsigned long long> smem_set{0};
  set_smem_once(k_velocity_fwd_tma<TX, R, MINB>, B, smem_set);
  k_velocity_fwd_tma<TX, R, MINB><<<grid, dim3(32, TX), B, st>>>(maps, g, f, ps, zchunk, nzc,
                                                                rec, status);
}

int fwd_tma_tile(int cfg) { return cfg == 3 ? 8 : 4; }

void launch_stress_fwd_tma(int cfg, dim3 grid, cudaStream_t st, const Maps<11> &maps,
                           const Geo &g, const Fields &f, const Psi &ps, int zchunk, int nzc,
                           const SrcArgs &src, const ShellMap &shell, int *status) {
  switch (cfg) {
    case 1: stress_launch<4, 3, 7>(grid, st, maps, g, f, ps, zchunk, nzc, src, shell, status); break;
    case 2: stress_launch<4, 4, 6>(grid, st, maps, g, f, ps, zchunk, nzc, src, shell, status); break;
    case 3: stress_launch<8, 4, 1>(grid, st, maps, g, f, ps, zchunk, nzc, src, shell, status); break;
    default: stress_launch<4, 4, 1>(grid, st, maps, g, f, ps, zchunk, nzc, src, shell, status); break;
  }
}

void launch_velocity_fwd_tma(int cfg, dim3 grid, cudaStream_t st, const Maps<9> &maps,
                             const Geo &g, const Fields &f, const Psi &ps, int zchunk, int nzc,
                             const RecFuse &rec, int *status) {
  switch (cfg) {
    case 1: velocity_launch<4, 3, 7>(grid, st, maps, g, f, ps, zchunk, nzc, rec, status); break;
    case 2: velocity_launch<4, 4, 6>(grid, st, maps, g, f, ps, zchunk, nzc, rec, status); break;
    case 3: velocity_launch<8, 4, 1>(grid, st, maps, g, f, ps, zchunk, nzc, rec, status); break;
    default: velocity_launch<4, 4, 1>(grid, st, maps, g, f, ps, zchunk, nzc, rec, status); break;
  }
}

}  // namespace efwi
