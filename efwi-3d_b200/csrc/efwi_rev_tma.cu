// Reverse sweep of the reference gradient with TMA-staged planes (same
// arithmetic and fusion as efwi_rev.cu: K1 = velocity(rev) + velocity_adj,
// K2 = add_source(sub) + stress(rev) + stress_adj).
//
// K1 ring: halo  sxz syz sxx sxy syy | asxz asyz asxx asxy asyy aszz
//          point vz vx vy avz avx avy | model buoyancy lambda mu rho-image
//          z queues: szz sxz syz aszz asxx asyy asxz asyz
// K2 ring: halo  vz vx vy avz avx avy
//          point szz sxx syy sxz sxy syz aszz asxx asyy asxz asxy asyz |
//          model lambda mu buoyancy lambda-image mu-image
//          z queues: vz vx vy avz avx avy
// Restated reference kernels: velocity.cu:102-131, stress.cu:103-135,
// velocity_adj.cu:59-144, stress_adj.cu:52-142.
//
// Fused epilogues (efwi_fuse.cuh): K1 restores the reverse velocities at
// the boundary-shell points (to_bnd of the velocities) and adds the adjoint
// source at the receiver cells to the adjoint velocities (res_injection);
// K2 restores the reverse stresses at the shell points.  Values written are
// those the separate kernels would leave, bit for bit.
#include "efwi_common.cuh"
#include "efwi_fuse.cuh"
#include "efwi_kernels.h"
#include "efwi_tma.cuh"

namespace efwi {

namespace {

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

// Register queue of four consecutive z planes of one field.
struct Q4 {
  float a, b, c, d;
  __device__ __forceinline__ void shift(float h) { a = b; b = c; c = d; d = h; }
};

}  // namespace

// Box layout of K1 by MODE: 0 = reverse velocity + adjoint velocity fused;
// 1 = reverse velocity + rho image only; 2 = adjoint velocity only (the
// two halves of mode 0 as separate launches, run 1 then 2).
template <int MODE>
struct K1L {
  static constexpr bool REV = MODE != 2, ADJ = MODE != 1;
  static constexpr int NH = MODE == 0 ? 11 : (MODE == 1 ? 5 : 6);
  static constexpr int NPF = MODE == 2 ? 3 : 6;  // field point boxes
  static constexpr int NM = MODE == 0 ? 4 : (MODE == 1 ? 2 : 3);
  static constexpr int NP = NPF + NM;
  static constexpr int N = NH + NP;
  static constexpr int HA = MODE == 2 ? 0 : 5;  // first adjoint-stress halo box
  static constexpr int PA = MODE == 2 ? 0 : 3;  // first adjoint-velocity point box
  static constexpr int MB = NPF, ML = NPF + 1, MM = NPF + 2;  // buoyancy, lambda, mu
  static constexpr int MG = MODE == 0 ? NPF + 3 : NPF + 1;     // rho image
};

template <int TX, int R, int MINB, int MODE>
__global__ void __launch_bounds__(32 * TX, MINB)
k_rev_velocity_tma(const __grid_constant__ Maps<K1L<MODE>::N> maps, Geo g, Fields f, Fields a,
                   Psi ps, float *grho, int zchunk, int nzc, int do_rev, int do_adj,
                   ShellMap shell, RecFuse inj, int *status) {
  using L = K1L<MODE>;
  using Ring = PlaneRing<L::NH, L::NP, L::NM, TX, R>;
  extern __shared__ __align__(128) unsigned char smem[];
  Ring ring;
  ring.bind(smem);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int y0 = blockIdx.x * 32, x0 = blockIdx.y * TX;
  const int zc = blockIdx.z % nzc;
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
    for (int q = 0; q < nq && q < R; ++q) ring.issue(maps, q, y0, x0, z0 + q, z0 + q);

  const int sz = (int)g.sz;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;
  const bool xin = x >= np && x <= nx - 1 - np, yin = y >= np && y <= ny - 1 - np;
  const bool xs = slab_s(x, nx, np), ys = slab_s(y, ny, np);
  Coef cx{1.f, 0.f, 0.f, 1.f, 0.f, 0.f}, cy = cx;
  if (act) { cx = coef(g.cx, nx, x); cy = coef(g.cy, ny, y); }
  const float *psz = ps.z, *psx = ps.x, *psy = ps.y;
  float *pz = ps.z, *px = ps.x, *py = ps.y;

  int i = act ? (int)cell(g, z0, x, y) : 0;
  Q4 szz{}, sxz{}, syz{}, aszz{}, asxx{}, asyy{}, asxz{}, asyz{};
  if (act && L::REV) {
    szz = {f.szz[i - sz], f.szz[i], f.szz[i + sz], f.szz[i + 2 * sz]};
    sxz = {f.sxz[i - 2 * sz], f.sxz[i - sz], f.sxz[i], f.sxz[i + sz]};
    syz = {f.syz[i - 2 * sz], f.syz[i - sz], f.syz[i], f.syz[i + sz]};
  }
  if (act && L::ADJ) {
    aszz = {a.szz[i - sz], a.szz[i], a.szz[i + sz], a.szz[i + 2 * sz]};
    asxx = {a.sxx[i - sz], a.sxx[i], a.sxx[i + sz], a.sxx[i + 2 * sz]};
    asyy = {a.syy[i - sz], a.syy[i], a.syy[i + sz], a.syy[i + 2 * sz]};
    asxz = {a.sxz[i - 2 * sz], a.sxz[i - sz], a.sxz[i], a.sxz[i + sz]};
    asyz = {a.syz[i - 2 * sz], a.syz[i - sz], a.syz[i], a.syz[i + sz]};
  }
  const int off = (ty + TMA_HX) * TMA_BOXY + tx + TMA_HY;
  const int pt = ty * 32 + tx;
  // row entry of the shell map and receiver-plane index, one plane ahead
  const bool use_shell = L::REV && shell.rows && act, use_inj = L::ADJ && inj.a.plane;
  int srow = use_shell ? shell.rows[z0 * nx + x] : -1;
  int rmap = use_inj ? inj.a.plane[z0] : -1;

  for (int q = 0; q < nq; ++q, i += sz) {
    const int z = z0 + q;
    const int srow_n = (use_shell && q + 1 < nq) ? shell.rows[(z + 1) * nx + x] : -1;
    const int rmap_n = (use_inj && q + 1 < nq) ? inj.a.plane[z + 1] : -1;
    float h0 = 0.f, h1 = 0.f, h2 = 0.f, h3 = 0.f, h4 = 0.f, h5 = 0.f, h6 = 0.f, h7 = 0.f;
    if (act && q + 1 < nq) {
      if (L::REV) { h0 = f.szz[i + 3 * sz]; h1 = f.sxz[i + 2 * sz]; h2 = f.syz[i + 2 * sz]; }
      if (L::ADJ) {
        h3 = a.szz[i + 3 * sz]; h4 = a.sxx[i + 3 * sz]; h5 = a.syy[i + 3 * sz];
        h6 = a.sxz[i + 2 * sz]; h7 = a.syz[i + 2 * sz];
      }
      if (q + 2 < nq) {  // heads of the plane after next (z + 4 <= nz - 1)
        if (L::REV) {
          prefetch_l2(f.szz + i + 4 * sz); prefetch_l2(f.sxz + i + 3 * sz); prefetch_l2(f.syz + i + 3 * sz);
        }
        if (L::ADJ) {
          prefetch_l2(a.szz + i + 4 * sz); prefetch_l2(a.sxx + i + 4 * sz); prefetch_l2(a.syy + i + 4 * sz);
          prefetch_l2(a.sxz + i + 3 * sz); prefetch_l2(a.syz + i + 3 * sz);
        }
      }
    }
    // fused epilogue operands of this plane, loaded before the wait so that
    // their latency overlaps it: the stored shell velocities (to_bnd) and the
    // receiver map index (res_injection)
    int sk = -1;
    float rvz = 0.f, rvx = 0.f, rvy = 0.f;
    if (use_shell) {
      sk = shell_index(shell, srow, y);
      if (sk >= 0) {
        const int n = shell.npts;
        rvz = shell.store[6 * n + sk]; rvx = shell.store[7 * n + sk];
        rvy = shell.store[8 * n + sk];
      }
    }
    const bool got = ring.wait(q);
    if (act && got) {
      const float b = ring.point(q, L::MB)[pt];
      const float avz0 = ring.point(q, L::PA)[pt], avx0 = ring.point(q, L::PA + 1)[pt],
                  avy0 = ring.point(q, L::PA + 2)[pt];
      if (L::REV && do_rev) {
        const bool inr = xin && yin && z >= np && z <= nz - 1 - np;
        float nvz = 0.f, nvx = 0.f, nvy = 0.f;
        if (inr) {
        const BoxView bsxz{ring.halo(q, 0) + off}, bsyz{ring.halo(q, 1) + off},
            bsxx{ring.halo(q, 2) + off}, bsxy{ring.halo(q, 3) + off}, bsyy{ring.halo(q, 4) + off};
        const float sxy_0 = bsxy.c(), sxy_xm1 = bsxy.x(-1);
        const float dz_ = dplus(szz.a, szz.b, szz.c, szz.d) * idz +
                          dminus(bsxz.x(-2), bsxz.x(-1), sxz.c, bsxz.x(1)) * idx +
                          dminus(bsyz.y(-2), bsyz.y(-1), syz.c, bsyz.y(1)) * idy;
        const float dx_ = dminus(sxz.a, sxz.b, sxz.c, sxz.d) * idz +
                          dplus(bsxx.x(-1), bsxx.c(), bsxx.x(1), bsxx.x(2)) * idx +
                          dminus(bsxy.y(-2), bsxy.y(-1), sxy_0, bsxy.y(1)) * idy;
        const float dy_ = dminus(syz.a, syz.b, syz.c, syz.d) * idz +
                          (EFWI_C1 * (sxy_0 - sxy_xm1) - EFWI_C2 * (sxy_xm1 - bsxy.x(-2))) * idx +
                          dplus(bsyy.y(-1), bsyy.c(), bsyy.y(1), bsyy.y(2)) * idy;
        nvz = ring.point(q, 0)[pt] - dz_ * b * dt;
        nvx = ring.point(q, 1)[pt] - dx_ * b * dt;
        nvy = ring.point(q, 2)[pt] - dy_ * b * dt;
        const float nb2 = -(b * b);
        grho[i] = ring.point(q, L::MG)[pt] -
                    (avz0 * dz_ * dt * nb2 + avx0 * dx_ * dt * nb2 + avy0 * dy_ * dt * nb2);
        }
        // to_bnd: the shell points take the stored velocities of the step
        if (sk >= 0) { nvz = rvz; nvx = rvx; nvy = rvy; }
        if (inr || sk >= 0) { f.vz[i] = nvz; f.vx[i] = nvx; f.vy[i] = nvy; }
      }
      if (L::ADJ && do_adj) {
        const BoxView basxz{ring.halo(q, L::HA) + off}, basyz{ring.halo(q, L::HA + 1) + off},
            basxx{ring.halo(q, L::HA + 2) + off}, basxy{ring.halo(q, L::HA + 3) + off},
            basyy{ring.halo(q, L::HA + 4) + off}, baszz{ring.halo(q, L::HA + 5) + off};
        const bool zs = slab_s(z, nz, np);
        // outside the z slab the profile is K = 1, a = 0 (b unused there)
        const Coef cz = zs ? coef(g.cz, nz, z) : Coef{1.f, 0.f, 0.f, 1.f, 0.f, 0.f};
        const float l = ring.point(q, L::ML)[pt], u = ring.point(q, L::MM)[pt], l2u = l + 2.0f * u;
        float nax, naz, nay;  // the new adjoint velocities (before res_injection)
        {  // adjoint vx
          const float dszz_dx = -dplus(baszz.x(-1), aszz.b, baszz.x(1), baszz.x(2)) * idx;
          const float dsxx_dx = -dplus(basxx.x(-1), asxx.b, basxx.x(1), basxx.x(2)) * idx;
          const float dsyy_dx = -dplus(basyy.x(-1), asyy.b, basyy.x(1), basyy.x(2)) * idx;
          const float dsxz_dz = -dminus(asxz.a, asxz.b, asxz.c, asxz.d) * idz;
          const float dsxy_dy = -dminus(basxy.y(-2), basxy.y(-1), basxy.c(), basxy.y(1)) * idy;
          float acc = l2u * dsxx_dx * cx.K * dt + l * dszz_dx * cx.K * dt +
                      l * dsyy_dx * cx.K * dt + u * cz.Kh * dsxz_dz * dt +
                      u * cy.Kh * dsxy_dy * dt;
          if (xs) acc += cx.a * (nxp(g, psx + PSI_VA * g.slab_x, z, x, y) * idx);
          if (zs) acc += cz.ah * (nzm(g, psz + PSI_VB1 * g.slab_z, z, x, y) * idz);
          if (ys) acc += cy.ah * (nym(g, psy + PSI_VB2 * g.slab_y, z, x, y) * idy);
          const float v = avx0 + acc;
          nax = v;
          if (xs) { const long long k = PSI_SAA * g.slab_x + psi_x_idx(g, z, x, y); px[k] = cx.bh * px[k] + b * v * dt; }
          if (zs) { const long long k = PSI_SAB1 * g.slab_z + psi_z_idx(g, z, x, y); pz[k] = cz.b * pz[k] + b * v * dt; }
          if (ys) { const long long k = PSI_SAB2 * g.slab_y + psi_y_idx(g, z, x, y); py[k] = cy.b * py[k] + b * v * dt; }
        }
        {  // adjoint vz
          const float dszz_dz = -dplus(aszz.a, aszz.b, aszz.c, aszz.d) * idz;
          const float dsxx_dz = -dplus(asxx.a, asxx.b, asxx.c, asxx.d) * idz;
          const float dsyy_dz = -dplus(asyy.a, asyy.b, asyy.c, asyy.d) * idz;
          const float dsxz_dx = -dminus(basxz.x(-2), basxz.x(-1), asxz.c, basxz.x(1)) * idx;
          const float dsyz_dy = -dminus(basyz.y(-2), basyz.y(-1), asyz.c, basyz.y(1)) * idy;
          float acc = l2u * dszz_dz * cz.K * dt + l * dsxx_dz * cz.K * dt +
                      l * dsyy_dz * cz.K * dt + u * cy.Kh * dsyz_dy * dt +
                      u * cx.Kh * dsxz_dx * dt;
          if (zs) acc += cz.a * (nzp(g, psz + PSI_VA * g.slab_z, z, x, y) * idz);
          if (ys) acc += cy.ah * (nym(g, psy + PSI_VB1 * g.slab_y, z, x, y) * idy);
          if (xs) acc += cx.ah * (nxm(g, psx + PSI_VB1 * g.slab_x, z, x, y) * idx);
          const float v = avz0 + acc;
          naz = v;
          if (xs) { const long long k = PSI_SAB1 * g.slab_x + psi_x_idx(g, z, x, y); px[k] = cx.b * px[k] + b * v * dt; }
          if (zs) { const long long k = PSI_SAA * g.slab_z + psi_z_idx(g, z, x, y); pz[k] = cz.bh * pz[k] + b * v * dt; }
          if (ys) { const long long k = PSI_SAB1 * g.slab_y + psi_y_idx(g, z, x, y); py[k] = cy.b * py[k] + b * v * dt; }
        }
        {  // adjoint vy
          const float dsyy_dy = -dplus(basyy.y(-1), asyy.b, basyy.y(1), basyy.y(2)) * idy;
          const float dsxx_dy = -dplus(basxx.y(-1), asxx.b, basxx.y(1), basxx.y(2)) * idy;
          const float dszz_dy = -dplus(baszz.y(-1), aszz.b, baszz.y(1), baszz.y(2)) * idy;
          const float dsxy_dx = -dminus(basxy.x(-2), basxy.x(-1), basxy.c(), basxy.x(1)) * idx;
          const float dsyz_dz = -dminus(asyz.a, asyz.b, asyz.c, asyz.d) * idz;
          float acc = l2u * dsyy_dy * cy.K * dt + l * dsxx_dy * cy.K * dt +
                      l * dszz_dy * cy.K * dt + u * cx.Kh * dsxy_dx * dt +
                      u * cz.Kh * dsyz_dz * dt;
          if (ys) acc += cy.a * (nyp(g, psy + PSI_VA * g.slab_y, z, x, y) * idy);
          if (xs) acc += cx.ah * (nxm(g, psx + PSI_VB2 * g.slab_x, z, x, y) * idx);
          if (zs) acc += cz.ah * (nzm(g, psz + PSI_VB2 * g.slab_z, z, x, y) * idz);
          const float v = avy0 + acc;
          nay = v;
          if (xs) { const long long k = PSI_SAB2 * g.slab_x + psi_x_idx(g, z, x, y); px[k] = cx.b * px[k] + b * v * dt; }
          if (zs) { const long long k = PSI_SAB2 * g.slab_z + psi_z_idx(g, z, x, y); pz[k] = cz.bh * pz[k] + b * v * dt; }
          if (ys) { const long long k = PSI_SAA * g.slab_y + psi_y_idx(g, z, x, y); py[k] = cy.b * py[k] + b * v * dt; }
        }
        if (rmap >= 0) {  // res_injection after the adjoint update
          const int ur = inj.a.map[(long long)rmap * inj.a.nxpy + x * g.sx + y];
          if (ur >= 0) inject_cell(inj.a, inj.tm, inj.it, ur, naz, nax, nay);
        }
        a.vx[i] = nax; a.vz[i] = naz; a.vy[i] = nay;
      }
    }
    szz.shift(h0); sxz.shift(h1); syz.shift(h2); aszz.shift(h3);
    asxx.shift(h4); asyy.shift(h5); asxz.shift(h6); asyz.shift(h7);
    srow = srow_n;
    rmap = rmap_n;
    if (__syncthreads_or(!got)) {
      ring_abort(ring, q, nq, R, tid, status);
      return;
    }
    if (tid == 0 && q + R < nq) {
      fence_proxy_async_smem();
      ring.issue(maps, q + R, y0, x0, z0 + q + R, z0 + q + R);
    }
  }
}

template <int TX, int R, int MINB>
__global__ void __launch_bounds__(32 * TX, MINB)
k_rev_stress_tma(const __grid_constant__ Maps<23> maps, Geo g, Fields f, Fields a, Psi ps,
                 float *glam, float *gmu, int zchunk, int nzc, int do_rev, int do_adj,
                 SrcArgs src, ShellMap shell, int *status) {
  using Ring = PlaneRing<6, 17, 5, TX, R>;
  extern __shared__ __align__(128) unsigned char smem[];
  Ring ring;
  ring.bind(smem);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int y0 = blockIdx.x * 32, x0 = blockIdx.y * TX;
  const int zc = blockIdx.z % nzc;
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
    for (int q = 0; q < nq && q < R; ++q) ring.issue(maps, q, y0, x0, z0 + q, z0 + q);

  const int sz = (int)g.sz;
  const float dt = g.dt, idz = g.idz, idx = g.idx, idy = g.idy;
  const bool xin = x >= np && x <= nx - 1 - np, yin = y >= np && y <= ny - 1 - np;
  const bool xs = slab_s(x, nx, np), ys = slab_s(y, ny, np);
  Coef cx{1.f, 0.f, 0.f, 1.f, 0.f, 0.f}, cy = cx;
  if (act) { cx = coef(g.cx, nx, x); cy = coef(g.cy, ny, y); }
  const long long src_cell = (do_rev && src.cell) ? src.cell[0] : -1;
  const float src_amp = (do_rev && src.stf) ? src.stf[src.it] : 0.f;
  const float *psz = ps.z, *psx = ps.x, *psy = ps.y;
  float *pz = ps.z, *px = ps.x, *py = ps.y;

  int i = act ? (int)cell(g, z0, x, y) : 0;
  Q4 vz{}, vx{}, vy{}, avz{}, avx{}, avy{};
  if (act) {
    vz = {f.vz[i - 2 * sz], f.vz[i - sz], f.vz[i], f.vz[i + sz]};
    vx = {f.vx[i - sz], f.vx[i], f.vx[i + sz], f.vx[i + 2 * sz]};
    vy = {f.vy[i - sz], f.vy[i], f.vy[i + sz], f.vy[i + 2 * sz]};
    avz = {a.vz[i - 2 * sz], a.vz[i - sz], a.vz[i], a.vz[i + sz]};
    avx = {a.vx[i - sz], a.vx[i], a.vx[i + sz], a.vx[i + 2 * sz]};
    avy = {a.vy[i - sz], a.vy[i], a.vy[i + sz], a.vy[i + 2 * sz]};
  }
  const int off = (ty + TMA_HX) * TMA_BOXY + tx + TMA_HY;
  const int pt = ty * 32 + tx;
  // row entry of the shell map, one plane ahead
  const bool use_shell = shell.rows && act;
  int srow = use_shell ? shell.rows[z0 * nx + x] : -1;

  for (int q = 0; q < nq; ++q, i += sz) {
    const int z = z0 + q;
    const int srow_n = (use_shell && q + 1 < nq) ? shell.rows[(z + 1) * nx + x] : -1;
    float h0 = 0.f, h1 = 0.f, h2 = 0.f, h3 = 0.f, h4 = 0.f, h5 = 0.f;
    if (act && q + 1 < nq) {
      h0 = f.vz[i + 2 * sz]; h1 = f.vx[i + 3 * sz]; h2 = f.vy[i + 3 * sz];
      h3 = a.vz[i + 2 * sz]; h4 = a.vx[i + 3 * sz]; h5 = a.vy[i + 3 * sz];
      if (q + 2 < nq) {
        prefetch_l2(f.vz + i + 3 * sz); prefetch_l2(f.vx + i + 4 * sz); prefetch_l2(f.vy + i + 4 * sz);
        prefetch_l2(a.vz + i + 3 * sz); prefetch_l2(a.vx + i + 4 * sz); prefetch_l2(a.vy + i + 4 * sz);
      }
    }
    // the stored shell stresses of this plane (to_bnd), loaded before the
    // wait so that their latency overlaps it
    int sk = -1;
    float rst[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (use_shell) {
      sk = shell_index(shell, srow, y);
      if (sk >= 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) rst[k] = shell.store[k * shell.npts + sk];
      }
    }
    const bool got = ring.wait(q);
    if (act && got) {
      const BoxView bvz{ring.halo(q, 0) + off}, bvx{ring.halo(q, 1) + off},
          bvy{ring.halo(q, 2) + off};
      const BoxView bavz{ring.halo(q, 3) + off}, bavx{ring.halo(q, 4) + off},
          bavy{ring.halo(q, 5) + off};
      const float l = ring.point(q, 12)[pt], u = ring.point(q, 13)[pt], l2u = l + 2.0f * u;
      const float azz0 = ring.point(q, 6)[pt], axx0 = ring.point(q, 7)[pt],
                  ayy0 = ring.point(q, 8)[pt];
      const float axz0 = ring.point(q, 9)[pt], axy0 = ring.point(q, 10)[pt],
                  ayz0 = ring.point(q, 11)[pt];
      if (do_rev) {
        float szz = ring.point(q, 0)[pt], sxx = ring.point(q, 1)[pt], syy = ring.point(q, 2)[pt];
        if ((long long)i == src_cell) {
          const double am = 2250000.0 * (double)src_amp * (double)dt;
          szz = (float)((double)szz - am);
          sxx = (float)((double)sxx - am);
          syy = (float)((double)syy - am);
        }
        const bool inr = xin && yin && z >= np && z <= nz - 1 - np;
        float nsxz = 0.f, nsxy = 0.f, nsyz = 0.f;
        if (inr) {
          const float ezz = dminus(vz.a, vz.b, vz.c, vz.d) * idz;
          const float exx = dminus(bvx.x(-2), bvx.x(-1), vx.b, bvx.x(1)) * idx;
          const float eyy = dminus(bvy.y(-2), bvy.y(-1), vy.b, bvy.y(1)) * idy;
          szz = szz - (l2u * ezz + l * exx + l * eyy) * dt;
          sxx = sxx - (l * ezz + l2u * exx + l * eyy) * dt;
          syy = syy - (l * ezz + l * exx + l2u * eyy) * dt;
          const float dvx_dz = dplus(vx.a, vx.b, vx.c, vx.d) * idz;
          const float dvx_dy = dplus(bvx.y(-1), vx.b, bvx.y(1), bvx.y(2)) * idy;
          const float dvz_dx = dplus(bvz.x(-1), vz.c, bvz.x(1), bvz.x(2)) * idx;
          const float dvz_dy = dplus(bvz.y(-1), vz.c, bvz.y(1), bvz.y(2)) * idy;
          const float dvy_dx = dplus(bvy.x(-1), vy.b, bvy.x(1), bvy.x(2)) * idx;
          const float dvy_dz = dplus(vy.a, vy.b, vy.c, vy.d) * idz;
          nsxz = ring.point(q, 3)[pt] - u * (dvx_dz + dvz_dx) * dt;
          nsxy = ring.point(q, 4)[pt] - u * (dvx_dy + dvy_dx) * dt;
          nsyz = ring.point(q, 5)[pt] - u * (dvy_dz + dvz_dy) * dt;
          glam[i] = ring.point(q, 15)[pt] - (azz0 + axx0 + ayy0) * (ezz + exx + eyy) * dt;
          gmu[i] = ring.point(q, 16)[pt] -
                     (2.0f * azz0 * ezz + 2.0f * axx0 * exx + 2.0f * ayy0 * eyy +
                      axz0 * (dvx_dz + dvz_dx) + ayz0 * (dvy_dz + dvz_dy) +
                      axy0 * (dvy_dx + dvx_dy)) * dt;
        }
        // to_bnd: the shell points take the stored stresses of the step
        if (sk >= 0) {
          szz = rst[0]; nsxz = rst[1]; sxx = rst[2]; syy = rst[3]; nsxy = rst[4]; nsyz = rst[5];
        }
        if (inr || sk >= 0) { f.sxz[i] = nsxz; f.sxy[i] = nsxy; f.syz[i] = nsyz; }
        f.szz[i] = szz; f.sxx[i] = sxx; f.syy[i] = syy;
      }
      if (do_adj) {
        const bool zs = slab_s(z, nz, np);
        // outside the z slab the profile is K = 1, a = 0 (b unused there)
        const Coef cz = zs ? coef(g.cz, nz, z) : Coef{1.f, 0.f, 0.f, 1.f, 0.f, 0.f};
        const float b = ring.point(q, 14)[pt];
        {  // sxz
          const float dvz_dx = -dplus(bavz.x(-1), avz.c, bavz.x(1), bavz.x(2)) * idx;
          const float dvx_dz = -dplus(avx.a, avx.b, avx.c, avx.d) * idz;
          float acc = dvz_dx * cx.K * b * dt + dvx_dz * cz.K * b * dt;
          if (xs) acc += cx.a * (nxp(g, psx + PSI_SAB1 * g.slab_x, z, x, y) * idx);
          if (zs) acc += cz.a * (nzp(g, psz + PSI_SAB1 * g.slab_z, z, x, y) * idz);
          const float s = axz0 + acc;
          a.sxz[i] = s;
          if (xs) { const long long k = PSI_VB1 * g.slab_x + psi_x_idx(g, z, x, y); px[k] = cx.bh * px[k] + s * u * dt; }
          if (zs) { const long long k = PSI_VB1 * g.slab_z + psi_z_idx(g, z, x, y); pz[k] = cz.bh * pz[k] + s * u * dt; }
        }
        {  // sxy
          const float dvy_dx = -dplus(bavy.x(-1), avy.b, bavy.x(1), bavy.x(2)) * idx;
          const float dvx_dy = -dplus(bavx.y(-1), avx.b, bavx.y(1), bavx.y(2)) * idy;
          float acc = dvy_dx * cx.K * b * dt + dvx_dy * cy.K * b * dt;
          if (xs) acc += cx.a * (nxp(g, psx + PSI_SAB2 * g.slab_x, z, x, y) * idx);
          if (ys) acc += cy.a * (nyp(g, psy + PSI_SAB2 * g.slab_y, z, x, y) * idy);
          const float s = axy0 + acc;
          a.sxy[i] = s;
          if (ys) { const long long k = PSI_VB2 * g.slab_y + psi_y_idx(g, z, x, y); py[k] = cy.bh * py[k] + s * u * dt; }
          if (xs) { const long long k = PSI_VB2 * g.slab_x + psi_x_idx(g, z, x, y); px[k] = cx.bh * px[k] + s * u * dt; }
        }
        {  // syz
          const float dvz_dy = -dplus(bavz.y(-1), avz.c, bavz.y(1), bavz.y(2)) * idy;
          const float dvy_dz = -dplus(avy.a, avy.b, avy.c, avy.d) * idz;
          float acc = dvz_dy * cy.K * b * dt + dvy_dz * cz.K * b * dt;
          if (ys) acc += cy.a * (nyp(g, psy + PSI_SAB1 * g.slab_y, z, x, y) * idy);
          if (zs) acc += cz.a * (nzp(g, psz + PSI_SAB2 * g.slab_z, z, x, y) * idz);
          const float s = ayz0 + acc;
          a.syz[i] = s;
          if (ys) { const long long k = PSI_VB1 * g.slab_y + psi_y_idx(g, z, x, y); py[k] = cy.bh * py[k] + s * u * dt; }
          if (zs) { const long long k = PSI_VB2 * g.slab_z + psi_z_idx(g, z, x, y); pz[k] = cz.bh * pz[k] + s * u * dt; }
        }
        {  // normal stresses
          const float dvx_dx = -dminus(bavx.x(-2), bavx.x(-1), avx.b, bavx.x(1)) * idx;
          const float dvz_dz = -dminus(avz.a, avz.b, avz.c, avz.d) * idz;
          const float dvy_dy = -dminus(bavy.y(-2), bavy.y(-1), avy.b, bavy.y(1)) * idy;
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
    vz.shift(h0); vx.shift(h1); vy.shift(h2); avz.shift(h3); avx.shift(h4); avy.shift(h5);
    srow = srow_n;
    if (__syncthreads_or(!got)) {
      ring_abort(ring, q, nq, R, tid, status);
      return;
    }
    if (tid == 0 && q + R < nq) {
      fence_proxy_async_smem();
      ring.issue(maps, q + R, y0, x0, z0 + q + R, z0 + q + R);
    }
  }
}


// Launch configurations of the reverse TMA kernels (32 x 4 tiles): (ring
// depth, minimum resident CTAs per SM).  32 x 8 tiles were measured slower
// (0.227 / 0.243 ms against 0.198 / 0.200 ms per launch at 152^3).
int rev_tma_tile(int) { return 4; }
template <int R, int MINB, int MODE = 0, int TX = 4>
static void revv_launch(dim3 grid, cudaStream_t st, const Maps<K1L<MODE>::N> &maps, const Geo &g,
                        const Fields &f, const Fields &a, const Psi &ps, float *grho, int zchunk,
                        int nzc, int do_rev, int do_adj, const ShellMap &shell,
                        const RecFuse &inj, int *status) {
  using L = K1L<MODE>;
  constexpr int B = PlaneRing<L::NH, L::NP, L::NM, TX, R>::BYTES;
  static std::atomic<unsigned long long> smem_set{0};
  set_smem_once(k_rev_velocity_tma<TX, R, MINB, MODE>, B, smem_set);
  k_rev_velocity_tma<TX, R, MINB, MODE><<<grid, dim3(32, TX), B, st>>>(
      maps, g, f, a, ps, grho, zchunk, nzc, do_rev, do_adj, shell, inj, status);
}

template <int R, int MINB, int TX = 4>
static void revs_launch(dim3 grid, cudaStream_t st, const Maps<23> &maps, const Geo &g,
                        const Fields &f, const Fields &a, const Psi &ps, float *glam, float *gmu,
                        int zchunk, int nzc, int do_rev, int do_adj, const SrcArgs &src,
                        const ShellMap &shell, int *status) {
  constexpr int B = PlaneRing<6, 17, 5, TX, R>::BYTES;
  static std::atomic<unsigned long long> smem_set{0};
  set_smem_once(k_rev_stress_tma<TX, R, MINB>, B, smem_set);
  k_rev_stress_tma<TX, R, MINB><<<grid, dim3(32, TX), B, st>>>(maps, g, f, a, ps, glam, gmu, zchunk,
                                                            nzc, do_rev, do_adj, src, shell,
                                                            status);
}

void launch_rev_velocity_tma(int cfg, dim3 grid, cudaStream_t st, const Maps<21> &maps,
                             const Geo &g, const Fields &f, const Fields &a, const Psi &ps,
                             float *grho, int zchunk, int nzc, int do_rev, int do_adj,
                             const ShellMap &shell, const RecFuse &inj, int *status) {
  switch (cfg) {
    case 1: revv_launch<2, 4>(grid, st, maps, g, f, a, ps, grho, zchunk, nzc, do_rev, do_adj, shell, inj, status); break;
    case 2: revv_launch<3, 4>(grid, st, maps, g, f, a, ps, grho, zchunk, nzc, do_rev, do_adj, shell, inj, status); break;
    case 3: revv_launch<2, 1>(grid, st, maps, g, f, a, ps, grho, zchunk, nzc, do_rev, do_adj, shell, inj, status); break;
    case 4: revv_launch<2, 5>(grid, st, maps, g, f, a, ps, grho, zchunk, nzc, do_rev, do_adj, shell, inj, status); break;
    case 5: revv_launch<2, 6>(grid, st, maps, g, f, a, ps, grho, zchunk, nzc, do_rev, do_adj, shell, inj, status); break;
    default: revv_launch<3, 1>(grid, st, maps, g, f, a, ps, grho, zchunk, nzc, do_rev, do_adj, shell, inj, status); break;
  }
}

// Split K1 (cfg 6: rings of 2 planes; cfg 7: 3 planes): the reverse
// velocity half, then the adjoint velocity half.
void launch_rev_velocity_split_tma(int cfg, dim3 grid, cudaStream_t st, const Maps<13> &rev_maps,
                                   const Maps<12> &adj_maps, const Geo &g, const Fields &f,
                                   const Fields &a, const Psi &ps, float *grho, int zchunk,
                                   int nzc, int do_rev, int do_adj, const ShellMap &shell,
                                   const RecFuse &inj, int *status) {
  if (cfg == 7) {
    if (do_rev) revv_launch<3, 8, 1>(grid, st, rev_maps, g, f, a, ps, grho, zchunk, nzc, 1, 0, shell, RecFuse{}, status);
    if (do_adj) revv_launch<3, 4, 2>(grid, st, adj_maps, g, f, a, ps, grho, zchunk, nzc, 0, 1, ShellMap{}, inj, status);
  } else {
    if (do_rev) revv_launch<2, 8, 1>(grid, st, rev_maps, g, f, a, ps, grho, zchunk, nzc, 1, 0, shell, RecFuse{}, status);
    if (do_adj) revv_launch<2, 5, 2>(grid, st, adj_maps, g, f, a, ps, grho, zchunk, nzc, 0, 1, ShellMap{}, inj, status);
  }
}

void launch_rev_stress_tma(int cfg, dim3 grid, cudaStream_t st, const Maps<23> &maps,
                           const Geo &g, const Fields &f, const Fields &a, const Psi &ps,
                           float *glam, float *gmu, int zchunk, int nzc, int do_rev, int do_adj,
                           const SrcArgs &src, const ShellMap &shell, int *status) {
  switch (cfg) {
    case 1: revs_launch<2, 5>(grid, st, maps, g, f, a, ps, glam, gmu, zchunk, nzc, do_rev, do_adj, src, shell, status); break;
    case 2: revs_launch<3, 4>(grid, st, maps, g, f, a, ps, glam, gmu, zchunk, nzc, do_rev, do_adj, src, shell, status); break;
    case 3: revs_launch<2, 1>(grid, st, maps, g, f, a, ps, glam, gmu, zchunk, nzc, do_rev, do_adj, src, shell, status); break;
    case 4: revs_launch<2, 6>(grid, st, maps, g, f, a, ps, glam, gmu, zchunk, nzc, do_rev, do_adj, src, shell, status); break;
    case 5: revs_launch<2, 7>(grid, st, maps, g, f, a, ps, glam, gmu, zchunk, nzc, do_rev, do_adj, src, shell, status); break;
    case 6: revs_launch<2, 5>(grid, st, maps, g, f, a, ps, glam, gmu, zchunk, nzc, do_rev, do_adj, src, shell, status); break;
    case 7: revs_launch<3, 4>(grid, st, maps, g, f, a, ps, glam, gmu, zchunk, nzc, do_rev, do_adj, src, shell, status); break;
    default: revs_launch<3, 1>(grid, st, maps, g, f, a, ps, glam, gmu, zchunk, nzc, do_rev, do_adj, src, shell, status); break;
  }
}

}  // namespace efwi
