// EFWI-3D oracle: FP64 CPU restatement of the reference elastic solver.
//
// TEST INFRASTRUCTURE ONLY.  Nothing on the product path links, imports or
// executes this file; tests/, the smoke check and bench.py's cpu_baseline leg
// use it as the checker.  It is a statement-by-statement restatement, in
// double precision and in the torch-native [z][x][y] (y fastest) layout, of:
//
//   forward stress       Ops/FWI/Src_3d/stress.cu:36-97
//   forward velocity     Ops/FWI/Src_3d/velocity.cu:35-96   (quirks Q1 :79, Q2 :46)
//   reverse stress       Ops/FWI/Src_3d/stress.cu:103-135   (lambda/mu imaging)
//   reverse velocity     Ops/FWI/Src_3d/velocity.cu:102-131 (rho imaging)
//   adjoint stress       Ops/FWI/Src_3d/stress_adj.cu:52-142
//   adjoint velocity     Ops/FWI/Src_3d/velocity_adj.cu:59-144
//   C-PML coefficients   Ops/FWI/Src_3d/utilities.cu:204-320 (cpmlInit, VpAve forced to 3000)
//   point source         Ops/FWI/Src_3d/utilities.cu:423-479 (Gaussian weights underflow: point)
//   receivers            Ops/FWI/Src_3d/utilities.cu:481-507 (recording / res_injection)
//   boundary shell       Ops/FWI/Src_3d/Boundary.cu:14-42, utilities.cu:323-420
//   misfit + windows     Ops/FWI/Src_3d/utilities.cu:130-166, 524-614; libCUFD.cu:371-440
//   source taper         Ops/FWI/Src_3d/Src_Rec.cu:146 (ratio 0.001)
//   step ordering        Ops/FWI/Src_3d/libCUFD.cu:312-354 (forward), 500-612 (reverse)
//
// It also holds the exact discrete adjoint of the same forward scheme
// (mode 1), which has no reference counterpart; it is checked here by a
// dot-product test and by finite differences.
//
// All volumes are [nz][nx][ny] float64, C order.  Grid sizes are the padded
// sizes; source and receiver indices are padded-grid indices.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
typedef struct {
  int nz, nx, ny, npml, nt;
  double dz, dx, dy, dt, f0;
} OracleGrid;

typedef struct {
  int z_src, x_src, y_src, nrec;
  const int *z_rec, *x_rec, *y_rec;
  // Optional per-trace time windows (seconds) and weights, used when the
  // caller asks for windowed misfit (reference `if_win`).  May be NULL.
  const double *win_start, *win_end, *weights;
  double src_weight;
} OracleShot;
}

namespace {

const double kC1 = 9.0 / 8.0;
const double kC2 = 1.0 / 24.0;
const double kPi = 3.141592653589793238462643383279502884197169;

struct Profile {
  std::vector<double> K, a, b, Kh, ah, bh;
};

// Restates cpmlInit (utilities.cu:204-320): damping d0 with VpAve = 3000,
// R = 8e-4, N = 8, K_max = 2, alpha_max = pi*f0, profile 0.25x + 0.75x^8,
// evaluated at integer and half points from both edges.
Profile cpml_profile(int n, int npml, double dh, double f0, double dt) {
  Profile p;
  p.K.assign(n, 1.0); p.Kh.assign(n, 1.0);
  p.a.assign(n, 0.0); p.ah.assign(n, 0.0);
  p.b.assign(n, 0.0); p.bh.assign(n, 0.0);
  std::vector<double> d(n, 0.0), dh_(n, 0.0), al(n, 0.0), alh(n, 0.0);
  const double R = 0.0008, Kmax = 2.0, npow = 8.0, vp = 3000.0;
  const double amax = 2.0 * kPi * (f0 / 2.0);
  const double L = npml * dh;
  const double d0 = -(npow + 1.0) * vp * std::log(R) / (2.0 * L);
  auto prof = [&](double depth, double &dd, double &KK, double &aa) {
    double x = depth / L;
    dd = d0 * (0.25 * x + 0.75 * std::pow(x, npow));
    KK = 1.0 + (Kmax - 1.0) * std::pow(x, npow);
    aa = amax * (1.0 - x);
  };
  for (int i = 0; i < n; ++i) {
    double depth = (npml - i) * dh;
    if (depth >= 0.0) prof(depth, d[i], p.K[i], al[i]);
    depth = (npml - i - 0.5) * dh;
    if (depth >= 0.0) prof(depth, dh_[i], p.Kh[i], alh[i]);
    depth = (npml - n + i) * dh;
    if (depth >= 0.0) prof(depth, d[i], p.K[i], al[i]);
    depth = (npml - n + i + 0.5) * dh;
    if (depth >= 0.0) prof(depth, dh_[i], p.Kh[i], alh[i]);
    if (al[i] < 0.0) al[i] = 0.0;
    if (alh[i] < 0.0) alh[i] = 0.0;
    p.b[i] = std::exp(-(d[i] / p.K[i] + al[i]) * dt);
    p.bh[i] = std::exp(-(dh_[i] / p.Kh[i] + alh[i]) * dt);
    if (std::fabs(d[i]) > 1.0e-6)
      p.a[i] = d[i] * (p.b[i] - 1.0) / (p.K[i] * (d[i] + p.K[i] * al[i]));
    if (std::fabs(dh_[i]) > 1.0e-6)
      p.ah[i] = dh_[i] * (p.bh[i] - 1.0) / (p.Kh[i] * (dh_[i] + p.Kh[i] * alh[i]));
  }
  return p;
}

// Time taper of cuda_window without per-trace windows (utilities.cu:578-614).
// The window is data weighting, not part of the stencil, so it is restated
// with the reference's float time variables and double sin/cos: a sample
// then falls on the same side of every window edge as in the reference.
// Returns the amplitude w (the data is multiplied by w*w); `ok` is false
// when the reference kernel would leave the data untouched.
double taper_plain(int it, int nt, double dt_, double ratio_, bool &ok) {
  const float dt = (float)dt_, ratio = (float)ratio_;
  const float t = it * dt, t0 = 0.0f, t3 = nt * dt, off = nt * dt * ratio;
  ok = !(2.0 * off >= t3 - t0);
  if (!ok) return 1.0;
  const float t1 = t0 + off, t2 = t3 - off;
  if (t >= t0 && t < t1) return (float)std::sin(kPi / 2.0 * (t - t0) / (t1 - t0));
  if (t >= t1 && t < t2) return 1.0;
  if (t >= t2 && t < t3) return (float)std::cos(kPi / 2.0 * (t - t2) / (t3 - t2));
  return 0.0;
}

// Windowed variant (utilities.cu:524-576): returns the full multiplier
// w*w*weight*src_weight, or 1 when the reference leaves the trace untouched.
double taper_win(int it, int nt, double dt_, double ratio_, double t0_, double t3_,
                 double weight, double srcw) {
  const float dt = (float)dt_, ratio = (float)ratio_;
  if (ratio > 0.5f) return 1.0;
  const float t = it * dt, tmax = nt * dt;
  float t0 = (float)t0_, t3 = (float)t3_;
  if (t0 < 0.0f) t0 = 0.0f;
  if (t0 > tmax) t0 = tmax;
  if (t3 < 0.0f) t3 = 0.0f;
  if (t3 > tmax) t3 = tmax;
  const float off = (t3 - t0) * ratio;
  if (off <= 0.0f) return 1.0;
  const float t1 = t0 + off, t2 = t3 - off;
  double w;
  if (t >= t0 && t < t1) w = (float)std::sin(kPi / 2.0 * (t - t0) / (t1 - t0));
  else if (t >= t1 && t < t2) w = 1.0;
  else if (t >= t2 && t < t3) w = (float)std::cos(kPi / 2.0 * (t - t2) / (t3 - t2));
  else w = 0.0;
  return w * w * weight * srcw;
}

typedef std::vector<double> Vec;

struct Solver {
  int nz, nx, ny, np, nt;
  double dz, dx, dy, dt;
  long sz, sx;
  size_t N;
  Profile pz, px, py;
  const double *lam, *mu;
  Vec B;
  // forward fields
  Vec vz, vx, vy, szz, sxx, syy, sxz, sxy, syz;
  // stress-kernel memory variables (also adjoint psi in reference mode)
  Vec m_vz_z, m_vz_x, m_vz_y, m_vx_z, m_vx_x, m_vx_y, m_vy_z, m_vy_x, m_vy_y;
  // velocity-kernel memory variables
  Vec m_szz_z, m_sxx_x, m_syy_y, m_sxz_z, m_sxz_x, m_sxy_x, m_sxy_y, m_syz_y, m_syz_z;
  // adjoint fields
  Vec avz, avx, avy, aszz, asxx, asyy, asxz, asxy, asyz;

  Solver(const OracleGrid &g, const double *lam_, const double *mu_, const double *rho)
      : nz(g.nz), nx(g.nx), ny(g.ny), np(g.npml), nt(g.nt), dz(g.dz), dx(g.dx),
        dy(g.dy), dt(g.dt), lam(lam_), mu(mu_) {
    sz = (long)nx * ny; sx = ny;
    N = (size_t)nz * nx * ny;
    pz = cpml_profile(nz, np, dz, g.f0, dt);
    px = cpml_profile(nx, np, dx, g.f0, dt);
    py = cpml_profile(ny, np, dy, g.f0, dt);
    // Buoyancy: 1/rho on [2, n-3]^3, 1/1000 elsewhere (Model.cu:65-76).
    B.assign(N, 1.0 / 1000.0);
    for (int z = 2; z <= nz - 3; ++z)
      for (int x = 2; x <= nx - 3; ++x)
        for (int y = 2; y <= ny - 3; ++y) {
          size_t i = idx(z, x, y);
          B[i] = 1.0 / rho[i];
        }
    Vec *all[] = {&vz, &vx, &vy, &szz, &sxx, &syy, &sxz, &sxy, &syz,
                  &m_vz_z, &m_vz_x, &m_vz_y, &m_vx_z, &m_vx_x, &m_vx_y, &m_vy_z, &m_vy_x, &m_vy_y,
                  &m_szz_z, &m_sxx_x, &m_syy_y, &m_sxz_z, &m_sxz_x, &m_sxy_x, &m_sxy_y, &m_syz_y, &m_syz_z,
                  &avz, &avx, &avy, &aszz, &asxx, &asyy, &asxz, &asxy, &asyz};
    for (Vec *v : all) v->assign(N, 0.0);
  }

  size_t idx(int z, int x, int y) const { return ((size_t)z * nx + x) * ny + y; }

  // Staggered 4th-order differences.  Dm: half point below i; Dp: above.
  static double Dm(const double *f, size_t i, long s) {
    return kC1 * (f[i] - f[i - s]) - kC2 * (f[i + s] - f[i - 2 * s]);
  }
  static double Dp(const double *f, size_t i, long s) {
    return kC1 * (f[i + s] - f[i]) - kC2 * (f[i + 2 * s] - f[i - s]);
  }
  // Quirk Q1 (velocity.cu:79): the c2 term of dsxy/dx uses sxy[i-s].
  static double Dq(const double *f, size_t i, long s) {
    return kC1 * (f[i] - f[i - s]) - kC2 * (f[i - s] - f[i - 2 * s]);
  }

  bool slabS(int i, int n) const { return i < np || i > n - np - 1; }
  // Quirk Q2 (velocity.cu:46,50,...): x/y slabs of the velocity kernel end one
  // cell short on the high side.
  bool slabV(int i, int n) const { return i < np || i > n - np; }

  void zero_all() {
    Vec *all[] = {&vz, &vx, &vy, &szz, &sxx, &syy, &sxz, &sxy, &syz};
    for (Vec *v : all) std::fill(v->begin(), v->end(), 0.0);
    zero_psi();
  }
  void zero_psi() {
    Vec *all[] = {&m_vz_z, &m_vz_x, &m_vz_y, &m_vx_z, &m_vx_x, &m_vx_y, &m_vy_z, &m_vy_x, &m_vy_y,
                  &m_szz_z, &m_sxx_x, &m_syy_y, &m_sxz_z, &m_sxz_x, &m_sxy_x, &m_sxy_y, &m_syz_y, &m_syz_z};
    for (Vec *v : all) std::fill(v->begin(), v->end(), 0.0);
  }
  void zero_adj() {
    Vec *all[] = {&avz, &avx, &avy, &aszz, &asxx, &asyy, &asxz, &asxy, &asyz};
    for (Vec *v : all) std::fill(v->begin(), v->end(), 0.0);
  }

  // ---------------------------------------------------------------- forward
  void stress_fwd() {
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 2; z <= nz - 3; ++z)
      for (int x = 2; x <= nx - 3; ++x)
        for (int y = 2; y <= ny - 3; ++y) {
          size_t i = idx(z, x, y);
          double ezz = Dm(vz.data(), i, sz) / dz;
          double exx = Dm(vx.data(), i, sx) / dx;
          double eyy = Dm(vy.data(), i, 1) / dy;
          if (slabS(z, nz)) { m_vz_z[i] = pz.b[z] * m_vz_z[i] + pz.a[z] * ezz; ezz = ezz / pz.K[z] + m_vz_z[i]; }
          if (slabS(x, nx)) { m_vx_x[i] = px.b[x] * m_vx_x[i] + px.a[x] * exx; exx = exx / px.K[x] + m_vx_x[i]; }
          if (slabS(y, ny)) { m_vy_y[i] = py.b[y] * m_vy_y[i] + py.a[y] * eyy; eyy = eyy / py.K[y] + m_vy_y[i]; }
          double l = lam[i], m = mu[i];
          szz[i] += ((l + 2.0 * m) * ezz + l * exx + l * eyy) * dt;
          sxx[i] += (l * ezz + (l + 2.0 * m) * exx + l * eyy) * dt;
          syy[i] += (l * ezz + l * exx + (l + 2.0 * m) * eyy) * dt;
          double dvx_dz = Dp(vx.data(), i, sz) / dz, dvx_dy = Dp(vx.data(), i, 1) / dy;
          double dvz_dx = Dp(vz.data(), i, sx) / dx, dvz_dy = Dp(vz.data(), i, 1) / dy;
          double dvy_dx = Dp(vy.data(), i, sx) / dx, dvy_dz = Dp(vy.data(), i, sz) / dz;
          if (slabS(z, nz)) {
            m_vx_z[i] = pz.bh[z] * m_vx_z[i] + pz.ah[z] * dvx_dz; dvx_dz = dvx_dz / pz.Kh[z] + m_vx_z[i];
            m_vy_z[i] = pz.bh[z] * m_vy_z[i] + pz.ah[z] * dvy_dz; dvy_dz = dvy_dz / pz.Kh[z] + m_vy_z[i];
          }
          if (slabS(x, nx)) {
            m_vz_x[i] = px.bh[x] * m_vz_x[i] + px.ah[x] * dvz_dx; dvz_dx = dvz_dx / px.Kh[x] + m_vz_x[i];
            m_vy_x[i] = px.bh[x] * m_vy_x[i] + px.ah[x] * dvy_dx; dvy_dx = dvy_dx / px.Kh[x] + m_vy_x[i];
          }
          if (slabS(y, ny)) {
            m_vz_y[i] = py.bh[y] * m_vz_y[i] + py.ah[y] * dvz_dy; dvz_dy = dvz_dy / py.Kh[y] + m_vz_y[i];
            m_vx_y[i] = py.bh[y] * m_vx_y[i] + py.ah[y] * dvx_dy; dvx_dy = dvx_dy / py.Kh[y] + m_vx_y[i];
          }
          sxz[i] += m * (dvx_dz + dvz_dx) * dt;
          sxy[i] += m * (dvx_dy + dvy_dx) * dt;
          syz[i] += m * (dvy_dz + dvz_dy) * dt;
        }
  }

  void velocity_fwd() {
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 2; z <= nz - 3; ++z)
      for (int x = 2; x <= nx - 3; ++x)
        for (int y = 2; y <= ny - 3; ++y) {
          size_t i = idx(z, x, y);
          double b = B[i];
          double dszz_dz = Dp(szz.data(), i, sz) / dz;
          double dsxz_dx = Dm(sxz.data(), i, sx) / dx;
          double dsyz_dy = Dm(syz.data(), i, 1) / dy;
          if (slabS(z, nz)) { m_szz_z[i] = pz.bh[z] * m_szz_z[i] + pz.ah[z] * dszz_dz; dszz_dz = dszz_dz / pz.Kh[z] + m_szz_z[i]; }
          if (slabV(x, nx)) { m_sxz_x[i] = px.b[x] * m_sxz_x[i] + px.a[x] * dsxz_dx; dsxz_dx = dsxz_dx / px.K[x] + m_sxz_x[i]; }
          if (slabV(y, ny)) { m_syz_y[i] = py.b[y] * m_syz_y[i] + py.a[y] * dsyz_dy; dsyz_dy = dsyz_dy / py.K[y] + m_syz_y[i]; }
          vz[i] += (dszz_dz + dsxz_dx + dsyz_dy) * b * dt;

          double dsxz_dz = Dm(sxz.data(), i, sz) / dz;
          double dsxx_dx = Dp(sxx.data(), i, sx) / dx;
          double dsxy_dy = Dm(sxy.data(), i, 1) / dy;
          if (slabS(z, nz)) { m_sxz_z[i] = pz.b[z] * m_sxz_z[i] + pz.a[z] * dsxz_dz; dsxz_dz = dsxz_dz / pz.K[z] + m_sxz_z[i]; }
          if (slabV(x, nx)) { m_sxx_x[i] = px.bh[x] * m_sxx_x[i] + px.ah[x] * dsxx_dx; dsxx_dx = dsxx_dx / px.Kh[x] + m_sxx_x[i]; }
          if (slabV(y, ny)) { m_sxy_y[i] = py.b[y] * m_sxy_y[i] + py.a[y] * dsxy_dy; dsxy_dy = dsxy_dy / py.K[y] + m_sxy_y[i]; }
          vx[i] += (dsxz_dz + dsxx_dx + dsxy_dy) * b * dt;

          double dsyz_dz = Dm(syz.data(), i, sz) / dz;
          double dsxy_dx = Dq(sxy.data(), i, sx) / dx;
          double dsyy_dy = Dp(syy.data(), i, 1) / dy;
          if (slabS(z, nz)) { m_syz_z[i] = pz.b[z] * m_syz_z[i] + pz.a[z] * dsyz_dz; dsyz_dz = dsyz_dz / pz.K[z] + m_syz_z[i]; }
          if (slabV(x, nx)) { m_sxy_x[i] = px.b[x] * m_sxy_x[i] + px.a[x] * dsxy_dx; dsxy_dx = dsxy_dx / px.K[x] + m_sxy_x[i]; }
          if (slabV(y, ny)) { m_syy_y[i] = py.bh[y] * m_syy_y[i] + py.ah[y] * dsyy_dy; dsyy_dy = dsyy_dy / py.Kh[y] + m_syy_y[i]; }
          vy[i] += (dsyz_dz + dsxy_dx + dsyy_dy) * b * dt;
        }
  }

  // Source illumination of the current state S_k (after forward step k-1):
  // squared model derivatives of the stress stage of step k (when
  // do_stress) and of the velocity stage of step k-1 (Shin et al. 2001
  // pseudo-Hessian); same modified derivatives as stress_fwd/velocity_fwd,
  // with the stress memory variables advanced as the stress stage would.
  void illum(double *hl, double *hm, double *hb, bool do_stress) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 2; z <= nz - 3; ++z)
      for (int x = 2; x <= nx - 3; ++x)
        for (int y = 2; y <= ny - 3; ++y) {
          size_t i = idx(z, x, y);
          const double dt2 = dt * dt;
          if (do_stress) {
            double ezz = Dm(vz.data(), i, sz) / dz, exx = Dm(vx.data(), i, sx) / dx, eyy = Dm(vy.data(), i, 1) / dy;
            double dvx_dz = Dp(vx.data(), i, sz) / dz, dvx_dy = Dp(vx.data(), i, 1) / dy;
            double dvz_dx = Dp(vz.data(), i, sx) / dx, dvz_dy = Dp(vz.data(), i, 1) / dy;
            double dvy_dx = Dp(vy.data(), i, sx) / dx, dvy_dz = Dp(vy.data(), i, sz) / dz;
            if (slabS(z, nz)) {
              ezz = ezz / pz.K[z] + (pz.b[z] * m_vz_z[i] + pz.a[z] * ezz);
              dvx_dz = dvx_dz / pz.Kh[z] + (pz.bh[z] * m_vx_z[i] + pz.ah[z] * dvx_dz);
              dvy_dz = dvy_dz / pz.Kh[z] + (pz.bh[z] * m_vy_z[i] + pz.ah[z] * dvy_dz);
            }
            if (slabS(x, nx)) {
              exx = exx / px.K[x] + (px.b[x] * m_vx_x[i] + px.a[x] * exx);
              dvz_dx = dvz_dx / px.Kh[x] + (px.bh[x] * m_vz_x[i] + px.ah[x] * dvz_dx);
              dvy_dx = dvy_dx / px.Kh[x] + (px.bh[x] * m_vy_x[i] + px.ah[x] * dvy_dx);
            }
            if (slabS(y, ny)) {
              eyy = eyy / py.K[y] + (py.b[y] * m_vy_y[i] + py.a[y] * eyy);
              dvz_dy = dvz_dy / py.Kh[y] + (py.bh[y] * m_vz_y[i] + py.ah[y] * dvz_dy);
              dvx_dy = dvx_dy / py.Kh[y] + (py.bh[y] * m_vx_y[i] + py.ah[y] * dvx_dy);
            }
            double div = ezz + exx + eyy;
            double exz = dvx_dz + dvz_dx, exy = dvx_dy + dvy_dx, eyz = dvy_dz + dvz_dy;
            hl[i] += 3.0 * div * div * dt2;
            hm[i] += (4.0 * (ezz * ezz + exx * exx + eyy * eyy) + exz * exz + exy * exy + eyz * eyz) * dt2;
          }
          double q[3];
          {
            double a = Dp(szz.data(), i, sz) / dz, b = Dm(sxz.data(), i, sx) / dx, c = Dm(syz.data(), i, 1) / dy;
            if (slabS(z, nz)) a = a / pz.Kh[z] + m_szz_z[i];
            if (slabV(x, nx)) b = b / px.K[x] + m_sxz_x[i];
            if (slabV(y, ny)) c = c / py.K[y] + m_syz_y[i];
            q[0] = a + b + c;
          }
          {
            double a = Dm(sxz.data(), i, sz) / dz, b = Dp(sxx.data(), i, sx) / dx, c = Dm(sxy.data(), i, 1) / dy;
            if (slabS(z, nz)) a = a / pz.K[z] + m_sxz_z[i];
            if (slabV(x, nx)) b = b / px.Kh[x] + m_sxx_x[i];
            if (slabV(y, ny)) c = c / py.K[y] + m_sxy_y[i];
            q[1] = a + b + c;
          }
          {
            double a = Dm(syz.data(), i, sz) / dz, b = Dq(sxy.data(), i, sx) / dx, c = Dp(syy.data(), i, 1) / dy;
            if (slabS(z, nz)) a = a / pz.K[z] + m_syz_z[i];
            if (slabV(x, nx)) b = b / px.K[x] + m_sxy_x[i];
            if (slabV(y, ny)) c = c / py.Kh[y] + m_syy_y[i];
            q[2] = a + b + c;
          }
          hb[i] += (q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) * dt2;
        }
  }

  // ------------------------------------------------ reference-mode reverse
  // Reverse velocity step on [npml, n-1-npml]^3 with rho imaging
  // (velocity.cu:102-131).
  void velocity_rev(double *grho) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = np; z <= nz - 1 - np; ++z)
      for (int x = np; x <= nx - 1 - np; ++x)
        for (int y = np; y <= ny - 1 - np; ++y) {
          size_t i = idx(z, x, y);
          double b = B[i];
          double dz_ = Dp(szz.data(), i, sz) / dz + Dm(sxz.data(), i, sx) / dx + Dm(syz.data(), i, 1) / dy;
          vz[i] -= dz_ * b * dt;
          double dx_ = Dm(sxz.data(), i, sz) / dz + Dp(sxx.data(), i, sx) / dx + Dm(sxy.data(), i, 1) / dy;
          vx[i] -= dx_ * b * dt;
          double dy_ = Dm(syz.data(), i, sz) / dz + Dq(sxy.data(), i, sx) / dx + Dp(syy.data(), i, 1) / dy;
          vy[i] -= dy_ * b * dt;
          grho[i] += -(avz[i] * dz_ * dt * (-b * b) + avx[i] * dx_ * dt * (-b * b) + avy[i] * dy_ * dt * (-b * b));
        }
  }

  // Reverse stress step with lambda/mu imaging (stress.cu:103-135).
  void stress_rev(double *glam, double *gmu) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = np; z <= nz - 1 - np; ++z)
      for (int x = np; x <= nx - 1 - np; ++x)
        for (int y = np; y <= ny - 1 - np; ++y) {
          size_t i = idx(z, x, y);
          double ezz = Dm(vz.data(), i, sz) / dz, exx = Dm(vx.data(), i, sx) / dx, eyy = Dm(vy.data(), i, 1) / dy;
          double l = lam[i], m = mu[i];
          szz[i] -= ((l + 2.0 * m) * ezz + l * exx + l * eyy) * dt;
          sxx[i] -= (l * ezz + (l + 2.0 * m) * exx + l * eyy) * dt;
          syy[i] -= (l * ezz + l * exx + (l + 2.0 * m) * eyy) * dt;
          double dvx_dz = Dp(vx.data(), i, sz) / dz, dvx_dy = Dp(vx.data(), i, 1) / dy;
          double dvz_dx = Dp(vz.data(), i, sx) / dx, dvz_dy = Dp(vz.data(), i, 1) / dy;
          double dvy_dx = Dp(vy.data(), i, sx) / dx, dvy_dz = Dp(vy.data(), i, sz) / dz;
          sxz[i] -= m * (dvx_dz + dvz_dx) * dt;
          sxy[i] -= m * (dvx_dy + dvy_dx) * dt;
          syz[i] -= m * (dvy_dz + dvz_dy) * dt;
          glam[i] += -(aszz[i] + asxx[i] + asyy[i]) * (ezz + exx + eyy) * dt;
          gmu[i] += -(2.0 * aszz[i] * ezz + 2.0 * asxx[i] * exx + 2.0 * asyy[i] * eyy +
                      asxz[i] * (dvx_dz + dvz_dx) + asyz[i] * (dvy_dz + dvz_dy) +
                      asxy[i] * (dvy_dx + dvx_dy)) * dt;
        }
  }

  // Reference adjoint velocity (velocity_adj.cu:59-144).  The adjoint psi
  // re-use the forward memory arrays, as the reference does.
  void velocity_adj_ref() {
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 2; z <= nz - 3; ++z)
      for (int x = 2; x <= nx - 3; ++x)
        for (int y = 2; y <= ny - 3; ++y) {
          size_t i = idx(z, x, y);
          double l = lam[i], m = mu[i], b = B[i];
          // vx
          double dpsixx_dx = -Dp(m_vx_x.data(), i, sx) / dx;
          double dszz_dx = -Dp(aszz.data(), i, sx) / dx, dsxx_dx = -Dp(asxx.data(), i, sx) / dx,
                 dsyy_dx = -Dp(asyy.data(), i, sx) / dx;
          double dpsixz_dz = -Dm(m_vx_z.data(), i, sz) / dz, dsxz_dz = -Dm(asxz.data(), i, sz) / dz;
          double dpsixy_dy = -Dm(m_vx_y.data(), i, 1) / dy, dsxy_dy = -Dm(asxy.data(), i, 1) / dy;
          avx[i] += (px.a[x] * dpsixx_dx + (l + 2.0 * m) * dsxx_dx / px.K[x] * dt +
                     l * dszz_dx / px.K[x] * dt + l * dsyy_dx / px.K[x] * dt +
                     m / pz.Kh[z] * dsxz_dz * dt + pz.ah[z] * dpsixz_dz +
                     m / py.Kh[y] * dsxy_dy * dt + py.ah[y] * dpsixy_dy);
          if (slabS(x, nx)) m_sxx_x[i] = px.bh[x] * m_sxx_x[i] + b * avx[i] * dt;
          if (slabS(z, nz)) m_sxz_z[i] = pz.b[z] * m_sxz_z[i] + b * avx[i] * dt;
          if (slabS(y, ny)) m_sxy_y[i] = py.b[y] * m_sxy_y[i] + b * avx[i] * dt;
          // vz
          double dpsizz_dz = -Dp(m_vz_z.data(), i, sz) / dz;
          double dszz_dz = -Dp(aszz.data(), i, sz) / dz, dsxx_dz = -Dp(asxx.data(), i, sz) / dz,
                 dsyy_dz = -Dp(asyy.data(), i, sz) / dz;
          double dpsizx_dx = -Dm(m_vz_x.data(), i, sx) / dx, dsxz_dx = -Dm(asxz.data(), i, sx) / dx;
          double dpsizy_dy = -Dm(m_vz_y.data(), i, 1) / dy, dsyz_dy = -Dm(asyz.data(), i, 1) / dy;
          avz[i] += (pz.a[z] * dpsizz_dz + (l + 2.0 * m) * dszz_dz / pz.K[z] * dt +
                     l * dsxx_dz / pz.K[z] * dt + l * dsyy_dz / pz.K[z] * dt +
                     m / py.Kh[y] * dsyz_dy * dt + py.ah[y] * dpsizy_dy +
                     m / px.Kh[x] * dsxz_dx * dt + px.ah[x] * dpsizx_dx);
          if (slabS(x, nx)) m_sxz_x[i] = px.b[x] * m_sxz_x[i] + b * avz[i] * dt;
          if (slabS(z, nz)) m_szz_z[i] = pz.bh[z] * m_szz_z[i] + b * avz[i] * dt;
          if (slabS(y, ny)) m_syz_y[i] = py.b[y] * m_syz_y[i] + b * avz[i] * dt;
          // vy
          double dpsiyy_dy = -Dp(m_vy_y.data(), i, 1) / dy;
          double dsyy_dy = -Dp(asyy.data(), i, 1) / dy, dsxx_dy = -Dp(asxx.data(), i, 1) / dy,
                 dszz_dy = -Dp(aszz.data(), i, 1) / dy;
          double dpsiyx_dx = -Dm(m_vy_x.data(), i, sx) / dx, dsxy_dx = -Dm(asxy.data(), i, sx) / dx;
          double dpsiyz_dz = -Dm(m_vy_z.data(), i, sz) / dz, dsyz_dz = -Dm(asyz.data(), i, sz) / dz;
          avy[i] += (py.a[y] * dpsiyy_dy + (l + 2.0 * m) * dsyy_dy / py.K[y] * dt +
                     l * dsxx_dy / py.K[y] * dt + l * dszz_dy / py.K[y] * dt +
                     m / px.Kh[x] * dsxy_dx * dt + px.ah[x] * dpsiyx_dx +
                     m / pz.Kh[z] * dsyz_dz * dt + pz.ah[z] * dpsiyz_dz);
          if (slabS(x, nx)) m_sxy_x[i] = px.b[x] * m_sxy_x[i] + b * avy[i] * dt;
          if (slabS(z, nz)) m_syz_z[i] = pz.bh[z] * m_syz_z[i] + b * avy[i] * dt;
          if (slabS(y, ny)) m_syy_y[i] = py.b[y] * m_syy_y[i] + b * avy[i] * dt;
        }
  }

  // Reference adjoint stress (stress_adj.cu:52-142).
  void stress_adj_ref() {
#pragma omp parallel for collapse(2) schedule(static)
    for (int z = 2; z <= nz - 3; ++z)
      for (int x = 2; x <= nx - 3; ++x)
        for (int y = 2; y <= ny - 3; ++y) {
          size_t i = idx(z, x, y);
          double l = lam[i], m = mu[i], b = B[i];
          // sxz
          double dphi_x = -Dp(m_sxz_x.data(), i, sx) / dx, dvz_dx = -Dp(avz.data(), i, sx) / dx;
          double dphi_z = -Dp(m_sxz_z.data(), i, sz) / dz, dvx_dz = -Dp(avx.data(), i, sz) / dz;
          asxz[i] += px.a[x] * dphi_x + dvz_dx / px.K[x] * b * dt + pz.a[z] * dphi_z + dvx_dz / pz.K[z] * b * dt;
          if (slabS(x, nx)) m_vz_x[i] = px.bh[x] * m_vz_x[i] + asxz[i] * m * dt;
          if (slabS(z, nz)) m_vx_z[i] = pz.bh[z] * m_vx_z[i] + asxz[i] * m * dt;
          // sxy
          double dphi_xy_x = -Dp(m_sxy_x.data(), i, sx) / dx, dvy_dx = -Dp(avy.data(), i, sx) / dx;
          double dphi_xy_y = -Dp(m_sxy_y.data(), i, 1) / dy, dvx_dy = -Dp(avx.data(), i, 1) / dy;
          asxy[i] += px.a[x] * dphi_xy_x + dvy_dx / px.K[x] * b * dt + py.a[y] * dphi_xy_y + dvx_dy / py.K[y] * b * dt;
          if (slabS(y, ny)) m_vx_y[i] = py.bh[y] * m_vx_y[i] + asxy[i] * m * dt;
          if (slabS(x, nx)) m_vy_x[i] = px.bh[x] * m_vy_x[i] + asxy[i] * m * dt;
          // syz
          double dphi_yz_y = -Dp(m_syz_y.data(), i, 1) / dy, dvz_dy = -Dp(avz.data(), i, 1) / dy;
          double dphi_yz_z = -Dp(m_syz_z.data(), i, sz) / dz, dvy_dz = -Dp(avy.data(), i, sz) / dz;
          asyz[i] += py.a[y] * dphi_yz_y + dvz_dy / py.K[y] * b * dt + pz.a[z] * dphi_yz_z + dvy_dz / pz.K[z] * b * dt;
          if (slabS(y, ny)) m_vz_y[i] = py.bh[y] * m_vz_y[i] + asyz[i] * m * dt;
          if (slabS(z, nz)) m_vy_z[i] = pz.bh[z] * m_vy_z[i] + asyz[i] * m * dt;
          // normal stresses
          double dphi_xx = -Dm(m_sxx_x.data(), i, sx) / dx, dvx_dx = -Dm(avx.data(), i, sx) / dx;
          double dphi_zz = -Dm(m_szz_z.data(), i, sz) / dz, dvz_dz = -Dm(avz.data(), i, sz) / dz;
          double dphi_yy = -Dm(m_syy_y.data(), i, 1) / dy, dvy_dy = -Dm(avy.data(), i, 1) / dy;
          asxx[i] += px.ah[x] * dphi_xx + b * dvx_dx / px.Kh[x] * dt;
          aszz[i] += pz.ah[z] * dphi_zz + b * dvz_dz / pz.Kh[z] * dt;
          asyy[i] += py.ah[y] * dphi_yy + b * dvy_dy / py.Kh[y] * dt;
          if (slabS(x, nx)) m_vx_x[i] = px.b[x] * m_vx_x[i] + l * aszz[i] * dt + (l + 2.0 * m) * asxx[i] * dt + l * asyy[i] * dt;
          if (slabS(z, nz)) m_vz_z[i] = pz.b[z] * m_vz_z[i] + (l + 2.0 * m) * aszz[i] * dt + l * asxx[i] * dt + l * asyy[i] * dt;
          if (slabS(y, ny)) m_vy_y[i] = py.b[y] * m_vy_y[i] + l * aszz[i] * dt + l * asxx[i] * dt + (l + 2.0 * m) * asyy[i] * dt;
        }
  }
};

// Boundary shell: every point of the box [npml-2, n-npml+1]^3 that lies in
// one of the six 5-cell layers at its faces (Boundary.cu:14-20,
// utilities.cu:323-420).  Stored once per point (the reference stores edge
// points once per face; the values are equal).
std::vector<size_t> shell_points(const Solver &s) {
  std::vector<size_t> pts;
  int lo = s.np - 2;
  int hz = s.nz - s.np + 1, hx = s.nx - s.np + 1, hy = s.ny - s.np + 1;
  for (int z = lo; z <= hz; ++z)
    for (int x = lo; x <= hx; ++x)
      for (int y = lo; y <= hy; ++y) {
        bool in = (z <= lo + 4 || z >= hz - 4 || x <= lo + 4 || x >= hx - 4 || y <= lo + 4 || y >= hy - 4);
        if (in) pts.push_back(s.idx(z, x, y));
      }
  return pts;
}

void taper_stf(const double *stf, int nt, double dt, std::vector<double> &out) {
  out.resize(nt);
  for (int it = 0; it < nt; ++it) {
    bool ok;
    double w = taper_plain(it, nt, dt, 0.001, ok);
    out[it] = ok ? stf[it] * w * w : stf[it];
  }
}

// Runs one shot forward; records traces[3][nrec][nt] (x, y, z components).
// When `shell` is non-null, stores the 9-field shell before every step.
void run_forward(Solver &s, const OracleShot &sh, const double *stf_raw, double *traces,
                 std::vector<double> *shell, const std::vector<size_t> *pts) {
  s.zero_all();
  std::vector<double> stf;
  taper_stf(stf_raw, s.nt, s.dt, stf);
  const int nt = s.nt, nr = sh.nrec;
  std::fill(traces, traces + (size_t)3 * nr * nt, 0.0);
  size_t isrc = s.idx(sh.z_src, sh.x_src, sh.y_src);
  const Vec *F[9] = {&s.szz, &s.sxz, &s.sxx, &s.syy, &s.sxy, &s.syz, &s.vz, &s.vx, &s.vy};
  size_t np = pts ? pts->size() : 0;
  for (int it = 0; it <= nt - 2; ++it) {
    if (shell) {
      double *dst = shell->data() + (size_t)it * 9 * np;
      for (int f = 0; f < 9; ++f)
        for (size_t k = 0; k < np; ++k) dst[f * np + k] = (*F[f])[(*pts)[k]];
    }
    s.stress_fwd();
    double amp = 1500.0 * 1500.0 * stf[it] * s.dt;
    s.szz[isrc] += amp; s.sxx[isrc] += amp; s.syy[isrc] += amp;
    s.velocity_fwd();
    for (int r = 0; r < nr; ++r) {
      size_t i = s.idx(sh.z_rec[r], sh.x_rec[r], sh.y_rec[r]);
      traces[((size_t)0 * nr + r) * nt + it + 1] = s.vx[i];
      traces[((size_t)1 * nr + r) * nt + it + 1] = s.vy[i];
      traces[((size_t)2 * nr + r) * nt + it + 1] = s.vz[i];
    }
  }
}

// Misfit of one shot (libCUFD.cu:371-440): window obs and syn, residual with
// sample 0 zeroed, sum of squares, window the residual again.  `res` gets
// the adjoint source in [3][nrec][nt].
double misfit(const OracleShot &sh, int nt, double dt, bool if_win, const double *obs,
              const double *syn, double *res) {
  const int nr = sh.nrec;
  const double ratio = 0.005;
  double J = 0.0;
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < nr; ++r)
      for (int it = 0; it < nt; ++it) {
        double mult;
        if (if_win) {
          double w0 = sh.win_start ? sh.win_start[r] : 0.0;
          double w1 = sh.win_end ? sh.win_end[r] : 0.0;
          double wt = sh.weights ? sh.weights[r] : 1.0;
          mult = taper_win(it, nt, dt, ratio, w0, w1, wt, sh.src_weight);
        } else {
          bool ok;
          double w = taper_plain(it, nt, dt, ratio, ok);
          mult = ok ? w * w : 1.0;
        }
        size_t k = ((size_t)c * nr + r) * nt + it;
        double rr = (it == 0) ? 0.0 : obs[k] * mult - syn[k] * mult;
        J += rr * rr;
        res[k] = rr * mult;
      }
  return J;
}

}  // namespace

// =========================================================== exact adjoint
// The forward step is linear in the 27-component state (9 fields + 18 memory
// variables) for fixed (lambda, mu, B).  The exact discrete adjoint runs the
// transposed step backwards; imaging is the derivative of each step with
// respect to the model, contracted with the adjoint state.
namespace {

struct ExactAdj {
  Solver &s;
  // adjoint of every forward variable, same naming with prefix 'a'
  Vec a_vz, a_vx, a_vy, a_szz, a_sxx, a_syy, a_sxz, a_sxy, a_syz;
  Vec a_m_vz_z, a_m_vz_x, a_m_vz_y, a_m_vx_z, a_m_vx_x, a_m_vx_y, a_m_vy_z, a_m_vy_x, a_m_vy_y;
  Vec a_m_szz_z, a_m_sxx_x, a_m_syy_y, a_m_sxz_z, a_m_sxz_x, a_m_sxy_x, a_m_sxy_y, a_m_syz_y, a_m_syz_z;
  explicit ExactAdj(Solver &s_) : s(s_) {
    Vec *all[] = {&a_vz, &a_vx, &a_vy, &a_szz, &a_sxx, &a_syy, &a_sxz, &a_sxy, &a_syz,
                  &a_m_vz_z, &a_m_vz_x, &a_m_vz_y, &a_m_vx_z, &a_m_vx_x, &a_m_vx_y, &a_m_vy_z, &a_m_vy_x, &a_m_vy_y,
                  &a_m_szz_z, &a_m_sxx_x, &a_m_syy_y, &a_m_sxz_z, &a_m_sxz_x, &a_m_sxy_x, &a_m_sxy_y, &a_m_syz_y, &a_m_syz_z};
    for (Vec *v : all) v->assign(s.N, 0.0);
  }

  // Scatter helpers: adjoint of y = Dm(f, i, st)/h, i.e. accumulate g into
  // the five stencil points of f.
  static void tDm(double *af, size_t i, long st, double g) {
    af[i] += kC1 * g; af[i - st] -= kC1 * g; af[i + st] -= kC2 * g; af[i - 2 * st] += kC2 * g;
  }
  static void tDp(double *af, size_t i, long st, double g) {
    af[i + st] += kC1 * g; af[i] -= kC1 * g; af[i + 2 * st] -= kC2 * g; af[i - st] += kC2 * g;
  }
  static void tDq(double *af, size_t i, long st, double g) {
    af[i] += kC1 * g; af[i - st] -= kC1 * g; af[i - st] -= kC2 * g; af[i - 2 * st] += kC2 * g;
  }

  // Transpose of velocity_fwd.  The forward reads stresses at neighbours and
  // writes v and psi at the cell, so the adjoint gathers are written here
  // as serial scatters (serial loop: the scatters overlap between cells).
  // Imaging: d(step)/dB contracted with the adjoint, accumulated in gB.
  void velocity_T(double *gB) {
    const int nz = s.nz, nx = s.nx, ny = s.ny;
    const double dt = s.dt;
    for (int z = 2; z <= nz - 3; ++z)
      for (int x = 2; x <= nx - 3; ++x)
        for (int y = 2; y <= ny - 3; ++y) {
          size_t i = s.idx(z, x, y);
          double b = s.B[i];
          // ---- vy (forward: vy += (dsyz_dz' + dsxy_dx' + dsyy_dy') * b * dt)
          {
            double g = a_vy[i];  // adjoint of the new vy; vy_old keeps g (identity)
            // forward values needed for imaging
            double d1 = Solver::Dm(s.syz.data(), i, s.sz) / s.dz;
            double d2 = Solver::Dq(s.sxy.data(), i, s.sx) / s.dx;
            double d3 = Solver::Dp(s.syy.data(), i, 1) / s.dy;
            double p1 = 0, p2 = 0, p3 = 0;  // modified derivatives
            // psi_new values for this step are stored in s (after forward step)
            if (s.slabS(z, nz)) p1 = d1 / s.pz.K[z] + s.m_syz_z[i]; else p1 = d1;
            if (s.slabV(x, nx)) p2 = d2 / s.px.K[x] + s.m_sxy_x[i]; else p2 = d2;
            if (s.slabV(y, ny)) p3 = d3 / s.py.Kh[y] + s.m_syy_y[i]; else p3 = d3;
            if (gB) gB[i] += g * (p1 + p2 + p3) * dt;
            double gd = g * b * dt;  // adjoint of each modified derivative
            // d' = d/K + psi_new ; psi_new = bb*psi_old + aa*d
            double gd1 = gd, gd2 = gd, gd3 = gd;
            if (s.slabS(z, nz)) { a_m_syz_z[i] += gd1; gd1 = gd1 / s.pz.K[z]; }
            if (s.slabV(x, nx)) { a_m_sxy_x[i] += gd2; gd2 = gd2 / s.px.K[x]; }
            if (s.slabV(y, ny)) { a_m_syy_y[i] += gd3; gd3 = gd3 / s.py.Kh[y]; }
            // psi_new adjoint -> psi_old and d
            if (s.slabS(z, nz)) { double gp = a_m_syz_z[i]; gd1 += s.pz.a[z] * gp; a_m_syz_z[i] = s.pz.b[z] * gp; }
            if (s.slabV(x, nx)) { double gp = a_m_sxy_x[i]; gd2 += s.px.a[x] * gp; a_m_sxy_x[i] = s.px.b[x] * gp; }
            if (s.slabV(y, ny)) { double gp = a_m_syy_y[i]; gd3 += s.py.ah[y] * gp; a_m_syy_y[i] = s.py.bh[y] * gp; }
            tDm(a_syz.data(), i, s.sz, gd1 / s.dz);
            tDq(a_sxy.data(), i, s.sx, gd2 / s.dx);
            tDp(a_syy.data(), i, 1, gd3 / s.dy);
          }
          // ---- vx
          {
            double g = a_vx[i];
            double d1 = Solver::Dm(s.sxz.data(), i, s.sz) / s.dz;
            double d2 = Solver::Dp(s.sxx.data(), i, s.sx) / s.dx;
            double d3 = Solver::Dm(s.sxy.data(), i, 1) / s.dy;
            double p1 = s.slabS(z, nz) ? d1 / s.pz.K[z] + s.m_sxz_z[i] : d1;
            double p2 = s.slabV(x, nx) ? d2 / s.px.Kh[x] + s.m_sxx_x[i] : d2;
            double p3 = s.slabV(y, ny) ? d3 / s.py.K[y] + s.m_sxy_y[i] : d3;
            if (gB) gB[i] += g * (p1 + p2 + p3) * dt;
            double gd = g * b * dt, gd1 = gd, gd2 = gd, gd3 = gd;
            if (s.slabS(z, nz)) { a_m_sxz_z[i] += gd1; gd1 /= s.pz.K[z]; double gp = a_m_sxz_z[i]; gd1 += s.pz.a[z] * gp; a_m_sxz_z[i] = s.pz.b[z] * gp; }
            if (s.slabV(x, nx)) { a_m_sxx_x[i] += gd2; gd2 /= s.px.Kh[x]; double gp = a_m_sxx_x[i]; gd2 += s.px.ah[x] * gp; a_m_sxx_x[i] = s.px.bh[x] * gp; }
            if (s.slabV(y, ny)) { a_m_sxy_y[i] += gd3; gd3 /= s.py.K[y]; double gp = a_m_sxy_y[i]; gd3 += s.py.a[y] * gp; a_m_sxy_y[i] = s.py.b[y] * gp; }
            tDm(a_sxz.data(), i, s.sz, gd1 / s.dz);
            tDp(a_sxx.data(), i, s.sx, gd2 / s.dx);
            tDm(a_sxy.data(), i, 1, gd3 / s.dy);
          }
          // ---- vz
          {
            double g = a_vz[i];
            double d1 = Solver::Dp(s.szz.data(), i, s.sz) / s.dz;
            double d2 = Solver::Dm(s.sxz.data(), i, s.sx) / s.dx;
            double d3 = Solver::Dm(s.syz.data(), i, 1) / s.dy;
            double p1 = s.slabS(z, nz) ? d1 / s.pz.Kh[z] + s.m_szz_z[i] : d1;
            double p2 = s.slabV(x, nx) ? d2 / s.px.K[x] + s.m_sxz_x[i] : d2;
            double p3 = s.slabV(y, ny) ? d3 / s.py.K[y] + s.m_syz_y[i] : d3;
            if (gB) gB[i] += g * (p1 + p2 + p3) * dt;
            double gd = g * b * dt, gd1 = gd, gd2 = gd, gd3 = gd;
            if (s.slabS(z, nz)) { a_m_szz_z[i] += gd1; gd1 /= s.pz.Kh[z]; double gp = a_m_szz_z[i]; gd1 += s.pz.ah[z] * gp; a_m_szz_z[i] = s.pz.bh[z] * gp; }
            if (s.slabV(x, nx)) { a_m_sxz_x[i] += gd2; gd2 /= s.px.K[x]; double gp = a_m_sxz_x[i]; gd2 += s.px.a[x] * gp; a_m_sxz_x[i] = s.px.b[x] * gp; }
            if (s.slabV(y, ny)) { a_m_syz_y[i] += gd3; gd3 /= s.py.K[y]; double gp = a_m_syz_y[i]; gd3 += s.py.a[y] * gp; a_m_syz_y[i] = s.py.b[y] * gp; }
            tDp(a_szz.data(), i, s.sz, gd1 / s.dz);
            tDm(a_sxz.data(), i, s.sx, gd2 / s.dx);
            tDm(a_syz.data(), i, 1, gd3 / s.dy);
          }
        }
  }

  // Transpose of stress_fwd, with lambda/mu imaging.
  void stress_T(double *glam, double *gmu) {
    const int nz = s.nz, nx = s.nx, ny = s.ny;
    const double dt = s.dt;
    for (int z = 2; z <= nz - 3; ++z)
      for (int x = 2; x <= nx - 3; ++x)
        for (int y = 2; y <= ny - 3; ++y) {
          size_t i = s.idx(z, x, y);
          double l = s.lam[i], m = s.mu[i];
          // shear part: sxz += m (dvx_dz' + dvz_dx') dt etc.
          {
            double gxz = a_sxz[i], gxy = a_sxy[i], gyz = a_syz[i];
            double d_vx_z = Solver::Dp(s.vx.data(), i, s.sz) / s.dz, d_vx_y = Solver::Dp(s.vx.data(), i, 1) / s.dy;
            double d_vz_x = Solver::Dp(s.vz.data(), i, s.sx) / s.dx, d_vz_y = Solver::Dp(s.vz.data(), i, 1) / s.dy;
            double d_vy_x = Solver::Dp(s.vy.data(), i, s.sx) / s.dx, d_vy_z = Solver::Dp(s.vy.data(), i, s.sz) / s.dz;
            bool zs = s.slabS(z, nz), xs = s.slabS(x, nx), ys = s.slabS(y, ny);
            double p_vx_z = zs ? d_vx_z / s.pz.Kh[z] + s.m_vx_z[i] : d_vx_z;
            double p_vy_z = zs ? d_vy_z / s.pz.Kh[z] + s.m_vy_z[i] : d_vy_z;
            double p_vz_x = xs ? d_vz_x / s.px.Kh[x] + s.m_vz_x[i] : d_vz_x;
            double p_vy_x = xs ? d_vy_x / s.px.Kh[x] + s.m_vy_x[i] : d_vy_x;
            double p_vz_y = ys ? d_vz_y / s.py.Kh[y] + s.m_vz_y[i] : d_vz_y;
            double p_vx_y = ys ? d_vx_y / s.py.Kh[y] + s.m_vx_y[i] : d_vx_y;
            if (gmu) gmu[i] += (gxz * (p_vx_z + p_vz_x) + gxy * (p_vx_y + p_vy_x) + gyz * (p_vy_z + p_vz_y)) * dt;
            double g_vx_z = gxz * m * dt, g_vz_x = gxz * m * dt;
            double g_vx_y = gxy * m * dt, g_vy_x = gxy * m * dt;
            double g_vy_z = gyz * m * dt, g_vz_y = gyz * m * dt;
            auto psiT = [&](bool on, Vec &am, double Kk, double aa, double bb, double &gd) {
              if (!on) return;
              am[i] += gd; gd /= Kk; double gp = am[i]; gd += aa * gp; am[i] = bb * gp;
            };
            psiT(zs, a_m_vx_z, s.pz.Kh[z], s.pz.ah[z], s.pz.bh[z], g_vx_z);
            psiT(zs, a_m_vy_z, s.pz.Kh[z], s.pz.ah[z], s.pz.bh[z], g_vy_z);
            psiT(xs, a_m_vz_x, s.px.Kh[x], s.px.ah[x], s.px.bh[x], g_vz_x);
            psiT(xs, a_m_vy_x, s.px.Kh[x], s.px.ah[x], s.px.bh[x], g_vy_x);
            psiT(ys, a_m_vz_y, s.py.Kh[y], s.py.ah[y], s.py.bh[y], g_vz_y);
            psiT(ys, a_m_vx_y, s.py.Kh[y], s.py.ah[y], s.py.bh[y], g_vx_y);
            tDp(a_vx.data(), i, s.sz, g_vx_z / s.dz);
            tDp(a_vx.data(), i, 1, g_vx_y / s.dy);
            tDp(a_vz.data(), i, s.sx, g_vz_x / s.dx);
            tDp(a_vz.data(), i, 1, g_vz_y / s.dy);
            tDp(a_vy.data(), i, s.sx, g_vy_x / s.dx);
            tDp(a_vy.data(), i, s.sz, g_vy_z / s.dz);
          }
          // normal part
          {
            double gzz = a_szz[i], gxx = a_sxx[i], gyy = a_syy[i];
            double ezz = Solver::Dm(s.vz.data(), i, s.sz) / s.dz;
            double exx = Solver::Dm(s.vx.data(), i, s.sx) / s.dx;
            double eyy = Solver::Dm(s.vy.data(), i, 1) / s.dy;
            bool zs = s.slabS(z, nz), xs = s.slabS(x, nx), ys = s.slabS(y, ny);
            double pz_ = zs ? ezz / s.pz.K[z] + s.m_vz_z[i] : ezz;
            double px_ = xs ? exx / s.px.K[x] + s.m_vx_x[i] : exx;
            double py_ = ys ? eyy / s.py.K[y] + s.m_vy_y[i] : eyy;
            double div = pz_ + px_ + py_;
            if (glam) glam[i] += (gzz + gxx + gyy) * div * dt;
            if (gmu) gmu[i] += 2.0 * (gzz * pz_ + gxx * px_ + gyy * py_) * dt;
            double g_ez = ((l + 2.0 * m) * gzz + l * gxx + l * gyy) * dt;
            double g_ex = (l * gzz + (l + 2.0 * m) * gxx + l * gyy) * dt;
            double g_ey = (l * gzz + l * gxx + (l + 2.0 * m) * gyy) * dt;
            if (zs) { a_m_vz_z[i] += g_ez; g_ez /= s.pz.K[z]; double gp = a_m_vz_z[i]; g_ez += s.pz.a[z] * gp; a_m_vz_z[i] = s.pz.b[z] * gp; }
            if (xs) { a_m_vx_x[i] += g_ex; g_ex /= s.px.K[x]; double gp = a_m_vx_x[i]; g_ex += s.px.a[x] * gp; a_m_vx_x[i] = s.px.b[x] * gp; }
            if (ys) { a_m_vy_y[i] += g_ey; g_ey /= s.py.K[y]; double gp = a_m_vy_y[i]; g_ey += s.py.a[y] * gp; a_m_vy_y[i] = s.py.b[y] * gp; }
            tDm(a_vz.data(), i, s.sz, g_ez / s.dz);
            tDm(a_vx.data(), i, s.sx, g_ex / s.dx);
            tDm(a_vy.data(), i, 1, g_ey / s.dy);
          }
        }
  }
};

// Forward state snapshot (fields + memory variables).
struct State {
  std::vector<Vec> v;
};
State snap(Solver &s) {
  Vec *all[] = {&s.vz, &s.vx, &s.vy, &s.szz, &s.sxx, &s.syy, &s.sxz, &s.sxy, &s.syz,
                &s.m_vz_z, &s.m_vz_x, &s.m_vz_y, &s.m_vx_z, &s.m_vx_x, &s.m_vx_y, &s.m_vy_z, &s.m_vy_x, &s.m_vy_y,
                &s.m_szz_z, &s.m_sxx_x, &s.m_syy_y, &s.m_sxz_z, &s.m_sxz_x, &s.m_sxy_x, &s.m_sxy_y, &s.m_syz_y, &s.m_syz_z};
  State st;
  for (Vec *p : all) st.v.push_back(*p);
  return st;
}
void restore(Solver &s, const State &st) {
  Vec *all[] = {&s.vz, &s.vx, &s.vy, &s.szz, &s.sxx, &s.syy, &s.sxz, &s.sxy, &s.syz,
                &s.m_vz_z, &s.m_vz_x, &s.m_vz_y, &s.m_vx_z, &s.m_vx_x, &s.m_vx_y, &s.m_vy_z, &s.m_vy_x, &s.m_vy_y,
                &s.m_szz_z, &s.m_sxx_x, &s.m_syy_y, &s.m_sxz_z, &s.m_sxz_x, &s.m_sxy_x, &s.m_sxy_y, &s.m_syz_y, &s.m_syz_z};
  for (size_t k = 0; k < st.v.size(); ++k) *all[k] = st.v[k];
}

}  // namespace

extern "C" {

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// C-PML profile of one axis: K, a, b, K_half, a_half, b_half (length n each).
void oracle_cpml(int n, int npml, double dh, double f0, double dt, double *out6) {
  Profile p = cpml_profile(n, npml, dh, f0, dt);
  const Vec *v[6] = {&p.K, &p.a, &p.b, &p.Kh, &p.ah, &p.bh};
  for (int k = 0; k < 6; ++k) std::copy(v[k]->begin(), v[k]->end(), out6 + (size_t)k * n);
}

// Tapered source-time function (Src_Rec.cu:146).
void oracle_taper_stf(const double *stf, int nt, double dt, double *out) {
  std::vector<double> v;
  taper_stf(stf, nt, dt, v);
  std::copy(v.begin(), v.end(), out);
}

// Forward modelling of `nshot` shots.  stf: [nshot][nt] untapered rows.
// traces: concatenation over shots of [3][nrec_s][nt] (x, y, z components).
int oracle_forward(const OracleGrid *g, const double *lam, const double *mu, const double *rho,
                   int nshot, const OracleShot *shots, const double *stf, double *traces) {
  Solver s(*g, lam, mu, rho);
  size_t off = 0;
  for (int k = 0; k < nshot; ++k) {
    run_forward(s, shots[k], stf + (size_t)k * g->nt, traces + off, nullptr, nullptr);
    off += (size_t)3 * shots[k].nrec * g->nt;
  }
  return 0;
}

// Source illumination (diagonal pseudo-Hessian, Shin et al. 2001) summed
// over the shots: for every state S_k, k = 1 .. nt-1, the squared
// derivatives of the forward step with respect to lambda, mu and rho
// (Solver::illum; rho through B = 1/rho on [2, n-3]^3, (dB/drho)^2 = 1/rho^4).
int oracle_illumination(const OracleGrid *g, const double *lam, const double *mu,
                        const double *rho, int nshot, const OracleShot *shots, const double *stf,
                        double *hl, double *hm, double *hr) {
  Solver s(*g, lam, mu, rho);
  const size_t N = s.N;
  std::fill(hl, hl + N, 0.0);
  std::fill(hm, hm + N, 0.0);
  std::vector<double> hb(N, 0.0);
  const int nt = g->nt;
  for (int k = 0; k < nshot; ++k) {
    const OracleShot &sh = shots[k];
    s.zero_all();
    std::vector<double> st;
    taper_stf(stf + (size_t)k * nt, nt, s.dt, st);
    size_t isrc = s.idx(sh.z_src, sh.x_src, sh.y_src);
    for (int it = 0; it <= nt - 2; ++it) {
      s.stress_fwd();
      double amp = 1500.0 * 1500.0 * st[it] * s.dt;
      s.szz[isrc] += amp; s.sxx[isrc] += amp; s.syy[isrc] += amp;
      s.velocity_fwd();
      s.illum(hl, hm, hb.data(), it + 1 <= nt - 2);
    }
  }
  for (int z = 0; z < s.nz; ++z)
    for (int x = 0; x < s.nx; ++x)
      for (int y = 0; y < s.ny; ++y) {
        size_t i = s.idx(z, x, y);
        bool in = z >= 2 && z <= s.nz - 3 && x >= 2 && x <= s.nx - 3 && y >= 2 && y <= s.ny - 3;
        hr[i] = in ? hb[i] / (rho[i] * rho[i] * rho[i] * rho[i]) : 0.0;
      }
  return 0;
}

// Gradient of the windowed L2 misfit.  obs uses the traces layout.
// mode 0: the reference algorithm (boundary-shell reconstruction, reference
//         adjoint kernels, interior-only imaging); gradients w.r.t. lambda,
//         mu, rho in the reference's convention.
// mode 1: exact discrete adjoint of the forward scheme (full state stored),
//         gradients are dJ/dlambda, dJ/dmu, dJ/drho of J as returned.
// res_out (optional, traces layout): adjoint source of each shot.
int oracle_gradient(const OracleGrid *g, const double *lam, const double *mu, const double *rho,
                    int nshot, const OracleShot *shots, const double *stf, const double *obs,
                    int mode, int if_win, double *misfit_out, double *glam, double *gmu,
                    double *grho, double *res_out) {
  Solver s(*g, lam, mu, rho);
  const int nt = g->nt;
  const size_t N = s.N;
  std::fill(glam, glam + N, 0.0);
  std::fill(gmu, gmu + N, 0.0);
  std::fill(grho, grho + N, 0.0);
  double J = 0.0;
  size_t off = 0;
  std::vector<size_t> pts = shell_points(s);
  for (int k = 0; k < nshot; ++k) {
    const OracleShot &sh = shots[k];
    const int nr = sh.nrec;
    size_t ntr = (size_t)3 * nr * nt;
    std::vector<double> syn(ntr), res(ntr), stf_t;
    taper_stf(stf + (size_t)k * nt, nt, s.dt, stf_t);
    size_t isrc = s.idx(sh.z_src, sh.x_src, sh.y_src);
    std::vector<size_t> irec(nr);
    for (int r = 0; r < nr; ++r) irec[r] = s.idx(sh.z_rec[r], sh.x_rec[r], sh.y_rec[r]);
    if (mode == 0) {
      std::vector<double> shell((size_t)nt * 9 * pts.size());
      run_forward(s, sh, stf + (size_t)k * nt, syn.data(), &shell, &pts);
      J += misfit(sh, nt, s.dt, if_win != 0, obs + off, syn.data(), res.data());
      if (res_out) std::copy(res.begin(), res.end(), res_out + off);
      s.zero_adj();
      s.zero_psi();
      auto inject = [&](int it) {
        for (int r = 0; r < nr; ++r) {
          s.avx[irec[r]] += res[((size_t)0 * nr + r) * nt + it];
          s.avy[irec[r]] += res[((size_t)1 * nr + r) * nt + it];
          s.avz[irec[r]] += res[((size_t)2 * nr + r) * nt + it];
        }
      };
      Vec *Fs[6] = {&s.szz, &s.sxz, &s.sxx, &s.syy, &s.sxy, &s.syz};
      Vec *Fv[3] = {&s.vz, &s.vx, &s.vy};
      const size_t np = pts.size();
      s.velocity_adj_ref();
      inject(nt - 1);
      s.stress_adj_ref();
      for (int it = nt - 2; it >= 0; --it) {
        const double *src = shell.data() + (size_t)it * 9 * np;
        s.velocity_rev(grho);
        for (int f = 0; f < 3; ++f)
          for (size_t q = 0; q < np; ++q) (*Fv[f])[pts[q]] = src[(6 + f) * np + q];
        double amp = 1500.0 * 1500.0 * stf_t[it] * s.dt;
        s.szz[isrc] -= amp; s.sxx[isrc] -= amp; s.syy[isrc] -= amp;
        s.stress_rev(glam, gmu);
        for (int f = 0; f < 6; ++f)
          for (size_t q = 0; q < np; ++q) (*Fs[f])[pts[q]] = src[f * np + q];
        s.velocity_adj_ref();
        inject(it);
        s.stress_adj_ref();
      }
    } else {
      // Exact adjoint with every forward state stored.  Forward step t maps
      // state S_t to S_{t+1}: stress update, source, velocity update.
      // Receivers read v of S_{t+1} at sample t+1.
      s.zero_all();
      std::vector<State> states;
      states.reserve(nt);
      for (int it = 0; it <= nt - 2; ++it) {
        states.push_back(snap(s));
        s.stress_fwd();
        double amp = 1500.0 * 1500.0 * stf_t[it] * s.dt;
        s.szz[isrc] += amp; s.sxx[isrc] += amp; s.syy[isrc] += amp;
        // stress-stage state is needed by the velocity transpose
        s.velocity_fwd();
        for (int r = 0; r < nr; ++r) {
          syn[((size_t)0 * nr + r) * nt + it + 1] = s.vx[irec[r]];
          syn[((size_t)1 * nr + r) * nt + it + 1] = s.vy[irec[r]];
          syn[((size_t)2 * nr + r) * nt + it + 1] = s.vz[irec[r]];
        }
      }
      for (int r = 0; r < nr; ++r)
        for (int c = 0; c < 3; ++c) syn[((size_t)c * nr + r) * nt] = 0.0;
      J += misfit(sh, nt, s.dt, if_win != 0, obs + off, syn.data(), res.data());
      if (res_out) std::copy(res.begin(), res.end(), res_out + off);
      // dJ/dsyn = -2 * res (res already carries the second window factor).
      ExactAdj A(s);
      std::vector<double> gB(N, 0.0);
      for (int it = nt - 2; it >= 0; --it) {
        // adjoint of the receiver read at sample it+1
        for (int r = 0; r < nr; ++r) {
          A.a_vx[irec[r]] += -2.0 * res[((size_t)0 * nr + r) * nt + it + 1];
          A.a_vy[irec[r]] += -2.0 * res[((size_t)1 * nr + r) * nt + it + 1];
          A.a_vz[irec[r]] += -2.0 * res[((size_t)2 * nr + r) * nt + it + 1];
        }
        // recover the state after the stress stage of step it
        restore(s, states[it]);
        s.stress_fwd();
        double amp = 1500.0 * 1500.0 * stf_t[it] * s.dt;
        s.szz[isrc] += amp; s.sxx[isrc] += amp; s.syy[isrc] += amp;
        // velocity transpose needs sigma_{t+1} (current) and psi_v after the
        // update; run the velocity step on a copy to get psi_v new.
        State mid = snap(s);
        s.velocity_fwd();
        State after = snap(s);
        // put sigma/psi_v(new) in place, v irrelevant for velocity_T
        restore(s, mid);
        // psi_v new values
        Vec *pv[9] = {&s.m_szz_z, &s.m_sxx_x, &s.m_syy_y, &s.m_sxz_z, &s.m_sxz_x, &s.m_sxy_x, &s.m_sxy_y, &s.m_syz_y, &s.m_syz_z};
        for (int q = 0; q < 9; ++q) *pv[q] = after.v[18 + q];
        A.velocity_T(gB.data());
        // stress transpose needs v_t (before stress) and psi_s after update
        restore(s, states[it]);
        State st0 = snap(s);
        s.stress_fwd();
        Vec *ps[9] = {&s.m_vz_z, &s.m_vz_x, &s.m_vz_y, &s.m_vx_z, &s.m_vx_x, &s.m_vx_y, &s.m_vy_z, &s.m_vy_x, &s.m_vy_y};
        std::vector<Vec> psnew;
        for (int q = 0; q < 9; ++q) psnew.push_back(*ps[q]);
        restore(s, st0);
        for (int q = 0; q < 9; ++q) *ps[q] = psnew[q];
        A.stress_T(glam, gmu);
      }
      // rho enters through B = 1/rho on [2, n-3]^3 only.
      for (int z = 2; z <= s.nz - 3; ++z)
        for (int x = 2; x <= s.nx - 3; ++x)
          for (int y = 2; y <= s.ny - 3; ++y) {
            size_t i = s.idx(z, x, y);
            grho[i] += -gB[i] / (rho[i] * rho[i]);
          }
    }
    off += ntr;
  }
  *misfit_out = J;
  return 0;
}

// Applies one forward step (stress, source amplitude `amp`, velocity) to a
// full 27-component state in place; used by the dot-product test.
int oracle_step(const OracleGrid *g, const double *lam, const double *mu, const double *rho,
                int z_src, int x_src, int y_src, double amp, double *state27) {
  Solver s(*g, lam, mu, rho);
  Vec *all[] = {&s.vz, &s.vx, &s.vy, &s.szz, &s.sxx, &s.syy, &s.sxz, &s.sxy, &s.syz,
                &s.m_vz_z, &s.m_vz_x, &s.m_vz_y, &s.m_vx_z, &s.m_vx_x, &s.m_vx_y, &s.m_vy_z, &s.m_vy_x, &s.m_vy_y,
                &s.m_szz_z, &s.m_sxx_x, &s.m_syy_y, &s.m_sxz_z, &s.m_sxz_x, &s.m_sxy_x, &s.m_sxy_y, &s.m_syz_y, &s.m_syz_z};
  for (int k = 0; k < 27; ++k) std::copy(state27 + (size_t)k * s.N, state27 + (size_t)(k + 1) * s.N, all[k]->begin());
  s.stress_fwd();
  size_t i = s.idx(z_src, x_src, y_src);
  s.szz[i] += amp; s.sxx[i] += amp; s.syy[i] += amp;
  s.velocity_fwd();
  for (int k = 0; k < 27; ++k) std::copy(all[k]->begin(), all[k]->end(), state27 + (size_t)k * s.N);
  return 0;
}

// Transposed step applied to a 27-component adjoint state (linear part of
// oracle_step, source excluded); the forward state is irrelevant for the
// transpose of a linear map, so only the model is needed.
int oracle_step_T(const OracleGrid *g, const double *lam, const double *mu, const double *rho,
                  double *astate27) {
  Solver s(*g, lam, mu, rho);
  ExactAdj A(s);
  Vec *all[] = {&A.a_vz, &A.a_vx, &A.a_vy, &A.a_szz, &A.a_sxx, &A.a_syy, &A.a_sxz, &A.a_sxy, &A.a_syz,
                &A.a_m_vz_z, &A.a_m_vz_x, &A.a_m_vz_y, &A.a_m_vx_z, &A.a_m_vx_x, &A.a_m_vx_y, &A.a_m_vy_z, &A.a_m_vy_x, &A.a_m_vy_y,
                &A.a_m_szz_z, &A.a_m_sxx_x, &A.a_m_syy_y, &A.a_m_sxz_z, &A.a_m_sxz_x, &A.a_m_sxy_x, &A.a_m_sxy_y, &A.a_m_syz_y, &A.a_m_syz_z};
  for (int k = 0; k < 27; ++k) std::copy(astate27 + (size_t)k * s.N, astate27 + (size_t)(k + 1) * s.N, all[k]->begin());
  A.velocity_T(nullptr);
  A.stress_T(nullptr, nullptr);
  for (int k = 0; k < 27; ++k) std::copy(all[k]->begin(), all[k]->end(), astate27 + (size_t)k * s.N);
  return 0;
}

}  // extern "C"
