// Driver that runs the reference's own kernel bodies on the CPU.
//
// TEST INFRASTRUCTURE ONLY.  Linked by oracle/Makefile with the reference's
// Src_3d kernel sources compiled through ref_shim.h into
// oracle/_ref/libefwi_ref.so.  This file is new code: it emulates CUDA
// launches (every block and thread of the reference's launch geometry) and
// follows the call order of cufd (Ops/FWI/Src_3d/libCUFD.cu):
//   set-up        :67-91   transpose to z-fastest, Model, Cpml, Src_Rec
//   forward loop  :312-354 from_bnd, stress, add_source, velocity, recording
//   misfit        :371-440 cuda_window, gpuMinus, sum of squares, window again
//   reverse loop  :500-612 velocity_adj, res_injection, stress_adj pre-step,
//                          then velocity(rev), to_bnd, add_source(sub),
//                          stress(rev), to_bnd, velocity_adj, res_injection,
//                          stress_adj per step
//   gradients     :636-652 transpose back to [z][x][y]
// The one reference kernel not run is cuda_cal_objective (a single-block
// shared-memory tree reduction, utilities.cu:145-166): the sum of squares is
// taken here in double instead.
#include "ref_shim.h"

#include <algorithm>
#include <cstdint>
#ifdef _OPENMP
#include <omp.h>
#endif

REF_TLS dim3 blockIdx;
REF_TLS dim3 threadIdx;
REF_TLS dim3 blockDim;
REF_TLS dim3 gridDim;

// ---- reference kernel interfaces (Src_3d/*.cu, compiled through the shim)
void stress(float *d_vz, float *d_vx, float *d_vy, float *d_szz, float *d_sxx, float *d_sxz,
            float *d_syy, float *d_sxy, float *d_syz, float *d_mem_dvz_dz, float *d_mem_dvz_dx,
            float *d_mem_dvz_dy, float *d_mem_dvx_dz, float *d_mem_dvx_dx, float *d_mem_dvx_dy,
            float *d_mem_dvy_dz, float *d_mem_dvy_dx, float *d_mem_dvy_dy, float *d_Lambda,
            float *d_Mu, float *d_Den, float *d_K_z, float *d_a_z, float *d_b_z, float *d_K_z_half,
            float *d_a_z_half, float *d_b_z_half, float *d_K_x, float *d_a_x, float *d_b_x,
            float *d_K_x_half, float *d_a_x_half, float *d_b_x_half, float *d_K_y, float *d_a_y,
            float *d_b_y, float *d_K_y_half, float *d_a_y_half, float *d_b_y_half, int nz, int nx,
            int ny, float dt, float dz, float dx, float dy, int nPml, bool isFor,
            float *d_szz_adj, float *d_sxx_adj, float *d_sxz_adj, float *d_syy_adj,
            float *d_sxy_adj, float *d_syz_adj, float *d_LambdaGrad, float *d_MuGrad);
void velocity(float *d_vz, float *d_vx, float *d_vy, float *d_szz, float *d_sxx, float *d_sxz,
              float *d_syy, float *d_sxy, float *d_syz, float *d_mem_dszz_dz, float *d_mem_dsxz_dx,
              float *d_mem_dsxz_dz, float *d_mem_dsxx_dx, float *d_mem_dsxy_dx,
              float *d_mem_dsxy_dy, float *d_mem_dsyy_dy, float *d_mem_dsyz_dy,
              float *d_mem_dsyz_dz, float *d_Lambda, float *d_Mu, float *d_Byc, float *d_K_z,
              float *d_a_z, float *d_b_z, float *d_K_z_half, float *d_a_z_half, float *d_b_z_half,
              float *d_K_x, float *d_a_x, float *d_b_x, float *d_K_x_half, float *d_a_x_half,
              float *d_b_x_half, float *d_K_y, float *d_a_y, float *d_b_y, float *d_K_y_half,
              float *d_a_y_half, float *d_b_y_half, int nz, int nx, int ny, float dt, float dz,
              float dx, float dy, int nPml, bool isFor, float *d_vz_adj, float *d_vx_adj,
              float *d_vy_adj, float *d_DenGrad);
void stress_adj(float *d_vz, float *d_vx, float *d_vy, float *d_szz, float *d_sxx, float *d_sxz,
                float *d_syy, float *d_sxy, float *d_syz, float *d_mem_dszz_dz,
                float *d_mem_dsxz_dx, float *d_mem_dsxz_dz, float *d_mem_dsxx_dx,
                float *d_mem_dsxy_dx, float *d_mem_dsxy_dy, float *d_mem_dsyy_dy,
                float *d_mem_dsyz_dy, float *d_mem_dsyz_dz, float *d_mem_dvz_dz,
                float *d_mem_dvz_dx, float *d_mem_dvz_dy, float *d_mem_dvx_dz,
                float *d_mem_dvx_dx, float *d_mem_dvx_dy, float *d_mem_dvy_dz,
                float *d_mem_dvy_dx, float *d_mem_dvy_dy, float *d_Lambda, float *d_Mu,
                float *d_Den, float *d_Byc, float *d_K_z_half, float *d_a_z_half,
                float *d_b_z_half, float *d_K_x_half, float *d_a_x_half, float *d_b_x_half,
                float *d_K_y_half, float *d_a_y_half, float *d_b_y_half, float *d_K_z,
                float *d_a_z, float *d_b_z, float *d_K_x, float *d_a_x, float *d_b_x,
                float *d_K_y, float *d_a_y, float *d_b_y, int nz, int nx, int ny, float dt,
                float dz, float dx, float dy, int nPml);
void velocity_adj(float *d_vz, float *d_vx, float *d_vy, float *d_szz, float *d_sxx,
                  float *d_sxz, float *d_syy, float *d_sxy, float *d_syz, float *d_mem_dszz_dz,
                  float *d_mem_dsxz_dx, float *d_mem_dsxz_dz, float *d_mem_dsxx_dx,
                  float *d_mem_dsxy_dx, float *d_mem_dsxy_dy, float *d_mem_dsyy_dy,
                  float *d_mem_dsyz_dy, float *d_mem_dsyz_dz, float *d_mem_dvz_dz,
                  float *d_mem_dvz_dx, float *d_mem_dvz_dy, float *d_mem_dvx_dz,
                  float *d_mem_dvx_dx, float *d_mem_dvx_dy, float *d_mem_dvy_dz,
                  float *d_mem_dvy_dx, float *d_mem_dvy_dy, float *d_Lambda, float *d_Mu,
                  float *d_Den, float *d_Byc, float *d_K_z_half, float *d_a_z_half,
                  float *d_b_z_half, float *d_K_x_half, float *d_a_x_half, float *d_b_x_half,
                  float *d_K_y_half, float *d_a_y_half, float *d_b_y_half, float *d_K_z,
                  float *d_a_z, float *d_b_z, float *d_K_x, float *d_a_x, float *d_b_x,
                  float *d_K_y, float *d_a_y, float *d_b_y, int nz, int nx, int ny, float dt,
                  float dz, float dx, float dy, int nPml);
void cpmlInit(float *K, float *a, float *b, float *K_half, float *a_half, float *b_half, int N,
              int nPml, float dh, float f0, float dt, float VpAve);
void aveBycInit(float *d_Rho, float *d_Byc, int nz, int nx, int ny);
void src_rec_gauss_amp(float *gauss_amp, int nz, int nx, int ny);
void add_source(float *d_szz, float *d_sxx, float *d_syy, float amp, int nz, int nx, int ny,
                bool isFor, int z_loc, int x_loc, int y_loc, float dt, float *gauss_amp);
void recording(float *d_vz, float *d_vx, float *d_vy, int nz, int nx, float *d_data_x,
               float *d_data_y, float *d_data_z, int iShot, int it, int nSteps, int nrec,
               int *d_z_rec, int *d_x_rec, int *d_y_rec);
void res_injection(float *d_vx_adj, float *d_vy_adj, float *d_vz_adj, int nz, int nx,
                   float *d_res_x, float *d_res_y, float *d_res_z, int it, float dt, int nSteps,
                   int nrec, int *d_z_rec, int *d_x_rec, int *d_y_rec);
void from_bnd(float *d_field, float *d_bnd, int nz, int nx, int ny, int nzBnd, int nxBnd,
              int nyBnd, int len_Bnd_vec, int nLayerStore, int indT, int nPml, int nSteps);
void to_bnd(float *d_field, float *d_bnd, int nz, int nx, int ny, int nzBnd, int nxBnd,
            int nyBnd, int len_Bnd_vec, int nLayerStore, int indT, int nPml, int nSteps);
void cuda_window(int nt, int nrec, float dt, float *d_win_start, float *d_win_end,
                 float *d_weights, float src_weight, float ratio, float *data);
void cuda_window(int nt, int nrec, float dt, float ratio, float *data);
void gpuMinus(float *d_out, float *d_in1, float *d_in2, int nx, int ny);

extern "C" {
typedef struct {
  int nz, nx, ny, npml, nt;
  float dz, dx, dy, dt, f0;
} RefGrid;

typedef struct {
  int z_src, x_src, y_src, nrec;
  const int *z_rec, *x_rec, *y_rec;
  const float *win_start, *win_end, *weights;
  float src_weight;
} RefShot;
}

namespace {

// Runs `body` once per emulated CUDA thread of the launch <<<g, b>>>.
template <class F>
void launch(dim3 g, dim3 b, F body) {
  long nblk = (long)g.x * g.y * g.z;
#pragma omp parallel for schedule(dynamic, 1)
  for (long k = 0; k < nblk; ++k) {
    gridDim = g;
    blockDim = b;
    blockIdx = dim3(k % g.x, (k / g.x) % g.y, k / ((long)g.x * g.y));
    for (unsigned tz = 0; tz < b.z; ++tz)
      for (unsigned ty = 0; ty < b.y; ++ty)
        for (unsigned tx = 0; tx < b.x; ++tx) {
          threadIdx = dim3(tx, ty, tz);
          body();
        }
  }
}

// Zero-initialised float buffer with slack after the end, so that the
// reference kernels' reads of model values before their bounds test
// (stress_adj.cu:47-49, velocity_adj.cu:55-57) stay inside the allocation.
struct Buf {
  std::vector<float> v;
  Buf() {}
  explicit Buf(size_t n, size_t slack) : v(n + slack, 0.0f) {}
  float *p() { return v.data(); }
  void zero() { std::fill(v.begin(), v.end(), 0.0f); }
};

struct Ref {
  int nz, nx, ny, np, nt;
  float dz, dx, dy, dt, f0;
  size_t N;
  dim3 blocks, threads;
  Buf L, M, R, Byc;
  Buf vz, vx, vy, szz, sxx, sxz, syy, sxy, syz;
  Buf avz, avx, avy, aszz, asxx, asxz, asyy, asxy, asyz;
  Buf m_vz_z, m_vz_x, m_vz_y, m_vx_z, m_vx_x, m_vx_y, m_vy_z, m_vy_x, m_vy_y;
  Buf m_szz_z, m_sxx_x, m_syy_y, m_sxz_z, m_sxz_x, m_sxy_x, m_sxy_y, m_syz_y, m_syz_z;
  Buf gL, gM, gR;
  std::vector<float> Kz, az, bz, Kzh, azh, bzh, Kx, ax, bx, Kxh, axh, bxh, Ky, ay, by, Kyh, ayh, byh;
  std::vector<float> gauss;
  int nzB, nxB, nyB, lenB;

  Ref(const RefGrid &g, const float *lam, const float *mu, const float *rho)
      : nz(g.nz), nx(g.nx), ny(g.ny), np(g.npml), nt(g.nt), dz(g.dz), dx(g.dx), dy(g.dy),
        dt(g.dt), f0(g.f0) {
    N = (size_t)nz * nx * ny;
    size_t slack = (size_t)64 * nz + 64;
    Buf *all[] = {&L, &M, &R, &Byc, &vz, &vx, &vy, &szz, &sxx, &sxz, &syy, &sxy, &syz,
                  &avz, &avx, &avy, &aszz, &asxx, &asxz, &asyy, &asxy, &asyz,
                  &m_vz_z, &m_vz_x, &m_vz_y, &m_vx_z, &m_vx_x, &m_vx_y, &m_vy_z, &m_vy_x, &m_vy_y,
                  &m_szz_z, &m_sxx_x, &m_syy_y, &m_sxz_z, &m_sxz_x, &m_sxy_x, &m_sxy_y, &m_syz_y, &m_syz_z,
                  &gL, &gM, &gR};
    for (Buf *b : all) *b = Buf(N, slack);
    // [z][x][y] -> z-fastest, as libCUFD.cu:72-80.
    for (int z = 0; z < nz; ++z)
      for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
          size_t src = ((size_t)z * nx + x) * ny + y, dst = (size_t)y * nx * nz + (size_t)x * nz + z;
          L.v[dst] = lam[src]; M.v[dst] = mu[src]; R.v[dst] = rho[src];
        }
    // Model.cu:65,76
    std::fill(Byc.v.begin(), Byc.v.begin() + N, 1.0f / 1000.0f);
    dim3 mt(32, 32, 1), mb((nx + 31) / 32, (ny + 31) / 32, nz);
    float *pR = R.p(), *pB = Byc.p();
    int nz_ = nz, nx_ = nx, ny_ = ny;
    launch(mb, mt, [&] { aveBycInit(pR, pB, nz_, nx_, ny_); });
    // Cpml.cu:42-52 (VpAve is overwritten inside cpmlInit)
    auto prof = [&](int n, float h, std::vector<float> *v6[6]) {
      for (int k = 0; k < 6; ++k) v6[k]->assign(n, 0.0f);
      cpmlInit(v6[0]->data(), v6[1]->data(), v6[2]->data(), v6[3]->data(), v6[4]->data(),
               v6[5]->data(), n, np, h, f0, dt, 3000.0f);
    };
    std::vector<float> *pz6[6] = {&Kz, &az, &bz, &Kzh, &azh, &bzh};
    std::vector<float> *px6[6] = {&Kx, &ax, &bx, &Kxh, &axh, &bxh};
    std::vector<float> *py6[6] = {&Ky, &ay, &by, &Kyh, &ayh, &byh};
    prof(nz, dz, pz6);
    prof(nx, dx, px6);
    prof(ny, dy, py6);
    gauss.assign(729, 0.0f);
    float *pg = gauss.data();
    launch(dim3(1, 1, 9), dim3(32, 32, 1), [&] { src_rec_gauss_amp(pg, 9, 9, 9); });
    threads = dim3(32, 1, 32);
    blocks = dim3((nx + 31) / 32, ny, (nz + 31) / 32);
    nzB = nz - 2 * np + 4; nxB = nx - 2 * np + 4; nyB = ny - 2 * np + 4;
    lenB = 2 * (5 * (nzB * nxB) + 5 * (nxB * nyB) + 5 * (nyB * nzB));
  }

  void zero_fwd() {
    Buf *all[] = {&vz, &vx, &vy, &szz, &sxx, &sxz, &syy, &sxy, &syz};
    for (Buf *b : all) b->zero();
  }
  void zero_adj() {
    Buf *all[] = {&avz, &avx, &avy, &aszz, &asxx, &asxz, &asyy, &asxy, &asyz};
    for (Buf *b : all) b->zero();
  }
  void zero_mem() {
    Buf *all[] = {&m_vz_z, &m_vz_x, &m_vz_y, &m_vx_z, &m_vx_x, &m_vx_y, &m_vy_z, &m_vy_x, &m_vy_y,
                  &m_szz_z, &m_sxx_x, &m_syy_y, &m_sxz_z, &m_sxz_x, &m_sxy_x, &m_sxy_y, &m_syz_y, &m_syz_z};
    for (Buf *b : all) b->zero();
  }

  void k_stress(bool isFor) {
    launch(blocks, threads, [&] {
      stress(vz.p(), vx.p(), vy.p(), szz.p(), sxx.p(), sxz.p(), syy.p(), sxy.p(), syz.p(),
             m_vz_z.p(), m_vz_x.p(), m_vz_y.p(), m_vx_z.p(), m_vx_x.p(), m_vx_y.p(), m_vy_z.p(),
             m_vy_x.p(), m_vy_y.p(), L.p(), M.p(), R.p(), Kz.data(), az.data(), bz.data(),
             Kzh.data(), azh.data(), bzh.data(), Kx.data(), ax.data(), bx.data(), Kxh.data(),
             axh.data(), bxh.data(), Ky.data(), ay.data(), by.data(), Kyh.data(), ayh.data(),
             byh.data(), nz, nx, ny, dt, dz, dx, dy, np, isFor, aszz.p(), asxx.p(), asxz.p(),
             asyy.p(), asxy.p(), asyz.p(), gL.p(), gM.p());
    });
  }
  void k_velocity(bool isFor) {
    launch(blocks, threads, [&] {
      velocity(vz.p(), vx.p(), vy.p(), szz.p(), sxx.p(), sxz.p(), syy.p(), sxy.p(), syz.p(),
               m_szz_z.p(), m_sxz_x.p(), m_sxz_z.p(), m_sxx_x.p(), m_sxy_x.p(), m_sxy_y.p(),
               m_syy_y.p(), m_syz_y.p(), m_syz_z.p(), L.p(), M.p(), Byc.p(), Kz.data(),
               az.data(), bz.data(), Kzh.data(), azh.data(), bzh.data(), Kx.data(), ax.data(),
               bx.data(), Kxh.data(), axh.data(), bxh.data(), Ky.data(), ay.data(), by.data(),
               Kyh.data(), ayh.data(), byh.data(), nz, nx, ny, dt, dz, dx, dy, np, isFor,
               avz.p(), avx.p(), avy.p(), gR.p());
    });
  }
  void k_velocity_adj() {
    launch(blocks, threads, [&] {
      velocity_adj(avz.p(), avx.p(), avy.p(), aszz.p(), asxx.p(), asxz.p(), asyy.p(), asxy.p(),
                   asyz.p(), m_szz_z.p(), m_sxz_x.p(), m_sxz_z.p(), m_sxx_x.p(), m_sxy_x.p(),
                   m_sxy_y.p(), m_syy_y.p(), m_syz_y.p(), m_syz_z.p(), m_vz_z.p(), m_vz_x.p(),
                   m_vz_y.p(), m_vx_z.p(), m_vx_x.p(), m_vx_y.p(), m_vy_z.p(), m_vy_x.p(),
                   m_vy_y.p(), L.p(), M.p(), R.p(), Byc.p(), Kzh.data(), azh.data(), bzh.data(),
                   Kxh.data(), axh.data(), bxh.data(), Kyh.data(), ayh.data(), byh.data(),
                   Kz.data(), az.data(), bz.data(), Kx.data(), ax.data(), bx.data(), Ky.data(),
                   ay.data(), by.data(), nz, nx, ny, dt, dz, dx, dy, np);
    });
  }
  void k_stress_adj() {
    launch(blocks, threads, [&] {
      stress_adj(avz.p(), avx.p(), avy.p(), aszz.p(), asxx.p(), asxz.p(), asyy.p(), asxy.p(),
                 asyz.p(), m_szz_z.p(), m_sxz_x.p(), m_sxz_z.p(), m_sxx_x.p(), m_sxy_x.p(),
                 m_sxy_y.p(), m_syy_y.p(), m_syz_y.p(), m_syz_z.p(), m_vz_z.p(), m_vz_x.p(),
                 m_vz_y.p(), m_vx_z.p(), m_vx_x.p(), m_vx_y.p(), m_vy_z.p(), m_vy_x.p(),
                 m_vy_y.p(), L.p(), M.p(), R.p(), Byc.p(), Kzh.data(), azh.data(), bzh.data(),
                 Kxh.data(), axh.data(), bxh.data(), Kyh.data(), ayh.data(), byh.data(),
                 Kz.data(), az.data(), bz.data(), Kx.data(), ax.data(), bx.data(), Ky.data(),
                 ay.data(), by.data(), nz, nx, ny, dt, dz, dx, dy, np);
    });
  }
  void k_source(float amp, bool isFor, int zs, int xs, int ys) {
    float *pg = gauss.data();
    launch(dim3(1, 1, 9), dim3(32, 32, 1), [&] {
      add_source(szz.p(), sxx.p(), syy.p(), amp, nz, nx, ny, isFor, zs, xs, ys, dt, pg);
    });
  }
  // 9 fields in the order of Bnd::field_from_bnd (Boundary.cu:59-96).
  Buf *shell_field(int f) {
    Buf *F[9] = {&szz, &sxz, &sxx, &syy, &sxy, &syz, &vz, &vx, &vy};
    return F[f];
  }
  void k_from_bnd(std::vector<float> *bnd, int it) {
    for (int f = 0; f < 9; ++f) {
      float *fld = shell_field(f)->p(), *b = bnd[f].data();
      launch(dim3((lenB + 31) / 32), dim3(32), [&] {
        from_bnd(fld, b, nz, nx, ny, nzB, nxB, nyB, lenB, 5, it, np, nt);
      });
    }
  }
  void k_to_bnd(std::vector<float> *bnd, int it, bool if_stress) {
    int f0_ = if_stress ? 0 : 6, f1 = if_stress ? 6 : 9;
    for (int f = f0_; f < f1; ++f) {
      float *fld = shell_field(f)->p(), *b = bnd[f].data();
      launch(dim3((lenB + 31) / 32), dim3(32), [&] {
        to_bnd(fld, b, nz, nx, ny, nzB, nxB, nyB, lenB, 5, it, np, nt);
      });
    }
  }
};

void tapered_stf(const Ref &r, const float *stf, std::vector<float> &out) {
  out.assign(stf, stf + r.nt);
  float *p = out.data();
  int nt = r.nt;
  float dt = r.dt;
  launch(dim3((nt + 31) / 32), dim3(32), [&] { cuda_window(nt, 1, dt, 0.001f, p); });
}

// Forward time loop of one shot; traces x/y/z as [nrec][nt] each.
void forward_shot(Ref &r, const RefShot &sh, const float *stf, float *tx, float *ty, float *tz,
                  std::vector<float> *bnd, std::vector<float> &src_t) {
  r.zero_fwd();
  r.zero_mem();
  tapered_stf(r, stf, src_t);
  const int nr = sh.nrec, nt = r.nt;
  std::vector<int> zr(nr), xr(nr), yr(nr);
  for (int k = 0; k < nr; ++k) { zr[k] = sh.z_rec[k]; xr[k] = sh.x_rec[k]; yr[k] = sh.y_rec[k]; }
  std::fill(tx, tx + (size_t)nr * nt, 0.0f);
  std::fill(ty, ty + (size_t)nr * nt, 0.0f);
  std::fill(tz, tz + (size_t)nr * nt, 0.0f);
  int nz = r.nz, nx = r.nx;
  for (int it = 0; it <= nt - 2; ++it) {
    if (bnd) r.k_from_bnd(bnd, it);
    r.k_stress(true);
    r.k_source(src_t[it], true, sh.z_src, sh.x_src, sh.y_src);
    r.k_velocity(true);
    int itp = it + 1;
    launch(dim3((nr + 31) / 32), dim3(32), [&] {
      recording(r.vz.p(), r.vx.p(), r.vy.p(), nz, nx, tx, ty, tz, 0, itp, nt, nr, zr.data(),
                xr.data(), yr.data());
    });
  }
}

}  // namespace

extern "C" {

int ref_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void ref_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

void ref_cpml(int n, int npml, float dh, float f0, float dt, float *out6) {
  cpmlInit(out6, out6 + n, out6 + 2 * n, out6 + 3 * n, out6 + 4 * n, out6 + 5 * n, n, npml, dh,
           f0, dt, 3000.0f);
}

void ref_taper_stf(const float *stf, int nt, float dt, float *out) {
  std::copy(stf, stf + nt, out);
  launch(dim3((nt + 31) / 32), dim3(32), [&] { cuda_window(nt, 1, dt, 0.001f, out); });
}

// traces: concatenation over shots of [3][nrec][nt] (x, y, z).
int ref_forward(const RefGrid *g, const float *lam, const float *mu, const float *rho, int nshot,
                const RefShot *shots, const float *stf, float *traces) {
  Ref r(*g, lam, mu, rho);
  size_t off = 0;
  std::vector<float> src_t;
  for (int k = 0; k < nshot; ++k) {
    size_t plane = (size_t)shots[k].nrec * g->nt;
    forward_shot(r, shots[k], stf + (size_t)k * g->nt, traces + off, traces + off + plane,
                 traces + off + 2 * plane, nullptr, src_t);
    off += 3 * plane;
  }
  return 0;
}

// Reference gradient (calc_id 1): misfit and lambda/mu/rho gradients in
// [z][x][y].  res_out (optional): adjoint source, traces layout.
int ref_gradient(const RefGrid *g, const float *lam, const float *mu, const float *rho, int nshot,
                 const RefShot *shots, const float *stf, const float *obs, int if_win,
                 double *misfit, float *glam, float *gmu, float *grho, float *res_out) {
  Ref r(*g, lam, mu, rho);
  const int nt = r.nt, nz = r.nz, nx = r.nx, ny = r.ny;
  std::vector<float> bnd[9];
  for (int f = 0; f < 9; ++f) bnd[f].assign((size_t)r.lenB * nt, 0.0f);
  double J = 0.0;
  size_t off = 0;
  std::vector<float> src_t;
  for (int k = 0; k < nshot; ++k) {
    const RefShot &sh = shots[k];
    const int nr = sh.nrec;
    size_t plane = (size_t)nr * nt;
    std::vector<float> syn(3 * plane), ob(obs + off, obs + off + 3 * plane), res(3 * plane, 0.0f);
    forward_shot(r, sh, stf + (size_t)k * nt, syn.data(), syn.data() + plane,
                 syn.data() + 2 * plane, bnd, src_t);
    std::vector<float> win0(nr, 0.0f), win1(nr, 0.0f), wts(nr, 1.0f);
    for (int q = 0; q < nr; ++q) {
      if (sh.win_start) win0[q] = sh.win_start[q];
      if (sh.win_end) win1[q] = sh.win_end[q];
      if (sh.weights) wts[q] = sh.weights[q];
    }
    float dt = r.dt, sw = sh.src_weight;
    dim3 tt(32, 32), bt((nt + 31) / 32, (nr + 31) / 32);
    auto window = [&](float *d) {
      if (if_win)
        launch(bt, tt, [&] { cuda_window(nt, nr, dt, win0.data(), win1.data(), wts.data(), sw, 0.005f, d); });
      else
        launch(bt, tt, [&] { cuda_window(nt, nr, dt, 0.005f, d); });
    };
    for (int c = 0; c < 3; ++c) {
      window(ob.data() + c * plane);
      window(syn.data() + c * plane);
    }
    for (int c = 0; c < 3; ++c) {
      float *o = res.data() + c * plane, *i1 = ob.data() + c * plane, *i2 = syn.data() + c * plane;
      launch(bt, tt, [&] { gpuMinus(o, i1, i2, nt, nr); });
      for (size_t q = 0; q < plane; ++q) J += (double)o[q] * (double)o[q];
    }
    for (int c = 0; c < 3; ++c) window(res.data() + c * plane);
    if (res_out) std::copy(res.begin(), res.end(), res_out + off);

    std::vector<int> zr(nr), xr(nr), yr(nr);
    for (int q = 0; q < nr; ++q) { zr[q] = sh.z_rec[q]; xr[q] = sh.x_rec[q]; yr[q] = sh.y_rec[q]; }
    float *rx = res.data(), *ry = res.data() + plane, *rz = res.data() + 2 * plane;
    auto inject = [&](int it) {
      launch(dim3((nr + 31) / 32), dim3(32), [&] {
        res_injection(r.avx.p(), r.avy.p(), r.avz.p(), nz, nx, rx, ry, rz, it, dt, nt, nr,
                      zr.data(), xr.data(), yr.data());
      });
    };
    r.zero_adj();
    r.zero_mem();
    r.k_velocity_adj();
    inject(nt - 1);
    r.k_stress_adj();
    for (int it = nt - 2; it >= 0; --it) {
      r.k_velocity(false);
      r.k_to_bnd(bnd, it, false);
      r.k_source(src_t[it], false, sh.z_src, sh.x_src, sh.y_src);
      r.k_stress(false);
      r.k_to_bnd(bnd, it, true);
      r.k_velocity_adj();
      inject(it);
      r.k_stress_adj();
    }
    off += 3 * plane;
  }
  (void)ny;
  // z-fastest -> [z][x][y], as libCUFD.cu:644-652.
  for (int z = 0; z < nz; ++z)
    for (int x = 0; x < nx; ++x)
      for (int y = 0; y < ny; ++y) {
        size_t dst = ((size_t)z * nx + x) * ny + y, src = (size_t)y * nx * nz + (size_t)x * nz + z;
        glam[dst] = r.gL.v[src]; gmu[dst] = r.gM.v[src]; grho[dst] = r.gR.v[src];
      }
  *misfit = J;
  return 0;
}

}  // extern "C"
