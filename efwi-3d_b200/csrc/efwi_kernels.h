// Kernel declarations shared by the kernel translation units and the C-ABI.
#pragma once
#include "efwi_common.cuh"
#include "efwi_tma.cuh"

namespace efwi {

// Point source of the shots of one launch.  cell[s]: linear index of the
// source of shot s (or -1); stf: tapered source-time functions [nshot][nt];
// `it`: time step.
struct SrcArgs {
  const long long *cell;
  const float *stf;
  int nt;
  int it;
  // when set, the step index is read from this device word instead of `it`
  // (a launch replayed from a CUDA graph step after step)
  const int *it_dev;
};

// Receivers of the shots of one launch, grouped by cell so that several
// receivers on one cell are handled by one thread in receiver order.
//   ucell[u]          linear cell index of unique receiver cell u
//   ushot[u]          shot (within the launch) of cell u
//   uptr[u]..uptr[u+1] range in rec[] of the receivers on cell u
//   rec[k]            trace row of the receiver: traces of shot s start at
//                     trace_off[s]; a row is (t*3 + c)*nrec_s + r.
struct RecArgs {
  const long long *ucell;
  const int *ushot;
  const int *uptr;
  const int *rec;       // receiver number r within its shot
  const long long *trace_off;
  const int *nrec;      // per shot
  int ncell;
  // Cell lookup for kernels that gather or inject in their own epilogue:
  // plane[s * nz + z] names a map [nx][py] of unique receiver cells u in
  // plane z of shot s (-1 elsewhere), or is -1 when the plane holds none;
  // plane == nullptr: no lookup (separate k_record / k_inject launches).
  const int *plane;
  const int *map;
  int nxpy;
};

// Boundary-shell save/restore inside the stencil kernels (efwi_fuse.cuh):
// rows[z * nx + x] is the index of the row's first shell point (bit 30 set
// when the row holds two runs, [ya0, ya1] and [yb0, yb1], instead of one
// run [ya0, yb1]) or -1; store is the [9][npts] shell of the current step
// in the reference's field order (Boundary.cu:59-96); rows == nullptr: no
// shell work.
struct ShellMap {
  const int *rows;
  float *store;
  int npts;
  int ya0, ya1, yb0, yb1;
};

// Receiver work fused into a launch: the receivers, the time-major trace
// array (recorded into by the forward velocity kernel at sample `it`, or
// read as the adjoint source by the reverse velocity kernel) and `it`;
// a.plane == nullptr: none.
struct RecFuse {
  RecArgs a;
  float *tm;
  int it;
};

// One domain of a multi-domain launch (a shot on its own window grid): its
// geometry, state, model, source and place in the concatenated tile list
// (tiles_y * tiles_x * nzc tiles from tile0).
struct Domain {
  Geo g;
  Fields f;
  Psi ps;
  const float *lam, *mu, *buoy;
  long long src_cell;
  const float *stf;  // tapered source-time function [nt]
  int nt;
  int tiles_y, tiles_x, nzc, tile0;
  long long trace_off;  // the shot's time-major traces [nt][3][nrec]
  int nrec;
};

// Persistent launches over several domains (L1-served stencils):
// stress + source, then velocity, for time step `it`; `blocks` CTAs
// (multi_blocks(bx): the SM count times the resident CTAs per SM).
int multi_blocks(int bx);
void launch_fwd_multi(int bx, int blocks, cudaStream_t st, const Domain *dom, int ndom, int ntiles,
                      int zchunk, int it);
// Receivers of windowed shots at sample `it`, or at 1 + *it_dev when it_dev
// is set.
__global__ void k_record_multi(const Domain *dom, const int *rec_dom, const int *rec_cell,
                               const int *rec_r, int nrec, float *traces_tm, int it,
                               const int *it_dev = nullptr);

// Host launchers of the stencil kernels (bx: x rows per CTA, 4 or 8; the
// CTA is 32 x bx threads).
void launch_stress_fwd(int bx, dim3 grid, cudaStream_t st, const Geo &g, const Fields &f,
                       const Psi &ps, const float *lam, const float *mu, int zchunk, int nzc,
                       const SrcArgs &src);
void launch_velocity_fwd(int bx, dim3 grid, cudaStream_t st, const Geo &g, const Fields &f,
                         const Psi &ps, const float *buoy, int zchunk, int nzc);
void launch_rev_velocity(int bx, dim3 grid, cudaStream_t st, const Geo &g, const Fields &f,
                         const Fields &a, const Psi &ps, const float *lam, const float *mu,
                         const float *buoy, float *grho, int zchunk, int nzc, int do_rev,
                         int do_adj);
void launch_rev_stress(int bx, dim3 grid, cudaStream_t st, const Geo &g, const Fields &f,
                       const Fields &a, const Psi &ps, const float *lam, const float *mu,
                       const float *buoy, float *glam, float *gmu, int zchunk, int nzc,
                       int do_rev, int do_adj, const SrcArgs &src);

// TMA-staged variants (efwi_fwd_tma.cu); `status` receives
// EFWI_STATUS_TIMEOUT if a pipeline wait ran out of time.
// cfg selects (tile, ring depth, min CTAs/SM); fwd_tma_tile(cfg) is the
// tile's x extent.
int fwd_tma_tile(int cfg);
// K_S maps: halo vz vx vy | point szz sxx syy sxz sxy syz | model lambda mu.
// With shell.rows set (one shot per launch), the state at the start of the
// step is stored into shell.store at the shell points.
void launch_stress_fwd_tma(int cfg, dim3 grid, cudaStream_t st, const Maps<11> &maps,
                           const Geo &g, const Fields &f, const Psi &ps, int zchunk, int nzc,
                           const SrcArgs &src, const ShellMap &shell, int *status);
// K_V maps: halo sxz syz sxx sxy syy | point vz vx vy | model buoyancy.
// With rec.a.plane set, the new velocities of receiver cells are recorded
// at sample rec.it.
void launch_velocity_fwd_tma(int cfg, dim3 grid, cudaStream_t st, const Maps<9> &maps,
                             const Geo &g, const Fields &f, const Psi &ps, int zchunk, int nzc,
                             const RecFuse &rec, int *status);

// Reverse sweep with TMA-staged planes (efwi_rev_tma.cu); rev_tma_tile(cfg)
// is the tile's x extent (4 or 8; the tile is 32 x that).
int rev_tma_tile(int cfg);
// K1 maps: halo sxz syz sxx sxy syy asxz asyz asxx asxy asyy aszz |
//          point vz vx vy avz avx avy | model buoyancy lambda mu grho.
// With shell.rows set (do_rev), the reverse velocities are restored at the
// shell points from shell.store; with inj.a.plane set (do_adj), the adjoint
// source inj.tm at sample inj.it is added to the adjoint velocities.
void launch_rev_velocity_tma(int cfg, dim3 grid, cudaStream_t st, const Maps<21> &maps,
                             const Geo &g, const Fields &f, const Fields &a, const Psi &ps,
                             float *grho, int zchunk, int nzc, int do_rev, int do_adj,
                             const ShellMap &shell, const RecFuse &inj, int *status);
// K1 as two launches (cfg 6, 7): reverse half maps halo sxz syz sxx sxy syy |
// point vz vx vy avz avx avy | model buoyancy rho-image; adjoint half maps
// halo asxz asyz asxx asxy asyy aszz | point avz avx avy | model buoyancy
// lambda mu.
void launch_rev_velocity_split_tma(int cfg, dim3 grid, cudaStream_t st, const Maps<13> &rev_maps,
                                   const Maps<12> &adj_maps, const Geo &g, const Fields &f,
                                   const Fields &a, const Psi &ps, float *grho, int zchunk,
                                   int nzc, int do_rev, int do_adj, const ShellMap &shell,
                                   const RecFuse &inj, int *status);
// K2 maps: halo vz vx vy avz avx avy | point szz sxx syy sxz sxy syz aszz
//          asxx asyy asxz asxy asyz | model lambda mu buoyancy glam gmu.
// With shell.rows set (do_rev), the reverse stresses are restored at the
// shell points from shell.store.
void launch_rev_stress_tma(int cfg, dim3 grid, cudaStream_t st, const Maps<23> &maps,
                           const Geo &g, const Fields &f, const Fields &a, const Psi &ps,
                           float *glam, float *gmu, int zchunk, int nzc, int do_rev, int do_adj,
                           const SrcArgs &src, const ShellMap &shell, int *status);

__global__ void k_prep_buoyancy(const float *rho, float *buoy, int nz, int nx, int ny, int py);
__global__ void k_window_slice(const float *src, float *dst, int nz, int nx, int pyg, int x0,
                               int y0, int nxw, int nyw, int pyw);
__global__ void k_pitch_copy(const float *src, float *dst, int nz, int nx, int ny, int py,
                             int to_pitched);
__global__ void k_record(Fields f, long long N, RecArgs rec, float *traces_tm, int it);
__global__ void k_inject(Fields a, long long N, RecArgs rec, const float *res_tm, int it,
                         float scale);
__global__ void k_shell_save(Fields f, const int *pts, int npts, float *dst);
__global__ void k_shell_restore(Fields f, const int *pts, int npts, const float *src, int stress);

struct MisfitArgs {
  int nt, nrec;
  float dt;
  int if_win;
  const float *win_start, *win_end, *weights;  // [nrec] (if_win)
  float src_weight;
  float *syn_w, *obs_w;  // optional [nt][3][nrec]: windowed synthetics and observed data
};
// obs [3][nrec][nt], syn_tm [nt][3][nrec] -> res_tm [nt][3][nrec];
// per-CTA partial sums of squares (double) in partial[].
__global__ void k_misfit(MisfitArgs m, const float *obs, const float *syn_tm, float *res_tm,
                         double *partial);
__global__ void k_reduce_sum(const double *partial, int n, double *out);
// [nt][3][nrec] -> [3][nrec][nt]
__global__ void k_traces_to_cr_t(const float *tm, float *out, int nt, int nrec);
// [3][nrec][nt] -> [nt][3][nrec]
__global__ void k_traces_to_tm(const float *in, float *tm, int nt, int nrec);

}  // namespace efwi
