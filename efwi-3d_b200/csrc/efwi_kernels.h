// Kernel declarations shared by the kernel translation units and the C-ABI.
#pragma once
#include "efwi_common.cuh"

namespace efwi {

// Point source of the shots of one launch.  cell[s]: linear index of the
// source of shot s (or -1); stf: tapered source-time functions [nshot][nt];
// `it`: time step.
struct SrcArgs {
  const long long *cell;
  const float *stf;
  int nt;
  int it;
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
};

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

__global__ void k_prep_buoyancy(const float *rho, float *buoy, int nz, int nx, int ny);
__global__ void k_record(Fields f, long long N, RecArgs rec, float *traces_tm, int it);
__global__ void k_inject(Fields a, long long N, RecArgs rec, const float *res_tm, int it);
__global__ void k_shell_save(Fields f, const int *pts, int npts, float *dst);
__global__ void k_shell_restore(Fields f, const int *pts, int npts, const float *src, int stress);

struct MisfitArgs {
  int nt, nrec;
  float dt;
  int if_win;
  const float *win_start, *win_end, *weights;  // [nrec] (if_win)
  float src_weight;
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
