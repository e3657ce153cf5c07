// Receiver gather, adjoint-source injection and boundary-shell save/restore
// in the stencil kernels' epilogues (the reference runs them as separate
// kernels every step: recording and res_injection, utilities.cu:481-507;
// from_bnd / to_bnd, utilities.cu:323-420 with Boundary.cu:59-138).
//
// Shell: the points of the reference's 5-cell boundary shell inside
// [2, n-3]^3 are stored per step as [9][npts] in (z, x, y) order.  A row
// (z, x) of the grid holds no shell point, one run of points y in
// [ya0, yb1], or two runs [ya0, ya1] and [yb0, yb1] (ShellMap), so a thread
// finds its cell's shell index in O(1) from one row entry that is uniform
// over its warp.  Receivers: a per-plane map of unique receiver cells
// (RecArgs::plane, RecArgs::map).
#pragma once
#include "efwi_common.cuh"
#include "efwi_kernels.h"

namespace efwi {

constexpr int SHELL_SPLIT = 1 << 30;

// Shell point index of a cell at y whose row entry is `row`, or -1.
__host__ __device__ __forceinline__ int shell_index(const ShellMap &s, int row, int y) {
  if (row < 0) return -1;
  const int base = row & ~SHELL_SPLIT;
  if (!(row & SHELL_SPLIT)) return (y >= s.ya0 && y <= s.yb1) ? base + y - s.ya0 : -1;
  if (y >= s.ya0 && y <= s.ya1) return base + y - s.ya0;
  if (y >= s.yb0 && y <= s.yb1) return base + (s.ya1 - s.ya0 + 1) + y - s.yb0;
  return -1;
}

// Unique receiver cell at (shot, z, x, y), or -1.
__device__ __forceinline__ int receiver_at(const RecArgs &r, int nz, int py, int shot, int z,
                                           int x, int y) {
  const int mp = r.plane[shot * nz + z];
  if (mp < 0) return -1;
  return r.map[(long long)mp * r.nxpy + x * py + y];
}

// recording (utilities.cu:481-495) of unique receiver cell u at sample it.
__device__ __forceinline__ void record_cell(const RecArgs &rec, float *traces_tm, int it, int u,
                                            float vz, float vx, float vy) {
  const int s = rec.ushot[u];
  const int nr = rec.nrec[s];
  float *t = traces_tm + rec.trace_off[s] + (long long)it * 3 * nr;
  for (int k = rec.uptr[u]; k < rec.uptr[u + 1]; ++k) {
    const int r = rec.rec[k];
    t[r] = vx;
    t[nr + r] = vy;
    t[2 * nr + r] = vz;
  }
}

// res_injection (utilities.cu:497-507) at unique receiver cell u: the
// receivers on the cell are added one after the other in receiver order.
__device__ __forceinline__ void inject_cell(const RecArgs &rec, const float *res_tm, int it, int u,
                                            float &vz, float &vx, float &vy) {
  const int s = rec.ushot[u];
  const int nr = rec.nrec[s];
  const float *t = res_tm + rec.trace_off[s] + (long long)it * 3 * nr;
  for (int k = rec.uptr[u]; k < rec.uptr[u + 1]; ++k) {
    const int r = rec.rec[k];
    vx += t[r];
    vy += t[nr + r];
    vz += t[2 * nr + r];
  }
}

}  // namespace efwi
