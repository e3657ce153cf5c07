// Receiver gather, adjoint-source injection and boundary-shell save/restore
// fused into the stencil kernels' epilogues (the reference runs them as
// separate kernels every step: recording and res_injection,
// utilities.cu:481-507; from_bnd / to_bnd, utilities.cu:323-420 with
// Boundary.cu:59-138).
//
// Shell: the points of the reference's 5-cell boundary shell inside
// [2, n-3]^3 are stored per step as [9][npts] in (z, x, y) order.  A row
// (z, x) of the grid holds either no shell point, a full run of points
// y in [ya0, yb1], or two runs [ya0, ya1] and [yb0, yb1]; rows[z * nx + x]
// gives the index of the row's first point (bit 30 set for a split row) or
// -1.  So a thread finds its cell's shell index in O(1) from one load that
// is uniform over its warp.
//
// Receivers: for the planes that hold receiver cells of a launch's shots,
// plane[s * nz + z] names a map [nx][py] of unique receiver cell numbers
// (RecArgs::ucell order, -1 elsewhere); other planes read -1.
#pragma once
#include "efwi_common.cuh"
#include "efwi_kernels.h"

namespace efwi {

constexpr int SHELL_SPLIT = 1 << 30;

struct ShellMap {
  const int *rows;  // [nz][nx] (nullptr: no shell work)
  float *store;     // [9][npts] of the current step
  int npts;
  int ya0, ya1, yb0, yb1;
};

struct RecMap {
  const int *plane;  // [nshot][nz] (nullptr: no receiver work)
  const int *map;    // [nmaps][nx][py]
  int nxpy;
};

// Shell point index of cell (z, x, y) from its row entry, or -1.
__device__ __forceinline__ int shell_index(const ShellMap &s, int row, int y) {
  if (row < 0) return -1;
  const int base = row & ~SHELL_SPLIT;
  if (!(row & SHELL_SPLIT)) return (y >= s.ya0 && y <= s.yb1) ? base + y - s.ya0 : -1;
  if (y >= s.ya0 && y <= s.ya1) return base + y - s.ya0;
  if (y >= s.yb0 && y <= s.yb1) return base + (s.ya1 - s.ya0 + 1) + y - s.yb0;
  return -1;
}

// Unique receiver cell at (shot, z, x, y), or -1.
__device__ __forceinline__ int receiver_at(const RecMap &m, int nz, int py, int shot, int z, int x,
                                           int y) {
  if (!m.plane) return -1;
  const int mp = m.plane[shot * nz + z];
  if (mp < 0) return -1;
  return m.map[(long long)mp * m.nxpy + x * py + y];
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

namespace efwi {

// Receiver work of one launch: the maps, the grouping, the time-major trace
// array (recorded into by the forward velocity kernel, read as the
// adjoint source by the reverse velocity kernel) and the sample index.
struct RecFuse {
  RecMap m;
  RecArgs a;
  float *tm;
  int it;
};

}  // namespace efwi
