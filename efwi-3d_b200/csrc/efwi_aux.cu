// Small kernels around the stencil sweeps: model preparation, receivers,
// adjoint-source injection, boundary-shell save/restore, misfit, trace
// layout conversion.
#include "efwi_common.cuh"
#include "efwi_kernels.h"
#include "efwi_window.cuh"

namespace efwi {

// Buoyancy 1/rho on [2, n-3]^3 and 1/1000 elsewhere (Model.cu:65,76 with
// aveBycInit, utilities.cu:117-128).  The reciprocal is formed in double as
// the reference does.
// rho is in the caller's [nz][nx][ny] layout; buoy has the y pitch py.
__global__ void k_prep_buoyancy(const float *rho, float *buoy, int nz, int nx, int ny, int py) {
  const long long n = (long long)nz * nx * ny;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % ny);
    const long long zx = i / ny;
    const int x = (int)(zx % nx);
    const int z = (int)(zx / nx);
    const bool in = z >= 2 && z <= nz - 3 && x >= 2 && x <= nx - 3 && y >= 2 && y <= ny - 3;
    buoy[zx * py + y] = in ? (float)(1.0 / (double)rho[i]) : (float)(1.0 / 1000.0);
  }
}

// Copies between the caller's [nz][nx][ny] volumes and pitched ones;
// `to_pitched` selects the direction.  The pad columns are zeroed.
__global__ void k_pitch_copy(const float *src, float *dst, int nz, int nx, int ny, int py,
                             int to_pitched) {
  const long long n = (long long)nz * nx * py;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % py);
    const long long zx = i / py;
    if (to_pitched) dst[i] = (y < ny) ? src[zx * ny + y] : 0.0f;
    else if (y < ny) dst[zx * ny + y] = src[i];
  }
}

// recording (utilities.cu:481-495): trace row (it*3 + c)*nrec + r gets
// vx, vy, vz (c = 0, 1, 2) at the receiver cell.
__global__ void k_record(Fields f, long long N, RecArgs rec, float *traces_tm, int it) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= rec.ncell) return;
  const int s = rec.ushot[u];
  const long long i = (long long)s * N + rec.ucell[u];
  const float vx = f.vx[i], vy = f.vy[i], vz = f.vz[i];
  const int nr = rec.nrec[s];
  float *t = traces_tm + rec.trace_off[s] + (long long)it * 3 * nr;
  for (int k = rec.uptr[u]; k < rec.uptr[u + 1]; ++k) {
    const int r = rec.rec[k];
    t[r] = vx;
    t[nr + r] = vy;
    t[2 * nr + r] = vz;
  }
}

// res_injection (utilities.cu:497-507): adjoint velocity += scale * residual
// (scale 1 in the reference algorithm; -2, the derivative of the squared
// residual, in the exact adjoint).  Receivers sharing a cell are added one
// after the other in receiver order (the reference's threads race on such a
// cell).
__global__ void k_inject(Fields a, long long N, RecArgs rec, const float *res_tm, int it,
                         float scale) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= rec.ncell) return;
  const int s = rec.ushot[u];
  const long long i = (long long)s * N + rec.ucell[u];
  const int nr = rec.nrec[s];
  const float *t = res_tm + rec.trace_off[s] + (long long)it * 3 * nr;
  float vx = a.vx[i], vy = a.vy[i], vz = a.vz[i];
  for (int k = rec.uptr[u]; k < rec.uptr[u + 1]; ++k) {
    const int r = rec.rec[k];
    vx += scale * t[r];
    vy += scale * t[nr + r];
    vz += scale * t[2 * nr + r];
  }
  a.vx[i] = vx; a.vy[i] = vy; a.vz[i] = vz;
}

// Shell fields in the reference's order (Boundary.cu:59-96).
__device__ __forceinline__ float *shell_field(const Fields &f, int k) {
  switch (k) {
    case 0: return f.szz;
    case 1: return f.sxz;
    case 2: return f.sxx;
    case 3: return f.syy;
    case 4: return f.sxy;
    case 5: return f.syz;
    case 6: return f.vz;
    case 7: return f.vx;
    default: return f.vy;
  }
}

// dst[9][npts] <- fields at the shell points.
__global__ void k_shell_save(Fields f, const int *pts, int npts, float *dst) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npts) return;
  const int p = pts[k];
#pragma unroll
  for (int q = 0; q < 9; ++q) dst[(long long)q * npts + k] = shell_field(f, q)[p];
}

// Stresses (fields 0-5) or velocities (6-8) <- shell storage.
__global__ void k_shell_restore(Fields f, const int *pts, int npts, const float *src, int stress) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npts) return;
  const int p = pts[k];
  const int q0 = stress ? 0 : 6, q1 = stress ? 6 : 9;
  for (int q = q0; q < q1; ++q) shell_field(f, q)[p] = src[(long long)q * npts + k];
}

// Fused misfit (libCUFD.cu:371-440): window obs and syn, residual with
// sample 0 zeroed (gpuMinus, utilities.cu:130-143), sum of squares, window
// the residual again.  A CTA handles a 32 (t) x 32 (r) tile of one
// component and transposes through shared memory so that both the
// [3][nrec][nt] observed data and the [nt][3][nrec] traces are read
// coalesced.  Partial sums are double and reduced in a fixed order.
__global__ void __launch_bounds__(256)
k_misfit(MisfitArgs m, const float *obs, const float *syn_tm, float *res_tm, double *partial) {
  __shared__ float so[32][33];
  __shared__ float ss[32][33];
  __shared__ double red[8];
  const int t0 = blockIdx.x * 32, r0 = blockIdx.y * 32, c = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int nt = m.nt, nr = m.nrec;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int rl = ty + 8 * k;
    const int r = r0 + rl, t = t0 + tx;
    so[rl][tx] = (r < nr && t < nt) ? obs[((long long)c * nr + r) * nt + t] : 0.0f;
    const int tl = ty + 8 * k;
    const int t2 = t0 + tl, r2 = r0 + tx;
    ss[tl][tx] = (r2 < nr && t2 < nt) ? syn_tm[((long long)t2 * 3 + c) * nr + r2] : 0.0f;
  }
  __syncthreads();
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int tl = ty + 8 * k, rl = tx;
    const int t = t0 + tl, r = r0 + rl;
    if (t < nt && r < nr) {
      const float mult = window_mult(m, t, r);
      // windowed traces rounded on their own, as the reference windows the
      // data in place before subtracting (cuda_window, then gpuMinus)
      const float ow = __fmul_rn(so[rl][tl], mult), sw = __fmul_rn(ss[tl][rl], mult);
      const float rr = (t == 0) ? 0.0f : ow - sw;
      acc += (double)rr * (double)rr;
      const long long o = ((long long)t * 3 + c) * nr + r;
      res_tm[o] = rr * mult;
      if (m.syn_w) m.syn_w[o] = sw;
      if (m.obs_w) m.obs_w[o] = ow;
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (tx == 0) red[ty] = acc;
  __syncthreads();
  if (ty == 0 && tx == 0) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += red[w];
    partial[((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
  }
}

// Single-CTA fixed-order sum.
__global__ void __launch_bounds__(256) k_reduce_sum(const double *partial, int n, double *out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += 256) s += partial[k];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// [nt][3][nrec] -> [3][nrec][nt]; grid (ceil(nt/32), ceil(nrec/32), 3), CTA 32x8.
__global__ void k_traces_to_cr_t(const float *tm, float *out, int nt, int nrec) {
  __shared__ float tile[32][33];
  const int t0 = blockIdx.x * 32, r0 = blockIdx.y * 32, c = blockIdx.z;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int tl = threadIdx.y + 8 * k, t = t0 + tl, r = r0 + threadIdx.x;
    tile[tl][threadIdx.x] = (t < nt && r < nrec) ? tm[((long long)t * 3 + c) * nrec + r] : 0.0f;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int rl = threadIdx.y + 8 * k, r = r0 + rl, t = t0 + threadIdx.x;
    if (t < nt && r < nrec) out[((long long)c * nrec + r) * nt + t] = tile[threadIdx.x][rl];
  }
}

// [3][nrec][nt] -> [nt][3][nrec]
__global__ void k_traces_to_tm(const float *in, float *tm, int nt, int nrec) {
  __shared__ float tile[32][33];
  const int t0 = blockIdx.x * 32, r0 = blockIdx.y * 32, c = blockIdx.z;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int rl = threadIdx.y + 8 * k, r = r0 + rl, t = t0 + threadIdx.x;
    tile[rl][threadIdx.x] = (t < nt && r < nrec) ? in[((long long)c * nrec + r) * nt + t] : 0.0f;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int tl = threadIdx.y + 8 * k, t = t0 + tl, r = r0 + threadIdx.x;
    if (t < nt && r < nrec) tm[((long long)t * 3 + c) * nrec + r] = tile[threadIdx.x][tl];
  }
}

}  // namespace efwi

namespace efwi {

// Copies the window [x0, x0+nxw) x [y0, y0+nyw) (all z) of a pitched global
// volume (nx, pyg) into a pitched window volume (nxw, pyw); pad columns 0.
__global__ void k_window_slice(const float *src, float *dst, int nz, int nx, int pyg, int x0,
                               int y0, int nxw, int nyw, int pyw) {
  const long long n = (long long)nz * nxw * pyw;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % pyw);
    const long long zx = i / pyw;
    const int x = (int)(zx % nxw), z = (int)(zx / nxw);
    dst[i] = y < nyw ? src[((long long)z * nx + x0 + x) * pyg + y0 + y] : 0.0f;
  }
}

}  // namespace efwi
