// Misfit and adjoint source of one shot without any device allocation.
//
// Some callers cannot call cudaMalloc: a host application whose device
// memory is reserved up front by another allocator (a framework's caching
// pool or a serving process that budgets every byte), where a fresh
// cudaMalloc fails or has to wait for memory to be released, and code on a
// latency-critical path where the device-wide synchronisation of cudaMalloc
// and cudaFree is not acceptable.  efwi_misfit_noalloc serves them: it
// needs no handle and allocates nothing; the caller passes every input and
// output, and the per-CTA partial sums live in the file-scope array below.
//
// The array has EFWI_NOALLOC_MAX_PARTIALS doubles (512 KiB); every GPU that
// loads the library holds it until the process exits.  One CTA handles a
// 32 (t) x 32 (r) tile of one component, so a call needs
// 3 * ceil(nt/32) * ceil(nrec/32) partials; larger requests are rejected
// with EFWI_ERR_TOO_LARGE.  The array is shared by all calls on a device and
// keeps the last call's contents; every slot a call reads is written by the
// same call first, so nothing needs clearing.  Calls that overlap on the GPU
// (on different streams, or from different threads) race on the array.
//
// Set-up: the first call on a device looks up the device address of the
// array with cudaGetSymbolAddress while that device is current and keeps it;
// that first call should come before any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/efwi.h"
#include "efwi_common.cuh"
#include "efwi_kernels.h"
#include "efwi_window.cuh"

namespace efwi {
namespace {

static __device__ __align__(256) double g_misfit_scratch[EFWI_NOALLOC_MAX_PARTIALS];

constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

// Same windowed residual as k_misfit, with observed data, synthetics and
// the adjoint source all in the [3][nrec][nt] traces layout.
__global__ void __launch_bounds__(256)
k_misfit_direct(MisfitArgs m, const float *obs, const float *syn, float *res, double *partial) {
  __shared__ double red[8];
  const int t = blockIdx.x * 32 + threadIdx.x;
  const int c = blockIdx.z;
  const int nt = m.nt, nr = m.nrec;
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int r = blockIdx.y * 32 + threadIdx.y + 8 * k;
    if (t < nt && r < nr) {
      const long long i = ((long long)c * nr + r) * nt + t;
      const float mult = window_mult(m, t, r);
      const float ow = __fmul_rn(obs[i], mult), sw = __fmul_rn(syn[i], mult);
      const float rr = (t == 0) ? 0.0f : ow - sw;
      acc += (double)rr * (double)rr;
      res[i] = rr * mult;
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (threadIdx.x == 0) red[threadIdx.y] = acc;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += red[w];
    partial[((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
  }
}

// Device address of the scratch array on the current device (looked up
// once per device).
cudaError_t scratch_address(double **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    double *p = nullptr;
    e = cudaGetSymbolAddress((void **)&p, g_misfit_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

}  // namespace
}  // namespace efwi

using namespace efwi;

extern "C" int efwi_misfit_noalloc(int nrec, int nt, float dt, int if_win,
                                   const float *win_start, const float *win_end,
                                   const float *weights, float src_weight, const float *obs,
                                   const float *syn, float *res, double *misfit, void *stream) {
  if (nrec < 0 || nt < 1 || !(dt > 0.0f) || !obs || !syn || !res || !misfit) return EFWI_ERR_ARG;
  if (if_win && (!win_start || !win_end || !weights)) return EFWI_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 grid((nt + 31) / 32, (nrec + 31) / 32, 3);
  const long long nb = (long long)grid.x * grid.y * grid.z;
  if (nb > EFWI_NOALLOC_MAX_PARTIALS) return EFWI_ERR_TOO_LARGE;
  double *scratch = nullptr;
  if (scratch_address(&scratch) != cudaSuccess) return EFWI_ERR_CUDA;
  if (nrec == 0) {
    if (cudaMemsetAsync(misfit, 0, sizeof(double), st) != cudaSuccess) return EFWI_ERR_CUDA;
    return EFWI_OK;
  }
  MisfitArgs m{};
  m.nt = nt;
  m.nrec = nrec;
  m.dt = dt;
  m.if_win = if_win ? 1 : 0;
  m.win_start = win_start;
  m.win_end = win_end;
  m.weights = weights;
  m.src_weight = src_weight;
  k_misfit_direct<<<grid, dim3(32, 8), 0, st>>>(m, obs, syn, res, scratch);
  k_reduce_sum<<<1, 256, 0, st>>>(scratch, (int)nb, misfit);
  return cudaGetLastError() == cudaSuccess ? EFWI_OK : EFWI_ERR_CUDA;
}
