// 3-D convolutions of the learned gradient preconditioner on BF16 tensor
// cores with FP32 accumulation (no reference counterpart).
//
// Layer: 3x3x3 kernel, stride 1, zero padding 1, 16 input and 16 output
// channels (narrower inputs and outputs are zero-padded to 16 by the
// caller).  Layouts:
//   activations  [D][H][W][16] bf16 (channels last: one voxel = 32 bytes)
//   weights      [27][16 co][16 ci] bf16, tap t = (dz+1)*9 + (dy+1)*3 + (dx+1)
//   bias         [16] f32
// The convolution is an implicit GEMM: per output voxel row of 16
// consecutive x, one warp accumulates sum over taps t and input channels of
// X[v + off_t][ci] W[t][co][ci] with mma.m16n8k16 (bf16 in, f32 accumulate):
// A = 16 voxels x 16 input channels of one tap (ldmatrix from the CTA's
// staged input tile), B = 16 input channels x 8 output channels, two
// n-tiles.  Voxels outside the volume read as zero.
//
//   k_conv3d_fwd     y = act(conv(x, W) + b), stored as bf16 and/or f32.
//                    With W'[t][a][b] = W[26-t][b][a] it also computes the
//                    gradient of the input (the transposed convolution).
//   k_conv3d_wgrad   dW[t][co][ci] = sum_v dy[v][co] x[v + off_t][ci]: one
//                    warp per tap, K = voxels (16 per mma), per-CTA partial
//                    sums reduced in a fixed order by k_reduce_partials.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace efwi {
namespace {

__device__ __forceinline__ void mma_bf16_16816(float c[4], const uint32_t a[4], uint32_t b0,
                                               uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16 *p) {
  return *reinterpret_cast<const uint32_t *>(p);
}
__device__ __forceinline__ uint32_t ld16(const __nv_bfloat16 *p) {
  return (uint32_t)(*reinterpret_cast<const unsigned short *>(p));
}

constexpr int kC = 16;              // channels
constexpr int kRowsFwd = 8;   // warps per CTA of k_conv3d_fwd: one y row each
constexpr int kTileX = 16;    // voxels per warp row
constexpr int kVoxPitch = 48; // bytes per staged voxel (32 of data): ldmatrix rows hit
                              // distinct banks
constexpr int kTileVox = 3 * (kRowsFwd + 2) * (kTileX + 2);

__device__ __forceinline__ void ldmatrix_x4(uint32_t a[4], uint32_t addr) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
               : "r"(addr));
}

// A CTA computes the voxels (z, y0 .. y0+7, x0 .. x0+15).  Its input with a
// 1-voxel halo (3 x 10 x 18 voxels) is staged in shared memory once; each
// warp then takes, per tap, the 16 x 16 A fragment of its row with one
// ldmatrix.x4 (matrices: voxels 0-7 / 8-15 x channels 0-7 / 8-15, which is
// the register order of the mma A operand).
__global__ void __launch_bounds__(32 * kRowsFwd)
k_conv3d_fwd(const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ w,
             const float *__restrict__ bias, int D, int H, int W, int relu,
             __nv_bfloat16 *__restrict__ yb, float *__restrict__ yf) {
  __shared__ __align__(16) uint32_t sw[27 * kC * kC / 2];  // [t][co][ci pair]
  __shared__ __align__(16) unsigned char sx[kTileVox * kVoxPitch];
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * kTileX, y0 = blockIdx.y * kRowsFwd, z = blockIdx.z;
  for (int k = tid; k < 27 * kC * kC / 2; k += blockDim.x) sw[k] = ld32(w + 2 * k);
  for (int c = tid; c < 2 * kTileVox; c += blockDim.x) {
    const int v = c >> 1, h = c & 1;
    const int xx = v % (kTileX + 2), t = v / (kTileX + 2);
    const int yy = t % (kRowsFwd + 2), zz = t / (kRowsFwd + 2);
    const int gz = z - 1 + zz, gy = y0 - 1 + yy, gx = x0 - 1 + xx;
    uint4 val = make_uint4(0u, 0u, 0u, 0u);
    if (gz >= 0 && gz < D && gy >= 0 && gy < H && gx >= 0 && gx < W)
      val = *reinterpret_cast<const uint4 *>(x + (((long long)gz * H + gy) * W + gx) * kC + h * 8);
    *reinterpret_cast<uint4 *>(sx + v * kVoxPitch + h * 16) = val;
  }
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5;
  const int y = y0 + warp;
  if (y >= H) return;  // no barrier follows
  const int g = lane >> 2, q = lane & 3;
  const uint32_t sxa = (uint32_t)__cvta_generic_to_shared(sx);
  const int lrow = ((lane >> 3) & 1) * 8 + (lane & 7);  // voxel of this lane's ldmatrix row
  const int lcol = (lane >> 4) * 16;                      // channel half (bytes)

  float c[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
  for (int dz = 0; dz < 3; ++dz) {
#pragma unroll
    for (int dy = 0; dy < 3; ++dy) {
#pragma unroll
      for (int dx = 0; dx < 3; ++dx) {
        const int t = dz * 9 + dy * 3 + dx;
        const int v0 = (dz * (kRowsFwd + 2) + warp + dy) * (kTileX + 2) + dx;
        uint32_t a[4];
        ldmatrix_x4(a, sxa + (uint32_t)((v0 + lrow) * kVoxPitch + lcol));
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) {
          const uint32_t *wb = sw + (t * kC + nt * 8 + g) * (kC / 2);
          mma_bf16_16816(c[nt], a, wb[q], wb[q + 4]);
        }
      }
    }
  }
  // epilogue: c[nt][0..1] -> voxel x0+g, channels nt*8 + 2q, +1; [2..3] -> voxel x0+g+8
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    const int co = nt * 8 + 2 * q;
    const float b0 = bias ? bias[co] : 0.f, b1 = bias ? bias[co + 1] : 0.f;
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
      const int xv = x0 + g + 8 * hh;
      if (xv >= W) continue;
      float o0 = c[nt][2 * hh] + b0, o1 = c[nt][2 * hh + 1] + b1;
      if (relu) { o0 = fmaxf(o0, 0.f); o1 = fmaxf(o1, 0.f); }
      const long long off = (((long long)z * H + y) * W + xv) * kC + co;
      if (yb) *reinterpret_cast<__nv_bfloat162 *>(yb + off) = __floats2bfloat162_rn(o0, o1);
      if (yf) { yf[off] = o0; yf[off + 1] = o1; }
    }
  }
}

// One CTA of 27 warps (warp t = tap t) sums dW over a contiguous range of
// voxel rows; partial[cta][t][co][ci].
__global__ void __launch_bounds__(27 * 32)
k_conv3d_wgrad(const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ dy,
               int D, int H, int W, float *__restrict__ partial) {
  const int lane = threadIdx.x & 31, t = threadIdx.x >> 5;
  const int g = lane >> 2, q = lane & 3;
  const int dz = t / 9 - 1, dyy = (t / 3) % 3 - 1, dx = t % 3 - 1;
  const int nxc = (W + 15) >> 4;
  const long long units = (long long)D * H * nxc;
  const long long u0 = units * blockIdx.x / gridDim.x, u1 = units * (blockIdx.x + 1) / gridDim.x;
  float c[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
  for (long long u = u0; u < u1; ++u) {
    const int xc = (int)(u % nxc);
    const long long zy = u / nxc;
    const int y = (int)(zy % H), z = (int)(zy / H);
    const int zz = z + dz, yy = y + dyy;
    if (zz < 0 || zz >= D || yy < 0 || yy >= H) continue;
    const int x0 = xc * 16;
    const __nv_bfloat16 *grow = dy + ((long long)z * H + y) * W * kC;
    const __nv_bfloat16 *xrow = x + ((long long)zz * H + yy) * W * kC;
    // A (co x voxel): register r holds voxels (2q, 2q+1) (+8 for r = 2, 3)
    // of channel g (r = 0, 2) or g + 8 (r = 1, 3).
    const int va = x0 + 2 * q, vb = va + 8;
    uint32_t a[4];
    {
      const bool a0 = va < W, a1 = va + 1 < W, b0 = vb < W, b1 = vb + 1 < W;
      const uint32_t p00 = a0 ? ld16(grow + va * kC + g) : 0u, p01 = a1 ? ld16(grow + (va + 1) * kC + g) : 0u;
      const uint32_t p10 = a0 ? ld16(grow + va * kC + g + 8) : 0u, p11 = a1 ? ld16(grow + (va + 1) * kC + g + 8) : 0u;
      const uint32_t p20 = b0 ? ld16(grow + vb * kC + g) : 0u, p21 = b1 ? ld16(grow + (vb + 1) * kC + g) : 0u;
      const uint32_t p30 = b0 ? ld16(grow + vb * kC + g + 8) : 0u, p31 = b1 ? ld16(grow + (vb + 1) * kC + g + 8) : 0u;
      a[0] = p00 | (p01 << 16);
      a[1] = p10 | (p11 << 16);
      a[2] = p20 | (p21 << 16);
      a[3] = p30 | (p31 << 16);
    }
    // B (voxel x ci): voxels 2q, 2q+1 (b0) and 2q+8, 2q+9 (b1), shifted by dx
    const int sa = va + dx, sb = vb + dx;
    const bool s0 = sa >= 0 && sa < W && va < W, s1 = sa + 1 >= 0 && sa + 1 < W && va + 1 < W;
    const bool s2 = sb >= 0 && sb < W && vb < W, s3 = sb + 1 >= 0 && sb + 1 < W && vb + 1 < W;
#pragma unroll
    for (int nt = 0; nt < 2; ++nt) {
      const int ci = nt * 8 + g;
      const uint32_t e0 = s0 ? ld16(xrow + sa * kC + ci) : 0u, e1 = s1 ? ld16(xrow + (sa + 1) * kC + ci) : 0u;
      const uint32_t e2 = s2 ? ld16(xrow + sb * kC + ci) : 0u, e3 = s3 ? ld16(xrow + (sb + 1) * kC + ci) : 0u;
      mma_bf16_16816(c[nt], a, e0 | (e1 << 16), e2 | (e3 << 16));
    }
  }
  // C (co x ci): c[nt][0..1] -> co g, ci nt*8 + 2q, +1; [2..3] -> co g + 8
  float *out = partial + ((long long)blockIdx.x * 27 + t) * kC * kC;
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    const int ci = nt * 8 + 2 * q;
    out[g * kC + ci] = c[nt][0];
    out[g * kC + ci + 1] = c[nt][1];
    out[(g + 8) * kC + ci] = c[nt][2];
    out[(g + 8) * kC + ci + 1] = c[nt][3];
  }
}

__global__ void k_reduce_partials(const float *__restrict__ partial, int nparts, int n,
                                  float *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int p = 0; p < nparts; ++p) s += partial[(long long)p * n + i];
  out[i] = s;
}

}  // namespace
}  // namespace efwi

using namespace efwi;

extern "C" int efwi_conv3d_forward(const void *x, const void *w, const float *bias, int D, int H,
                                   int W, int relu, void *y_bf16, float *y_f32, void *stream) {
  if (!x || !w || D < 1 || H < 1 || W < 1 || D > 65535 || (!y_bf16 && !y_f32)) return 1;
  if (((uintptr_t)x & 15) != 0) return 1;  // staged with 16-byte loads
  const dim3 grid((W + kTileX - 1) / kTileX, (H + kRowsFwd - 1) / kRowsFwd, D);
  k_conv3d_fwd<<<grid, 32 * kRowsFwd, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16 *)x, (const __nv_bfloat16 *)w, bias, D, H, W, relu,
      (__nv_bfloat16 *)y_bf16, y_f32);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

extern "C" int efwi_conv3d_wgrad(const void *x, const void *dy, int D, int H, int W,
                                 float *partial, int nparts, float *dw, void *stream) {
  if (!x || !dy || !partial || !dw || D < 1 || H < 1 || W < 1 || nparts < 1) return 1;
  cudaStream_t st = (cudaStream_t)stream;
  k_conv3d_wgrad<<<nparts, 27 * 32, 0, st>>>((const __nv_bfloat16 *)x, (const __nv_bfloat16 *)dy,
                                             D, H, W, partial);
  const int n = 27 * kC * kC;
  k_reduce_partials<<<(n + 255) / 256, 256, 0, st>>>(partial, nparts, n, dw);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
