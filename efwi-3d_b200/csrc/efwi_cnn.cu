// 3-D convolutions of the learned gradient preconditioner on BF16 tensor
// cores with FP32 accumulation (no reference counterpart).
//
// Layer: 3x3x3 kernel, stride 1, zero padding 1, 16 input and 16 output
// channels (narrower inputs and outputs are zero-padded to 16 by the
// caller).  Layouts:
//   activations  [D][H][W][16] bf16 (channels last: one voxel = 32 bytes)
//   weights      [27][16 co][16 ci] bf16, tap t = (dz+1)*9 + (dy+1)*3 + (dx+1)
//   bias         [16] f32
// Voxels outside the volume read as zero.  With W'[t][a][b] = W[26-t][b][a]
// the forward convolution also computes the gradient of the input (the
// transposed convolution).
//
// Kernels (efwi_conv3d_set_kernel / efwi_conv3d_set_wgrad_kernel choose):
//   k_conv3d_fwd_tc2  forward on tcgen05.mma (the default): per tile of
//                     128 voxels one MMA per tap, accumulator in tensor
//                     memory, input tiles staged by bulk tensor copies
//   k_conv3d_fwd_ws   the same, warp-specialised (copy + MMA warp, four
//                     epilogue warps)
//   k_conv3d_fwd_tc   the same MMAs, tiles staged by plain loads
//   k_conv3d_fwd      forward on mma.sync.m16n8k16: per output row of 16
//                     voxels one warp, A fragments by ldmatrix
//   k_conv3d_wgrad_tc dW[t][co][ci] = sum_u dy[u - off_t][co] x[u][ci] on
//                     tcgen05.mma (the default): eight taps stacked on the
//                     MMA's rows, K = voxels
//   k_conv3d_wgrad    the same on mma.sync: one warp per tap
// Both weight gradients leave per-CTA partial sums that k_reduce_partials
// adds in a fixed order.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>

#include "efwi_tma.cuh"

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


// ------------------------------------------------------------- tcgen05 form
// The forward convolution on the 5th-generation tensor cores: per tile of
// 128 voxels (8 x by 16 y at one z) and tap t, D[128 voxels][16 co] +=
// A_t[128][16 ci] B_t[16 ci][16 co] with one tcgen05.mma.kind::f16 (M 128,
// N 16, K 16; BF16 operands from shared memory, FP32 accumulator in TMEM).
// The CTA's input tile with its 1-voxel halo (3 x 18 x 10 voxels) is staged
// as two planes of 16-byte chunks (channels 0-7, channels 8-15), x fastest,
// so that A_t is the canonical K-major, non-swizzled operand at a shifted
// base: core matrices of 8 rows (8 consecutive x) x 16 bytes, the 16 rows
// of the tile one staged row apart (SBO = 10 x 16 B), the two K halves one
// plane apart (LBO).  B_t is staged the same way ([t][half][co][8 ci]).  One
// thread issues the 27 MMAs and commits them to an mbarrier; each warp then
// reads its 32 TMEM lanes (32 voxels x 16 fp32 columns) with tcgen05.ld.
// CTAs are persistent (the weights are staged once per CTA) and hold 32 TMEM
// columns each, allocated on entry and freed on exit.
constexpr int kTcX = 8, kTcY = 16;                   // tile: 128 voxels
constexpr int kTcSX = kTcX + 2, kTcSY = kTcY + 2;    // staged with the halo
constexpr int kTcVox = 3 * kTcSY * kTcSX;            // 540 staged voxels
constexpr int kTcPlane = kTcVox * 16;                // bytes of one channel-half plane
constexpr int kTcWBytes = 27 * 2 * kC * 16;          // staged weights
constexpr int kTcSmem = 2 * kTcPlane + kTcWBytes;

// Shared-memory matrix descriptor of tcgen05.mma: start address, leading
// (K) and stride (M/N) byte offsets, descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = 16, M = 128.
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) |
                              ((128u >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(kTcIdesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float v[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ int g_conv_status;  // EFWI_STATUS_TIMEOUT after a wait that ran out

// The 27 MMAs of one tile into the accumulator at TMEM address d: the
// descriptors of tap t are the tap-0 ones with the start address moved by
// the tap's offset (the 14-bit start field cannot carry: shared addresses
// stay below 256 KB), so the unrolled loop issues one add per operand.
__device__ __forceinline__ void tc_tile_mmas(uint32_t d, uint32_t sxa, uint32_t plane_bytes,
                                             uint32_t swa) {
  const uint64_t a0 = tc_desc(sxa, plane_bytes, kTcSX * 16);
  const uint64_t b0 = tc_desc(swa, kC * 16, 8 * 16);
#pragma unroll
  for (int t = 0; t < 27; ++t) {
    const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
    const uint64_t ao = (uint64_t)((dz * kTcSY + dy) * kTcSX + dx);  // 16-byte units
    const uint64_t bo = (uint64_t)(t * 2 * kC);                      // 16-byte units
    tc_mma(d, a0 + ao, b0 + bo, t > 0 ? 1u : 0u);
  }
}

__global__ void __launch_bounds__(128)
k_conv3d_fwd_tc(const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ w,
                const float *__restrict__ bias, int D, int H, int W, int relu,
                __nv_bfloat16 *__restrict__ yb, float *__restrict__ yf) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  unsigned char *sx = smem;                     // [half][z][y][x] x 16 B
  unsigned char *swt = smem + 2 * kTcPlane;     // [t][half][co] x 16 B
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int k = tid; k < 27 * 2 * kC; k += blockDim.x) {
    const int t = k / (2 * kC), r = k % (2 * kC), h = r / kC, co = r % kC;
    *reinterpret_cast<uint4 *>(swt + ((t * 2 + h) * kC + co) * 16) =
        *reinterpret_cast<const uint4 *>(w + (t * kC + co) * kC + h * 8);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(
                     smem_u32(&tmem_slot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t sxa = smem_u32(sx), swa = smem_u32(swt);
  float bv[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) bv[k] = bias ? bias[k] : 0.f;
  const int ntx = (W + kTcX - 1) / kTcX, nty = (H + kTcY - 1) / kTcY;
  const long long ntiles = (long long)ntx * nty * D;
  int phase = 0;
  bool ok = true;
  for (long long tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int tx = (int)(tile % ntx);
    const long long r = tile / ntx;
    const int ty = (int)(r % nty), z = (int)(r / nty);
    const int x0 = tx * kTcX, y0 = ty * kTcY;
    for (int c = tid; c < 2 * kTcVox; c += blockDim.x) {
      const int v = c >> 1, h = c & 1;
      const int xx = v % kTcSX, t2 = v / kTcSX;
      const int yy = t2 % kTcSY, zz = t2 / kTcSY;
      const int gz = z - 1 + zz, gy = y0 - 1 + yy, gx = x0 - 1 + xx;
      uint4 val = make_uint4(0u, 0u, 0u, 0u);
      if (gz >= 0 && gz < D && gy >= 0 && gy < H && gx >= 0 && gx < W)
        val = *reinterpret_cast<const uint4 *>(x + (((long long)gz * H + gy) * W + gx) * kC + h * 8);
      *reinterpret_cast<uint4 *>(sx + h * kTcPlane + v * 16) = val;
    }
    // the staged tile (generic-proxy writes) is read by the tensor cores
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      tc_tile_mmas(tmem, sxa, kTcPlane, swa);
      tc_commit(&bar);
    }
    // every thread decides on the same value: tcgen05.ld is warp-collective
    const bool got = __syncthreads_and(mbar_wait_bounded(&bar, (uint32_t)phase));
    phase ^= 1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (got) {
      float v[16];
      tc_ld16(tmem + ((uint32_t)(warp * 32) << 16), v);
      const int m = warp * 32 + lane;
      const int xv = x0 + (m & 7), yv = y0 + (m >> 3);
      if (xv < W && yv < H) {
        const long long off = (((long long)z * H + yv) * W + xv) * kC;
        float o[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          o[k] = v[k] + bv[k];
          if (relu) o[k] = fmaxf(o[k], 0.f);
        }
        if (yb) {
          uint32_t pk[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const __nv_bfloat162 b2 = __floats2bfloat162_rn(o[2 * k], o[2 * k + 1]);
            pk[k] = *reinterpret_cast<const uint32_t *>(&b2);
          }
          uint4 *dst = reinterpret_cast<uint4 *>(yb + off);
          dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
        if (yf) {
          float4 *dst = reinterpret_cast<float4 *>(yf + off);
#pragma unroll
          for (int k = 0; k < 4; ++k) dst[k] = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // TMEM and the staged tile are free again
    ok = got;
  }
  if (!ok && tid == 0) {
    atomicExch(&g_conv_status, EFWI_STATUS_TIMEOUT);
    mbar_wait_bounded(&bar, (uint32_t)(phase ^ 1));  // the MMAs still in flight, bounded
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
}


// The same tile and MMAs with the input staged by bulk tensor copies and
// the work software-pipelined: while the warps drain tile j's accumulator,
// the tensor cores already work on tile j+1 (two accumulators of 16 TMEM
// columns, used in turn) and the copy engine fills stages ahead.  With NS
// stages the copies of tile j+NS-1 are issued as soon as their stage is
// free: for NS = 3 right after tile j+1's MMAs (the stage last held tile
// j-1, whose MMAs completed in the previous iteration), for NS = 2 once tile
// j's MMAs completed.  The tensor map views x as [D][H][W][2 halves][8
// channels]; a box of 8 x 1 x 10 x 18 x 3 is one channel-half plane of the
// staged tile in exactly the layout above (zeros outside the volume), so
// each stage takes two copies.  Half planes start 128-byte aligned.
constexpr int kTc2Plane = (kTcPlane + 127) / 128 * 128;  // 8704
constexpr int kTc2Stage = 2 * kTc2Plane;
constexpr int kTc2Copy = 2 * kTcPlane;  // bytes the two copies deliver
template <int NS>
constexpr int tc2_smem() { return NS * kTc2Stage + kTcWBytes + 128; }  // + alignment slack

__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int c0, int c1, int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4),
      "r"(smem_u32(bar))
      : "memory");
}

template <int NS>
__global__ void __launch_bounds__(128)
k_conv3d_fwd_tc2(const __grid_constant__ CUtensorMap xmap, const __nv_bfloat16 *__restrict__ w,
                 const float *__restrict__ bias, int D, int H, int W, int relu,
                 __nv_bfloat16 *__restrict__ yb, float *__restrict__ yf) {
  static_assert(NS == 2 || NS == 3, "two or three stages");
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[NS];  // stage filled (copies landed)
  __shared__ __align__(8) uint64_t done[2];   // accumulator b complete
  __shared__ uint32_t tmem_slot;
  __shared__ int s_abort;
  unsigned char *smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  unsigned char *swt = smem + NS * kTc2Stage;  // [t][half][co] x 16 B
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntx = (W + kTcX - 1) / kTcX, nty = (H + kTcY - 1) / kTcY;
  const long long ntiles = (long long)ntx * nty * D;
  // tiles of this CTA: blockIdx.x + j * gridDim.x, j < nj
  const long long nj =
      (long long)blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  auto tile_origin = [&](long long j, int &x0, int &y0, int &z) {
    const long long tile = blockIdx.x + j * gridDim.x;
    x0 = (int)(tile % ntx) * kTcX;
    const long long r = tile / ntx;
    y0 = (int)(r % nty) * kTcY;
    z = (int)(r / nty);
  };
  const uint32_t swa = smem_u32(swt);
  uint32_t tmem = 0;
  // thread 0: copies of tile j into stage j % NS
  auto issue = [&](long long j) {
    int x0, y0, z;
    tile_origin(j, x0, y0, z);
    const int s = (int)(j % NS);
    mbar_arrive_expect_tx(&full[s], kTc2Copy);
    unsigned char *dst = smem + s * kTc2Stage;
    tma_load_5d(dst, &xmap, &full[s], 0, 0, x0 - 1, y0 - 1, z - 1);
    tma_load_5d(dst + kTc2Plane, &xmap, &full[s], 0, 1, x0 - 1, y0 - 1, z - 1);
  };
  // thread 0: the 27 MMAs of tile j into accumulator j & 1, once its stage landed
  auto mma = [&](long long j) -> bool {
    const int s = (int)(j % NS);
    if (!mbar_wait_bounded(&full[s], (uint32_t)((j / NS) & 1))) return false;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    tc_tile_mmas(tmem + (uint32_t)((j & 1) * kC), smem_u32(smem + s * kTc2Stage), kTc2Plane, swa);
    tc_commit(&done[j & 1]);
    return true;
  };
  long long n_tma = 0, n_mma = 0;  // thread 0: tiles whose copies / MMAs were issued
  if (tid == 0) {
    for (int s = 0; s < NS; ++s) mbar_init(&full[s], 1);
    mbar_init(&done[0], 1);
    mbar_init(&done[1], 1);
    fence_mbar_init();
    s_abort = 0;
    for (; n_tma < 2 && n_tma < nj; ++n_tma) issue(n_tma);
  }
  for (int k = tid; k < 27 * 2 * kC; k += blockDim.x) {
    const int t = k / (2 * kC), r = k % (2 * kC), h = r / kC, co = r % kC;
    *reinterpret_cast<uint4 *>(swt + ((t * 2 + h) * kC + co) * 16) =
        *reinterpret_cast<const uint4 *>(w + (t * kC + co) * kC + h * 8);
  }
  float bv[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) bv[q] = bias ? bias[q] : 0.f;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(
                     smem_u32(&tmem_slot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_proxy_async_smem();  // the staged weights are read by the tensor cores
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  tmem = tmem_slot;
  if (tid == 0 && nj > 0) {
    if (mma(0)) n_mma = 1;
    else s_abort = 1;
  }
  __syncthreads();
  bool ok = !s_abort;
  for (long long j = 0; j < nj && ok; ++j) {
    if (tid == 0 && !s_abort) {
      // accumulator (j+1)&1 was drained in iteration j-1
      if (j + 1 < nj) {
        if (mma(j + 1)) n_mma = j + 2;
        else s_abort = 1;
      }
      if (NS == 3 && !s_abort && j + 2 < nj) {
        issue(j + 2);
        n_tma = j + 3;
      }
    }
    // every thread takes the same branch: tcgen05.ld is warp-collective
    const bool got =
        __syncthreads_and(mbar_wait_bounded(&done[j & 1], (uint32_t)((j >> 1) & 1)));
    if (NS == 2 && tid == 0 && got && !s_abort && j + 2 < nj) {
      issue(j + 2);  // stage j % 2: tile j's MMAs completed
      n_tma = j + 3;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (got) {
      int x0, y0, z;
      tile_origin(j, x0, y0, z);
      float v[16];
      tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((j & 1) * kC), v);
      const int m = warp * 32 + lane;
      const int xv = x0 + (m & 7), yv = y0 + (m >> 3);
      if (xv < W && yv < H) {
        const long long off = (((long long)z * H + yv) * W + xv) * kC;
        float o[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          o[q] = v[q] + bv[q];
          if (relu) o[q] = fmaxf(o[q], 0.f);
        }
        if (yb) {
          uint32_t pk[8];
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const __nv_bfloat162 b2 = __floats2bfloat162_rn(o[2 * q], o[2 * q + 1]);
            pk[q] = *reinterpret_cast<const uint32_t *>(&b2);
          }
          uint4 *dst = reinterpret_cast<uint4 *>(yb + off);
          dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
        if (yf) {
          float4 *dst = reinterpret_cast<float4 *>(yf + off);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            dst[q] = make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();  // accumulator j & 1 is free again; s_abort is published
    ok = got && !s_abort;
  }
  if (!ok && tid == 0) {
    atomicExch(&g_conv_status, EFWI_STATUS_TIMEOUT);
    // bounded waits for what may still be in flight: the copies of tiles
    // whose MMAs were never issued, and the last MMAs issued
    for (long long j = n_mma; j < n_tma; ++j)
      mbar_wait_bounded(&full[j % NS], (uint32_t)((j / NS) & 1));
    if (n_mma > 0) mbar_wait_bounded(&done[(n_mma - 1) & 1], (uint32_t)(((n_mma - 1) >> 1) & 1));
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
}


// Warp-specialised form of the copy-staged kernel: warp 0 (one elected
// thread) fills NS stages with bulk tensor copies and issues each tile's 27
// MMAs into one of two accumulators; warps 1-4 drain the accumulators
// (warp w reads TMEM lanes 32 (w % 4) .. + 31, so the four cover the 128
// rows).  The roles meet only at mbarriers -- stage full (copies landed),
// stage empty (its MMAs completed, committed by the MMA thread), accumulator
// full (committed) and accumulator empty (one arrival per epilogue warp
// after its tcgen05.ld) -- so no warp waits for the CTA at a barrier per
// tile.  Every wait is bounded: a role that gives up sets the status flag
// and a shared abort word that the other roles test once per tile; before
// TMEM is freed, thread 0 waits (bounded) for the copies and MMAs it issued.
constexpr int kWsThreads = 160;

__device__ __forceinline__ void mbar_arrive1(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <int NS>
__global__ void __launch_bounds__(kWsThreads)
k_conv3d_fwd_ws(const __grid_constant__ CUtensorMap xmap, const __nv_bfloat16 *__restrict__ w,
                const float *__restrict__ bias, int D, int H, int W, int relu,
                __nv_bfloat16 *__restrict__ yb, float *__restrict__ yf) {
  static_assert(NS >= 2 && NS <= 4, "two to four stages");
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t full[NS], empty[NS], tfull[2], tempty[2];
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int s_abort;
  unsigned char *smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  unsigned char *swt = smem + NS * kTc2Stage;  // [t][half][co] x 16 B
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntx = (W + kTcX - 1) / kTcX, nty = (H + kTcY - 1) / kTcY;
  const long long ntiles = (long long)ntx * nty * D;
  const long long nj =
      (long long)blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  auto tile_origin = [&](long long j, int &x0, int &y0, int &z) {
    const long long tile = blockIdx.x + j * gridDim.x;
    x0 = (int)(tile % ntx) * kTcX;
    const long long r = tile / ntx;
    y0 = (int)(r % nty) * kTcY;
    z = (int)(r / nty);
  };
  auto give_up = [&]() {
    s_abort = 1;
    atomicExch(&g_conv_status, EFWI_STATUS_TIMEOUT);
  };
  auto issue = [&](long long j) {  // thread 0: copies of tile j into stage j % NS
    int x0, y0, z;
    tile_origin(j, x0, y0, z);
    const int s = (int)(j % NS);
    mbar_arrive_expect_tx(&full[s], kTc2Copy);
    unsigned char *dst = smem + s * kTc2Stage;
    tma_load_5d(dst, &xmap, &full[s], 0, 0, x0 - 1, y0 - 1, z - 1);
    tma_load_5d(dst + kTc2Plane, &xmap, &full[s], 0, 1, x0 - 1, y0 - 1, z - 1);
  };
  long long jt = 0, jm = 0;  // thread 0: tiles whose copies / MMAs were issued
  if (tid == 0) {
    for (int s = 0; s < NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], 4);
    }
    fence_mbar_init();
    s_abort = 0;
    for (; jt < NS && jt < nj; ++jt) issue(jt);
  }
  for (int k = tid; k < 27 * 2 * kC; k += blockDim.x) {
    const int t = k / (2 * kC), r = k % (2 * kC), h = r / kC, co = r % kC;
    *reinterpret_cast<uint4 *>(swt + ((t * 2 + h) * kC + co) * 16) =
        *reinterpret_cast<const uint4 *>(w + (t * kC + co) * kC + h * 8);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(
                     smem_u32(&tmem_slot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_proxy_async_smem();  // the staged weights are read by the tensor cores
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t swa = smem_u32(swt);

  if (warp == 0) {
    if (lane == 0) {  // copies and MMAs
      for (long long j = 0; j < nj; ++j) {
        if (s_abort) break;
        const int s = (int)(j % NS), b = (int)(j & 1);
        if (!mbar_wait_bounded(&full[s], (uint32_t)((j / NS) & 1))) { give_up(); break; }
        if (j >= 2 && !mbar_wait_bounded(&tempty[b], (uint32_t)(((j - 2) >> 1) & 1))) {
          give_up();
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tc_tile_mmas(tmem + (uint32_t)(b * kC), smem_u32(smem + s * kTc2Stage), kTc2Plane, swa);
        tc_commit(&tfull[b]);
        tc_commit(&empty[s]);
        jm = j + 1;
        // refill the stage of tile j-1 (its MMAs were issued one tile ago)
        if (j >= 1 && jt < nj) {
          const long long jp = j - 1;
          if (!mbar_wait_bounded(&empty[jp % NS], (uint32_t)((jp / NS) & 1))) { give_up(); break; }
          issue(jt);
          ++jt;
        }
      }
    }
  } else if (warp <= 4) {  // epilogue: TMEM lanes 32 (warp % 4) .. + 31
    const int q = warp & 3;
    float bv[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) bv[k] = bias ? bias[k] : 0.f;
    for (long long j = 0; j < nj; ++j) {
      if (s_abort) break;
      const int b = (int)(j & 1);
      bool ok = mbar_wait_bounded(&tfull[b], (uint32_t)((j >> 1) & 1));
      ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld is warp-collective
      if (!ok) {
        if (lane == 0) give_up();
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      float v[16];
      tc_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kC), v);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive1(&tempty[b]);
      int x0, y0, z;
      tile_origin(j, x0, y0, z);
      const int m = q * 32 + lane;
      const int xv = x0 + (m & 7), yv = y0 + (m >> 3);
      if (xv < W && yv < H) {
        const long long off = (((long long)z * H + yv) * W + xv) * kC;
        float o[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          o[k] = v[k] + bv[k];
          if (relu) o[k] = fmaxf(o[k], 0.f);
        }
        if (yb) {
          uint32_t pk[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const __nv_bfloat162 b2 = __floats2bfloat162_rn(o[2 * k], o[2 * k + 1]);
            pk[k] = *reinterpret_cast<const uint32_t *>(&b2);
          }
          uint4 *dst = reinterpret_cast<uint4 *>(yb + off);
          dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        }
        if (yf) {
          float4 *dst = reinterpret_cast<float4 *>(yf + off);
#pragma unroll
          for (int k = 0; k < 4; ++k)
            dst[k] = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
        }
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    // bounded waits for what thread 0 issued and nobody consumed: copies of
    // tiles whose MMAs were never issued, and the last MMAs (their commit)
    for (long long j = jm; j < jt; ++j) mbar_wait_bounded(&full[j % NS], (uint32_t)((j / NS) & 1));
    if (jm > 0) mbar_wait_bounded(&empty[(jm - 1) % NS], (uint32_t)(((jm - 1) / NS) & 1));
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
}
// Weight gradient on tcgen05: dW[t][co][ci] = sum_u dy[u - off_t][co] x[u][ci]
// (u = v + off_t).  A unit is 8 (x) x 16 (y) voxels u on each of up to 8
// consecutive z planes (the dy planes of one z are reused for the next);
// its K = 16 slices are two staged rows of 8 voxels.  B = x[u][ci] staged as
// [row][ci][8 x] (256-byte row blocks: ci halves 128 B apart, the second K
// row one block on).  A stacks taps on M: rows (j, co), j = 3a + b standing
// for dy = 1 - a, dz = 1 - b, read from dy staged as [row][plane][co][8 x]
// with the three planes z-1, z, z+1 in consecutive 256-byte blocks, so the
// 16 row groups of taps j = 0..7 lie 128 B apart (a uniform stride) and the
// second K row is three blocks on.  One staged copy per x shift dx keeps the
// operands 16-byte aligned; per K slice and shift one MMA covers taps 0..7
// and a second, one block later, taps 1..8 (only its last 16 rows, tap 8,
// are kept).  Six accumulators of 16 TMEM columns sum over all units of a
// CTA; the CTA's 27 x 16 x 16 sums go to partial[cta] for the fixed-order
// reduction.  Every wait is bounded; on a timeout the CTA sets the status
// flag and writes NaN partial sums.
constexpr int kWgRows = 16;                           // y rows of a unit
constexpr int kWgZ = 8;                               // z planes a unit marches
constexpr int kWgX = 8;                               // x voxels of a unit
constexpr int kWgXBytes = kWgRows * 256;              // staged x: [row][ci][8]
constexpr int kWgDyBytes = (kWgRows + 2) * 3 * 256;   // staged dy per shift
constexpr int kWgSmem = kWgXBytes + 3 * kWgDyBytes + 128;
constexpr int kWgThreads = 128;

__global__ void __launch_bounds__(kWgThreads)
k_conv3d_wgrad_tc(const __nv_bfloat16 *__restrict__ x, const __nv_bfloat16 *__restrict__ dy,
                  int D, int H, int W, float *__restrict__ partial) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  unsigned char *smem = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  unsigned char *sxs = smem;                  // [row][ci][8 x]
  unsigned char *sdy = smem + kWgXBytes;      // [dx][row][plane][co][8 x]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nxw = (W + kWgX - 1) / kWgX, nyb = (H + kWgRows - 1) / kWgRows;
  const long long nunits = (long long)nxw * nyb * ((D + kWgZ - 1) / kWgZ);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(
                     smem_u32(&tmem_slot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t xa = smem_u32(sxs), da = smem_u32(sdy);
  int phase = 0;
  bool ok = true, any = false;
  // dy of plane gz into plane slot b of every shift copy (zeros outside)
  auto stage_dy_plane = [&](int b, int gz, int x0, int y0) {
    for (int c = tid; c < 3 * (kWgRows + 2) * kWgX * 2; c += blockDim.x) {
      const int h = c & 1;
      int rest = c >> 1;
      const int k = rest % kWgX;
      rest /= kWgX;
      const int r = rest % (kWgRows + 2), sh = rest / (kWgRows + 2);
      const int gy = y0 - 1 + r, gx = x0 + k - (sh - 1);
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (gz >= 0 && gz < D && gy >= 0 && gy < H && gx >= 0 && gx < W)
        v = *reinterpret_cast<const uint4 *>(dy + (((long long)gz * H + gy) * W + gx) * kC + h * 8);
      const unsigned short *e = reinterpret_cast<const unsigned short *>(&v);
      unsigned short *dst =
          reinterpret_cast<unsigned short *>(sdy + sh * kWgDyBytes + (r * 3 + b) * 256) + k;
#pragma unroll
      for (int q = 0; q < 8; ++q) dst[(h * 8 + q) * kWgX] = e[q];
    }
  };
  for (long long unit = blockIdx.x; unit < nunits && ok; unit += gridDim.x) {
    const int xw = (int)(unit % nxw);
    const long long r0 = unit / nxw;
    const int yb = (int)(r0 % nyb), zc = (int)(r0 / nyb);
    const int x0 = xw * kWgX, y0 = yb * kWgRows;
    const int zb = zc * kWgZ, ze = min(zb + kWgZ, D);
    for (int z = zb; z < ze && ok; ++z) {
      if (z == zb) {
        for (int b = 0; b < 3; ++b) stage_dy_plane(b, z - 1 + b, x0, y0);
      } else {
        // planes z-1, z of the new window are planes 1, 2 of the last one:
        // each thread moves its own 16-byte pieces, then plane z+1 arrives
        for (int c = tid; c < 3 * (kWgRows + 2) * 16; c += blockDim.x) {
          const int piece = c & 15, rs = c >> 4;  // rs = shift * (rows) + row
          uint4 *blk = reinterpret_cast<uint4 *>(sdy + (rs / (kWgRows + 2)) * kWgDyBytes +
                                                 (rs % (kWgRows + 2)) * 3 * 256);
          const uint4 p1 = blk[16 + piece], p2 = blk[32 + piece];
          blk[piece] = p1;
          blk[16 + piece] = p2;
        }
        __syncthreads();  // plane slot 2 is rewritten below by other threads
        stage_dy_plane(2, z + 1, x0, y0);
      }
      // x: voxel (row, k) of plane z, 8 channels per item
      for (int c = tid; c < kWgRows * kWgX * 2; c += blockDim.x) {
        const int h = c & 1, k = (c >> 1) % kWgX, row = (c >> 1) / kWgX;
        const int gy = y0 + row, gx = x0 + k;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (gy < H && gx < W)
          v = *reinterpret_cast<const uint4 *>(x + (((long long)z * H + gy) * W + gx) * kC + h * 8);
        const unsigned short *e = reinterpret_cast<const unsigned short *>(&v);
        unsigned short *dst = reinterpret_cast<unsigned short *>(sxs + row * 256) + k;
#pragma unroll
        for (int q = 0; q < 8; ++q) dst[(h * 8 + q) * kWgX] = e[q];
      }
      fence_proxy_async_smem();  // staged by the threads, read by the tensor cores
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
        for (int r = 0; r < kWgRows; r += 2) {
          const uint64_t bd = tc_desc(xa + (uint32_t)(r * 256), 256, 128);
#pragma unroll
          for (int sh = 0; sh < 3; ++sh) {
            const uint32_t a0 = da + (uint32_t)(sh * kWgDyBytes + r * 3 * 256);
            const uint32_t acc = (any || r > 0) ? 1u : 0u;
            tc_mma(tmem + (uint32_t)(2 * sh * kC), tc_desc(a0, 768, 128), bd, acc);
            tc_mma(tmem + (uint32_t)((2 * sh + 1) * kC), tc_desc(a0 + 256, 768, 128), bd, acc);
          }
        }
        tc_commit(&bar);
      }
      any = true;
      // the staged planes are read by the MMAs: wait before changing them
      ok = __syncthreads_and(mbar_wait_bounded(&bar, (uint32_t)phase));
      phase ^= 1;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
  }
  if (!ok && tid == 0) {
    atomicExch(&g_conv_status, EFWI_STATUS_TIMEOUT);
    mbar_wait_bounded(&bar, (uint32_t)(phase ^ 1));  // the MMAs still in flight, bounded
  }
  // the CTA's sums: accumulator 2s holds taps j = 0..7 of shift s in rows
  // 16 j + co, accumulator 2s + 1 tap j = 8 in rows 112..127; column = ci
  float *out = partial + (long long)blockIdx.x * 27 * kC * kC;
  const float nan = __int_as_float(0x7fc00000);
#pragma unroll 1
  for (int acc = 0; acc < 6; ++acc) {
    float v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = 0.f;
    if (any && ok) tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(acc * kC), v);
    const int row = warp * 32 + lane, co = row & 15;
    const int j = (acc & 1) ? 8 : row >> 4;
    if ((acc & 1) && row < 112) continue;
    const int a = j / 3, b = j % 3, s = acc >> 1;
    const int t = (2 - b) * 9 + (2 - a) * 3 + s;  // (dz+1)*9 + (dy+1)*3 + (dx+1)
    float *o = out + ((long long)t * kC + co) * kC;
#pragma unroll
    for (int q = 0; q < 16; ++q) o[q] = ok ? v[q] : nan;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(tmem) : "memory");
}

}  // namespace
}  // namespace efwi

using namespace efwi;

namespace {
// 0: mma.sync; 1: tcgen05, tile staged by loads; 2 / 3: tcgen05, tiles
// staged by bulk tensor copies two / three stages deep; 4 / 5: the same,
// warp-specialised (copy + MMA warp, four epilogue warps), two / three stages
std::atomic<int> g_conv_kernel{2};
std::atomic<unsigned long long> g_tc_smem_set{0}, g_tc2_smem_set{0}, g_tc3_smem_set{0},
    g_ws2_smem_set{0}, g_ws3_smem_set{0};
int g_sm_count[64] = {0};
std::atomic<PFN_cuTensorMapEncodeTiled_v12000> g_conv_encode{nullptr};

PFN_cuTensorMapEncodeTiled_v12000 conv_encoder() {
  PFN_cuTensorMapEncodeTiled_v12000 f = g_conv_encode.load();
  if (f) return f;
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
          cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !fn)
    return nullptr;
  f = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  g_conv_encode.store(f);
  return f;
}

// x [D][H][W][16] bf16 as a 5-D tensor (8 channels, 2 halves, W, H, D) with
// boxes of one channel half over the 10 x 18 x 3 staged voxels.
bool conv_map(CUtensorMap *m, const void *x, int D, int H, int W) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = conv_encoder();
  if (!enc) return false;
  cuuint64_t dims[5] = {8, 2, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)D};
  cuuint64_t strides[4] = {16, 32, 32ull * W, 32ull * W * H};
  cuuint32_t box[5] = {8, 1, (cuuint32_t)kTcSX, (cuuint32_t)kTcSY, 3};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void *>(x), dims, strides, box,
             es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace

extern "C" int efwi_conv3d_set_kernel(int form) {
  if (form < 0 || form > 5) return 1;
  g_conv_kernel.store(form);
  return 0;
}

extern "C" int efwi_conv3d_status(int *timed_out, void *stream) {
  if (!timed_out) return 1;
  int v = 0, zero = 0;
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemcpyFromSymbolAsync(&v, g_conv_status, sizeof(int), 0, cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaMemcpyToSymbolAsync(g_conv_status, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return 2;
  *timed_out = v != 0;
  return 0;
}

extern "C" int efwi_conv3d_forward(const void *x, const void *w, const float *bias, int D, int H,
                                   int W, int relu, void *y_bf16, float *y_f32, void *stream) {
  if (!x || !w || D < 1 || H < 1 || W < 1 || D > 65535 || (!y_bf16 && !y_f32)) return 1;
  if (((uintptr_t)x & 15) != 0) return 1;  // staged with 16-byte loads
  cudaStream_t st = (cudaStream_t)stream;
  const int form = g_conv_kernel.load();
  if (form != 0 && ((uintptr_t)w & 15) == 0 && ((uintptr_t)y_bf16 & 15) == 0 &&
      ((uintptr_t)y_f32 & 15) == 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 2;
    int &sms = g_sm_count[dev & 63];
    if (!sms && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return 2;
    const long long tiles = (long long)((W + kTcX - 1) / kTcX) * ((H + kTcY - 1) / kTcY) * D;
    if (form >= 2) {
      CUtensorMap map;
      if (!conv_map(&map, x, D, H, W)) return 2;
      if (form >= 4) {  // warp-specialised: two stages at 4 CTAs per SM, or three at 3
        const __nv_bfloat16 *wb = (const __nv_bfloat16 *)w;
        if (form == 4) {
          set_smem_once(k_conv3d_fwd_ws<2>, tc2_smem<2>(), g_ws2_smem_set);
          const int blocks = (int)std::min<long long>(tiles, 4LL * sms);
          k_conv3d_fwd_ws<2><<<blocks, kWsThreads, tc2_smem<2>(), st>>>(
              map, wb, bias, D, H, W, relu, (__nv_bfloat16 *)y_bf16, y_f32);
        } else {
          set_smem_once(k_conv3d_fwd_ws<3>, tc2_smem<3>(), g_ws3_smem_set);
          const int blocks = (int)std::min<long long>(tiles, 3LL * sms);
          k_conv3d_fwd_ws<3><<<blocks, kWsThreads, tc2_smem<3>(), st>>>(
              map, wb, bias, D, H, W, relu, (__nv_bfloat16 *)y_bf16, y_f32);
        }
      } else if (form == 2) {  // two stages, 49 KB of shared memory: 4 CTAs per SM
        set_smem_once(k_conv3d_fwd_tc2<2>, tc2_smem<2>(), g_tc2_smem_set);
        const int blocks = (int)std::min<long long>(tiles, 4LL * sms);
        k_conv3d_fwd_tc2<2><<<blocks, 128, tc2_smem<2>(), st>>>(
            map, (const __nv_bfloat16 *)w, bias, D, H, W, relu, (__nv_bfloat16 *)y_bf16, y_f32);
      } else {  // three stages, 66 KB: 3 CTAs per SM
        set_smem_once(k_conv3d_fwd_tc2<3>, tc2_smem<3>(), g_tc3_smem_set);
        const int blocks = (int)std::min<long long>(tiles, 3LL * sms);
        k_conv3d_fwd_tc2<3><<<blocks, 128, tc2_smem<3>(), st>>>(
            map, (const __nv_bfloat16 *)w, bias, D, H, W, relu, (__nv_bfloat16 *)y_bf16, y_f32);
      }
    } else {
      set_smem_once(k_conv3d_fwd_tc, kTcSmem, g_tc_smem_set);
      const int blocks = (int)std::min<long long>(tiles, 6LL * sms);
      k_conv3d_fwd_tc<<<blocks, 128, kTcSmem, st>>>((const __nv_bfloat16 *)x,
                                                    (const __nv_bfloat16 *)w, bias, D, H, W, relu,
                                                    (__nv_bfloat16 *)y_bf16, y_f32);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
  }
  const dim3 grid((W + kTileX - 1) / kTileX, (H + kRowsFwd - 1) / kRowsFwd, D);
  k_conv3d_fwd<<<grid, 32 * kRowsFwd, 0, st>>>(
      (const __nv_bfloat16 *)x, (const __nv_bfloat16 *)w, bias, D, H, W, relu,
      (__nv_bfloat16 *)y_bf16, y_f32);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

namespace {
std::atomic<int> g_wgrad_kernel{1};  // 1: tcgen05, 0: mma.sync
std::atomic<unsigned long long> g_wg_smem_set{0};
}  // namespace

extern "C" int efwi_conv3d_set_wgrad_kernel(int tcgen05) {
  g_wgrad_kernel.store(tcgen05 ? 1 : 0);
  return 0;
}

extern "C" int efwi_conv3d_wgrad(const void *x, const void *dy, int D, int H, int W,
                                 float *partial, int nparts, float *dw, void *stream) {
  if (!x || !dy || !partial || !dw || D < 1 || H < 1 || W < 1 || nparts < 1) return 1;
  cudaStream_t st = (cudaStream_t)stream;
  // the tcgen05 form stages with 16-byte loads; unaligned inputs take mma.sync
  if (g_wgrad_kernel.load() == 1 && ((uintptr_t)x & 15) == 0 && ((uintptr_t)dy & 15) == 0) {
    set_smem_once(k_conv3d_wgrad_tc, kWgSmem, g_wg_smem_set);
    k_conv3d_wgrad_tc<<<nparts, kWgThreads, kWgSmem, st>>>(
        (const __nv_bfloat16 *)x, (const __nv_bfloat16 *)dy, D, H, W, partial);
  } else {
    k_conv3d_wgrad<<<nparts, 27 * 32, 0, st>>>((const __nv_bfloat16 *)x,
                                               (const __nv_bfloat16 *)dy, D, H, W, partial);
  }
  const int n = 27 * kC * kC;
  k_reduce_partials<<<(n + 255) / 256, 256, 0, st>>>(partial, nparts, n, dw);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
