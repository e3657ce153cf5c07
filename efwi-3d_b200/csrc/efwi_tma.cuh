// Bulk tensor copies (TMA) into a ring of shared-memory plane slots.
//
// A CTA owns a 32 (y) x TX (x) column tile and marches z.  For every z plane
// the fields that need x/y neighbours are brought into shared memory as
// boxes of 40 (y) x (TX + 4) (x) floats by cp.async.bulk.tensor.3d, one
// mbarrier per ring slot.  The y box starts 4 cells before the tile so that
// its first element sits on a 16-byte boundary (the tile itself starts at a
// multiple of 32); the x box starts 2 rows before the tile.  Loads only, no
// cluster multicast.
//
// Every wait on an mbarrier is bounded by the global timer; a CTA that runs
// out of time records EFWI_STATUS_TIMEOUT in the status word, waits (again
// bounded) for its copies in flight and leaves, so a broken pipeline never
// hangs the GPU.
#pragma once
#include <cuda.h>
#include <stdint.h>

#include <atomic>

namespace efwi {

constexpr int TMA_BOXY = 40;     // y extent of a box (32 + 2 x 4 halo)
constexpr int TMA_HY = 4;        // y offset of the tile inside the box
constexpr int TMA_HX = 2;        // x offset of the tile inside the box
constexpr unsigned long long TMA_WAIT_NS = 2000000000ULL;  // 2 s

enum { EFWI_STATUS_OK = 0, EFWI_STATUS_TIMEOUT = 1 };

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) writes to the same slots.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// One try: the thread may be suspended up to TMA_SUSPEND_NS while the
// phase is incomplete, instead of spinning and taking issue slots.
constexpr uint32_t TMA_SUSPEND_NS = 2000;
// Hint that the line holding *p will be read soon: bring it into L2 (no
// register is written; the z-queue heads of the next plane use it).
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(TMA_SUSPEND_NS)
      : "memory");
  return ok != 0;
}

// Bounded wait: true when the phase completed, false after TMA_WAIT_NS.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > TMA_WAIT_NS) return false;
  }
  return true;
}

// Raises a kernel's dynamic shared-memory limit once per device: the
// attribute belongs to the device's context, so a process that drives
// several GPUs sets it on each (bit d of `done` stands for device d).  The
// bit is set only when the call succeeded; a failure stays pending as the
// runtime's last error, which the launch wrapper's check reports for the
// launch that needed the attribute.
template <class K>
inline void set_smem_once(K kernel, int bytes, std::atomic<unsigned long long> &done) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  const unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) ==
      cudaSuccess)
    done.fetch_or(bit, std::memory_order_acq_rel);
}

// 3-D tiled bulk tensor load of one box into shared memory (no multicast).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// Tensor maps of the staged fields: the first NH have halo boxes
// (TMA_BOXY x (TX + 4)), the rest point boxes (32 x TX).
template <int NF>
struct Maps {
  CUtensorMap m[NF];
};

// Ring of R plane slots in dynamic shared memory.  A slot holds NH halo
// boxes (fields read at x/y neighbours) followed by NP point boxes (fields
// read at the thread's own cell), all of one z plane.  The last NM point
// fields are model volumes shared by the shots of a batch; their plane
// coordinate is z instead of shot * nz + z.
template <int NH, int NP, int NM, int TX, int R>
struct PlaneRing {
  static constexpr int BOXX = TX + 2 * TMA_HX;
  static constexpr int HBOX = TMA_BOXY * BOXX;  // floats of a halo box
  static constexpr int PBOX = 32 * TX;          // floats of a point box
  static constexpr int SLOT_FLOATS = NH * HBOX + NP * PBOX;
  static constexpr int SLOT_BYTES = SLOT_FLOATS * 4;
  static constexpr int BYTES = R * SLOT_BYTES + R * 8;
  static_assert((HBOX * 4) % 128 == 0 && (PBOX * 4) % 128 == 0,
                "box starts must stay 128-byte aligned");

  float *buf;
  uint64_t *bar;

  __device__ __forceinline__ void bind(unsigned char *smem) {
    buf = reinterpret_cast<float *>(smem);
    bar = reinterpret_cast<uint64_t *>(smem + R * SLOT_BYTES);
  }
  __device__ __forceinline__ void init() {
    for (int s = 0; s < R; ++s) mbar_init(&bar[s], 1);
    fence_mbar_init();
  }
  // Issued by one thread: relative plane q, plane index `plane` of the
  // stacked shot volumes and `mplane` of the model volumes, tile origin
  // (y0, x0).
  __device__ __forceinline__ void issue(const Maps<NH + NP> &maps, int q, int y0, int x0,
                                        int plane, int mplane) {
    const int s = q % R;
    mbar_arrive_expect_tx(&bar[s], SLOT_BYTES);
    float *slot = buf + s * SLOT_FLOATS;
#pragma unroll
    for (int f = 0; f < NH; ++f)
      tma_load_3d(slot + f * HBOX, &maps.m[f], &bar[s], y0 - TMA_HY, x0 - TMA_HX, plane);
#pragma unroll
    for (int f = 0; f < NP; ++f)
      tma_load_3d(slot + NH * HBOX + f * PBOX, &maps.m[NH + f], &bar[s], y0, x0,
                  f < NP - NM ? plane : mplane);
  }
  __device__ __forceinline__ bool wait(int q) { return mbar_wait_bounded(&bar[q % R], (q / R) & 1); }
  __device__ __forceinline__ const float *halo(int q, int f) const {
    return buf + (q % R) * SLOT_FLOATS + f * HBOX;
  }
  __device__ __forceinline__ const float *point(int q, int f) const {
    return buf + (q % R) * SLOT_FLOATS + NH * HBOX + f * PBOX;
  }
};

// Leaves a CTA whose pipeline timed out: records the status, waits (bounded)
// for the copies it still has in flight, then every thread returns.  Best
// effort: if that wait runs out as well, a copy may still land in shared
// memory after the CTA has left (in another CTA's buffers), so once the
// status word reads EFWI_STATUS_TIMEOUT the host reports the whole call as
// failed and none of its device results may be used; every call zeroes the
// state, memory variables, images and traces it uses before its first
// kernel, so no stale value carries into the next call.
template <class Ring>
__device__ __forceinline__ void ring_abort(Ring &ring, int q, int nq, int R, int tid, int *status) {
  if (tid == 0) {
    atomicExch(status, EFWI_STATUS_TIMEOUT);
    for (int k = q; k < nq && k < q + R; ++k) ring.wait(k);
  }
  __syncthreads();
}

// Shared-memory accessor of one box around the thread's cell.
struct BoxView {
  const float *p;  // points at the thread's cell
  __device__ __forceinline__ float c() const { return p[0]; }
  __device__ __forceinline__ float x(int k) const { return p[k * TMA_BOXY]; }
  __device__ __forceinline__ float y(int k) const { return p[k]; }
};

}  // namespace efwi
