// C ABI of the engine (include/efwi.h): handle, workspace and the time
// loops of the forward and gradient calls.
//
// Structure of a call (compare cufd, Ops/FWI/Src_3d/libCUFD.cu:37-799):
//   - the model, coefficients and survey stay resident in HBM across calls
//     (the reference re-creates them, re-allocates 45 volumes and re-reads
//     the survey on every call, libCUFD.cu:52-205);
//   - forward-only calls advance up to `max_batch` shots per launch;
//   - the reference gradient runs shot by shot with the boundary shell
//     stored in HBM, and accumulates the images in shot order;
//   - the exact gradient runs shot by shot with binomial checkpoints of the
//     whole state in HBM under a byte budget (efwi_revolve.h).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "../../include/efwi.h"
#include "efwi_exact.h"
#include "efwi_fuse.cuh"
#include "efwi_kernels.h"
#include "efwi_revolve.h"

using namespace efwi;

namespace {

enum KClass {
  K_STRESS_FWD = 0,
  K_VELOCITY_FWD,
  K_REV_VELOCITY,
  K_REV_STRESS,
  K_RECORD,
  K_INJECT,
  K_SHELL_SAVE,
  K_SHELL_RESTORE,
  K_MISFIT,
  K_ADJ_STRESS,
  K_ADJ_VELOCITY,
  K_CHECKPOINT,
  K_OTHER,
  K_NCLASS
};
const char *kKernelNames[K_NCLASS] = {"stress_fwd", "velocity_fwd", "rev_velocity", "rev_stress",
                                      "record", "inject", "shell_save", "shell_restore",
                                      "misfit", "adj_stress", "adj_velocity", "checkpoint",
                                      "other"};

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  bool borrowed = false;  // a view of another handle's buffer: never freed here
  ~DevBuf() { if (p && !borrowed) cudaFree(p); }
  void view(const DevBuf &o) {
    if (p && !borrowed) cudaFree(p);
    p = o.p;
    bytes = o.bytes;
    borrowed = true;
  }
  void release() {
    if (p && !borrowed) cudaFree(p);
    p = nullptr;
    bytes = 0;
    borrowed = false;
  }
  cudaError_t ensure(size_t n) {
    if (n <= bytes) return cudaSuccess;
    if (p && !borrowed) cudaFree(p);
    p = nullptr; bytes = 0; borrowed = false;
    cudaError_t e = cudaMalloc(&p, n);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  template <class T> T *as() const { return static_cast<T *>(p); }
};

struct ShotHost {
  long long src_cell = -1;
  int nrec = 0;
  std::vector<long long> rec_cell;
  std::vector<float> win0, win1, wts;
  float src_w = 1.0f;
};

struct Pending {
  int cls;
  cudaEvent_t a, b;
};

// CUDA graph of one time loop, replayed while the launch parameters the
// loop bakes in (buffer addresses, tensor maps, tuning, time axis: the key)
// are unchanged -- across the shots of a call and across calls.
struct GraphCache {
  std::string key;
  cudaGraphExec_t exec = nullptr;
  long long launches[K_NCLASS] = {0};  // kernel launches of one replay, by class
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    key.clear();
  }
  ~GraphCache() { reset(); }
};

// Byte image of the values that make up a graph's key: scalars, pointers
// and padding-free structs (Fields, Psi, tensor maps) as they are; the
// structs with padding field by field.
struct KeyBytes {
  std::string s;
  template <class T>
  KeyBytes &add(const T &v) {
    s.append(reinterpret_cast<const char *>(&v), sizeof(T));
    return *this;
  }
  KeyBytes &rec(const RecArgs &r) {
    // the fused kernels read no count, only whether there are receivers
    const int n = r.plane ? (r.ncell > 0) : r.ncell;
    return add(r.ucell).add(r.ushot).add(r.uptr).add(r.rec).add(r.trace_off).add(r.nrec).add(n)
        .add(r.plane).add(r.map).add(r.nxpy);
  }
  KeyBytes &src(const SrcArgs &a) { return add(a.cell).add(a.stf).add(a.nt); }
  KeyBytes &shell(const ShellMap &m) {
    return add(m.rows).add(m.store).add(m.npts).add(m.ya0).add(m.ya1).add(m.yb0).add(m.yb1);
  }
  KeyBytes &geo(const Geo &g) {
    return add(g.nz).add(g.nx).add(g.ny).add(g.np).add(g.N).add(g.sz).add(g.sx).add(g.dt)
        .add(g.idz).add(g.idx).add(g.idy).add(g.slab_z).add(g.slab_x).add(g.slab_y).add(g.cz)
        .add(g.cx).add(g.cy);
  }
};

}  // namespace

struct EfwiHandle {
  EfwiGrid grid{};
  Geo geo{};
  long long N = 0;  // cells of one pitched volume
  int py = 0;       // y pitch
  int if_win = 0, bx = 4, zchunk = 8, max_batch = 4;
  int variant = 1;  // 0: L1-served stencils, 1: TMA-staged planes
  int fcfg = 0, rcfg = 0;  // launch configurations of the TMA kernels
  int zchunk_rev = 8;      // z planes per CTA of the reverse kernels
  int nt_limit = 0;        // > 0: time loops stop early (timing probes)
  std::string err;

  DevBuf coef, lam, mu, buoy;
  bool model_set = false;

  std::vector<ShotHost> shots;
  DevBuf stf, src_cell;
  bool survey_set = false;

  DevBuf pts;
  int npts = 0;
  // row table of the shell points for the save/restore fused into the TMA
  // stencil kernels (efwi_fuse.cuh); shell_fused false: separate kernels
  DevBuf shell_rows;
  ShellMap shm{};
  bool shell_fused = false;
  DevBuf recmap;  // per-plane receiver maps of the current batch

  DevBuf fields, psi, adj, traces_tm, res_tm, shell, partial, jdev, recbuf, winbuf, scalar, grad;
  DevBuf status;  // pipeline status word (EFWI_STATUS_*)

  // exact gradient: checkpoint slots and the two adjoint memory-variable sets
  DevBuf ckpt, apsi;
  // shot windows: per-domain volumes and tables; stream for graph capture
  DevBuf wvol, wtab, wstep;
  // windowed gradients: one sub-handle per window shape (its own grid and
  // C-PML), scratch for the window's observed data and images
  std::map<std::pair<int, int>, EfwiHandle *> wsub;
  DevBuf wobs, wimg, wsel;
  std::vector<float> stf_host;  // untapered source-time functions [nshot][nt]
  cudaStream_t cap_stream = nullptr;
  // shot windows on the TMA kernels: window groups run on their own streams
  cudaStream_t wst[8] = {};
  cudaEvent_t wev[9] = {};
  // shot lanes of reference-mode calls: sub-handles with their own
  // workspace and stream, each running a contiguous share of the shots
  int lanes = 2;
  std::vector<EfwiHandle *> lane;
  cudaStream_t own_st = nullptr;  // a lane's stream
  cudaEvent_t lane_fork = nullptr;
  long long ck_budget = 4LL << 30;  // bytes of checkpoint slots
  long long ck_forward_steps = 0;   // forward steps of the last exact gradient
  // optional outputs of the misfit: windowed synthetics / observed data
  float *scr_syn = nullptr, *scr_obs = nullptr, *scr_res = nullptr;
  // optional output of exact gradients: dJ/dstf [n][nt] of the call's shots
  float *gstf = nullptr;
  DevBuf stf_w2;  // taper factor w^2 of the source-time functions [nt]
  DevBuf scr_tm;
  int ck_slots = 0;                 // slots it used

  // time loops of reference-mode gradients and forward batches as CUDA
  // graphs (efwi_set_graphs; kernel-event sampling runs them eagerly)
  bool use_graphs = true;
  GraphCache g_fwd, g_rev;

  int prof_sample = 0;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<Pending> pending;
  long long launches[K_NCLASS] = {0};
  long long timed[K_NCLASS] = {0};
  double ms[K_NCLASS] = {0};
};

namespace {

int fail(EfwiHandle *h, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (h) h->err = buf;
  return code;
}

#define CK_CUDA(h, call)                                                              \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(h, e_ == cudaErrorMemoryAllocation ? EFWI_ERR_NOMEM : EFWI_ERR_CUDA, \
                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

// Reference C-PML profile (utilities.cu:204-320), evaluated with the
// reference's float variables and double intermediates.
void cpml_profile(int n, int npml, float dh, float f0, float dt, float *out6) {
  float *K = out6, *a = out6 + n, *b = out6 + 2 * n, *Kh = out6 + 3 * n, *ah = out6 + 4 * n,
        *bh = out6 + 5 * n;
  const double kPi = 3.141592653589793238462643383279502884197169;
  const float Rc = 0.0008f, Kmax = 2.0f, npow = 8.0f, vp = 3000.0f;
  const float amax = (float)(2.0 * kPi * (f0 / 2.0));
  const float L = npml * dh;
  const float d0 = (float)(-(npow + 1) * vp * std::log((double)Rc) / (2.0 * L));
  std::vector<float> d(n, 0.f), dhh(n, 0.f), al(n, 0.f), alh(n, 0.f);
  for (int i = 0; i < n; ++i) { K[i] = 1.f; Kh[i] = 1.f; a[i] = 0.f; ah[i] = 0.f; b[i] = 0.f; bh[i] = 0.f; }
  auto prof = [&](float depth, float &dd, float &KK, float &aa) {
    const float x = depth / L;
    dd = d0 * (float)(0.25 * x + 0.75 * std::pow((double)x, (double)npow));
    KK = (float)(1.0 + (Kmax - 1.0) * std::pow((double)x, (double)npow));
    aa = (float)(amax * (1.0 - x));
  };
  for (int i = 0; i < n; ++i) {
    float depth = (npml - i) * dh;
    if (depth >= 0.f) prof(depth, d[i], K[i], al[i]);
    depth = (float)((npml - i - 0.5) * dh);
    if (depth >= 0.f) prof(depth, dhh[i], Kh[i], alh[i]);
    depth = (npml - n + i) * dh;
    if (depth >= 0.f) prof(depth, d[i], K[i], al[i]);
    depth = (float)((npml - n + i + 0.5) * dh);
    if (depth >= 0.f) prof(depth, dhh[i], Kh[i], alh[i]);
    if (al[i] < 0.f) al[i] = 0.f;
    if (alh[i] < 0.f) alh[i] = 0.f;
    b[i] = std::exp(-(d[i] / K[i] + al[i]) * dt);
    bh[i] = std::exp(-(dhh[i] / Kh[i] + alh[i]) * dt);
    if (std::fabs(d[i]) > 1.0e-6) a[i] = (float)(d[i] * (b[i] - 1.0) / (K[i] * (d[i] + K[i] * al[i])));
    if (std::fabs(dhh[i]) > 1.0e-6)
      ah[i] = (float)(dhh[i] * (bh[i] - 1.0) / (Kh[i] * (dhh[i] + Kh[i] * alh[i])));
  }
}

// Source taper: cuda_window with nrec = 1 and ratio 0.001 (Src_Rec.cu:146,
// utilities.cu:578-614).
void taper_stf(const float *in, int nt, float dt, float *out) {
  const double kPi = 3.141592653589793238462643383279502884197169;
  const float ratio = 0.001f;
  const float t0 = 0.0f, t3 = nt * dt, off = nt * dt * ratio;
  const bool ok = !(2.0 * off >= t3 - t0);
  const float t1 = t0 + off, t2 = t3 - off;
  for (int it = 0; it < nt; ++it) {
    if (!ok) { out[it] = in[it]; continue; }
    const float t = it * dt;
    float w;
    if (t >= t0 && t < t1) w = (float)std::sin(kPi / 2.0 * (t - t0) / (t1 - t0));
    else if (t >= t1 && t < t2) w = 1.0f;
    else if (t >= t2 && t < t3) w = (float)std::cos(kPi / 2.0 * (t - t2) / (t3 - t2));
    else w = 0.0f;
    out[it] = in[it] * (w * w);
  }
}

// Shell points (Boundary.cu:14-20, utilities.cu:323-420): the box
// [npml-2, n-npml+1]^3 minus its part more than 4 cells inside every face.
// Points outside [2, n-3]^3 never change (they stay zero), so they are left
// out.
std::vector<int> shell_points(const EfwiGrid &g, int py) {
  std::vector<int> pts;
  const int lo = g.npml - 2;
  const int hz = g.nz - g.npml + 1, hx = g.nx - g.npml + 1, hy = g.ny - g.npml + 1;
  for (int z = std::max(lo, 2); z <= std::min(hz, g.nz - 3); ++z)
    for (int x = std::max(lo, 2); x <= std::min(hx, g.nx - 3); ++x)
      for (int y = std::max(lo, 2); y <= std::min(hy, g.ny - 3); ++y) {
        const bool in = z <= lo + 4 || z >= hz - 4 || x <= lo + 4 || x >= hx - 4 ||
                        y <= lo + 4 || y >= hy - 4;
        if (in) pts.push_back((int)(((long long)z * g.nx + x) * py + y));
      }
  return pts;
}

// Row table of the shell points (efwi_fuse.cuh): for every row (z, x) the
// index of its first point, with SHELL_SPLIT set when the row holds the two
// runs [ya0, ya1] and [yb0, yb1] instead of the one run [ya0, yb1].  Checked
// against the list point by point (a bijection between the cells the table
// names and the points); false when the points do not have that form.
bool shell_rows(const EfwiGrid &g, int py, const std::vector<int> &pts, std::vector<int> *rows,
                ShellMap *m) {
  rows->assign((size_t)g.nz * g.nx, -1);
  const int lo = g.npml - 2, hy = g.ny - g.npml + 1;
  m->ya0 = std::max(lo, 2);
  m->yb1 = std::min(hy, g.ny - 3);
  m->ya1 = std::min(lo + 4, m->yb1);
  m->yb0 = std::max(hy - 4, m->ya0);
  const bool can_split = m->ya1 + 1 < m->yb0;
  const long long nsplit = (m->ya1 - m->ya0 + 1) + (m->yb1 - m->yb0 + 1);
  m->npts = (int)pts.size();
  if (pts.size() >= (size_t)SHELL_SPLIT) return false;
  size_t k = 0;
  while (k < pts.size()) {
    const int zx = pts[k] / py;
    size_t e = k;
    while (e < pts.size() && pts[e] / py == zx) ++e;
    const long long cnt = (long long)(e - k);
    if (pts[k] % py != m->ya0) return false;
    if (cnt == m->yb1 - m->ya0 + 1) (*rows)[zx] = (int)k;
    else if (can_split && cnt == nsplit) (*rows)[zx] = (int)k | SHELL_SPLIT;
    else return false;
    k = e;
  }
  long long named = 0;
  for (long long zx = 0; zx < (long long)g.nz * g.nx; ++zx) {
    const int row = (*rows)[zx];
    if (row < 0) continue;
    for (int y = 0; y < g.ny; ++y) {
      const int q = shell_index(*m, row, y);
      if (q < 0) continue;
      if (q >= (int)pts.size() || pts[q] != (int)(zx * py + y)) return false;
      ++named;
    }
  }
  return named == (long long)pts.size();
}

// out[c][j][t] = obs[c][sel[j]][t]: the observed data of the receivers
// that lie inside a window (traces layout [3][nrec][nt]).
__global__ void k_gather_rows(const float *obs, const int *sel, int nsel, int nrec, int nt,
                              float *out) {
  const long long n = 3LL * nsel * nt;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(i % nt);
    const long long cj = i / nt;
    const int j = (int)(cj % nsel), c = (int)(cj / nsel);
    out[i] = obs[((long long)c * nrec + sel[j]) * nt + t];
  }
}

// g[z][x0 + x][y0 + y] += w[z][x][y] (caller layouts, no pitch).
__global__ void k_window_add(float *g, const float *w, int nz, int nx, int ny, int x0, int y0,
                             int nxw, int nyw) {
  const long long n = (long long)nz * nxw * nyw;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % nyw);
    const long long zx = i / nyw;
    const int x = (int)(zx % nxw), z = (int)(zx / nxw);
    g[((long long)z * nx + x0 + x) * ny + y0 + y] += w[i];
  }
}

// Step counter of a time loop replayed from a graph of one step.
__global__ void k_step_advance(int *it) { if (threadIdx.x == 0 && blockIdx.x == 0) ++*it; }

__global__ void k_add(float *__restrict__ dst, const float *__restrict__ src, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] += src[i];
}

__global__ void k_max_vp(const float *lam, const float *mu, const float *rho, long long n,
                         unsigned int *out) {
  float m = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float v = sqrtf((lam[i] + 2.0f * mu[i]) / rho[i]);
    if (v > m) m = v;
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

cudaEvent_t next_event(EfwiHandle *h) {
  if (h->ev_used == h->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    h->ev_pool.push_back(e);
  }
  return h->ev_pool[h->ev_used++];
}

// Launch bracket: counts launches and, on sampled steps, records events.
struct Timer {
  EfwiHandle *h;
  int cls;
  cudaStream_t s;
  bool on;
  cudaEvent_t a{}, b{};
  Timer(EfwiHandle *h_, int cls_, cudaStream_t s_, int it) : h(h_), cls(cls_), s(s_) {
    h->launches[cls]++;
    // steps it = s/2, s/2 + s, ...: the first and last steps of a sweep
    // (it = 0 has no adjoint update) stay out of the sample when s > 1;
    // launches outside the time loop (it < 0) are always timed
    on = h->prof_sample > 0 && (it < 0 || it % h->prof_sample == h->prof_sample / 2);
    if (on) { a = next_event(h); b = next_event(h); cudaEventRecord(a, s); }
  }
  ~Timer() {
    if (on) { cudaEventRecord(b, s); h->pending.push_back({cls, a, b}); }
  }
};

int check_launch(EfwiHandle *h, const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(h, EFWI_ERR_CUDA, "launch of %s failed: %s", what, cudaGetErrorString(e));
  return EFWI_OK;
}

// Runs `body(stream)` -- a time loop of kernel launches with no host
// synchronisation -- through the graph cache `gc`: replays the cached graph
// when its key matches, otherwise captures body on the handle's capture
// stream, instantiates it and replays it.  Launches are counted per replay.
// Eager (body on st) when graphs are off or kernel events are sampled.
template <class Body>
int run_graphed(EfwiHandle *h, GraphCache &gc, const std::string &key, cudaStream_t st,
                Body body) {
  if (!h->use_graphs || h->prof_sample > 0) return body(st);
  if (!h->cap_stream) CK_CUDA(h, cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking));
  if (!gc.exec || gc.key != key) {
    gc.reset();
    long long before[K_NCLASS];
    std::memcpy(before, h->launches, sizeof(before));
    cudaGraph_t graph = nullptr;
    CK_CUDA(h, cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeThreadLocal));
    const int rc = body(h->cap_stream);
    cudaError_t ec = cudaStreamEndCapture(h->cap_stream, &graph);
    for (int k = 0; k < K_NCLASS; ++k) {
      gc.launches[k] = h->launches[k] - before[k];
      h->launches[k] = before[k];
    }
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      return rc;
    }
    if (ec == cudaSuccess) ec = cudaGraphInstantiate(&gc.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (ec != cudaSuccess) {
      gc.reset();
      return fail(h, EFWI_ERR_CUDA, "graph of a time loop: %s", cudaGetErrorString(ec));
    }
    gc.key = key;
  }
  CK_CUDA(h, cudaGraphLaunch(gc.exec, st));
  for (int k = 0; k < K_NCLASS; ++k) h->launches[k] += gc.launches[k];
  return EFWI_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int get_encoder(EfwiHandle *h) {
  if (g_encode) return EFWI_OK;
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
    return fail(h, EFWI_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
  return EFWI_OK;
}

// Tensor map of S stacked pitched volumes [S*nz][nx][py]; halo boxes of
// 40 (y) x (bx + 4) (x) x 1 plane, or point boxes of 32 x bx x 1.
// Tensor map of one field over volumes of pitch py, nx rows and nzs planes.
int make_map_dims(EfwiHandle *h, CUtensorMap *m, const float *base, int py, int nx, long long nzs,
                  bool halo, int bx) {
  int rc = get_encoder(h);
  if (rc) return rc;
  if (((uintptr_t)base & 15) != 0 || (py & 3) != 0)
    return fail(h, EFWI_ERR_ARG, "tensor map base or pitch not 16-byte aligned");
  cuuint64_t dims[3] = {(cuuint64_t)py, (cuuint64_t)nx, (cuuint64_t)nzs};
  cuuint64_t strides[2] = {(cuuint64_t)py * 4, (cuuint64_t)nx * py * 4};
  cuuint32_t box[3] = {halo ? (cuuint32_t)TMA_BOXY : 32u,
                       (cuuint32_t)(halo ? bx + 2 * TMA_HX : bx), 1};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(h, EFWI_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return EFWI_OK;
}

int make_map(EfwiHandle *h, CUtensorMap *m, const float *base, int S, bool halo, int bx) {
  return make_map_dims(h, m, base, h->py, h->grid.nx, (long long)h->grid.nz * S, halo, bx);
}

// Resets the status word at the start of a call.
int status_reset(EfwiHandle *h, cudaStream_t st) {
  CK_CUDA(h, h->status.ensure(sizeof(int)));
  CK_CUDA(h, cudaMemsetAsync(h->status.p, 0, sizeof(int), st));
  return EFWI_OK;
}

// Reads the status word (synchronises the stream).
int status_check(EfwiHandle *h, cudaStream_t st) {
  int v = 0;
  CK_CUDA(h, cudaMemcpyAsync(&v, h->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK_CUDA(h, cudaStreamSynchronize(st));
  if (v != EFWI_STATUS_OK) return fail(h, EFWI_ERR_CUDA, "a bulk-copy pipeline wait timed out");
  return EFWI_OK;
}

struct FwdMaps {
  Maps<11> s;  // vz vx vy | szz sxx syy sxz sxy syz | lam mu
  Maps<9> v;   // sxz syz sxx sxy syy | vz vx vy | buoy
};

Fields fields_at(float *base, long long N, int S) {
  // volumes of a batch of S shots: 9 arrays of S*N floats
  Fields f;
  const long long v = N * S;
  f.vz = base; f.vx = base + v; f.vy = base + 2 * v;
  f.szz = base + 3 * v; f.sxx = base + 4 * v; f.syy = base + 5 * v;
  f.sxz = base + 6 * v; f.sxy = base + 7 * v; f.syz = base + 8 * v;
  return f;
}

long long psi_per_shot(const Geo &g) { return 6 * (g.slab_z + g.slab_x + g.slab_y); }

Psi psi_at(float *base, const Geo &g, int S) {
  Psi p;
  p.z = base;
  p.x = base + (long long)S * 6 * g.slab_z;
  p.y = p.x + (long long)S * 6 * g.slab_x;
  return p;
}

// Receivers of a batch, grouped by (shot, cell).
struct RecHost {
  std::vector<long long> ucell, trace_off;
  std::vector<int> ushot, uptr, rec, nrec;
};

RecHost group_receivers(const EfwiHandle *h, const int *ids, int S, long long *total_floats) {
  RecHost r;
  long long off = 0;
  for (int s = 0; s < S; ++s) {
    const ShotHost &sh = h->shots[ids[s]];
    r.trace_off.push_back(off);
    r.nrec.push_back(sh.nrec);
    off += 3LL * sh.nrec * h->grid.nt;
    std::vector<std::pair<long long, int>> cr;
    for (int k = 0; k < sh.nrec; ++k) cr.push_back({sh.rec_cell[k], k});
    std::sort(cr.begin(), cr.end());
    for (size_t k = 0; k < cr.size(); ++k) {
      if (k == 0 || cr[k].first != cr[k - 1].first) {
        r.ucell.push_back(cr[k].first);
        r.ushot.push_back(s);
        r.uptr.push_back((int)r.rec.size());
      }
      r.rec.push_back(cr[k].second);
    }
  }
  r.uptr.push_back((int)r.rec.size());
  *total_floats = off;
  return r;
}

// Uploads the grouping into h->recbuf and returns device views.
int upload_receivers(EfwiHandle *h, const RecHost &r, cudaStream_t st, RecArgs *out) {
  auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t b0 = al(r.ucell.size() * 8), b1 = al(r.trace_off.size() * 8),
               b2 = al(r.ushot.size() * 4), b3 = al(r.uptr.size() * 4), b4 = al(r.rec.size() * 4 + 4),
               b5 = al(r.nrec.size() * 4);
  CK_CUDA(h, h->recbuf.ensure(b0 + b1 + b2 + b3 + b4 + b5));
  char *p = h->recbuf.as<char>();
  CK_CUDA(h, cudaMemcpyAsync(p, r.ucell.data(), r.ucell.size() * 8, cudaMemcpyHostToDevice, st));
  CK_CUDA(h, cudaMemcpyAsync(p + b0, r.trace_off.data(), r.trace_off.size() * 8, cudaMemcpyHostToDevice, st));
  CK_CUDA(h, cudaMemcpyAsync(p + b0 + b1, r.ushot.data(), r.ushot.size() * 4, cudaMemcpyHostToDevice, st));
  CK_CUDA(h, cudaMemcpyAsync(p + b0 + b1 + b2, r.uptr.data(), r.uptr.size() * 4, cudaMemcpyHostToDevice, st));
  if (!r.rec.empty())
    CK_CUDA(h, cudaMemcpyAsync(p + b0 + b1 + b2 + b3, r.rec.data(), r.rec.size() * 4, cudaMemcpyHostToDevice, st));
  CK_CUDA(h, cudaMemcpyAsync(p + b0 + b1 + b2 + b3 + b4, r.nrec.data(), r.nrec.size() * 4, cudaMemcpyHostToDevice, st));
  out->ucell = (const long long *)p;
  out->trace_off = (const long long *)(p + b0);
  out->ushot = (const int *)(p + b0 + b1);
  out->uptr = (const int *)(p + b0 + b1 + b2);
  out->rec = (const int *)(p + b0 + b1 + b2 + b3);
  out->nrec = (const int *)(p + b0 + b1 + b2 + b3 + b4);
  out->ncell = (int)r.ucell.size();
  // Per-plane maps of the unique receiver cells for the gather / injection
  // fused into the TMA stencil kernels; none for the L1 kernels, or when
  // the receivers spread over so many planes that the maps would pass
  // 64 Mi cells (the separate kernels run then).
  out->plane = nullptr;
  out->map = nullptr;
  const int nz = h->grid.nz;
  const long long nxpy = (long long)h->grid.nx * h->py;
  out->nxpy = (int)nxpy;
  const int S = (int)r.trace_off.size();
  if (h->variant == 1 && !r.ucell.empty()) {
    std::vector<int> plane((size_t)S * nz, -1);
    int nmaps = 0;
    for (size_t u = 0; u < r.ucell.size(); ++u) {
      int &m = plane[(size_t)r.ushot[u] * nz + (int)(r.ucell[u] / nxpy)];
      if (m < 0) m = nmaps++;
    }
    if ((long long)nmaps * nxpy <= (64LL << 20)) {
      std::vector<int> maps((size_t)nmaps * nxpy, -1);
      for (size_t u = 0; u < r.ucell.size(); ++u) {
        const int m = plane[(size_t)r.ushot[u] * nz + (int)(r.ucell[u] / nxpy)];
        maps[(size_t)m * nxpy + (size_t)(r.ucell[u] % nxpy)] = (int)u;
      }
      const size_t pb = al(plane.size() * 4);
      CK_CUDA(h, h->recmap.ensure(pb + maps.size() * 4));
      char *q = h->recmap.as<char>();
      CK_CUDA(h, cudaMemcpyAsync(q, plane.data(), plane.size() * 4, cudaMemcpyHostToDevice, st));
      CK_CUDA(h, cudaMemcpyAsync(q + pb, maps.data(), maps.size() * 4, cudaMemcpyHostToDevice, st));
      out->plane = (const int *)q;
      out->map = (const int *)(q + pb);
    }
  }
  return EFWI_OK;
}

int check_ready(EfwiHandle *h, int n, const int *ids) {
  if (!h) return EFWI_ERR_ARG;
  if (!h->model_set) return fail(h, EFWI_ERR_STATE, "efwi_set_model has not been called");
  if (!h->survey_set) return fail(h, EFWI_ERR_STATE, "efwi_set_survey has not been called");
  if (n < 0 || (n > 0 && !ids)) return fail(h, EFWI_ERR_ARG, "invalid shot list");
  for (int k = 0; k < n; ++k)
    if (ids[k] < 0 || ids[k] >= (int)h->shots.size())
      return fail(h, EFWI_ERR_ARG, "shot id %d out of range [0, %d)", ids[k], (int)h->shots.size());
  return EFWI_OK;
}

dim3 stencil_grid(const EfwiHandle *h, int S, int bx, int zchunk, int *nzc) {
  *nzc = (h->grid.nz + zchunk - 1) / zchunk;
  return dim3((h->grid.ny + 31) / 32, (h->grid.nx + bx - 1) / bx, (unsigned)(S * *nzc));
}

int nt_eff(const EfwiHandle *h) {
  return h->nt_limit > 0 && h->nt_limit < h->grid.nt ? std::max(h->nt_limit, 2) : h->grid.nt;
}

// One forward time step of a batch: stress (+ source), velocity, receivers.
// With `shell` set (one shot), the boundary shell of the step's starting
// state is stored there first.  On the TMA kernels the shell store and the
// receiver gather run in the stencil kernels' epilogues; otherwise as
// separate launches.
int forward_step(EfwiHandle *h, Fields f, Psi ps, int S, const SrcArgs &src, const RecArgs &rec,
                 float *traces_tm, cudaStream_t st, int it, const FwdMaps *maps,
                 float *shell = nullptr) {
  int nzc;
  const int bx = maps ? fwd_tma_tile(h->fcfg) : h->bx;
  const dim3 grid = stencil_grid(h, S, bx, h->zchunk, &nzc);
  int *status = h->status.as<int>();
  ShellMap shm{};
  if (shell && h->npts > 0) {
    if (maps && h->shell_fused) {
      shm = h->shm;
      shm.store = shell;
    } else {
      Timer t(h, K_SHELL_SAVE, st, it);
      k_shell_save<<<(h->npts + 255) / 256, 256, 0, st>>>(f, h->pts.as<int>(), h->npts, shell);
    }
  }
  RecFuse rf{};
  const bool rec_fused = maps && rec.ncell > 0 && rec.plane;
  if (rec_fused) rf = RecFuse{rec, traces_tm, it + 1};
  {
    Timer t(h, K_STRESS_FWD, st, it);
    if (maps)
      launch_stress_fwd_tma(h->fcfg, grid, st, maps->s, h->geo, f, ps, h->zchunk, nzc, src, shm,
                            status);
    else
      launch_stress_fwd(h->bx, grid, st, h->geo, f, ps, h->lam.as<float>(), h->mu.as<float>(),
                        h->zchunk, nzc, src);
  }
  {
    Timer t(h, K_VELOCITY_FWD, st, it);
    if (maps)
      launch_velocity_fwd_tma(h->fcfg, grid, st, maps->v, h->geo, f, ps, h->zchunk, nzc, rf,
                              status);
    else
      launch_velocity_fwd(h->bx, grid, st, h->geo, f, ps, h->buoy.as<float>(), h->zchunk, nzc);
  }
  if (rec.ncell > 0 && !rec_fused) {
    Timer t(h, K_RECORD, st, it);
    k_record<<<(rec.ncell + 127) / 128, 128, 0, st>>>(f, h->N, rec, traces_tm, it + 1);
  }
  return check_launch(h, "forward step");
}

// Tensor maps of the forward kernels over the batch volumes f.
int make_fwd_maps(EfwiHandle *h, const Fields &f, int S, FwdMaps *maps) {
  const float *sm[11] = {f.vz, f.vx, f.vy, f.szz, f.sxx, f.syy, f.sxz, f.sxy, f.syz,
                         h->lam.as<float>(), h->mu.as<float>()};
  const float *vm[9] = {f.sxz, f.syz, f.sxx, f.sxy, f.syy, f.vz, f.vx, f.vy, h->buoy.as<float>()};
  const int bxf = fwd_tma_tile(h->fcfg);
  for (int k = 0; k < 11; ++k) {
    int rc = make_map(h, &maps->s.m[k], sm[k], k < 9 ? S : 1, k < 3, bxf);
    if (rc) return rc;
  }
  for (int k = 0; k < 9; ++k) {
    int rc = make_map(h, &maps->v.m[k], vm[k], k < 8 ? S : 1, k < 5, bxf);
    if (rc) return rc;
  }
  return EFWI_OK;
}

// Zeroed state, receivers, source rows and tensor maps of a batch of S
// shots (ids) whose traces go to traces_tm (time-major, zeroed here).
struct Batch {
  Fields f;
  Psi ps;
  RecArgs rec;
  SrcArgs src;
  FwdMaps maps;
  const FwdMaps *mp = nullptr;
};

int prepare_batch(EfwiHandle *h, const int *ids, int S, float *traces_tm, long long ntr,
                  cudaStream_t st, Batch *b) {
  const long long N = h->N;
  CK_CUDA(h, h->fields.ensure(sizeof(float) * 9 * N * S));
  CK_CUDA(h, h->psi.ensure(sizeof(float) * psi_per_shot(h->geo) * S));
  CK_CUDA(h, cudaMemsetAsync(h->fields.p, 0, sizeof(float) * 9 * N * S, st));
  CK_CUDA(h, cudaMemsetAsync(h->psi.p, 0, sizeof(float) * psi_per_shot(h->geo) * S, st));
  CK_CUDA(h, cudaMemsetAsync(traces_tm, 0, sizeof(float) * ntr, st));
  b->f = fields_at(h->fields.as<float>(), N, S);
  b->ps = psi_at(h->psi.as<float>(), h->geo, S);

  long long tot;
  RecHost rh = group_receivers(h, ids, S, &tot);
  int rc = upload_receivers(h, rh, st, &b->rec);
  if (rc) return rc;

  // per-batch source arrays: cells and tapered stf rows, staged in scalar buf
  const int nt = h->grid.nt;
  CK_CUDA(h, h->scalar.ensure(sizeof(long long) * S + sizeof(float) * (size_t)S * nt + 256));
  std::vector<long long> cells(S);
  for (int s = 0; s < S; ++s) cells[s] = h->shots[ids[s]].src_cell;
  long long *dcell = h->scalar.as<long long>();
  float *dstf = (float *)((char *)h->scalar.p + ((sizeof(long long) * S + 255) & ~size_t(255)));
  CK_CUDA(h, cudaMemcpyAsync(dcell, cells.data(), sizeof(long long) * S, cudaMemcpyHostToDevice, st));
  for (int s = 0; s < S; ++s)
    CK_CUDA(h, cudaMemcpyAsync(dstf + (size_t)s * nt, h->stf.as<float>() + (size_t)ids[s] * nt,
                               sizeof(float) * nt, cudaMemcpyDeviceToDevice, st));
  b->src = SrcArgs{dcell, dstf, nt, 0};
  b->mp = nullptr;
  if (h->variant == 1) {
    rc = make_fwd_maps(h, b->f, S, &b->maps);
    if (rc) return rc;
    b->mp = &b->maps;
  }
  return EFWI_OK;
}

// Forward of a batch of S shots (ids) into traces_tm (time-major, zeroed
// here).  When `shell` is set (S must be 1) the boundary shell is stored
// before every step.
int run_forward_batch(EfwiHandle *h, const int *ids, int S, float *traces_tm, long long ntr,
                      RecArgs *rec_out, float *shell, cudaStream_t st) {
  Batch b;
  int rc = prepare_batch(h, ids, S, traces_tm, ntr, st, &b);
  if (rc) return rc;
  if (rec_out) *rec_out = b.rec;
  const int npts = h->npts;
  const int ntl = nt_eff(h);
  auto loop = [&](cudaStream_t s) -> int {
    for (int it = 0; it <= ntl - 2; ++it) {
      b.src.it = it;
      const int r = forward_step(h, b.f, b.ps, S, b.src, b.rec, traces_tm, s, it, b.mp,
                                 shell ? shell + (size_t)it * 9 * npts : nullptr);
      if (r) return r;
    }
    return check_launch(h, "forward");
  };
  KeyBytes key;
  key.add(b.f).add(b.ps).rec(b.rec).src(b.src).add(S).add(ntl).add(traces_tm).add(shell)
      .add(npts).add(h->fcfg).add(h->zchunk).add(h->bx).add(h->variant).geo(h->geo)
      .shell(h->shm).add(h->shell_fused).add(h->status.p).add(h->lam.p).add(h->mu.p)
      .add(h->buoy.p);
  if (b.mp) key.add(b.maps);
  return run_graphed(h, h->g_fwd, key.s, st, loop);
}

int resolve_profile(EfwiHandle *h) {
  for (const Pending &p : h->pending) {
    float t = 0.f;
    cudaError_t e = cudaEventSynchronize(p.b);
    if (e != cudaSuccess) return fail(h, EFWI_ERR_CUDA, "profile event: %s", cudaGetErrorString(e));
    cudaEventElapsedTime(&t, p.a, p.b);
    h->ms[p.cls] += t;
    h->timed[p.cls]++;
  }
  h->pending.clear();
  h->ev_used = 0;
  return EFWI_OK;
}

// Misfit of one shot: fills res_tm and adds the sum of squares to *jdev.
// With efwi_set_scratch outputs set, also writes the windowed synthetics
// and observed data of the shot at traces offset `off`.
int misfit_shot(EfwiHandle *h, const ShotHost &sh, const float *obs, const float *syn_tm,
                float *res_tm, double *jdev, cudaStream_t st, long long off) {
  const int nt = h->grid.nt, nr = sh.nrec;
  if (nr == 0) return EFWI_OK;
  dim3 grid((nt + 31) / 32, (nr + 31) / 32, 3);
  const int nb = grid.x * grid.y * grid.z;
  CK_CUDA(h, h->partial.ensure(sizeof(double) * nb));
  MisfitArgs m{};
  m.nt = nt; m.nrec = nr; m.dt = h->grid.dt; m.if_win = h->if_win; m.src_weight = sh.src_w;
  if (h->if_win) {
    CK_CUDA(h, h->winbuf.ensure(sizeof(float) * 3 * nr));
    float *w = h->winbuf.as<float>();
    CK_CUDA(h, cudaMemcpyAsync(w, sh.win0.data(), sizeof(float) * nr, cudaMemcpyHostToDevice, st));
    CK_CUDA(h, cudaMemcpyAsync(w + nr, sh.win1.data(), sizeof(float) * nr, cudaMemcpyHostToDevice, st));
    CK_CUDA(h, cudaMemcpyAsync(w + 2 * nr, sh.wts.data(), sizeof(float) * nr, cudaMemcpyHostToDevice, st));
    m.win_start = w; m.win_end = w + nr; m.weights = w + 2 * nr;
  }
  const long long ntr = 3LL * nr * nt;
  if (h->scr_syn || h->scr_obs) {
    CK_CUDA(h, h->scr_tm.ensure(sizeof(float) * 2 * ntr));
    m.syn_w = h->scr_tm.as<float>();
    m.obs_w = m.syn_w + ntr;
  }
  {
    Timer t(h, K_MISFIT, st, -1);
    k_misfit<<<grid, dim3(32, 8), 0, st>>>(m, obs, syn_tm, res_tm, h->partial.as<double>());
    k_reduce_sum<<<1, 256, 0, st>>>(h->partial.as<double>(), nb, jdev);
  }
  const dim3 tg((nt + 31) / 32, (nr + 31) / 32, 3);
  if (h->scr_syn) k_traces_to_cr_t<<<tg, dim3(32, 8), 0, st>>>(m.syn_w, h->scr_syn + off, nt, nr);
  if (h->scr_obs) k_traces_to_cr_t<<<tg, dim3(32, 8), 0, st>>>(m.obs_w, h->scr_obs + off, nt, nr);
  if (h->scr_res) k_traces_to_cr_t<<<tg, dim3(32, 8), 0, st>>>(res_tm, h->scr_res + off, nt, nr);
  return check_launch(h, "misfit");
}

// Floats of one checkpoint: 9 fields and the memory variables of one shot.
long long state_floats(const EfwiHandle *h) { return 9 * h->N + psi_per_shot(h->geo); }

// Checkpoint slots the budget allows for a run of `blocks` states
// (S_0 is the zero state and needs none).
int checkpoint_slots(const EfwiHandle *h, int blocks) {
  const long long per = state_floats(h) * (long long)sizeof(float);
  long long s = per > 0 ? h->ck_budget / per : 0;
  if (s > blocks - 1) s = blocks - 1;
  return (int)std::max(s, 0LL);
}

// Adjoint kernels' arguments over the engine's single-shot buffers.
ExactArgs exact_args(EfwiHandle *h, const Fields &f, const Psi &ps, const Fields &a, int par,
                     float *g0, float *g1) {
  ExactArgs A;
  A.g = h->geo;
  A.f = f;
  A.ps = ps;
  A.a = a;
  const long long P = psi_per_shot(h->geo);
  A.lin = psi_at(h->apsi.as<float>() + par * P, h->geo, 1);
  A.lout = psi_at(h->apsi.as<float>() + (1 - par) * P, h->geo, 1);
  A.lam = h->lam.as<float>();
  A.mu = h->mu.as<float>();
  A.buoy = h->buoy.as<float>();
  A.g0 = g0;
  A.g1 = g1;
  return A;
}

// Exact gradient of one shot (EFWI_MODE_EXACT).  Forward states are
// recomputed from binomial checkpoints (efwi_revolve.h); the first sweep
// records the traces, then the misfit gives the adjoint source and block k
// (k = nt-1 .. 0, state S_k current) runs
//   transpose of stress stage k (+ lambda, mu images)      if k <= nt-2
//   adjoint source -2 * res at sample k                    if k >= 1
//   transpose of velocity stage k-1 (+ buoyancy image)     if k >= 1.
// glam, gmu, gB: pitched image accumulators.  With `adj_source` set, obs
// holds the adjoint source itself (the derivative of some objective with
// respect to the traces, traces layout): no misfit is formed and the source
// is injected as it is, so the images are J^T applied to it.
int exact_shot(EfwiHandle *h, int id, const float *obs, double *jdev, float *res_out,
               float *glam, float *gmu, float *gB, cudaStream_t st, bool adj_source = false,
               long long scratch_off = 0, float *gstf_row = nullptr) {
  const int nt = h->grid.nt;
  const int ntl = nt_eff(h);
  const long long N = h->N;
  const long long P = psi_per_shot(h->geo);
  const ShotHost &sh = h->shots[id];
  const long long ntr = 3LL * sh.nrec * nt;
  CK_CUDA(h, h->traces_tm.ensure(sizeof(float) * std::max(ntr, 1LL)));
  CK_CUDA(h, h->res_tm.ensure(sizeof(float) * std::max(ntr, 1LL)));
  CK_CUDA(h, h->adj.ensure(sizeof(float) * 9 * N));
  CK_CUDA(h, h->apsi.ensure(sizeof(float) * 2 * P));

  const int slots = checkpoint_slots(h, ntl);
  CkPlan plan;
  plan.build(ntl, slots, 64LL * ntl + 4096);
  if (plan.too_long || plan.forward_steps > 16LL * ntl)
    return fail(h, EFWI_ERR_TOO_LARGE,
                "checkpoint budget of %lld bytes (%d slots of %lld bytes) is too small for %d steps",
                h->ck_budget, slots, state_floats(h) * 4, ntl);
  const long long SF = state_floats(h);
  CK_CUDA(h, h->ckpt.ensure(sizeof(float) * std::max(1LL, (long long)plan.slots_used * SF)));
  h->ck_forward_steps = plan.forward_steps;
  h->ck_slots = plan.slots_used;

  Batch b;
  int rc = prepare_batch(h, &id, 1, h->traces_tm.as<float>(), ntr, st, &b);
  if (rc) return rc;
  Fields a = fields_at(h->adj.as<float>(), N, 1);
  CK_CUDA(h, cudaMemsetAsync(h->adj.p, 0, sizeof(float) * 9 * N, st));
  CK_CUDA(h, cudaMemsetAsync(h->apsi.p, 0, sizeof(float) * 2 * P, st));
  RecArgs norec = b.rec;
  norec.ncell = 0;
  float *state = h->fields.as<float>();  // [9N fields][P memory variables]
  float *psi = h->psi.as<float>();
  float *ck = h->ckpt.as<float>();
  int nzc;
  const int zc = h->zchunk_rev;
  const int bxe = h->bx;
  const dim3 grid = stencil_grid(h, 1, bxe, zc, &nzc);
  // adjoint kernels with bulk-copy staged planes (TMA variant): tensor maps
  // over this shot's buffers
  const bool etma = h->variant == 1 && (bxe == 4 || bxe == 8);
  Maps<11> mes;
  Maps<10> mev;
  if (etma) {
    const float *hs[11] = {a.szz, a.sxx, a.syy, a.sxz, a.sxy, a.syz, h->lam.as<float>(),
                           h->mu.as<float>(), b.f.vz, b.f.vx, b.f.vy};
    const float *hv[10] = {a.vz, a.vx, a.vy, h->buoy.as<float>(), b.f.sxz, b.f.sxx, b.f.sxy,
                           b.f.syz, b.f.syy, b.f.szz};
    for (int k2 = 0; k2 < 11 && rc == 0; ++k2) rc = make_map(h, &mes.m[k2], hs[k2], 1, true, bxe);
    for (int k2 = 0; k2 < 10 && rc == 0; ++k2) rc = make_map(h, &mev.m[k2], hv[k2], 1, true, bxe);
    if (rc) return rc;
  }
  int *status = h->status.as<int>();
  int par_s = 0, par_v = 0;
  bool first = true;
  for (const CkAction &act : plan.actions) {
    if (act.op == CK_ADVANCE) {
      for (int it = act.a; it < act.b; ++it) {
        b.src.it = it;
        rc = forward_step(h, b.f, b.ps, 1, b.src, first ? b.rec : norec, h->traces_tm.as<float>(),
                          st, it, b.mp);
        if (rc) return rc;
      }
    } else if (act.op == CK_STORE) {
      Timer t(h, K_CHECKPOINT, st, -1);
      float *dst = ck + (long long)act.a * SF;
      CK_CUDA(h, cudaMemcpyAsync(dst, state, sizeof(float) * 9 * N, cudaMemcpyDeviceToDevice, st));
      CK_CUDA(h, cudaMemcpyAsync(dst + 9 * N, psi, sizeof(float) * P, cudaMemcpyDeviceToDevice, st));
    } else if (act.op == CK_RESTORE) {
      Timer t(h, K_CHECKPOINT, st, -1);
      if (act.a < 0) {
        CK_CUDA(h, cudaMemsetAsync(state, 0, sizeof(float) * 9 * N, st));
        CK_CUDA(h, cudaMemsetAsync(psi, 0, sizeof(float) * P, st));
      } else {
        const float *src = ck + (long long)act.a * SF;
        CK_CUDA(h, cudaMemcpyAsync(state, src, sizeof(float) * 9 * N, cudaMemcpyDeviceToDevice, st));
        CK_CUDA(h, cudaMemcpyAsync(psi, src + 9 * N, sizeof(float) * P, cudaMemcpyDeviceToDevice, st));
      }
    } else {  // CK_BLOCK
      const int k = act.a;
      if (first && adj_source) {
        first = false;
        if (sh.nrec > 0) {
          k_traces_to_tm<<<dim3((nt + 31) / 32, (sh.nrec + 31) / 32, 3), dim3(32, 8), 0, st>>>(
              obs, h->res_tm.as<float>(), nt, sh.nrec);
          h->launches[K_OTHER]++;
        }
      }
      if (first) {
        first = false;
        rc = misfit_shot(h, sh, obs, h->traces_tm.as<float>(), h->res_tm.as<float>(), jdev, st,
                         scratch_off);
        if (rc) return rc;
        if (res_out && sh.nrec > 0) {
          k_traces_to_cr_t<<<dim3((nt + 31) / 32, (sh.nrec + 31) / 32, 3), dim3(32, 8), 0, st>>>(
              h->res_tm.as<float>(), res_out, nt, sh.nrec);
          h->launches[K_OTHER]++;
        }
      }
      if (k <= ntl - 2 && gstf_row) {
        // the source of step k adds to the stresses after the stress stage
        // of step k: its adjoint is read before that stage's transpose
        k_stf_gradient<<<1, 32, 0, st>>>(a, b.src.cell, h->stf_w2.as<float>(), gstf_row, k,
                                         2250000.0f * h->grid.dt);
        h->launches[K_OTHER]++;
      }
      if (k <= ntl - 2) {
        Timer t(h, K_ADJ_STRESS, st, k);
        const ExactArgs A = exact_args(h, b.f, b.ps, a, par_s, glam, gmu);
        if (etma) launch_adj_stress_tma(bxe, grid, st, mes, A, zc, status);
        else launch_adj_stress_exact(bxe, grid, st, A, zc, nzc);
        par_s ^= 1;
      }
      if (k >= 1) {
        if (b.rec.ncell > 0) {
          Timer t(h, K_INJECT, st, k);
          k_inject<<<(b.rec.ncell + 127) / 128, 128, 0, st>>>(a, N, b.rec, h->res_tm.as<float>(), k,
                                                              adj_source ? 1.0f : -2.0f);
        }
        Timer t(h, K_ADJ_VELOCITY, st, k);
        const ExactArgs A = exact_args(h, b.f, b.ps, a, par_v, gB, nullptr);
        if (etma) launch_adj_velocity_tma(bxe, grid, st, mev, A, zc, status);
        else launch_adj_velocity_exact(bxe, grid, st, A, zc, nzc);
        par_v ^= 1;
      }
    }
  }
  return check_launch(h, "exact gradient");
}

// Traces of the windows (time-major, per window at trace_off) into the
// caller's [3][nrec][nt] layout per shot; synchronises the stream.
int window_traces(EfwiHandle *h, const std::vector<Domain> &dom, float *traces, cudaStream_t st) {
  const int nt = h->grid.nt;
  const float *ttm = h->traces_tm.as<float>();
  long long off = 0;
  for (const Domain &d : dom) {
    if (d.nrec > 0) {
      k_traces_to_cr_t<<<dim3((nt + 31) / 32, (d.nrec + 31) / 32, 3), dim3(32, 8), 0, st>>>(
          ttm + d.trace_off, traces + off, nt, d.nrec);
      h->launches[K_OTHER]++;
    }
    off += 3LL * d.nrec * nt;
  }
  int rc = check_launch(h, "window forward");
  if (rc) return rc;
  CK_CUDA(h, cudaStreamSynchronize(st));
  return EFWI_OK;
}

// Tensor maps of the forward TMA kernels over one window's state and
// sliced model.
int make_window_maps(EfwiHandle *h, const Domain &d, int bxf, FwdMaps *maps) {
  const Fields &f = d.f;
  const float *sm[11] = {f.vz, f.vx, f.vy, f.szz, f.sxx, f.syy, f.sxz, f.sxy, f.syz, d.lam, d.mu};
  const float *vm[9] = {f.sxz, f.syz, f.sxx, f.sxy, f.syy, f.vz, f.vx, f.vy, d.buoy};
  for (int k = 0; k < 11; ++k) {
    int rc = make_map_dims(h, &maps->s.m[k], sm[k], d.g.sx, d.g.nx, d.g.nz, k < 3, bxf);
    if (rc) return rc;
  }
  for (int k = 0; k < 9; ++k) {
    int rc = make_map_dims(h, &maps->v.m[k], vm[k], d.g.sx, d.g.nx, d.g.nz, k < 5, bxf);
    if (rc) return rc;
  }
  return EFWI_OK;
}

// Time loop of the windows on the TMA kernels.  Each window is its own
// single-domain grid with its own tensor maps (kernel parameters, which a
// table of many domains in one launch cannot carry).  Contiguous groups of
// windows, balanced by cells, advance on up to 8 streams (the default
// number of hardware queues); every group records its own receivers after
// its velocity updates, so the groups never wait on one another inside the
// loop.  Each launch covers a whole window, so one stream already fills the
// GPU; the other streams fill the tails between launches.
int window_loop_tma(EfwiHandle *h, const std::vector<Domain> &dom, const std::vector<int> &rec_dom,
                    const Domain *ddom, const int *drd, const int *drc, const int *drr,
                    long long *dsrc, float *ttm, int ntl, bool use_graph, cudaStream_t st) {
  const int n = (int)dom.size();
  int rc = status_reset(h, st);
  if (rc) return rc;
  std::vector<long long> srcs(n);
  for (int k = 0; k < n; ++k) srcs[k] = dom[k].src_cell;
  CK_CUDA(h, cudaMemcpyAsync(dsrc, srcs.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, st));
  const int bxf = fwd_tma_tile(h->fcfg);
  std::vector<FwdMaps> maps(n);
  for (int k = 0; k < n; ++k) {
    rc = make_window_maps(h, dom[k], bxf, &maps[k]);
    if (rc) return rc;
  }
  // groups [gbeg[g], gbeg[g+1]) of at least one window each
  const int G = std::min(n, 8);
  std::vector<long long> cum(n + 1, 0);
  for (int k = 0; k < n; ++k) cum[k + 1] = cum[k] + dom[k].g.N;
  std::vector<int> gbeg(G + 1, n);
  gbeg[0] = 0;
  for (int g = 1; g < G; ++g) {
    int k = gbeg[g - 1] + 1;
    while (k < n - (G - g) && cum[k] * G < cum[n] * g) ++k;
    gbeg[g] = k;
  }
  // receivers are listed window by window: rstart[k] is window k's first
  std::vector<int> rstart(n + 1, 0);
  for (int d : rec_dom) rstart[d + 1]++;
  for (int k = 0; k < n; ++k) rstart[k + 1] += rstart[k];
  for (int g = 0; g < G; ++g)
    if (!h->wst[g]) CK_CUDA(h, cudaStreamCreateWithFlags(&h->wst[g], cudaStreamNonBlocking));
  for (int e = 0; e < 9; ++e)
    if (!h->wev[e]) CK_CUDA(h, cudaEventCreateWithFlags(&h->wev[e], cudaEventDisableTiming));
  CK_CUDA(h, cudaEventRecord(h->wev[8], st));
  for (int g = 0; g < G; ++g) CK_CUDA(h, cudaStreamWaitEvent(h->wst[g], h->wev[8], 0));
  int *status = h->status.as<int>();
  const int nt = h->grid.nt;
  std::vector<dim3> grids(n);
  std::vector<int> nzcs(n);
  for (int k = 0; k < n; ++k) {
    const Geo &g = dom[k].g;
    nzcs[k] = (g.nz + h->zchunk - 1) / h->zchunk;
    grids[k] = dim3((g.ny + 31) / 32, (g.nx + bxf - 1) / bxf, nzcs[k]);
  }
  long long nrec_launch = 0;
  // one time step of every group (it_dev: the step read from device memory)
  auto step = [&](int it, const int *it_dev) {
    for (int g = 0; g < G; ++g) {
      cudaStream_t s = h->wst[g];
      for (int k = gbeg[g]; k < gbeg[g + 1]; ++k) {
        const Domain &d = dom[k];
        const SrcArgs src{dsrc + k, d.stf, nt, it, it_dev};
        launch_stress_fwd_tma(h->fcfg, grids[k], s, maps[k].s, d.g, d.f, d.ps, h->zchunk, nzcs[k],
                              src, ShellMap{}, status);
        launch_velocity_fwd_tma(h->fcfg, grids[k], s, maps[k].v, d.g, d.f, d.ps, h->zchunk,
                                nzcs[k], RecFuse{}, status);
      }
      const int r0 = rstart[gbeg[g]], r1 = rstart[gbeg[g + 1]];
      if (r1 > r0) {
        k_record_multi<<<(r1 - r0 + 127) / 128, 128, 0, s>>>(ddom, drd + r0, drc + r0, drr + r0,
                                                               r1 - r0, ttm, it + 1, it_dev);
        ++nrec_launch;
      }
    }
  };
  const long long steps = std::max(ntl - 1, 0);
  if (use_graph && steps > 0) {
    // The step as a CUDA graph (the groups are its parallel branches, forked
    // from and joined to the capture stream), replayed once per time step;
    // the step index lives in a device word that the graph's last node
    // advances.
    if (!h->cap_stream) CK_CUDA(h, cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking));
    CK_CUDA(h, h->wstep.ensure(sizeof(int)));
    int *it_dev = h->wstep.as<int>();
    CK_CUDA(h, cudaMemsetAsync(it_dev, 0, sizeof(int), st));
    cudaStream_t cs = h->cap_stream;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CK_CUDA(h, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaError_t ec = cudaEventRecord(h->wev[8], cs);
    for (int g = 0; g < G && ec == cudaSuccess; ++g) ec = cudaStreamWaitEvent(h->wst[g], h->wev[8], 0);
    if (ec == cudaSuccess) step(0, it_dev);
    for (int g = 0; g < G && ec == cudaSuccess; ++g) {
      ec = cudaEventRecord(h->wev[g], h->wst[g]);
      if (ec == cudaSuccess) ec = cudaStreamWaitEvent(cs, h->wev[g], 0);
    }
    if (ec == cudaSuccess) {
      k_step_advance<<<1, 32, 0, cs>>>(it_dev);
      ec = cudaGetLastError();
    }
    const cudaError_t ee = cudaStreamEndCapture(cs, &graph);
    if (ec == cudaSuccess) ec = ee;
    if (ec == cudaSuccess) ec = cudaGraphInstantiate(&exec, graph, 0);
    for (long long s = 0; s < steps && ec == cudaSuccess; ++s) ec = cudaGraphLaunch(exec, st);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (ec != cudaSuccess)
      return fail(h, EFWI_ERR_CUDA, "graph of the window time step: %s", cudaGetErrorString(ec));
    nrec_launch *= steps;
    h->launches[K_OTHER] += steps;
  } else {
    for (int it = 0; it <= ntl - 2; ++it) step(it, nullptr);
    for (int g = 0; g < G; ++g) {
      CK_CUDA(h, cudaEventRecord(h->wev[g], h->wst[g]));
      CK_CUDA(h, cudaStreamWaitEvent(st, h->wev[g], 0));
    }
  }
  h->launches[K_STRESS_FWD] += steps * n;
  h->launches[K_VELOCITY_FWD] += steps * n;
  h->launches[K_RECORD] += nrec_launch;
  rc = check_launch(h, "window forward (TMA)");
  if (rc) return rc;
  return status_check(h, st);
}

}  // namespace

extern "C" {

const char *efwi_version(void) { return "efwi-b200 0.1 (sm_100a)"; }

int efwi_kernel_count(void) { return K_NCLASS; }

const char *efwi_kernel_name(int k) { return (k >= 0 && k < K_NCLASS) ? kKernelNames[k] : ""; }

const char *efwi_last_error(const EfwiHandle *h) { return h ? h->err.c_str() : "null handle"; }

int efwi_create(const EfwiGrid *g, EfwiHandle **out) {
  if (!g || !out) return EFWI_ERR_ARG;
  *out = nullptr;
  EfwiHandle *h = new EfwiHandle();
  if (g->nz < 5 || g->nx < 5 || g->ny < 5 || g->nt < 2 || g->npml < 2 || 2 * g->npml > g->nz ||
      2 * g->npml > g->nx || 2 * g->npml > g->ny || !(g->dt > 0) || !(g->dz > 0) ||
      !(g->dx > 0) || !(g->dy > 0)) {
    int rc = fail(h, EFWI_ERR_ARG, "invalid grid nz=%d nx=%d ny=%d npml=%d nt=%d", g->nz, g->nx,
                  g->ny, g->npml, g->nt);
    *out = h;
    return rc;
  }
  h->grid = *g;
  h->py = (g->ny + 3) & ~3;
  h->N = (long long)g->nz * g->nx * h->py;
  if (h->N >= (1LL << 31)) {
    *out = h;
    return fail(h, EFWI_ERR_ARG, "grid of %lld cells exceeds 2^31", h->N);
  }
  Geo &G = h->geo;
  G.nz = g->nz; G.nx = g->nx; G.ny = g->ny; G.np = g->npml;
  G.N = h->N; G.sz = (long long)g->nx * h->py; G.sx = h->py;
  G.dt = g->dt; G.idz = 1.0f / g->dz; G.idx = 1.0f / g->dx; G.idy = 1.0f / g->dy;
  G.slab_z = 2LL * g->npml * g->nx * g->ny;
  G.slab_x = (long long)g->nz * 2 * g->npml * g->ny;
  G.slab_y = (long long)g->nz * g->nx * 2 * g->npml;
  *out = h;
  const int nmax = g->nz + g->nx + g->ny;
  std::vector<float> c(6 * nmax);
  cpml_profile(g->nz, g->npml, g->dz, g->f0, g->dt, c.data());
  cpml_profile(g->nx, g->npml, g->dx, g->f0, g->dt, c.data() + 6 * g->nz);
  cpml_profile(g->ny, g->npml, g->dy, g->f0, g->dt, c.data() + 6 * (g->nz + g->nx));
  // The kernels multiply by 1/K and 1/K_half instead of dividing by K.
  {
    const int ns[3] = {g->nz, g->nx, g->ny};
    float *row = c.data();
    for (int ax = 0; ax < 3; ++ax) {
      for (int i = 0; i < ns[ax]; ++i) {
        row[CK * ns[ax] + i] = 1.0f / row[CK * ns[ax] + i];
        row[CKH * ns[ax] + i] = 1.0f / row[CKH * ns[ax] + i];
      }
      row += 6 * ns[ax];
    }
  }
  CK_CUDA(h, h->coef.ensure(sizeof(float) * c.size()));
  CK_CUDA(h, cudaMemcpy(h->coef.p, c.data(), sizeof(float) * c.size(), cudaMemcpyHostToDevice));
  G.cz = h->coef.as<float>();
  G.cx = G.cz + 6 * g->nz;
  G.cy = G.cx + 6 * g->nx;
  std::vector<int> pts = shell_points(*g, h->py);
  h->npts = (int)pts.size();
  if (!pts.empty()) {
    CK_CUDA(h, h->pts.ensure(sizeof(int) * pts.size()));
    CK_CUDA(h, cudaMemcpy(h->pts.p, pts.data(), sizeof(int) * pts.size(), cudaMemcpyHostToDevice));
    std::vector<int> rows;
    h->shell_fused = shell_rows(*g, h->py, pts, &rows, &h->shm);
    if (h->shell_fused) {
      CK_CUDA(h, h->shell_rows.ensure(sizeof(int) * rows.size()));
      CK_CUDA(h, cudaMemcpy(h->shell_rows.p, rows.data(), sizeof(int) * rows.size(),
                            cudaMemcpyHostToDevice));
      h->shm.rows = h->shell_rows.as<int>();
    }
  }
  return EFWI_OK;
}

void efwi_destroy(EfwiHandle *h) {
  if (!h) return;
  for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
  if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
  for (cudaStream_t s : h->wst)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : h->wev)
    if (e) cudaEventDestroy(e);
  for (EfwiHandle *c : h->lane) efwi_destroy(c);
  for (auto &w : h->wsub) efwi_destroy(w.second);
  if (h->own_st) cudaStreamDestroy(h->own_st);
  if (h->lane_fork) cudaEventDestroy(h->lane_fork);
  delete h;
}

int efwi_set_options(EfwiHandle *h, int if_win, int tile_bx, int zchunk, int max_batch) {
  if (!h) return EFWI_ERR_ARG;
  if (tile_bx != 0 && tile_bx != 4 && tile_bx != 8) return fail(h, EFWI_ERR_ARG, "tile_bx must be 4 or 8");
  if (zchunk < 0 || max_batch < 0) return fail(h, EFWI_ERR_ARG, "negative zchunk/max_batch");
  h->if_win = if_win ? 1 : 0;
  if (tile_bx) h->bx = tile_bx;
  if (zchunk) h->zchunk = zchunk;
  if (max_batch) h->max_batch = max_batch;
  return EFWI_OK;
}

int efwi_set_tuning(EfwiHandle *h, int fwd_cfg, int zchunk_fwd, int rev_cfg, int zchunk_rev) {
  if (!h) return EFWI_ERR_ARG;
  if (fwd_cfg < 0 || fwd_cfg > 3 || rev_cfg < 0 || rev_cfg > 7 || zchunk_fwd < 0 || zchunk_rev < 0)
    return fail(h, EFWI_ERR_ARG, "invalid tuning (forward cfg 0-3, reverse cfg 0-7, zchunk >= 0)");
  h->fcfg = fwd_cfg;
  h->rcfg = rev_cfg;
  if (zchunk_fwd) h->zchunk = zchunk_fwd;
  if (zchunk_rev) h->zchunk_rev = zchunk_rev;
  return EFWI_OK;
}

int efwi_set_lanes(EfwiHandle *h, int lanes) {
  if (!h) return EFWI_ERR_ARG;
  if (lanes < 1 || lanes > 8) return fail(h, EFWI_ERR_ARG, "lanes must be in [1, 8]");
  h->lanes = lanes;
  while ((int)h->lane.size() > lanes - 1) {  // frees the dropped lanes' workspace
    efwi_destroy(h->lane.back());
    h->lane.pop_back();
  }
  return EFWI_OK;
}

int efwi_set_nt_limit(EfwiHandle *h, int nt_limit) {
  if (!h || nt_limit < 0) return EFWI_ERR_ARG;
  h->nt_limit = nt_limit;
  return EFWI_OK;
}

int efwi_set_graphs(EfwiHandle *h, int on) {
  if (!h) return EFWI_ERR_ARG;
  h->use_graphs = on != 0;
  if (!h->use_graphs) {
    h->g_fwd.reset();
    h->g_rev.reset();
  }
  return EFWI_OK;
}

int efwi_set_variant(EfwiHandle *h, int variant) {
  if (!h) return EFWI_ERR_ARG;
  if (variant != 0 && variant != 1) return fail(h, EFWI_ERR_ARG, "variant must be 0 or 1");
  h->variant = variant;
  return EFWI_OK;
}

int efwi_set_model(EfwiHandle *h, const float *lam, const float *mu, const float *rho, void *stream) {
  if (!h) return EFWI_ERR_ARG;
  if (!lam || !mu || !rho) return fail(h, EFWI_ERR_ARG, "null model pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t bytes = sizeof(float) * h->N;
  CK_CUDA(h, h->lam.ensure(bytes));
  CK_CUDA(h, h->mu.ensure(bytes));
  CK_CUDA(h, h->buoy.ensure(bytes));
  const EfwiGrid &G = h->grid;
  k_pitch_copy<<<1184, 256, 0, st>>>(lam, h->lam.as<float>(), G.nz, G.nx, G.ny, h->py, 1);
  k_pitch_copy<<<1184, 256, 0, st>>>(mu, h->mu.as<float>(), G.nz, G.nx, G.ny, h->py, 1);
  CK_CUDA(h, cudaMemsetAsync(h->buoy.p, 0, bytes, st));
  k_prep_buoyancy<<<1184, 256, 0, st>>>(rho, h->buoy.as<float>(), G.nz, G.nx, G.ny, h->py);
  h->launches[K_OTHER] += 3;
  // CFL check of the reference (2D formula with min(dz, dx)).
  CK_CUDA(h, h->jdev.ensure(64));
  unsigned int *vmax = (unsigned int *)h->jdev.p;
  CK_CUDA(h, cudaMemsetAsync(vmax, 0, sizeof(unsigned int), st));
  k_max_vp<<<592, 256, 0, st>>>(lam, mu, rho, (long long)G.nz * G.nx * G.ny, vmax);
  h->launches[K_OTHER]++;
  int rc = check_launch(h, "set_model");
  if (rc) return rc;
  unsigned int bits = 0;
  CK_CUDA(h, cudaMemcpyAsync(&bits, vmax, sizeof(bits), cudaMemcpyDeviceToHost, st));
  CK_CUDA(h, cudaStreamSynchronize(st));
  float vm;
  std::memcpy(&vm, &bits, sizeof(vm));
  const float dh = h->grid.dz < h->grid.dx ? h->grid.dz : h->grid.dx;
  const float courant = vm * h->grid.dt * sqrtf(2.0f) * (1.0f / 24.0f + 9.0f / 8.0f) / dh;
  h->model_set = false;
  if (!(courant <= 1.0f)) return fail(h, EFWI_ERR_CFL, "Courant_number = %g", courant);
  h->model_set = true;
  return EFWI_OK;
}

int efwi_set_survey(EfwiHandle *h, int nshot, const EfwiShot *shots, const float *stf) {
  if (!h) return EFWI_ERR_ARG;
  if (nshot < 0 || (nshot > 0 && (!shots || !stf))) return fail(h, EFWI_ERR_ARG, "invalid survey");
  const EfwiGrid &g = h->grid;
  std::vector<ShotHost> out(nshot);
  for (int k = 0; k < nshot; ++k) {
    const EfwiShot &s = shots[k];
    if (s.z_src < 2 || s.z_src > g.nz - 3 || s.x_src < 2 || s.x_src > g.nx - 3 || s.y_src < 2 ||
        s.y_src > g.ny - 3)
      return fail(h, EFWI_ERR_ARG, "shot %d: source (%d, %d, %d) outside the updated region", k,
                  s.z_src, s.x_src, s.y_src);
    if (s.nrec < 0 || (s.nrec > 0 && (!s.z_rec || !s.x_rec || !s.y_rec)))
      return fail(h, EFWI_ERR_ARG, "shot %d: invalid receivers", k);
    ShotHost &o = out[k];
    o.src_cell = ((long long)s.z_src * g.nx + s.x_src) * h->py + s.y_src;
    o.nrec = s.nrec;
    o.rec_cell.resize(s.nrec);
    for (int r = 0; r < s.nrec; ++r) {
      const int z = s.z_rec[r], x = s.x_rec[r], y = s.y_rec[r];
      if (z < 0 || z >= g.nz || x < 0 || x >= g.nx || y < 0 || y >= g.ny)
        return fail(h, EFWI_ERR_ARG, "shot %d receiver %d at (%d, %d, %d) outside the grid", k, r, z, x, y);
      o.rec_cell[r] = ((long long)z * g.nx + x) * h->py + y;
    }
    o.win0.assign(s.nrec, 0.f);
    o.win1.assign(s.nrec, 0.f);
    o.wts.assign(s.nrec, 1.f);
    for (int r = 0; r < s.nrec; ++r) {
      if (s.win_start) o.win0[r] = s.win_start[r];
      if (s.win_end) o.win1[r] = s.win_end[r];
      if (s.weights) o.wts[r] = s.weights[r];
    }
    o.src_w = s.src_weight;
  }
  {
    std::vector<float> ones(g.nt, 1.0f), w2(g.nt);
    taper_stf(ones.data(), g.nt, g.dt, w2.data());
    CK_CUDA(h, h->stf_w2.ensure(sizeof(float) * g.nt));
    CK_CUDA(h, cudaMemcpy(h->stf_w2.p, w2.data(), sizeof(float) * g.nt, cudaMemcpyHostToDevice));
  }
  std::vector<float> tap((size_t)nshot * g.nt);
  for (int k = 0; k < nshot; ++k) taper_stf(stf + (size_t)k * g.nt, g.nt, g.dt, tap.data() + (size_t)k * g.nt);
  if (nshot > 0) {
    CK_CUDA(h, h->stf.ensure(sizeof(float) * tap.size()));
    CK_CUDA(h, cudaMemcpy(h->stf.p, tap.data(), sizeof(float) * tap.size(), cudaMemcpyHostToDevice));
  }
  h->stf_host.assign(stf, stf + (size_t)nshot * g.nt);
  h->shots.swap(out);
  h->survey_set = true;
  return EFWI_OK;
}

int efwi_forward(EfwiHandle *h, int n, const int *ids, float *traces, void *stream) {
  int rc = check_ready(h, n, ids);
  if (rc) return rc;
  if (n > 0 && !traces) return fail(h, EFWI_ERR_ARG, "null traces");
  cudaStream_t st = (cudaStream_t)stream;
  const int nt = h->grid.nt;
  long long out_off = 0;
  rc = status_reset(h, st);
  if (rc) return rc;
  for (int b0 = 0; b0 < n; b0 += h->max_batch) {
    const int S = std::min(h->max_batch, n - b0);
    long long ntr = 0;
    for (int s = 0; s < S; ++s) ntr += 3LL * h->shots[ids[b0 + s]].nrec * nt;
    CK_CUDA(h, h->traces_tm.ensure(sizeof(float) * std::max(ntr, 1LL)));
    rc = run_forward_batch(h, ids + b0, S, h->traces_tm.as<float>(), ntr, nullptr, nullptr, st);
    if (rc) return rc;
    long long toff = 0;
    for (int s = 0; s < S; ++s) {
      const int nr = h->shots[ids[b0 + s]].nrec;
      if (nr > 0) {
        Timer t(h, K_OTHER, st, -1);
        k_traces_to_cr_t<<<dim3((nt + 31) / 32, (nr + 31) / 32, 3), dim3(32, 8), 0, st>>>(
            h->traces_tm.as<float>() + toff, traces + out_off, nt, nr);
      }
      toff += 3LL * nr * nt;
      out_off += 3LL * nr * nt;
    }
    rc = check_launch(h, "traces");
    if (rc) return rc;
  }
  return status_check(h, st);
}

// Misfit (and, with glam set, the images) of shots ids on stream st.  With
// copy_out unset the images stay in the handle's pitched accumulator
// (h->grad) instead of being copied to glam/gmu/grho; js_out (host, n),
// when given, receives the misfit of every shot.
static int gradient_impl(EfwiHandle *h, int n, const int *ids, const float *obs, int mode,
                         double *misfit, float *glam, float *gmu, float *grho, float *res_out,
                         cudaStream_t st, bool adj_source = false, bool copy_out = true,
                         double *js_out = nullptr) {
  const int nt = h->grid.nt;
  const long long N = h->N;
  const bool grad = glam != nullptr;
  {
    int rc0 = status_reset(h, st);
    if (rc0) return rc0;
  }
  float *out_lam = glam, *out_mu = gmu, *out_rho = grho;
  if (grad) {
    // images accumulate in pitched volumes, copied out at the end
    CK_CUDA(h, h->grad.ensure(sizeof(float) * 3 * N));
    CK_CUDA(h, cudaMemsetAsync(h->grad.p, 0, sizeof(float) * 3 * N, st));
    glam = h->grad.as<float>();
    gmu = glam + N;
    grho = glam + 2 * N;
  }
  CK_CUDA(h, h->jdev.ensure(sizeof(double) * (n + 8)));
  double *jdev = h->jdev.as<double>() + 1;
  if (n > 0) CK_CUDA(h, cudaMemsetAsync(jdev, 0, sizeof(double) * n, st));
  if (grad) CK_CUDA(h, h->adj.ensure(sizeof(float) * 9 * N));
  if (grad && mode == EFWI_MODE_REFERENCE)
    CK_CUDA(h, h->shell.ensure(sizeof(float) * 9 * (size_t)std::max(h->npts, 1) * nt));
  long long obs_off = 0;
  int n_done_exact = 0;
  if (grad && mode == EFWI_MODE_EXACT) {
    for (int k = 0; k < n; ++k) {
      const ShotHost &sh = h->shots[ids[k]];
      float *grow = h->gstf ? h->gstf + (size_t)k * nt : nullptr;
      if (grow) CK_CUDA(h, cudaMemsetAsync(grow, 0, sizeof(float) * nt, st));
      int rc = exact_shot(h, ids[k], obs + obs_off, jdev + k, res_out ? res_out + obs_off : nullptr,
                          glam, gmu, grho, st, adj_source, obs_off, grow);
      if (rc) return rc;
      obs_off += 3LL * sh.nrec * nt;
    }
    // grho holds the buoyancy image until here
    const EfwiGrid &G = h->grid;
    k_buoy_to_rho<<<1184, 256, 0, st>>>(grho, h->buoy.as<float>(), grho, G.nz, G.nx, G.ny, h->py);
    h->launches[K_OTHER]++;
    n_done_exact = n;
  }
  for (int k = n_done_exact; k < n; ++k) {
    const ShotHost &sh = h->shots[ids[k]];
    const long long ntr = 3LL * sh.nrec * nt;
    CK_CUDA(h, h->traces_tm.ensure(sizeof(float) * std::max(ntr, 1LL)));
    CK_CUDA(h, h->res_tm.ensure(sizeof(float) * std::max(ntr, 1LL)));
    RecArgs rec;
    int rc = run_forward_batch(h, ids + k, 1, h->traces_tm.as<float>(), ntr, &rec,
                               grad ? h->shell.as<float>() : nullptr, st);
    if (rc) return rc;
    rc = misfit_shot(h, sh, obs + obs_off, h->traces_tm.as<float>(), h->res_tm.as<float>(), jdev + k, st,
                     obs_off);
    if (rc) return rc;
    if (res_out && sh.nrec > 0) {
      k_traces_to_cr_t<<<dim3((nt + 31) / 32, (sh.nrec + 31) / 32, 3), dim3(32, 8), 0, st>>>(
          h->res_tm.as<float>(), res_out + obs_off, nt, sh.nrec);
      h->launches[K_OTHER]++;
    }
    obs_off += ntr;
    if (!grad) continue;
    // ---------------------------------------------------------- reverse
    Fields f = fields_at(h->fields.as<float>(), N, 1);
    Fields a = fields_at(h->adj.as<float>(), N, 1);
    Psi ps = psi_at(h->psi.as<float>(), h->geo, 1);
    CK_CUDA(h, cudaMemsetAsync(h->adj.p, 0, sizeof(float) * 9 * N, st));
    CK_CUDA(h, cudaMemsetAsync(h->psi.p, 0, sizeof(float) * psi_per_shot(h->geo), st));
    long long *dcell = h->scalar.as<long long>();
    float *dstf = (float *)((char *)h->scalar.p + 256);
    SrcArgs src{dcell, dstf, nt, 0};
    const int npts = h->npts;
    const float *shell = h->shell.as<float>();
    // Reverse kernels: TMA-staged (tile 32 x 4) or L1-served.
    Maps<21> m1;
    Maps<23> m2;
    Maps<13> m1r;
    Maps<12> m1a;
    const bool split = h->rcfg == 6 || h->rcfg == 7;
    const bool tma = h->variant == 1;
    const EfwiGrid &G = h->grid;
    if (tma) {
      const float *h1[11] = {f.sxz, f.syz, f.sxx, f.sxy, f.syy, a.sxz, a.syz, a.sxx, a.sxy, a.syy, a.szz};
      const float *p1[10] = {f.vz, f.vx, f.vy, a.vz, a.vx, a.vy, h->buoy.as<float>(),
                             h->lam.as<float>(), h->mu.as<float>(), grho};
      const float *h2[6] = {f.vz, f.vx, f.vy, a.vz, a.vx, a.vy};
      const float *p2[17] = {f.szz, f.sxx, f.syy, f.sxz, f.sxy, f.syz, a.szz, a.sxx, a.syy,
                             a.sxz, a.sxy, a.syz, h->lam.as<float>(), h->mu.as<float>(),
                             h->buoy.as<float>(), glam, gmu};
      const int bxm = rev_tma_tile(h->rcfg);
      for (int k2 = 0; k2 < 21 && rc == 0; ++k2)
        rc = make_map(h, &m1.m[k2], k2 < 11 ? h1[k2] : p1[k2 - 11], 1, k2 < 11, bxm);
      if (split) {
        const float *r1[13] = {f.sxz, f.syz, f.sxx, f.sxy, f.syy, f.vz, f.vx, f.vy,
                               a.vz, a.vx, a.vy, h->buoy.as<float>(), grho};
        const float *a1[12] = {a.sxz, a.syz, a.sxx, a.sxy, a.syy, a.szz, a.vz, a.vx, a.vy,
                               h->buoy.as<float>(), h->lam.as<float>(), h->mu.as<float>()};
        for (int k2 = 0; k2 < 13 && rc == 0; ++k2) rc = make_map(h, &m1r.m[k2], r1[k2], 1, k2 < 5, 4);
        for (int k2 = 0; k2 < 12 && rc == 0; ++k2) rc = make_map(h, &m1a.m[k2], a1[k2], 1, k2 < 6, 4);
      }
      for (int k2 = 0; k2 < 23 && rc == 0; ++k2)
        rc = make_map(h, &m2.m[k2], k2 < 6 ? h2[k2] : p2[k2 - 6], 1, k2 < 6, bxm);
      if (rc) return rc;
    }
    int nzc;
    const int bxr = tma ? rev_tma_tile(h->rcfg) : h->bx;
    const int zcr = tma ? h->zchunk_rev : h->zchunk;
    const dim3 grid = stencil_grid(h, 1, bxr, zcr, &nzc);
    (void)G;
    int *status = h->status.as<int>();
    // On the TMA kernels the shell restore and the adjoint-source injection
    // run in K1's and K2's epilogues; otherwise as separate launches.
    const bool shell_fused = tma && h->shell_fused && npts > 0;
    const bool inj_fused = tma && rec.ncell > 0 && rec.plane;
    auto shell_at = [&](int rev, int it) {
      ShellMap m{};
      if (shell_fused && rev) {
        m = h->shm;
        m.store = const_cast<float *>(shell) + (size_t)it * 9 * npts;
      }
      return m;
    };
    auto K1 = [&](int rev, int adj, int it) {
      Timer t(h, K_REV_VELOCITY, st, it);
      const ShellMap sm = shell_at(rev, it);
      RecFuse inj{};
      if (inj_fused && adj) inj = RecFuse{rec, h->res_tm.as<float>(), it};
      if (tma && split)
        launch_rev_velocity_split_tma(h->rcfg, grid, st, m1r, m1a, h->geo, f, a, ps, grho, zcr,
                                      nzc, rev, adj, sm, inj, status);
      else if (tma)
        launch_rev_velocity_tma(h->rcfg, grid, st, m1, h->geo, f, a, ps, grho, zcr, nzc, rev, adj,
                                sm, inj, status);
      else
        launch_rev_velocity(h->bx, grid, st, h->geo, f, a, ps, h->lam.as<float>(),
                            h->mu.as<float>(), h->buoy.as<float>(), grho, zcr, nzc, rev, adj);
    };
    auto K2 = [&](int rev, int adj, int it) {
      Timer t(h, K_REV_STRESS, st, it);
      src.it = it;
      if (tma)
        launch_rev_stress_tma(h->rcfg, grid, st, m2, h->geo, f, a, ps, glam, gmu, zcr, nzc, rev,
                              adj, src, shell_at(rev, it), status);
      else
        launch_rev_stress(h->bx, grid, st, h->geo, f, a, ps, h->lam.as<float>(), h->mu.as<float>(),
                          h->buoy.as<float>(), glam, gmu, zcr, nzc, rev, adj, src);
    };
    auto inject = [&](int it) {
      if (rec.ncell == 0 || inj_fused) return;
      Timer t(h, K_INJECT, st, it);
      k_inject<<<(rec.ncell + 127) / 128, 128, 0, st>>>(a, N, rec, h->res_tm.as<float>(), it, 1.0f);
    };
    auto restore = [&](int it, int stress) {
      if (npts == 0 || shell_fused) return;
      Timer t(h, K_SHELL_RESTORE, st, it);
      k_shell_restore<<<(npts + 255) / 256, 256, 0, st>>>(f, h->pts.as<int>(), npts, shell + (size_t)it * 9 * npts, stress);
    };
    const int ntl = nt_eff(h);
    auto loop = [&](cudaStream_t s) -> int {
      st = s;  // the launch helpers above use st
      K1(0, 1, ntl - 1);
      inject(ntl - 1);
      K2(0, 1, ntl - 1);
      for (int it = ntl - 2; it >= 0; --it) {
        const int adj = it > 0;  // the adjoint update of step 0 feeds no image
        K1(1, adj, it);
        if (adj) inject(it);
        restore(it, 0);
        K2(1, adj, it);
        restore(it, 1);
      }
      return check_launch(h, "reverse");
    };
    KeyBytes key;
    key.add(f).add(a).add(ps).add(grho).add(glam).add(gmu).add(shell).add(npts).rec(rec)
        .src(src).add(h->res_tm.p).add(h->rcfg).add(zcr).add(bxr).add(h->bx).add(tma)
        .add(split).add(shell_fused).add(inj_fused).add(ntl).geo(h->geo).shell(h->shm)
        .add(h->status.p).add(h->lam.p).add(h->mu.p).add(h->buoy.p);
    if (tma) key.add(m1).add(m2);
    if (tma && split) key.add(m1r).add(m1a);
    cudaStream_t caller = st;
    rc = run_graphed(h, h->g_rev, key.s, caller, loop);
    st = caller;
    if (rc) return rc;
  }
  if (grad && copy_out) {
    const EfwiGrid &G = h->grid;
    k_pitch_copy<<<1184, 256, 0, st>>>(glam, out_lam, G.nz, G.nx, G.ny, h->py, 0);
    k_pitch_copy<<<1184, 256, 0, st>>>(gmu, out_mu, G.nz, G.nx, G.ny, h->py, 0);
    k_pitch_copy<<<1184, 256, 0, st>>>(grho, out_rho, G.nz, G.nx, G.ny, h->py, 0);
    h->launches[K_OTHER] += 3;
    int rc = check_launch(h, "gradient copy-out");
    if (rc) return rc;
  }
  std::vector<double> js(std::max(n, 1), 0.0);
  if (n > 0) CK_CUDA(h, cudaMemcpyAsync(js.data(), jdev, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  CK_CUDA(h, cudaStreamSynchronize(st));
  double J = 0.0;
  for (int k = 0; k < n; ++k) J += js[k];
  if (misfit) *misfit = J;
  if (js_out) std::copy(js.begin(), js.begin() + n, js_out);
  {
    int rc1 = status_check(h, st);
    if (rc1) return rc1;
  }
  if (h->prof_sample > 0) return resolve_profile(h);
  return EFWI_OK;
}

// Copies h's configuration into lane c; c borrows h's model,
// coefficients, survey and shell points, which no call writes.
static int lane_sync(EfwiHandle *h, EfwiHandle *c) {
  c->grid = h->grid;
  c->geo = h->geo;
  c->N = h->N;
  c->py = h->py;
  c->if_win = h->if_win; c->bx = h->bx; c->zchunk = h->zchunk; c->max_batch = h->max_batch;
  c->variant = h->variant; c->fcfg = h->fcfg; c->rcfg = h->rcfg; c->zchunk_rev = h->zchunk_rev;
  c->nt_limit = h->nt_limit;
  c->use_graphs = h->use_graphs;
  c->prof_sample = 0;  // lane 0 alone records kernel events (the others count launches)
  c->coef.view(h->coef);
  c->lam.view(h->lam);
  c->mu.view(h->mu);
  c->buoy.view(h->buoy);
  c->model_set = h->model_set;
  c->shots = h->shots;
  c->stf.view(h->stf);
  c->src_cell.view(h->src_cell);
  c->stf_w2.view(h->stf_w2);
  c->survey_set = h->survey_set;
  c->pts.view(h->pts);
  c->npts = h->npts;
  c->shell_rows.view(h->shell_rows);
  c->shm = h->shm;
  c->shell_fused = h->shell_fused;
  c->lanes = 1;
  if (!c->own_st) CK_CUDA(c, cudaStreamCreateWithFlags(&c->own_st, cudaStreamNonBlocking));
  return EFWI_OK;
}

// Allocates the large per-shot workspace of a reference-mode call up front;
// false (with the workspace released and the error cleared) when the GPU
// has no room for it.
// Reference mode: state, images and the boundary-shell store; exact mode:
// state, images, the two adjoint memory-variable sets and `ck_bytes` of
// checkpoint slots.
static bool lane_reserve(EfwiHandle *c, bool grad, int mode = EFWI_MODE_REFERENCE,
                         long long ck_bytes = 0) {
  const long long N = c->N;
  const long long P = psi_per_shot(c->geo);
  cudaError_t e = c->fields.ensure(sizeof(float) * 9 * N);
  if (e == cudaSuccess) e = c->psi.ensure(sizeof(float) * P);
  if (grad && e == cudaSuccess) e = c->adj.ensure(sizeof(float) * 9 * N);
  if (grad && e == cudaSuccess) e = c->grad.ensure(sizeof(float) * 3 * N);
  if (grad && mode == EFWI_MODE_REFERENCE && e == cudaSuccess)
    e = c->shell.ensure(sizeof(float) * 9 * (size_t)std::max(c->npts, 1) * c->grid.nt);
  if (grad && mode == EFWI_MODE_EXACT && e == cudaSuccess)
    e = c->apsi.ensure(sizeof(float) * 2 * P);
  if (grad && mode == EFWI_MODE_EXACT && e == cudaSuccess && ck_bytes > 0)
    e = c->ckpt.ensure((size_t)ck_bytes);
  if (e == cudaSuccess) return true;
  cudaGetLastError();
  c->fields.release(); c->psi.release(); c->adj.release(); c->grad.release(); c->shell.release();
  c->apsi.release(); c->ckpt.release();
  return false;
}

// Reference-mode misfit / gradient of n >= 2 shots on up to h->lanes
// lanes: lane 0 is h on the caller's stream, lane l >= 1 a sub-handle with
// its own workspace and stream, driven by its own host thread.  Lane l
// takes the contiguous shots [n*l/L, n*(l+1)/L).  Kernels of different
// lanes share the GPU, which fills the tail waves and launch gaps of one
// shot's sequence with another shot's work.  The misfit is summed over
// the shots in order (as with one lane); the images are the lanes'
// accumulators added in lane order.
static int gradient_lanes(EfwiHandle *h, int n, const int *ids, const float *obs, double *misfit,
                          float *glam, float *gmu, float *grho, float *res_out, cudaStream_t st,
                          int mode = EFWI_MODE_REFERENCE) {
  const bool grad = glam != nullptr;
  const int nt = h->grid.nt;
  int L = std::min(h->lanes, n);
  if (h->variant == 1) {
    int rc = get_encoder(h);  // once, before any thread needs it
    if (rc) return rc;
  }
  // exact mode: every lane takes an equal share of the checkpoint budget
  const long long budget = h->ck_budget;
  auto share = [&](int lanes) { return budget / std::max(lanes, 1); };
  if (!lane_reserve(h, grad, mode, mode == EFWI_MODE_EXACT ? share(L) : 0)) L = 1;
  while ((int)h->lane.size() < L - 1) h->lane.push_back(new EfwiHandle());
  int got = 1;
  for (; got < L; ++got) {
    EfwiHandle *c = h->lane[got - 1];
    if (lane_sync(h, c)) return fail(h, EFWI_ERR_CUDA, "lane %d: %s", got, c->err.c_str());
    if (!lane_reserve(c, grad, mode, mode == EFWI_MODE_EXACT ? share(L) : 0)) break;
  }
  L = got;
  if (L < 2)
    return gradient_impl(h, n, ids, obs, mode, misfit, glam, gmu, grho, res_out, st);
  h->ck_budget = share(L);
  for (int l = 1; l < L; ++l) h->lane[l - 1]->ck_budget = share(L);
  std::vector<int> b(L + 1);
  for (int l = 0; l <= L; ++l) b[l] = (int)((long long)n * l / L);
  std::vector<long long> off(n + 1, 0);
  for (int k = 0; k < n; ++k) off[k + 1] = off[k] + 3LL * h->shots[ids[k]].nrec * nt;
  if (!h->lane_fork) CK_CUDA(h, cudaEventCreateWithFlags(&h->lane_fork, cudaEventDisableTiming));
  CK_CUDA(h, cudaEventRecord(h->lane_fork, st));
  int dev = 0;
  CK_CUDA(h, cudaGetDevice(&dev));
  for (int l = 1; l < L; ++l) {
    EfwiHandle *c = h->lane[l - 1];
    const long long o = off[b[l]];
    c->scr_syn = h->scr_syn ? h->scr_syn + o : nullptr;
    c->scr_obs = h->scr_obs ? h->scr_obs + o : nullptr;
    c->scr_res = h->scr_res ? h->scr_res + o : nullptr;
    c->gstf = h->gstf ? h->gstf + (size_t)b[l] * nt : nullptr;
    CK_CUDA(h, cudaStreamWaitEvent(c->own_st, h->lane_fork, 0));
  }
  // No return between the first thread's start and the joins below.
  std::vector<double> js(n, 0.0);
  std::vector<int> rcs(L, EFWI_OK);
  std::vector<std::thread> th;
  th.reserve(L - 1);
  auto run_lane = [&](int l) {
    EfwiHandle *c = h->lane[l - 1];
    const long long o = off[b[l]];
    if (cudaSetDevice(dev) != cudaSuccess) {
      rcs[l] = fail(c, EFWI_ERR_CUDA, "cudaSetDevice(%d) failed in lane %d", dev, l);
      return;
    }
    rcs[l] = gradient_impl(c, b[l + 1] - b[l], ids + b[l], obs + o, mode, nullptr, glam, gmu,
                           grho, res_out ? res_out + o : nullptr, c->own_st, false, false,
                           js.data() + b[l]);
  };
  for (int l = 1; l < L; ++l) {
    try {
      th.emplace_back(run_lane, l);
    } catch (...) {
      run_lane(l);  // no thread to spare: the lane runs here, before lane 0
    }
  }
  rcs[0] = gradient_impl(h, b[1], ids, obs, mode, nullptr, glam, gmu, grho, res_out, st, false,
                         false, js.data());
  for (std::thread &t : th) t.join();
  h->ck_budget = budget;
  for (int l = 1; l < L; ++l) {
    EfwiHandle *c = h->lane[l - 1];
    h->ck_forward_steps = std::max(h->ck_forward_steps, c->ck_forward_steps);
  }
  for (int l = 1; l < L; ++l) {
    EfwiHandle *c = h->lane[l - 1];
    if (h->prof_sample > 0) resolve_profile(c);
    for (int k = 0; k < K_NCLASS; ++k) {
      h->launches[k] += c->launches[k];
      h->timed[k] += c->timed[k];
      h->ms[k] += c->ms[k];
      c->launches[k] = 0; c->timed[k] = 0; c->ms[k] = 0;
    }
  }
  for (int l = 0; l < L; ++l)
    if (rcs[l]) {
      // A failed lane may have returned with kernels still queued on its
      // stream (and the others keep running): drain every lane's stream
      // before the workspaces can be freed or reused.
      cudaStreamSynchronize(st);
      for (int m = 1; m < L; ++m) cudaStreamSynchronize(h->lane[m - 1]->own_st);
      cudaGetLastError();
      if (l > 0) h->err = "lane " + std::to_string(l) + ": " + h->lane[l - 1]->err;
      return rcs[l];
    }
  if (grad) {
    float *acc = h->grad.as<float>();
    for (int l = 1; l < L; ++l)
      k_add<<<1184, 256, 0, st>>>(acc, h->lane[l - 1]->grad.as<float>(), 3 * h->N);
    const EfwiGrid &G = h->grid;
    k_pitch_copy<<<1184, 256, 0, st>>>(acc, glam, G.nz, G.nx, G.ny, h->py, 0);
    k_pitch_copy<<<1184, 256, 0, st>>>(acc + h->N, gmu, G.nz, G.nx, G.ny, h->py, 0);
    k_pitch_copy<<<1184, 256, 0, st>>>(acc + 2 * h->N, grho, G.nz, G.nx, G.ny, h->py, 0);
    h->launches[K_OTHER] += L - 1 + 3;
    int rc = check_launch(h, "lane images");
    if (rc) return rc;
    CK_CUDA(h, cudaStreamSynchronize(st));
  }
  double J = 0.0;
  for (int k = 0; k < n; ++k) J += js[k];
  if (misfit) *misfit = J;
  return EFWI_OK;
}

int efwi_misfit(EfwiHandle *h, int n, const int *ids, const float *obs, double *misfit, void *stream) {
  int rc = check_ready(h, n, ids);
  if (rc) return rc;
  if (n > 0 && !obs) return fail(h, EFWI_ERR_ARG, "null obs");
  if (h->lanes > 1 && n > 1)
    return gradient_lanes(h, n, ids, obs, misfit, nullptr, nullptr, nullptr, nullptr,
                          (cudaStream_t)stream);
  return gradient_impl(h, n, ids, obs, EFWI_MODE_REFERENCE, misfit, nullptr, nullptr, nullptr,
                       nullptr, (cudaStream_t)stream);
}

int efwi_gradient(EfwiHandle *h, int n, const int *ids, const float *obs, int mode, double *misfit,
                  float *glam, float *gmu, float *grho, float *res, void *stream) {
  int rc = check_ready(h, n, ids);
  if (rc) return rc;
  if (n > 0 && !obs) return fail(h, EFWI_ERR_ARG, "null obs");
  if (!glam || !gmu || !grho) return fail(h, EFWI_ERR_ARG, "null gradient output");
  if (mode != EFWI_MODE_REFERENCE && mode != EFWI_MODE_EXACT)
    return fail(h, EFWI_ERR_ARG, "gradient mode %d is not available", mode);
  if (h->lanes > 1 && n > 1)
    return gradient_lanes(h, n, ids, obs, misfit, glam, gmu, grho, res, (cudaStream_t)stream, mode);
  return gradient_impl(h, n, ids, obs, mode, misfit, glam, gmu, grho, res, (cudaStream_t)stream);
}

int efwi_forward_windows(EfwiHandle *h, int n, const int *ids, const EfwiWindow *win,
                         float *traces, int use_graph, void *stream) {
  int rc = check_ready(h, n, ids);
  if (rc) return rc;
  if (n > 0 && (!win || !traces)) return fail(h, EFWI_ERR_ARG, "null windows or traces");
  if (n == 0) return EFWI_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const EfwiGrid &G = h->grid;
  const int np = G.npml, nz = G.nz, nt = G.nt, bx = h->bx, zchunk = h->zchunk;
  auto al = [](long long v) { return (v + 63) & ~63LL; };  // 256-byte aligned float offsets
  std::vector<Domain> dom(n);
  std::vector<float> coefs;
  std::vector<long long> vol_off(n), cx_off(n), cy_off(n);
  std::vector<int> rec_dom, rec_cell, rec_r;
  long long vol = 0, tr = 0;
  int tiles = 0;
  for (int k = 0; k < n; ++k) {
    const EfwiWindow &w = win[k];
    const ShotHost &sh = h->shots[ids[k]];
    if (w.nx < 2 * np + 5 || w.ny < 2 * np + 5 || w.x0 < 0 || w.y0 < 0 || w.x0 + w.nx > G.nx ||
        w.y0 + w.ny > G.ny)
      return fail(h, EFWI_ERR_ARG, "window %d (%d+%d, %d+%d) invalid for grid %d x %d, npml %d", k,
                  w.x0, w.nx, w.y0, w.ny, G.nx, G.ny, np);
    const long long sc = sh.src_cell;
    const int sy = (int)(sc % h->py), sx = (int)((sc / h->py) % G.nx), sz = (int)(sc / h->py / G.nx);
    const int lx = sx - w.x0, ly = sy - w.y0;
    if (lx < 2 || lx > w.nx - 3 || ly < 2 || ly > w.ny - 3)
      return fail(h, EFWI_ERR_ARG, "shot %d: source outside the updated part of its window", ids[k]);
    Domain &d = dom[k];
    const int pyw = (w.ny + 3) & ~3;
    Geo &g = d.g;
    g = h->geo;
    g.nx = w.nx; g.ny = w.ny;
    g.N = (long long)nz * w.nx * pyw;
    g.sz = (long long)w.nx * pyw;
    g.sx = pyw;
    g.slab_z = 2LL * np * w.nx * w.ny;
    g.slab_x = (long long)nz * 2 * np * w.ny;
    g.slab_y = (long long)nz * w.nx * 2 * np;
    for (int ax = 0; ax < 2; ++ax) {
      const int m = ax == 0 ? w.nx : w.ny;
      std::vector<float> c(6 * m);
      cpml_profile(m, np, ax == 0 ? G.dx : G.dy, G.f0, G.dt, c.data());
      for (int i = 0; i < m; ++i) { c[CK * m + i] = 1.0f / c[CK * m + i]; c[CKH * m + i] = 1.0f / c[CKH * m + i]; }
      (ax == 0 ? cx_off : cy_off)[k] = (long long)coefs.size();
      coefs.insert(coefs.end(), c.begin(), c.end());
      while (coefs.size() % 64) coefs.push_back(0.f);
    }
    vol_off[k] = vol;
    vol += al(12 * g.N) + al(psi_per_shot(g));
    d.src_cell = ((long long)sz * w.nx + lx) * pyw + ly;
    d.stf = h->stf.as<float>() + (size_t)ids[k] * nt;
    d.nt = nt;
    d.tiles_y = (w.ny + 31) / 32;
    d.tiles_x = (w.nx + bx - 1) / bx;
    d.nzc = (nz + zchunk - 1) / zchunk;
    d.tile0 = tiles;
    tiles += d.tiles_y * d.tiles_x * d.nzc;
    d.trace_off = tr;
    d.nrec = sh.nrec;
    tr += 3LL * sh.nrec * nt;
    for (int r = 0; r < sh.nrec; ++r) {
      const long long c = sh.rec_cell[r];
      const int y = (int)(c % h->py), x = (int)((c / h->py) % G.nx), z = (int)(c / h->py / G.nx);
      const int xl = x - w.x0, yl = y - w.y0;
      if (xl < 0 || xl >= w.nx || yl < 0 || yl >= w.ny) continue;
      rec_dom.push_back(k);
      rec_cell.push_back((int)(((long long)z * w.nx + xl) * pyw + yl));
      rec_r.push_back(r);
    }
  }
  CK_CUDA(h, h->wvol.ensure(sizeof(float) * std::max(vol, 1LL)));
  CK_CUDA(h, h->traces_tm.ensure(sizeof(float) * std::max(tr, 1LL)));
  const long long nr = (long long)rec_dom.size();
  const size_t b_dom = ((sizeof(Domain) * n + 255) / 256) * 256, b_coef = sizeof(float) * coefs.size();
  const size_t b_rec = ((sizeof(int) * nr + 255) / 256) * 256;
  CK_CUDA(h, h->wtab.ensure(b_dom + b_coef + 3 * b_rec + sizeof(long long) * n + 256));
  char *tab = h->wtab.as<char>();
  float *dcoef = (float *)(tab + b_dom);
  int *drd = (int *)(tab + b_dom + b_coef), *drc = (int *)((char *)drd + b_rec),
      *drr = (int *)((char *)drc + b_rec);
  float *V = h->wvol.as<float>();
  CK_CUDA(h, cudaMemsetAsync(h->traces_tm.p, 0, sizeof(float) * std::max(tr, 1LL), st));
  for (int k = 0; k < n; ++k) {
    Domain &d = dom[k];
    float *base = V + vol_off[k];
    d.f = fields_at(base, d.g.N, 1);
    float *model = base + 9 * d.g.N;
    d.lam = model; d.mu = model + d.g.N; d.buoy = model + 2 * d.g.N;
    d.ps = psi_at(base + al(12 * d.g.N), d.g, 1);
    d.g.cx = dcoef + cx_off[k];
    d.g.cy = dcoef + cy_off[k];
    CK_CUDA(h, cudaMemsetAsync(base, 0, sizeof(float) * 9 * d.g.N, st));
    CK_CUDA(h, cudaMemsetAsync(base + al(12 * d.g.N), 0, sizeof(float) * psi_per_shot(d.g), st));
    const float *src[3] = {h->lam.as<float>(), h->mu.as<float>(), h->buoy.as<float>()};
    for (int v = 0; v < 3; ++v)
      k_window_slice<<<592, 256, 0, st>>>(src[v], model + v * d.g.N, nz, G.nx, h->py, win[k].x0,
                                          win[k].y0, win[k].nx, win[k].ny, d.g.sx);
    h->launches[K_OTHER] += 3;
  }
  CK_CUDA(h, cudaMemcpyAsync(tab, dom.data(), sizeof(Domain) * n, cudaMemcpyHostToDevice, st));
  CK_CUDA(h, cudaMemcpyAsync(dcoef, coefs.data(), b_coef, cudaMemcpyHostToDevice, st));
  if (nr > 0) {
    CK_CUDA(h, cudaMemcpyAsync(drd, rec_dom.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, st));
    CK_CUDA(h, cudaMemcpyAsync(drc, rec_cell.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, st));
    CK_CUDA(h, cudaMemcpyAsync(drr, rec_r.data(), sizeof(int) * nr, cudaMemcpyHostToDevice, st));
  }
  rc = check_launch(h, "window set-up");
  if (rc) return rc;
  const Domain *ddom = (const Domain *)tab;
  const int ntl = nt_eff(h);
  float *ttm = h->traces_tm.as<float>();
  if (h->variant == 1) {
    long long *dsrc = (long long *)((char *)drr + b_rec);
    rc = window_loop_tma(h, dom, rec_dom, ddom, drd, drc, drr, dsrc, ttm, ntl,
                         use_graph && h->prof_sample == 0, st);
    if (rc) return rc;
    return window_traces(h, dom, traces, st);
  }
  const int blocks = multi_blocks(bx);
  auto loop = [&](cudaStream_t s) {
    for (int it = 0; it <= ntl - 2; ++it) {
      launch_fwd_multi(bx, blocks, s, ddom, n, tiles, zchunk, it);
      if (nr > 0) k_record_multi<<<(int)((nr + 127) / 128), 128, 0, s>>>(ddom, drd, drc, drr, (int)nr, ttm, it + 1);
    }
  };
  if (use_graph) {
    if (!h->cap_stream) CK_CUDA(h, cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking));
    cudaStream_t cs = h->cap_stream;
    cudaEvent_t e0, e1;
    CK_CUDA(h, cudaEventCreateWithFlags(&e0, cudaEventDisableTiming));
    CK_CUDA(h, cudaEventCreateWithFlags(&e1, cudaEventDisableTiming));
    CK_CUDA(h, cudaEventRecord(e0, st));
    CK_CUDA(h, cudaStreamWaitEvent(cs, e0, 0));
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CK_CUDA(h, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    loop(cs);
    cudaError_t ec = cudaStreamEndCapture(cs, &graph);
    if (ec == cudaSuccess) ec = cudaGraphInstantiate(&exec, graph, 0);
    if (ec == cudaSuccess) ec = cudaGraphLaunch(exec, cs);
    if (ec == cudaSuccess) ec = cudaEventRecord(e1, cs);
    if (ec == cudaSuccess) ec = cudaStreamWaitEvent(st, e1, 0);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ec != cudaSuccess) return fail(h, EFWI_ERR_CUDA, "graph of the window time loop: %s", cudaGetErrorString(ec));
  } else {
    loop(st);
  }
  h->launches[K_STRESS_FWD] += ntl - 1;
  h->launches[K_VELOCITY_FWD] += ntl - 1;
  if (nr > 0) h->launches[K_RECORD] += ntl - 1;
  return window_traces(h, dom, traces, st);
}

int efwi_gradient_windows(EfwiHandle *h, int n, const int *ids, const EfwiWindow *win,
                          const float *obs, int mode, double *misfit, float *g_lam, float *g_mu,
                          float *g_rho, void *stream) {
  int rc = check_ready(h, n, ids);
  if (rc) return rc;
  if (n > 0 && (!win || !obs)) return fail(h, EFWI_ERR_ARG, "null windows or observed data");
  if (!g_lam || !g_mu || !g_rho) return fail(h, EFWI_ERR_ARG, "null gradient output");
  if (mode != EFWI_MODE_REFERENCE && mode != EFWI_MODE_EXACT)
    return fail(h, EFWI_ERR_ARG, "gradient mode %d is not available", mode);
  cudaStream_t st = (cudaStream_t)stream;
  const EfwiGrid &G = h->grid;
  const int np = G.npml, nt = G.nt;
  const long long ncell = (long long)G.nz * G.nx * G.ny;
  for (float *g : {g_lam, g_mu, g_rho}) CK_CUDA(h, cudaMemsetAsync(g, 0, sizeof(float) * ncell, st));
  double J = 0.0;
  long long obs_off = 0;
  for (int k = 0; k < n; ++k) {
    const EfwiWindow &w = win[k];
    const ShotHost &sh = h->shots[ids[k]];
    const long long ntr = 3LL * sh.nrec * nt;
    if (w.nx < 2 * np + 5 || w.ny < 2 * np + 5 || w.x0 < 0 || w.y0 < 0 || w.x0 + w.nx > G.nx ||
        w.y0 + w.ny > G.ny)
      return fail(h, EFWI_ERR_ARG, "window %d (%d+%d, %d+%d) invalid for grid %d x %d, npml %d", k,
                  w.x0, w.nx, w.y0, w.ny, G.nx, G.ny, np);
    // the window's engine: its own grid and C-PML, the handle's tuning
    EfwiHandle *&W = h->wsub[{w.nx, w.ny}];
    if (!W) {
      EfwiGrid gw = G;
      gw.nx = w.nx;
      gw.ny = w.ny;
      rc = efwi_create(&gw, &W);
      if (rc) {
        const std::string e = W ? W->err : std::string("efwi_create failed");
        efwi_destroy(W);
        W = nullptr;
        return fail(h, rc, "window %d: %s", k, e.c_str());
      }
    }
    W->if_win = h->if_win; W->bx = h->bx; W->zchunk = h->zchunk; W->max_batch = 1;
    W->variant = h->variant; W->fcfg = h->fcfg; W->rcfg = h->rcfg; W->zchunk_rev = h->zchunk_rev;
    W->nt_limit = h->nt_limit; W->use_graphs = h->use_graphs; W->ck_budget = h->ck_budget;
    W->lanes = 1;
    // model: the window of the resident model volumes (as efwi_forward_windows)
    CK_CUDA(W, W->lam.ensure(sizeof(float) * W->N));
    CK_CUDA(W, W->mu.ensure(sizeof(float) * W->N));
    CK_CUDA(W, W->buoy.ensure(sizeof(float) * W->N));
    const float *src[3] = {h->lam.as<float>(), h->mu.as<float>(), h->buoy.as<float>()};
    float *dst[3] = {W->lam.as<float>(), W->mu.as<float>(), W->buoy.as<float>()};
    for (int v = 0; v < 3; ++v)
      k_window_slice<<<592, 256, 0, st>>>(src[v], dst[v], G.nz, G.nx, h->py, w.x0, w.y0, w.nx,
                                          w.ny, W->py);
    h->launches[K_OTHER] += 3;
    W->model_set = true;
    // survey: the shot with window-relative coordinates and the receivers
    // inside the window
    const long long sc = sh.src_cell;
    const int sy = (int)(sc % h->py), sx = (int)((sc / h->py) % G.nx), sz = (int)(sc / h->py / G.nx);
    std::vector<int> zr, xr, yr, sel;
    for (int r = 0; r < sh.nrec; ++r) {
      const long long c = sh.rec_cell[r];
      const int y = (int)(c % h->py), x = (int)((c / h->py) % G.nx), z = (int)(c / h->py / G.nx);
      if (x < w.x0 || x >= w.x0 + w.nx || y < w.y0 || y >= w.y0 + w.ny) continue;
      zr.push_back(z); xr.push_back(x - w.x0); yr.push_back(y - w.y0); sel.push_back(r);
    }
    std::vector<float> w0, w1, wt;
    for (int r : sel) { w0.push_back(sh.win0[r]); w1.push_back(sh.win1[r]); wt.push_back(sh.wts[r]); }
    EfwiShot es{};
    es.z_src = sz; es.x_src = sx - w.x0; es.y_src = sy - w.y0;
    es.nrec = (int)sel.size();
    es.z_rec = zr.data(); es.x_rec = xr.data(); es.y_rec = yr.data();
    es.win_start = w0.data(); es.win_end = w1.data(); es.weights = wt.data();
    es.src_weight = sh.src_w;
    rc = efwi_set_survey(W, 1, &es, h->stf_host.data() + (size_t)ids[k] * nt);
    if (rc) return fail(h, rc, "window %d: %s", k, W->err.c_str());
    // observed data of those receivers
    const long long nw = 3LL * (long long)sel.size() * nt;
    CK_CUDA(h, h->wobs.ensure(sizeof(float) * std::max(nw, 1LL)));
    if (!sel.empty()) {
      CK_CUDA(h, h->wsel.ensure(sizeof(int) * sel.size()));
      CK_CUDA(h, cudaMemcpyAsync(h->wsel.p, sel.data(), sizeof(int) * sel.size(),
                                 cudaMemcpyHostToDevice, st));
      k_gather_rows<<<592, 256, 0, st>>>(obs + obs_off, h->wsel.as<int>(), (int)sel.size(),
                                         sh.nrec, nt, h->wobs.as<float>());
      h->launches[K_OTHER]++;
    }
    const long long nwc = (long long)G.nz * w.nx * w.ny;
    CK_CUDA(h, h->wimg.ensure(sizeof(float) * 3 * nwc));
    float *gw = h->wimg.as<float>();
    const int zero = 0;
    double Jk = 0.0;
    rc = efwi_gradient(W, 1, &zero, h->wobs.as<float>(), mode, &Jk, gw, gw + nwc, gw + 2 * nwc,
                       nullptr, st);
    if (rc) return fail(h, rc, "window %d: %s", k, W->err.c_str());
    float *outs[3] = {g_lam, g_mu, g_rho};
    for (int v = 0; v < 3; ++v)
      k_window_add<<<592, 256, 0, st>>>(outs[v], gw + v * nwc, G.nz, G.nx, G.ny, w.x0, w.y0, w.nx,
                                        w.ny);
    h->launches[K_OTHER] += 3;
    // One window's workspace at a time: the window engine keeps its grid,
    // coefficients and shell table, and gives back its state, shell store
    // and checkpoints (their graphs go with them).
    CK_CUDA(h, cudaStreamSynchronize(st));
    for (DevBuf *b : {&W->fields, &W->psi, &W->adj, &W->grad, &W->shell, &W->ckpt, &W->apsi,
                      &W->traces_tm, &W->res_tm})
      b->release();
    W->g_fwd.reset();
    W->g_rev.reset();
    for (int c = 0; c < K_NCLASS; ++c) {
      h->launches[c] += W->launches[c];
      W->launches[c] = 0;
    }
    J += Jk;
    obs_off += ntr;
  }
  rc = check_launch(h, "window gradients");
  if (rc) return rc;
  CK_CUDA(h, cudaStreamSynchronize(st));
  if (misfit) *misfit = J;
  return EFWI_OK;
}

int efwi_adjoint(EfwiHandle *h, int n, const int *ids, const float *adj_src, float *g_lam,
                 float *g_mu, float *g_rho, void *stream) {
  int rc = check_ready(h, n, ids);
  if (rc) return rc;
  if (n > 0 && !adj_src) return fail(h, EFWI_ERR_ARG, "null adjoint source");
  if (!g_lam || !g_mu || !g_rho) return fail(h, EFWI_ERR_ARG, "null gradient output");
  return gradient_impl(h, n, ids, adj_src, EFWI_MODE_EXACT, nullptr, g_lam, g_mu, g_rho, nullptr,
                       (cudaStream_t)stream, true);
}

int efwi_illumination(EfwiHandle *h, int n, const int *ids, float *h_lam, float *h_mu,
                      float *h_rho, void *stream) {
  int rc = check_ready(h, n, ids);
  if (rc) return rc;
  if (!h_lam || !h_mu || !h_rho) return fail(h, EFWI_ERR_ARG, "null illumination output");
  cudaStream_t st = (cudaStream_t)stream;
  const long long N = h->N;
  const int nt = h->grid.nt;
  rc = status_reset(h, st);
  if (rc) return rc;
  CK_CUDA(h, h->grad.ensure(sizeof(float) * 3 * N));
  CK_CUDA(h, cudaMemsetAsync(h->grad.p, 0, sizeof(float) * 3 * N, st));
  float *il = h->grad.as<float>(), *im = il + N, *ib = il + 2 * N;
  for (int b0 = 0; b0 < n; b0 += h->max_batch) {
    const int S = std::min(h->max_batch, n - b0);
    long long ntr = 0;
    for (int s = 0; s < S; ++s) ntr += 3LL * h->shots[ids[b0 + s]].nrec * nt;
    CK_CUDA(h, h->traces_tm.ensure(sizeof(float) * std::max(ntr, 1LL)));
    Batch b;
    rc = prepare_batch(h, ids + b0, S, h->traces_tm.as<float>(), ntr, st, &b);
    if (rc) return rc;
    RecArgs norec = b.rec;
    norec.ncell = 0;
    const int ntl = nt_eff(h);
    const dim3 grid((h->grid.ny + 31) / 32, (h->grid.nx + 3) / 4, (h->grid.nz - 4 + 7) / 8);
    for (int it = 0; it <= ntl - 2; ++it) {
      b.src.it = it;
      rc = forward_step(h, b.f, b.ps, S, b.src, norec, nullptr, st, it, b.mp);
      if (rc) return rc;
      Timer t(h, K_OTHER, st, it);
      k_illumination<<<grid, dim3(32, 4), 0, st>>>(h->geo, b.f, b.ps, S, h->buoy.as<float>(),
                                                   it + 1 <= ntl - 2, il, im, ib);
    }
  }
  const EfwiGrid &G = h->grid;
  k_buoy_to_rho_sq<<<1184, 256, 0, st>>>(ib, h->buoy.as<float>(), G.nz, G.nx, G.ny, h->py);
  k_pitch_copy<<<1184, 256, 0, st>>>(il, h_lam, G.nz, G.nx, G.ny, h->py, 0);
  k_pitch_copy<<<1184, 256, 0, st>>>(im, h_mu, G.nz, G.nx, G.ny, h->py, 0);
  k_pitch_copy<<<1184, 256, 0, st>>>(ib, h_rho, G.nz, G.nx, G.ny, h->py, 0);
  h->launches[K_OTHER] += 4;
  rc = check_launch(h, "illumination");
  if (rc) return rc;
  return status_check(h, st);
}

int efwi_set_stf_gradient(EfwiHandle *h, float *g_stf) {
  if (!h) return EFWI_ERR_ARG;
  h->gstf = g_stf;
  return EFWI_OK;
}

int efwi_set_scratch(EfwiHandle *h, float *syn_w, float *obs_w, float *res) {
  if (!h) return EFWI_ERR_ARG;
  h->scr_syn = syn_w;
  h->scr_obs = obs_w;
  h->scr_res = res;
  return EFWI_OK;
}

int efwi_set_checkpoint_budget(EfwiHandle *h, long long bytes) {
  if (!h || bytes < 0) return EFWI_ERR_ARG;
  h->ck_budget = bytes;
  return EFWI_OK;
}

long long efwi_state_bytes(const EfwiHandle *h) { return h ? state_floats(h) * 4 : -1; }

int efwi_checkpoint_stats(const EfwiHandle *h, long long *forward_steps, int *slots) {
  if (!h) return EFWI_ERR_ARG;
  if (forward_steps) *forward_steps = h->ck_forward_steps;
  if (slots) *slots = h->ck_slots;
  return EFWI_OK;
}

int efwi_checkpoint_plan(int nt, int slots, long long *forward_steps, int *slots_used,
                         int *repetitions, int *actions, int max_actions) {
  if (nt < 1 || slots < 0 || max_actions < 0) return -1;
  CkPlan plan;
  plan.build(nt, slots, actions ? max_actions : 64LL * nt + 4096);
  if (plan.too_long) return -1;
  if (forward_steps) *forward_steps = plan.forward_steps;
  if (slots_used) *slots_used = plan.slots_used;
  if (repetitions) *repetitions = plan.repetitions;
  if (actions)
    for (size_t k = 0; k < plan.actions.size(); ++k) {
      actions[3 * k] = plan.actions[k].op;
      actions[3 * k + 1] = plan.actions[k].a;
      actions[3 * k + 2] = plan.actions[k].b;
    }
  return (int)plan.actions.size();
}

int efwi_step(EfwiHandle *h, float *state, int transpose, void *stream) {
  if (!h) return EFWI_ERR_ARG;
  if (!h->model_set) return fail(h, EFWI_ERR_STATE, "efwi_set_model has not been called");
  if (!state) return fail(h, EFWI_ERR_ARG, "null state");
  cudaStream_t st = (cudaStream_t)stream;
  const long long N = h->N, P = psi_per_shot(h->geo);
  CK_CUDA(h, h->fields.ensure(sizeof(float) * 9 * N));
  CK_CUDA(h, h->psi.ensure(sizeof(float) * P));
  CK_CUDA(h, h->adj.ensure(sizeof(float) * 9 * N));
  CK_CUDA(h, h->apsi.ensure(sizeof(float) * 2 * P));
  CK_CUDA(h, cudaMemsetAsync(h->fields.p, 0, sizeof(float) * 9 * N, st));
  CK_CUDA(h, cudaMemsetAsync(h->psi.p, 0, sizeof(float) * P, st));
  Fields f = fields_at(h->fields.as<float>(), N, 1);
  Psi ps = psi_at(h->psi.as<float>(), h->geo, 1);
  int rc = status_reset(h, st);
  if (rc) return rc;
  if (!transpose) {
    k_state_convert<<<1184, 256, 0, st>>>(h->geo, state, f, ps, 1);
    FwdMaps maps;
    const FwdMaps *mp = nullptr;
    if (h->variant == 1) {
      rc = make_fwd_maps(h, f, 1, &maps);
      if (rc) return rc;
      mp = &maps;
    }
    RecArgs norec{};
    SrcArgs nosrc{nullptr, nullptr, h->grid.nt, 0};
    rc = forward_step(h, f, ps, 1, nosrc, norec, nullptr, st, 0, mp);
    if (rc) return rc;
    k_state_convert<<<1184, 256, 0, st>>>(h->geo, state, f, ps, 0);
  } else {
    Fields a = fields_at(h->adj.as<float>(), N, 1);
    Psi ap = psi_at(h->apsi.as<float>(), h->geo, 1);
    CK_CUDA(h, cudaMemsetAsync(h->adj.p, 0, sizeof(float) * 9 * N, st));
    CK_CUDA(h, cudaMemsetAsync(h->apsi.p, 0, sizeof(float) * 2 * P, st));
    k_state_convert<<<1184, 256, 0, st>>>(h->geo, state, a, ap, 1);
    int nzc;
    const dim3 grid = stencil_grid(h, 1, h->bx, h->zchunk_rev, &nzc);
    launch_adj_velocity_exact(h->bx, grid, st, exact_args(h, f, ps, a, 0, nullptr, nullptr), h->zchunk_rev, nzc);
    launch_adj_stress_exact(h->bx, grid, st, exact_args(h, f, ps, a, 0, nullptr, nullptr), h->zchunk_rev, nzc);
    Psi out = psi_at(h->apsi.as<float>() + P, h->geo, 1);
    k_state_convert<<<1184, 256, 0, st>>>(h->geo, state, a, out, 0);
  }
  h->launches[K_OTHER] += 2;
  rc = check_launch(h, "step");
  if (rc) return rc;
  return status_check(h, st);
}

int efwi_profile(EfwiHandle *h, int sample) {
  if (!h || sample < 0) return EFWI_ERR_ARG;
  h->prof_sample = sample;
  return EFWI_OK;
}

int efwi_profile_read(EfwiHandle *h, int n, long long *timed, double *ms, long long *launches) {
  if (!h) return EFWI_ERR_ARG;
  int rc = resolve_profile(h);
  if (rc) return rc;
  for (int k = 0; k < n && k < K_NCLASS; ++k) {
    if (timed) timed[k] = h->timed[k];
    if (ms) ms[k] = h->ms[k];
    if (launches) launches[k] = h->launches[k];
    h->timed[k] = 0; h->ms[k] = 0; h->launches[k] = 0;
  }
  return EFWI_OK;
}

}  // extern "C"
