/*
 * efwi.h -- C ABI of the B200 elastic wave-propagation engine (EFWI-3D
 * operator).  Plain pointers and sizes only; no torch types.
 *
 * Conventions
 *   - Volumes are float32 [nz][nx][ny] (y fastest), DEVICE pointers, on the
 *     padded grid: the caller's torch tensors are passed as they are (the
 *     reference transposed them on the host, Ops/FWI/Src_3d/libCUFD.cu:72-80).
 *   - Traces are float32 [3][nrec][nt] per shot (components x, y, z), the
 *     layout of the reference's Shot_{x,y,z}{id}.bin files
 *     (libCUFD.cu:709-720); several shots are concatenated in call order.
 *   - Source and receiver indices are padded-grid indices (the reference
 *     adds nPoints_pml to survey coordinates, Src_Rec.cu:78-118).
 *   - Every call returns EFWI_OK or an error code and never exits the
 *     process (the reference calls exit(1), utilities.h:22-30); the message
 *     is in efwi_last_error().
 *   - All device work of a call is enqueued on `stream` (a cudaStream_t, or
 *     NULL for the legacy default stream).  A handle is used from one host
 *     thread at a time.
 */
#ifndef EFWI_H_
#define EFWI_H_

#ifdef __cplusplus
extern "C" {
#endif

#define EFWI_OK 0
#define EFWI_ERR_ARG 1     /* invalid argument or survey */
#define EFWI_ERR_CUDA 2    /* CUDA runtime error */
#define EFWI_ERR_CFL 3     /* Courant number > 1 (utilities.cu:186-202) */
#define EFWI_ERR_STATE 4   /* call order: model or survey missing */
#define EFWI_ERR_NOMEM 5   /* device allocation failed */
#define EFWI_ERR_TOO_LARGE 6 /* request exceeds a fixed-size buffer (efwi_misfit_noalloc) */

#define EFWI_MODE_REFERENCE 0 /* the reference's gradient (libCUFD.cu:469-613) */
#define EFWI_MODE_EXACT 1     /* exact discrete adjoint of the forward scheme */

typedef struct EfwiHandle EfwiHandle;

/* Grid and time axis; the fields of the reference's para JSON
 * (Parameter.cpp:39-104: nz, nx, ny, dz, dx, dy, nSteps, dt, f0,
 * nPoints_pml). */
typedef struct {
  int nz, nx, ny;
  int npml;
  int nt;
  float dz, dx, dy, dt, f0;
} EfwiGrid;

/* One shot of the survey (Src_Rec.cu:74-206).  Host pointers, copied. */
typedef struct {
  int z_src, x_src, y_src;
  int nrec;
  const int *z_rec, *x_rec, *y_rec;
  const float *win_start, *win_end; /* [nrec] seconds; windowed misfit only; may be NULL */
  const float *weights;             /* [nrec] or NULL (all ones); windowed misfit only */
  float src_weight;                 /* windowed misfit only */
} EfwiShot;

/* Replaces: cufd set-up (libCUFD.cu:52-91) and Cpml (Cpml.cu:7-99). */
int efwi_create(const EfwiGrid *grid, EfwiHandle **out);
void efwi_destroy(EfwiHandle *h);
const char *efwi_last_error(const EfwiHandle *h);
const char *efwi_version(void);

/* Misfit windowing (para `if_win`, Parameter.cpp:146-150) and launch
 * shape: tile_bx in {4, 8} (x rows per CTA; 0 keeps), zchunk > 0 (z planes
 * per CTA; 0 keeps), max_batch >= 1 shots per forward launch (0 keeps). */
int efwi_set_options(EfwiHandle *h, int if_win, int tile_bx, int zchunk, int max_batch);

/* Kernel family of the stencil sweeps: 1 (default) stages the x/y-halo
 * operands of every z plane in shared memory with bulk tensor copies
 * (TMA); 0 reads them through L1.  Both give identical results.  No
 * reference counterpart (the reference has one plain kernel per update). */
int efwi_set_variant(EfwiHandle *h, int variant);

/* CUDA graphs of the time loops (default on): the forward time loop of a
 * batch and the reverse time loop of a reference-mode gradient shot are
 * captured once and replayed while their launch parameters (buffers,
 * tensor maps, tuning, time axis) are unchanged, across shots and calls.
 * on = 0 launches them one by one (results are bitwise the same).  Runs with
 * kernel-event sampling (efwi_profile) launch eagerly.  No reference
 * counterpart (the reference launches about 25 kernels per step from the
 * host, libCUFD.cu:312-354, 532-612). */
int efwi_set_graphs(EfwiHandle *h, int on);

/* Launch configuration of the TMA kernels (the autotuner's knobs; results
 * do not depend on them): fwd_cfg in 0..3 and rev_cfg in 0..7 select tile,
 * ring depth and occupancy target (rev_cfg 6, 7 run the reverse-velocity
 * kernel as two launches); zchunk_* > 0 sets the z planes per CTA (0 keeps).
 * No reference counterpart. */
int efwi_set_tuning(EfwiHandle *h, int fwd_cfg, int zchunk_fwd, int rev_cfg, int zchunk_rev);

/* Shot lanes of reference-mode efwi_misfit / efwi_gradient calls of two or
 * more shots (replaces the reference's serial shot loop on one GPU,
 * libCUFD.cu:220-798): lanes in [1, 8], default 2.  Lane 0 runs on the
 * caller's stream; every further lane has its own workspace (state,
 * boundary-shell store, images: about 9 floats per boundary-shell cell and
 * time step plus 21 volumes) and its own stream and host thread, and takes
 * a contiguous share of the shots, so kernels of different shots share
 * the GPU.  A lane whose workspace does not fit in device memory is
 * dropped for the call.  The misfit is identical to one lane; images
 * differ by the order of the per-shot sums only.  Kernel events of
 * efwi_profile are recorded on lane 0 only; launches are counted on all
 * lanes.  Lowering the count
 * frees the dropped lanes' workspace.  The call stays synchronous. */
int efwi_set_lanes(EfwiHandle *h, int lanes);

/* Timing probes: nt_limit > 0 stops the time loops after nt_limit steps
 * (results are then not meaningful); 0 restores the full axis.  No
 * reference counterpart. */
int efwi_set_nt_limit(EfwiHandle *h, int nt_limit);

/* Replaces: Model (Model.cu:15-80) and the CFL check compCourantNumber
 * (utilities.cu:186-202).  lam, mu, rho: device [nz][nx][ny]; copied. */
int efwi_set_model(EfwiHandle *h, const float *lam, const float *mu, const float *rho,
                   void *stream);

/* Replaces: Src_Rec (Src_Rec.cu:20-249).  stf: host [nshot][nt] source
 * time functions (untapered; the 0.001 taper of Src_Rec.cu:146 is applied
 * here).  Shot k of later calls is shots[k]. */
int efwi_set_survey(EfwiHandle *h, int nshot, const EfwiShot *shots, const float *stf);

/* Replaces: cufd with calc_id 2 (observed data, libCUFD.cu:312-368).
 * traces: device, concatenation over shot_ids of [3][nrec][nt]. */
int efwi_forward(EfwiHandle *h, int n, const int *shot_ids, float *traces, void *stream);

/* Replaces: cufd with calc_id 0 (misfit only, libCUFD.cu:371-420).
 * obs: device, traces layout.  misfit: host. */
int efwi_misfit(EfwiHandle *h, int n, const int *shot_ids, const float *obs, double *misfit,
                void *stream);

/* Replaces: cufd with calc_id 1 (misfit and gradients, libCUFD.cu:220-652).
 * g_lam, g_mu, g_rho: device [nz][nx][ny], overwritten.  mode:
 * EFWI_MODE_REFERENCE or EFWI_MODE_EXACT.  res (optional, device, traces
 * layout): receives the adjoint source of each shot.
 * EFWI_MODE_REFERENCE follows the reference's algorithm (boundary-shell
 * reconstruction and its adjoint kernels, libCUFD.cu:469-613).
 * EFWI_MODE_EXACT (no reference counterpart) returns dJ/dlambda, dJ/dmu and
 * dJ/drho of the returned misfit J, by the exact discrete adjoint of the
 * forward scheme with binomial checkpointing of the whole state under the
 * byte budget of efwi_set_checkpoint_budget; it returns EFWI_ERR_TOO_LARGE
 * when the budget would need more than 16 forward steps per time step. */
int efwi_gradient(EfwiHandle *h, int n, const int *shot_ids, const float *obs, int mode,
                  double *misfit, float *g_lam, float *g_mu, float *g_rho, float *res,
                  void *stream);

/* Shot windows (no reference counterpart): shot k runs on its own aperture
 * window of the padded grid,
 * x in [x0, x0 + nx), y in [y0, y0 + ny), all z, with its own C-PML of npml
 * cells inside the window edges; receivers outside the window record
 * zeros.  With the TMA variant (efwi_set_variant 1, the default) every
 * window runs the forward TMA kernels as its own grid (forward cfg and
 * zchunk of efwi_set_tuning), groups of windows on up to 8 internal
 * streams; use_graph is ignored.  With the L1 variant all windows of a
 * call advance together in one persistent launch per half-step (tile_bx
 * and zchunk of efwi_set_options); use_graph = 1 captures the whole time
 * loop in a CUDA graph and launches it once.  With the TMA variant,
 * use_graph = 1 captures one time step (every group, as parallel branches)
 * in a CUDA graph and replays it once per step, the step index read from a
 * device word.  All forms give the same bits.
 * traces: device, concatenation over shot_ids of [3][nrec][nt].  The call
 * synchronises the stream. */
typedef struct {
  int x0, y0, nx, ny;
} EfwiWindow;
int efwi_forward_windows(EfwiHandle *h, int n, const int *shot_ids, const EfwiWindow *windows,
                         float *traces, int use_graph, void *stream);

/* Misfit and gradients of shots on windows (no reference counterpart): shot
 * k on window k as in efwi_forward_windows (its own grid and C-PML, the
 * window of the resident model), by the gradient `mode` of efwi_gradient on
 * that grid; the receivers inside the window take part (obs: device, the
 * shots' full [3][nrec][nt] blocks), the images are added into the full
 * grid's g_lam, g_mu, g_rho (device, [nz][nx][ny], zeroed here) at the
 * window's place, and misfit is the sum over the windows.  Synchronises the
 * stream. */
int efwi_gradient_windows(EfwiHandle *h, int n, const int *shot_ids, const EfwiWindow *windows,
                          const float *obs, int mode, double *misfit, float *g_lam, float *g_mu,
                          float *g_rho, void *stream);

/* J^T applied to an adjoint source (no reference counterpart): the exact
 * adjoint of the forward modelling of the shots, with the device traces
 * adj_src (traces layout, the derivative of some objective with respect to
 * the synthetic traces) injected at the receivers, checkpointed as in
 * EFWI_MODE_EXACT.  g_lam, g_mu, g_rho as in efwi_gradient.  Serves
 * random-probe estimates of diag(J^T J) (E[(J^T w)^2] for white w). */
int efwi_adjoint(EfwiHandle *h, int n, const int *shot_ids, const float *adj_src, float *g_lam,
                 float *g_mu, float *g_rho, void *stream);

/* Source illumination: the diagonal pseudo-Hessian of Shin et al. (2001),
 * summed over the shots and time steps -- at every cell the squared
 * derivative of the forward step with respect to lambda, mu and rho
 * applied to the forward wavefield.  No reference counterpart.  Outputs:
 * device [nz][nx][ny], overwritten. */
int efwi_illumination(EfwiHandle *h, int n, const int *shot_ids, float *h_lam, float *h_mu,
                      float *h_rho, void *stream);

/* Exact-gradient checkpoints (no reference counterpart; the reference keeps
 * only the boundary shell, Boundary.cu).  bytes: HBM for checkpoint slots
 * (default 4 GiB); one slot holds one state of efwi_state_bytes(h) bytes.
 * efwi_checkpoint_stats: forward steps and slots of the last exact
 * gradient's shot.  efwi_checkpoint_plan (host only, no handle): the
 * schedule for nt time steps and `slots` slots -- total forward steps,
 * slots used, repetition number, and (if actions is not NULL) up to
 * max_actions (op, a, b) triples with op 0 advance a->b, 1 store slot a,
 * 2 restore slot a (-1: the zero state), 3 adjoint block a.  Returns the
 * number of actions, or -1 if they exceed max_actions. */
int efwi_set_checkpoint_budget(EfwiHandle *h, long long bytes);
long long efwi_state_bytes(const EfwiHandle *h);
int efwi_checkpoint_stats(const EfwiHandle *h, long long *forward_steps, int *slots);
int efwi_checkpoint_plan(int nt, int slots, long long *forward_steps, int *slots_used,
                         int *repetitions, int *actions, int max_actions);

/* One time step of the forward scheme without source (transpose = 0; the
 * linear map of stress.cu:36-97 then velocity.cu:35-96), or of its exact
 * transpose (transpose = 1), applied in place to a device state
 * [27][nz][nx][ny]: vz vx vy szz sxx syy sxz sxy syz, then the memory
 * variables m_vz_z m_vz_x m_vz_y m_vx_z m_vx_x m_vx_y m_vy_z m_vy_x m_vy_y
 * m_szz_z m_sxx_x m_syy_y m_sxz_z m_sxz_x m_sxy_x m_sxy_y m_syz_y m_syz_z
 * (full grids; only their C-PML slabs are read and written).  No reference
 * counterpart; it serves dot-product tests of the adjoint. */
int efwi_step(EfwiHandle *h, float *state, int transpose, void *stream);

/* Source-time-function gradient (the reference returns zeros,
 * Torch_Fwi.cpp:73,96): while g_stf (device [n][nt]) is set, every
 * EFWI_MODE_EXACT gradient also writes dJ/dstf of its n shots, row k for
 * shot_ids[k], with respect to the untapered stf rows given to
 * efwi_set_survey.  NULL disables. */
int efwi_set_stf_gradient(EfwiHandle *h, float *g_stf);

/* Scratch outputs (the reference's scratch_dir_name dumps,
 * libCUFD.cu:660-700): while set, every misfit of efwi_misfit /
 * efwi_gradient also writes the windowed synthetics (syn_w), the windowed
 * observed data (obs_w) and the adjoint source (res) of its shots -- device
 * buffers in the traces layout of that call's `obs`; NULL disables each. */
int efwi_set_scratch(EfwiHandle *h, float *syn_w, float *obs_w, float *res);

/* Misfit and adjoint source of one shot with no device allocation.  No
 * counterpart in the reference.  For callers that cannot call cudaMalloc
 * (device memory reserved up front by another allocator, or a
 * latency-critical path that cannot take cudaMalloc's device-wide
 * synchronisation); needs no handle.  obs, syn (inputs) and res (output) are
 * device [3][nrec][nt] traces of one shot; misfit is a device double
 * (output).  Windowed mode (if_win) takes device [nrec] win_start, win_end
 * (seconds) and weights; otherwise they may be NULL.  Same window, residual
 * and sum of squares as efwi_misfit / efwi_gradient.  Scratch: a file-scope
 * device array of EFWI_NOALLOC_MAX_PARTIALS doubles (512 KiB per GPU, held
 * until exit); requests needing more than that many 32 x 32 tiles
 * (3 * ceil(nt/32) * ceil(nrec/32)) return EFWI_ERR_TOO_LARGE.  The first
 * call on a device looks up the array's address and should come before any
 * stream capture.  Calls that overlap on the GPU race on the array.  The
 * address is kept per device for the life of the process: it assumes the
 * device's primary context is never destroyed (after cudaDeviceReset the
 * library must be reloaded before this entry point is called again). */
#define EFWI_NOALLOC_MAX_PARTIALS 65536
int efwi_misfit_noalloc(int nrec, int nt, float dt, int if_win, const float *win_start,
                        const float *win_end, const float *weights, float src_weight,
                        const float *obs, const float *syn, float *res, double *misfit,
                        void *stream);

/* Learned gradient preconditioner: 3x3x3 convolutions with 16 input and 16
 * output channels on BF16 tensor cores, FP32 accumulation (no reference
 * counterpart).  x, y_bf16: device [D][H][W][16] bf16 (channels last);
 * w: device [27][16 co][16 ci] bf16, tap (dz+1)*9 + (dy+1)*3 + (dx+1);
 * bias: device [16] f32 or NULL.  Zero padding of 1, stride 1.
 * efwi_conv3d_forward: y = relu?(conv(x, w) + bias) into y_bf16 and/or
 * y_f32 ([D][H][W][16] f32); with w'[t][a][b] = w[26-t][b][a] it gives the
 * gradient of the input.  efwi_conv3d_wgrad: dw[t][co][ci] = sum over
 * voxels of dy[v][co] x[v + off_t][ci] (f32), through `nparts` partial sums
 * of 27*256 floats each in `partial`, added in a fixed order.  Return 0, 1
 * (bad argument) or 2 (launch error). */
int efwi_conv3d_forward(const void *x, const void *w, const float *bias, int D, int H, int W,
                        int relu, void *y_bf16, float *y_f32, void *stream);
int efwi_conv3d_wgrad(const void *x, const void *dy, int D, int H, int W, float *partial,
                      int nparts, float *dw, void *stream);
/* Kernel form of efwi_conv3d_forward for this process: 0 = mma.sync;
 * 1 = tcgen05.mma with the accumulator in tensor memory (128 voxels x 16
 * channels per tile, one MMA per tap), tile staged by loads; 2 / 3 = the
 * same MMAs with the tiles staged by bulk tensor copies two / three stages
 * deep and the next tile's MMAs overlapping this tile's epilogue; 4 / 5 =
 * the same warp-specialised (one warp issues the copies and MMAs, four
 * drain the accumulators; mbarriers between them), two / three stages.  All
 * give the same sums up to FP32 rounding order.  The tcgen05 forms need w
 * and the outputs 16-byte aligned and fall back to mma.sync otherwise.
 * Returns 1 for an unknown form.  efwi_conv3d_status reads and clears the
 * flag the tcgen05 forms set when a bounded wait for the tensor cores or
 * the copies ran out (the call's outputs are then incomplete).  Default 2. */
int efwi_conv3d_set_kernel(int form);
int efwi_conv3d_status(int *timed_out, void *stream);
/* Kernel form of efwi_conv3d_wgrad for this process: 1 = tcgen05.mma (eight
 * taps stacked on the 128 rows of one MMA, K = 16 voxels, accumulators in
 * tensor memory; 16-byte aligned inputs; the default), 0 = mma.sync.  The
 * same sums up to FP32 rounding order; a bounded wait that ran out sets the
 * efwi_conv3d_status flag and leaves NaN in that CTA's partial sums. */
int efwi_conv3d_set_wgrad_kernel(int tcgen05);

/* Per-kernel timing with CUDA events on the call's stream (the time steps
 * it with it % sample == sample / 2; 0 disables).  efwi_profile_read fills, for each
 * kernel class k < n, the number of timed launches, their total time in
 * milliseconds and the total number of launches of the class, and resets
 * the counters.  Class names: efwi_kernel_name(k). */
int efwi_profile(EfwiHandle *h, int sample);
int efwi_profile_read(EfwiHandle *h, int n, long long *timed, double *ms, long long *launches);
const char *efwi_kernel_name(int k);
int efwi_kernel_count(void);

#ifdef __cplusplus
}
#endif
#endif /* EFWI_H_ */
