/*
 * wakis_b200 -- C ABI of the B200 (sm_100a) FIT leap-frog stepper and wake
 * integration.
 *
 * Every entry point takes plain pointers and sizes (device pointers for
 * field data, host pointers for descriptors), returns 0 on success, a
 * positive WK_E_* code for an argument error detected on the host, or a
 * negative value -(cudaError_t) for a CUDA error.  wk_last_error() returns a
 * thread-local message for the last failure.  No entry point allocates or
 * frees device memory: the caller (the Python host, through PyTorch) owns
 * every buffer.  All work is enqueued on the given stream (a cudaStream_t
 * passed as void*; NULL = legacy default stream) and is asynchronous.
 *
 * Field layout (same as upstream wakis/field.py:57-76,139-190): a field is a
 * flat array of 3*N elements, N = Nx*Ny*Nz, holding the x, y and z component
 * blocks; inside a block n = i + j*Nx + k*Nx*Ny.
 */
#ifndef WAKIS_B200_H
#define WAKIS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define WK_ABI_VERSION 1

#define WK_OK 0
#define WK_E_NULL 1      /* required pointer is NULL                     */
#define WK_E_SHAPE 2     /* non-positive or too large dimension          */
#define WK_E_DTYPE 3     /* unsupported dtype / id width                 */
#define WK_E_ALIGN 4     /* pointer not aligned to its element size      */
#define WK_E_RANGE 5     /* index (beam line, capture window) off-grid   */
#define WK_E_MODE 6      /* inconsistent mode flags                      */
#define WK_E_TIMEOUT 7   /* a device-side wait ran out (wk_read_status)  */

#define WK_F64 0
#define WK_F32 1
#define WK_F32C 2   /* FP32 state with bf16 compensation words (Ec, Hc);
                       coefficient tables FP64; Ez capture FP64          */

/* J source used by the E half-step (upstream computes E += dt*(B*H - ieps*J)
 * with J the stored current, solverFIT3D.py:492-503). */
#define WK_J_ZERO 0      /* J = 0 everywhere except the beam line           */
#define WK_J_SIGMA_E 1   /* J = sigma * E_old (the value upstream stored at
                            the end of the previous step), beam line aside  */
#define WK_J_ARRAY 2     /* J read from `J`; with use_conductivity the
                            kernel also writes J = sigma * E_new back       */

/*
 * Geometry, coefficients and state of one FIT grid.  Field-type arrays
 * (E, H, J, metrics, material table) hold `dtype` elements; with WK_F32C
 * the state (E, H, J) is float and the metrics and material table double.
 *
 * Metric tables (values as upstream's diagonal matrices hold them after the
 * boundary folding of wakis/boundaries.py:35-181, cast to dtype):
 *   L{x,y,z}[Nx|Ny|Nz], tL{x,y,z}[Nx|Ny|Nz]    primal / dual edge lengths
 *   iAx[j + k*Ny], iAy[i + k*Nx], iAz[i + j*Nx] inverse primal face areas
 *   itAx, itAy, itAz (same indexing)           inverse dual face areas
 * Materials: mat_id[n] (id_bytes = 1, 2 or 4 per cell) indexes
 *   mat_table[9*id + {0,1,2}] = ieps (x,y,z), {3,4,5} = imu, {6,7,8} = sigma.
 * Boundary faces, order x-lo, x-hi, y-lo, y-hi, z-lo, z-hi:
 *   pec_face[f] = 0 masks the tangential E columns of the curl on face f
 *   (C <- C*Dbc, boundaries.py:72-110); pmc_face[f] = 0 masks the tangential
 *   H rows (C <- Dbc*C, boundaries.py:112-150).  has_pec / has_pmc say
 *   whether the mask exists at all.  h_sum_desc = 1 sums the four terms of
 *   an H row in descending column order (the row order scipy leaves in
 *   the assembled H operator when exactly one of the two masks exists).
 */
typedef struct wk_fit_desc {
  int Nx, Ny, Nz;
  int dtype;               /* WK_F64 or WK_F32                               */
  void* E[2];              /* ping-pong state buffers, 3N each; E[par] live  */
  void* H[2];
  int par;                 /* index of the live buffers                      */
  void* J;                 /* 3N, used for WK_J_ARRAY                        */
  int j_mode;
  int use_conductivity;
  const void* mat_id;
  int id_bytes;
  const void* mat_table;
  int n_mat;
  const void *Lx, *Ly, *Lz, *tLx, *tLy, *tLz;
  const void *iAx, *iAy, *iAz, *itAx, *itAy, *itAz;
  int pec_face[6];
  int pmc_face[6];
  int has_pec, has_pmc;
  int h_sum_desc;
  double dt;               /* solver time step (exact in dtype)              */
  int dt_is_f32;           /* upstream dt is a float32 scalar               */
  /* Gaussian beam on the z line (ixs, iys), wakis/sources.py:76-110:
   * Jz(k) = ((q*v) * c0*exp(-(s-s0)^2/two_sig2) / dx_s) / dy_s,
   * s = zc[k] - v*t, t = step*dt.                                         */
  int beam_on;
  int ixs, iys;
  double b_qv, b_v, b_s0, b_c0, b_two_sig2, b_dx, b_dy;
  const double* zc;        /* Nz cell-centre z coordinates                   */
  /* Host-supplied line current instead of the Gaussian: with line_on, the
   * Jz of line (ixs, iys) at step s is line[(s - line_step0) * Nz + k]
   * (dtype elements, line_nsteps rows).                                     */
  int line_on;
  long long line_step0, line_nsteps;
  const void* line;
  /* Ez window capture before each step (wakis/routines.py:419-440):
   * cap[((a*cap_nj + b)*Nz + k)*cap_nt + (step - cap_step0)]
   *     = Ez(cap_i0+a, cap_j0+b, k)
   * Every step run must satisfy cap_step0 <= step < cap_step0 + cap_nt (and
   * line_step0 <= step < line_step0 + line_nsteps with line_on); the step
   * entry points return WK_E_RANGE otherwise.                               */
  int cap_on;
  int cap_i0, cap_j0, cap_ni, cap_nj;
  long long cap_nt, cap_step0;
  void* cap;               /* dtype elements                                 */
  int* status;             /* device status word (0 = ok), may be NULL       */
  /* Kernel choice for wk_fit_step (WK_KERNEL_* below).
   * tile_planes (0 = automatic) sets the planes per block of the TMA kernel
   * and the planes per thread of the two-pass kernels.  tile_rows sets the
   * tile shape of the TMA kernels and of the batched launches: 8 for 64x8
   * tiles, 16 for 32x16 tiles, 0 for the faster on B200 (64x8 in FP64 and
   * FP32; in WK_F32C 32x16 on planes of 256x256 cells or more, else 64x8;
   * 32x16 in the batched launches).                                        */
  int kernel;
  int tile_rows, tile_planes;
  /* WK_F32C only: per-component compensation words of E and H (bf16 bit
   * patterns, uint16, 3N each, ping-pong like E and H): the state is the
   * float value v plus the bf16 value c (the rounding error of the last
   * update).                                                               */
  void* Ec[2];
  void* Hc[2];
  /* Optional device step counter (may be NULL).  When set, the step index
   * of the s-th step of a call is *step_dev + s (step0 is ignored), so one
   * captured CUDA graph can be replayed for consecutive steps; the host
   * cannot check the capture/line ranges then, and the kernels skip capture
   * columns and line rows outside their buffers.  Only the TMA and two-pass
   * schedules (and WK_F32C) take it; every dimension must be >= 5.          */
  const long long* step_dev;
  /* 1 when the caller knows that every E entry tangential to a PEC-masked
   * face (and its WK_F32C compensation word) is +0 and stays +0 through the
   * steps of the call (no source and no stored J on such entries): the
   * full-domain TMA kernels then skip the PEC column masks of the H rows,
   * which would only replace +0 by +0.  0 (the default) always masks.      */
  int faces_clean;
  /* Bound of each mbarrier wait in the step loop of the TMA kernels, in
   * nanoseconds of the GPU's global timer; 0 (the default) = 100 ms.  A
   * negative value makes the first wait give up at once: the block then
   * records the timeout in *status, waits with the default bound for the
   * loads it issued and returns (a test of the timeout path, which leaves
   * the output of the step incomplete).                                   */
  long long wait_ns;
  /* Steps per launch of the TMA schedule: 2 = two steps per launch
   * (temporal blocking, k_tma2) where that kernel applies (every face
   * PEC-masked, faces_clean, J = 0 without conductivity or sigma*E with it,
   * no step_dev) and n_steps >= 4, else one; 1 = always one; 0 (the
   * default) = the faster on B200 for the state type: one step per launch
   * for FP64 and FP32 (k_tma2 halves the DRAM bytes but issues more
   * instructions per cell at a lower occupancy).  The result and its buffer
   * parity do not depend on it.                                            */
  int steps_per_launch;
  /* WK_F32C only.  0 (the default): the rows read the float parts v of the
   * neighbouring state and sum in float; the compensated add then keeps
   * the state to ~32 bits, but each increment carries the rounding of a
   * float row sum.  1: compensated stencil: the rows read the full pairs
   * v + c, the update factors are split into two floats and the increment
   * is formed with error-free float transformations (~44 bits), so that
   * long runs whose increments are large against the state (conductive
   * cells near the relaxation limit) follow the FP64 trajectory closely;
   * runs the two-pass kernels (WK_KERNEL_TMA is refused).                  */
  int comp_stencil;
} wk_fit_desc;

#define WK_KERNEL_AUTO 0   /* WK_KERNEL_TMA when its conditions hold, else
                              WK_KERNEL_TWOPASS when Nx, Ny, Nz >= 5, else
                              WK_KERNEL_CELL                                */
#define WK_KERNEL_CELL 1   /* one thread per cell, general row code, H of
                              the backward neighbours recomputed            */
#define WK_KERNEL_TWOPASS 4 /* H pass then E pass, each an interior launch
                              with single-coefficient rows plus a shell
                              launch; tile_planes = planes per thread (1, 2
                              or 4; 0 = 1 for FP64, 2 for FP32)
                              (WK_E_SHAPE if a dimension is below 5)        */
#define WK_KERNEL_TMA 6    /* fused step with TMA-loaded plane tiles in a
                              shared-memory ring (interior) + shell launch;
                              needs 16-byte row pitch (Nx*elem % 16 == 0),
                              N*elem % 16 == 0 and every dimension >= 5;
                              tile_planes = planes per block (0 = auto).
                              A load that does not arrive within a bounded
                              wait sets *status = 1 and the block returns. */
/* Kernel values 2, 3 and 5 (earlier schedules) are no longer accepted:
 * wk_fit_step returns WK_E_MODE for them.                                   */

/*
 * Add `inc` to the device counter *ctr (one thread, on `stream`): advances
 * wk_fit_desc.step_dev between replays of a captured step graph.  No
 * counterpart in the reference.
 */
int wk_counter_add(long long* ctr, long long inc, void* stream);

/*
 * Batched FP32-compensated stepping: many independent grids (each with its
 * own shape, dt, materials, beam and Ez capture) advanced by ONE persistent
 * cooperative launch per call.  Upstream runs one SolverFIT3D.wakesolve per
 * geometry (wakis/routines.py:231-482, each step SolverFIT3D._one_step,
 * wakis/solverFIT3D.py:482-503); the result of every instance equals that of
 * wk_fit_step on its own descriptor.
 *
 * Every instance is WK_F32C, has its four x/y faces PEC-masked (face mode 1:
 * all six faces; mode 2: the z faces are not, e.g. ABC, and the four
 * z-boundary planes take the general rows), id_bytes 1 or 2, J mode
 * WK_J_ZERO or WK_J_SIGMA_E, Nx % 4 == 0, at most 64 materials and
 * step_dev == NULL; all instances share the face mode, id width and J mode.
 * tile_planes of a descriptor sets the planes per work item (0 = 24) and
 * tile_rows its tile shape: 8 for 64x8 tiles, 16 (or 0) for 32x16 tiles
 * (fewer idle lanes where Nx lies just above a multiple of 64).
 *
 * wk_batch_workspace_bytes: device bytes the plan needs (-1 on an argument
 *   error, see wk_last_error).
 * wk_batch_prepare: checks the descriptors (an array of n_inst structs),
 *   encodes every instance's TMA descriptors for both buffer parities, forms
 *   the work lists and copies all of it into `workspace` (caller-owned
 *   device memory, 128-byte aligned, at least wk_batch_workspace_bytes),
 *   then waits for `stream`.  The live parity of instance q at step t is
 *   descs[q].par ^ ((t - t_ref) & 1).  Not for stream capture.
 * wk_batch_run: advances every instance by n_steps steps, step indices
 *   t = step0 + s (+ *step_dev when step_dev is not NULL, read on the device
 *   when a launch starts, so captured launches can be replayed), on
 *   `stream` (capturable).  plan->form WK_BATCH_PERSISTENT: one cooperative
 *   launch whose blocks claim the items of every step in order; an item
 *   waits only for its own instance's earlier work (per-instance completion
 *   counters, no grid-wide barrier), each wait bounded by wait_ns
 *   nanoseconds (<= 0: 2 s).  WK_BATCH_PHASES: up to six launches per step
 *   (wait_ns unused).  A wait or a tile load that runs out sets the status
 *   word of the instance concerned and the launch ends (wk_read_status).
 * No counterpart in the reference.
 */
#define WK_BATCH_PERSISTENT 0   /* one cooperative launch per wk_batch_run  */
#define WK_BATCH_PHASES 1       /* per step, one launch per list of items:
                                   64x8 and 32x16 tiles with TMA-loaded
                                   compensation words, the same with
                                   per-thread loads, H rows of the boundary
                                   planes, then their E rows                */
typedef struct wk_batch_plan {
  void* workspace;
  long long workspace_bytes;
  int n_inst;
  int n_items[2];          /* work items of the two phases of a step         */
  int grid;                /* persistent blocks (SMs x blocks per SM)        */
  int smem;                /* dynamic shared memory per block                */
  int variant;             /* kernel instantiation                           */
  int device;
  long long offsets[4];    /* instances, TMA descriptors, items (two phases) */
  int n_parts[5];          /* phase-A items: TMA-word 64x8 tiles, TMA-word
                              32x16 tiles, other 64x8 tiles, other 32x16
                              tiles, boundary-plane H rows                   */
  int form;                /* WK_BATCH_PERSISTENT (set by wk_batch_prepare)
                              or WK_BATCH_PHASES; the caller may change it  */
} wk_batch_plan;

long long wk_batch_workspace_bytes(const wk_fit_desc* descs, int n_inst);
int wk_batch_prepare(const wk_fit_desc* descs, int n_inst, long long t_ref, void* workspace,
                     long long workspace_bytes, wk_batch_plan* plan, void* stream);
int wk_batch_run(const wk_batch_plan* plan, int n_steps, long long step0,
                 const long long* step_dev, long long wait_ns, void* stream);

/*
 * Adjoint (reverse-mode) FIT step, used for gradients of a wake/impedance
 * loss with respect to per-cell eps_r and sigma.  No counterpart in the
 * reference: these are the transposes of the operators of
 * SolverFIT3D._one_step (wakis/solverFIT3D.py:482-503).  A^T (rows: E
 * entries, columns: H entries) and B0^T (rows: H, columns: E; B = diag(ieps)
 * B0) are CSR matrices (int64 row pointers, int32 columns, dtype values) in
 * the flat 3N ordering of the fields.  All vectors have 3N dtype entries.
 *   wk_adj_h:    lH_out = lH_in + dt * B0^T (ieps .* lE)
 *   wk_adj_e:    lE_out = decay .* lE_in - A^T lH      (decay = 1 - dt ieps sigma m)
 *   wk_adj_grad: for each listed cell c = cells[q] (flat index < N),
 *                gI[q] += sum_comp lE1 inc[comp*ncell + q]     (inc: FP64,
 *                         dt (B0 H' - J) of the listed entries),
 *                gS[q] += -dt sum_comp ieps lE1 E0[comp*ncell + q] smask
 *                         (when use_sigma; E0: dtype, the E of the listed
 *                         entries, ncell per component like inc)
 *                (double accumulators, one entry per listed cell).
 * lH_in may equal lH_out and lE_in may equal lE_out.
 */
int wk_adj_h(int dtype, const long long* rowptr, const int* col, const void* val,
             long long nrows, const void* lamE, const void* ieps, double dt,
             const void* lamH_in, void* lamH_out, void* stream);
int wk_adj_e(int dtype, const long long* rowptr, const int* col, const void* val,
             long long nrows, const void* lamH, const void* lamE_in, const void* decay,
             void* lamE_out, void* stream);
int wk_adj_grad(int dtype, const long long* cells, long long ncell, long long N,
                const void* lamE1, const double* inc, const void* E0, const void* ieps,
                const void* smask, int use_sigma, double dt, double* gI, double* gS,
                void* stream);

/*
 * The same two transposes without assembled matrices: stencils over the
 * compact coefficient tables of a solver descriptor (material ids and
 * table, separable metrics, PEC/PMC face masks, dt; the state buffers of
 * the descriptor are not read or written).  No counterpart in the
 * reference (transposes of SolverFIT3D._one_step, solverFIT3D.py:482-503).
 * dtype (WK_F64 / WK_F32) is the type of the adjoint vectors (3N entries
 * each); the coefficient tables keep the descriptor's type.
 *   wk_adj_h_fit: lH_out = lH_in + dt * B0^T (ieps .* lE)
 *   wk_adj_e_fit: lE_out = decay .* lE_in - A^T lH      (decay may be NULL: 1)
 * lH_in may equal lH_out and lE_in may equal lE_out.  Fewer than 2^31 cells.
 * fu / fw (3N entries of dtype) are the cell factors of wk_adj_factors:
 * with them the products of each cell are formed once per z-marching tile;
 * with NULL, or with d->kernel == WK_KERNEL_CELL, one thread per cell forms
 * the products of its neighbours from the tables itself (the cross-check:
 * the same values).
 */
int wk_adj_h_fit(const wk_fit_desc* d, int dtype, const void* fu, const void* lamE,
                 const void* lamH_in, void* lamH_out, void* stream);
int wk_adj_e_fit(const wk_fit_desc* d, int dtype, const void* fw, const void* lamH,
                 const void* lamE_in, const void* decay, void* lamE_out, void* stream);

/*
 * The cell factors of the two transposes, in the adjoint type dtype:
 *   fu[c N + n] = itA_c(n) pec_c(n) ieps_c(n)          (B0^T ieps)
 *   fw[c N + n] = dt iA_c(n) imu_c(n) pmc_c(n)          (A^T)
 * each product rounded as the stencils of wk_adj_h_fit / wk_adj_e_fit form
 * it.  They depend only on the descriptor's coefficient tables, so a
 * backward pass forms them once.  Either pointer may be NULL, not both.
 * No counterpart in the reference.
 */
int wk_adj_factors(const wk_fit_desc* d, int dtype, void* fu, void* fw, void* stream);

/*
 * Hard-source write of step `step` (+ *step_dev when not NULL) into
 * component `component` of a field (3N entries; dtype WK_F64, WK_F32 or
 * WK_F32C, the last with its bf16 compensation words `comp`) over the box
 * [i0,i1) x [j0,j1) x [k0,k1):
 *   F[c, i, j, k] = (A[t] * prof[(i-i0) + (j-j0)*ni + (k-k0)*ni*nj]) * B[t]
 * (FP64 products in that order, rounded once to the field's type; prof NULL:
 * no profile factor, B NULL: no second factor).  A and B hold n_steps FP64
 * values; a step outside [0, n_steps) writes nothing (and is rejected on the
 * host when step_dev is NULL).  Replaces the assignment of
 * PlaneWave / WavePacket / Dipole / Pulse .update(solver, t)
 * (wakis/sources.py:142-762) that emsolve makes before each step
 * (wakis/routines.py:207), with the per-step factors tabulated once.
 */
int wk_source_write(void* field, int dtype, void* comp, int Nx, int Ny, int Nz, int component,
                    int i0, int i1, int j0, int j1, int k0, int k1, const double* prof,
                    const double* A, const double* B, long long n_steps,
                    const long long* step_dev, long long step, void* stream);

/*
 * Frequency-domain monitor update: for f < nf and d < 3,
 * acc[f][d][n] += E_d[n] * phases[f] (complex double, interleaved re/im,
 * acc laid out [nf][3][N] in the flat field order).  Replaces the loop of
 * FieldMonitor.update (wakis/field_monitors.py:60-107); the caller forms
 * phases[f] = exp(-2j pi f_f t).  nf <= 64, acc 16-byte aligned.
 */
int wk_field_monitor(const void* E, int dtype, long long N, const double* phases, int nf,
                     double* acc, void* stream);

/*
 * Wait for `stream`, read the device status word that the step kernels
 * set (wk_fit_desc.status) and, with reset != 0, clear it.  Returns WK_OK
 * when it is 0 and WK_E_TIMEOUT when a TMA step kernel gave up waiting for
 * a tile load (the fields written since the last check are then
 * incomplete).  No counterpart in the reference (upstream's scipy step
 * cannot time out).
 */
int wk_read_status(int* status, int reset, void* stream);

/* ABI version (WK_ABI_VERSION). */
int wk_version(void);

/* Thread-local message for the last non-zero return. */
const char* wk_last_error(void);

/*
 * Zero the ghost entries of the live E and H buffers before the first step.
 * Replaces SolverFIT3D._set_ghosts_to_0 (wakis/solverFIT3D.py:820-840).
 */
int wk_zero_ghosts(const wk_fit_desc* d, void* stream);

/*
 * Advance `n_steps` leap-frog steps starting at global step index `step0`:
 * for each step, (beam line J, Ez capture,) H <- H - dt*A*E, then
 * E <- E + dt*(B*H - ieps*J) and, with WK_J_ARRAY and use_conductivity,
 * J <- sigma*E.  Reads the buffers E[par], H[par] and leaves the result in
 * E[par ^ (n_steps & 1)], H[par ^ (n_steps & 1)] (the caller flips `par`).
 * Replaces SolverFIT3D._one_step (wakis/solverFIT3D.py:482-503) together with
 * Beam.update (wakis/sources.py:76-110) and the per-step Ez save of
 * RoutinesMixin.wakesolve (wakis/routines.py:435-445).
 */
int wk_fit_step(const wk_fit_desc* d, int n_steps, long long step0, void* stream);

/*
 * Same update with the two half-steps as separate in-place kernels (H pass,
 * then E pass); the state stays in E[par], H[par].  Reference schedule used
 * to cross-check the fused kernel of wk_fit_step.
 */
int wk_fit_step_split(const wk_fit_desc* d, int n_steps, long long step0, void* stream);

/*
 * wk_fit_step that also times the interior kernels of every step with CUDA
 * events recorded on `stream` (the TMA kernel of WK_KERNEL_TMA, the H and E
 * pass kernels of WK_KERNEL_TWOPASS, the two compensated pass kernels of
 * WK_F32C; shell launches are not included), then waits for the stream.
 * *ms_interior = summed interior-kernel time in ms, *n_launches = launches
 * timed (0 for schedules without a separate interior kernel).  n_steps is
 * limited to 4096.  No counterpart in the reference: a measurement hook.
 */
int wk_fit_step_timed(const wk_fit_desc* d, int n_steps, long long step0, void* stream,
                      float* ms_interior, int* n_launches);

/*
 * Materialise J = sigma*E_live (dtype) into `J` (3N).  Replaces the
 * J.fromarray(sigma*E) of wakis/solverFIT3D.py:502-503 for callers that read
 * J between steps.
 */
int wk_sigma_e(const wk_fit_desc* d, void* J, void* stream);

/*
 * Longitudinal wake potential, calc_long_WP_3d / calc_long_WP
 * (wakis/wakeSolver.py:310-420, 422-554), for n_win transverse positions
 * processed in order w = 0..n_win-1:
 *   acc = carry ? WP_3d[w-1][n] : 0          (carry-over of upstream 485/536)
 *   for k: it = (long)((((z[k]+s[n])/v - zmin/v) - t0 + ti)/dt)
 *          (counter-moving: (((z[nz-1-k]-s[n])/(-v) - zmax/(-v)) - t0) + ti)
 *          if it < nt: acc += Ez(w, k_src, t_index[it]) * coef_k
 *   WP_3d[w][n] = acc / qnorm
 * Ez history: hist[(w_src*Nzh + kz)*hist_nt + t] (dtype hist_dtype), with
 * w_src = win_map[w], kz = k + k_off (reversed index for counter-moving),
 * t = key_order[it] (upstream sorts the '#%05d' keys as strings).
 * coef_k = dz[k] (counter-moving: -dz[k]).  All double except hist.
 * A key_order entry outside [0, hist_nt) adds nothing (the caller passes
 * nt <= the number of steps the history holds, as upstream reads only the
 * saved steps).
 */
int wk_wake_potential(const void* hist, int hist_dtype, long long hist_nt, int Nzh,
                      const int* win_map, int n_win, int carry,
                      const double* z, const double* dz, int nz, int k_off,
                      const double* s, int ns, const long long* key_order, long long nt,
                      double v, double zmin, double zmax, double t0, double ti, double dt,
                      double qnorm, int counter_moving, double* WP3d, void* stream);

/*
 * Transverse wake potential by Panofsky-Wenzel (wakis/wakeSolver.py:556-612):
 *   int_w[n] = (sum_{m<n} WP3d[w][m]) * ds  (numpy pairwise summation order)
 *   WPx[n] = -(int_{+1,0}[n] - int_{-1,0}[n]) / dxsum
 *   WPy[n] = -(int_{0,+1}[n] - int_{0,-1}[n]) / dysum
 * WP3d holds the 3x3 positions, w = (i+1)*3 + (j+1).
 */
int wk_trans_wake(const double* WP3d, int ns, double ds, double dxsum, double dysum,
                  double* WPx, double* WPy, void* stream);

/*
 * Streaming form of wk_wake_potential, for runs whose whole Ez history does
 * not fit in memory: the history arrives in chunks of steps, and each chunk
 * is added into an accumulator as it completes.
 *
 * wk_wake_accumulate: the steps step0 .. step0+n_steps-1 of the Ez window
 * history are in ring[(w_src*Nzh + kz)*ring_nt + (step - step0)] (the
 * capture layout of wk_fit_desc with cap_step0 = step0, n_steps <=
 * ring_nt).  Step m sits at position p = pos[m] of upstream's sorted key
 * list ('#%05d' keys sorted as strings; pos = NULL: p = m, exact below 10^5
 * steps); it adds Ez(w, k, m) * coef_k into acc[w][n] (double, n_win x ns,
 * zeroed by the caller before the first chunk) for every s sample n with
 * it(n, k) == p < nt, it and coef_k as in wk_wake_potential.
 * wk_wake_finalize: WP3d[w][n] = ((carry ? WP3d[w-1][n] : 0) + acc[w][n]) /
 * qnorm, windows in order.
 * The sums run in another order than upstream's (by step, and the carried
 * value added after instead of before), so WP3d agrees with
 * wk_wake_potential to rounding, not value for value.  No counterpart in
 * the reference (it keeps the whole history in an HDF5 file).
 */
int wk_wake_accumulate(const void* ring, int ring_dtype, long long ring_nt, int Nzh,
                       long long step0, int n_steps, const int* win_map, int n_win,
                       const double* z, const double* dz, int nz, int k_off, const double* s,
                       int ns, const long long* pos, long long nt, double v, double zmin,
                       double zmax, double t0, double ti, double dt, int counter_moving,
                       double* acc, void* stream);
int wk_wake_finalize(const double* acc, int n_win, int ns, int carry, double qnorm,
                     double* WP3d, void* stream);

/*
 * wk_trans_wake for long s axes: the same Panofsky-Wenzel quotient
 * (wakis/wakeSolver.py:556-612) with the prefix integrals formed by
 * segmented scans in double-double arithmetic (~106-bit running sums,
 * rounded once), O(ns) instead of the O(ns^2) per-sample pairwise sums;
 * the integrals differ from numpy's pairwise ones only by the rounding of
 * the latter.  `scratch` is caller-owned device memory of at least
 * wk_trans_wake_scan_scratch_bytes(ns) bytes, 16-byte aligned (the segment
 * sums).  No counterpart in the reference.
 */
long long wk_trans_wake_scan_scratch_bytes(int ns);
int wk_trans_wake_scan(const double* WP3d, int ns, double ds, double dxsum, double dysum,
                       double* WPx, double* WPy, void* scratch, long long scratch_bytes,
                       void* stream);

/*
 * wk_trans_wake_scan without caller scratch, for callers that cannot hand
 * this library device memory of its own: a host program whose device
 * memory is all reserved up front by another allocator (a framework's
 * caching pool, a fixed per-process budget) or a plugin loaded into such a
 * program, where a cudaMalloc here would fail or break the owner's
 * accounting.  This entry point allocates nothing: its segment sums live in
 * a 256 KiB array built into the library, which every GPU that loads the
 * library holds until the process exits.  The caller still passes WP3d,
 * WPx and WPy.  ns above 4096 * 65536 samples is rejected (WK_E_RANGE).
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  All calls share the array and it keeps the
 * last call's segment sums (each call writes every sum it reads before
 * reading it): calls that overlap on one GPU, on different streams, race on
 * it (each GPU has its own copy).  No counterpart in the reference.
 */
int wk_trans_wake_scan_noalloc(const double* WP3d, int ns, double ds, double dxsum,
                               double dysum, double* WPx, double* WPy, void* stream);

/*
 * Zero-padded DFT bins X[m] = sum_{n<len} x[n] * exp(-2*pi*i*m*n/N) for
 * m = 0..nbins-1 (the bins 0 <= f < fmax of np.fft.fft(x, n=N) kept by
 * calc_long_Z / calc_trans_Z, wakis/wakeSolver.py:679-766), for `nsig`
 * real signals of length `len` stored back to back.  out is complex
 * (re, im interleaved), out[(sig*nbins + m)*2 + {0,1}].
 */
int wk_dft_bins(const double* x, int nsig, long long len, long long N, int nbins,
                double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* WAKIS_B200_H */
