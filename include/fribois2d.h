/*
 * fribois2d.h -- C ABI of the B200-native FRiBoIS2D fluid time step.
 *
 * The reference (AleNit/FRiBoIS2D, Fortran 90 + MPI) has no plugin or FFI
 * boundary: its driver calls module subroutines on global state
 * (src/main.F90:51-97).  This header is the boundary a Fortran host binds
 * with ISO_C_BINDING (`bind(C)` interfaces) to replace
 * those subroutines with one GPU.  Conventions:
 *
 *  - every function returns an int status (FB_OK = 0); the reference aborts
 *    through stopcase/MPI_ABORT (src/stopcase.F90:4-31) instead;
 *  - arrays crossing the boundary are plain host `double*` / `int*` with an
 *    element count; fields are the reference's column-major A(j,k), j = 1..n2
 *    contiguous, k = 0..n3 (the k = 0 ghost row of the reference is kept),
 *    i.e. (n3+1) * n2 doubles;
 *  - all device memory is owned by the opaque context; one host thread per
 *    context; calls are synchronous unless stated otherwise.
 */
#ifndef FRIBOIS2D_H
#define FRIBOIS2D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replace stopcase calls) ----------------------------- */
#define FB_OK 0
#define FB_ERR_CFL 1          /* fluid_tsch.F90:43-55: CFL above cfllim / dt too small */
#define FB_ERR_MLS 2          /* MLSint.F90:157-163: MLS partition of unity violated */
#define FB_ERR_MARKER_OUT 3   /* lgrdistribution.F90:217-221: marker leaves the grid */
#define FB_ERR_INPUT 4        /* utils_proc.F90:174-219: malformed or missing input */
#define FB_ERR_CUDA 5         /* CUDA runtime / cuBLAS failure */
#define FB_ERR_STATE 6        /* bad argument for this context (id, size, order) */
#define FB_ERR_UNSUPPORTED 7  /* deck option not implemented on the device path */
#define FB_ERR_NUMERIC 8      /* a NaN/Inf or a singular set-up system was detected */
#define FB_ERR_TIMEOUT 9      /* a device-side wait gave up (bounded waits in the tensor-core kernels) */

typedef struct fb_ctx fb_ctx;     /* device context: one case on one GPU */
typedef struct fb_host fb_host;   /* host-side set-up of one case (no GPU) */
typedef struct fb_batch fb_batch; /* independent cases stepped together */
typedef struct fb_mlp fb_mlp;     /* small perceptron: learned coupling predictor */

/* ---- array ids for fb_get_array / fb_set_array / fb_host_array --------- */
/* fields, (n3+1) x n2 doubles, k = 0..n3 */
#define FB_Q2 0      /* v at (rc_j, zm_k)   declarations.F90:148 */
#define FB_Q3 1      /* w at (rm_j, zz_k)   */
#define FB_PR 2      /* pressure at (rm_j, zm_k) */
#define FB_DPH 3     /* pressure correction phi (after phcalc) or divergence (after divg) */
#define FB_RHS2 7    /* explicit v right-hand side (after invtr2; forcing added in place) */
#define FB_RHS3 8
#define FB_RU2 9     /* previous convective term of v (= hdnl2 output) */
#define FB_RU3 10    /* previous convective term of w (= hdnl3 output) */
/* inflow / outflow boundary arrays, n2 doubles (index j-1) */
#define FB_QB2S 20
#define FB_QB2N 21
#define FB_DQB2S 22
#define FB_DQB2N 23
#define FB_QB3S 24
#define FB_QB3N 25
#define FB_DQB3S 26
#define FB_DQB3N 27
#define FB_DQ2X2O 28
#define FB_DQ3X2O 29
/* 1-D grid data, n2 or n3 doubles (index j-1 / k-1) */
#define FB_RC 40
#define FB_RM 41
#define FB_ZZ 42
#define FB_ZM 43
#define FB_UDX2C 48
#define FB_UDX2M 49
#define FB_UDX3C 50
#define FB_UDX3M 51
#define FB_AMPHJ 64
#define FB_ACPHJ 65
#define FB_APPHJ 66
#define FB_AMPHK 67
#define FB_ACPHK 68
#define FB_APPHK 69
/* Poisson eigen data: wr (n3m), zmm and zmmt (n3m*n3m, column-major) */
#define FB_WR 80
#define FB_ZMM 81
#define FB_ZMMT 82
/* markers: nlm x 2 row-major (y, z) unless stated */
#define FB_LMCC 90
#define FB_LMVEL 91
#define FB_LMACC 92
#define FB_LMNOR 93
#define FB_LMA 94    /* nlm */
#define FB_VERT 95   /* (nlm+1) x 2 */
#define FB_PHI 96    /* nlm x 2 x 9: MLS transfer weights, (marker, direction, support node) */
#define FB_CL 97     /* nlm x 2 */
#define FB_PRESS 98  /* nlm: wall pressure from loads_transfer_c */
#define FB_TAU 99    /* nlm x 2: wall shear stress */
#define FB_BCERRV 100
#define FB_BCERRW 101
#define FB_RIGID 110   /* 18: cmp_n, cmv_n, cma_n, cmp_np1, cmv_np1, cma_np1 */
#define FB_SCALARS 111 /* 13: time, dt, dt_o, beta, al, ga, ro, cflm, q3avg, nbcv, nbcw, ddmin, pravg */
#define FB_FORCES 112  /* 8: forcecomp.out row: time, Fy, Fz, M, Fyp, Fzp, Fyv, Fzv */
#define FB_HMN 113     /* n3m x ldh (ldh = dims[5]): Poisson modal work array [mode][j], read only */
/* integer arrays for fb_get_iarray */
#define FB_LMIND 0     /* nlm x 2 x 2: nearest node per marker and direction */
#define FB_EULINS 1    /* nlm x 2 x 2 x 9: MLS support node indices (j, k) */

/* ---- history rows written by fb_advance -------------------------------- */
/* one row per step: forcecomp.out (rigid.F90:432) then rbkin.out (ttime.F90:146)
 *  [0] time (start of step)  [1] Fy  [2] Fz  [3] M  [4] Fyp [5] Fzp [6] Fyv [7] Fzv
 *  [8] time (end of step) [9..11] cmp_np1 [12..14] cmv_np1 [15..17] cma_np1
 *  [18] nbcv [19] nbcw [20] cflm (start of step) [21] dt
 *  with fb_set_report on, the ttime.F90 diagnostics of the end-of-step field
 *  (fluid_rep.out, ttime.F90:142): [22] cflm [23] dmax [24] ektot [25] vorti
 *  [26] vmax(1) [27] vmax(2) [28] vmin(1) [29] vmin(2); zero otherwise
 *  [30] fluid solves in the step (1 with loose coupling; the coupling
 *  iterations with fb_set_coupling) */
#define FB_HIST_COLS 31

/* ---- stage ids for fb_stage: one per reference subroutine --------------- */
#define FB_ST_CFL 0        /* cfl.F90 (fluid_tsch.F90:211-258) */
#define FB_ST_BOUCDQ 1     /* iobcs.F90:5-77 */
#define FB_ST_NL_RHS 2     /* HDNL.F90:5-171 + INVTR.F90:4-280, fused */
#define FB_ST_LGRDIST 6    /* lgrdistribution.F90:189-267 */
#define FB_ST_FORCING 7    /* forcing_MLS.F90:5-182 (forcing added to rhs2/rhs3) */
#define FB_ST_HELSOLVE 8   /* helsolve.F90:4-56 + solve_fluid.F90:4-255 */
#define FB_ST_DIVG 9       /* divergence.F90:88-115 */
#define FB_ST_PHCALC 10    /* phcalc_outflow.F90:4-71 */
#define FB_ST_UPDVP 11     /* updvp.F90:5-105 (updvp + prcalc, fused) */
#define FB_ST_PRSUBMEAN 13 /* updvp.F90:112-144 + iobcs.F90:81-108 (boucqt), fused */
#define FB_ST_CHECKBCS 15  /* ckbcs.F90:5-86 */
#define FB_ST_LOADS 16     /* loads_transfer.F90:93-281 */
#define FB_ST_RIGID 17     /* rigid.F90:4-138 on the device */

/* ---- set-up -------------------------------------------------------------
 * Replaces read_genin + fluid_pre + read_rigid + allocate_mls_local +
 * rigid_pre (main.F90:51-62; utils_proc.F90:45-222,519-578; fluid_pre.F90;
 * indic.F90; cordin.F90; coetar.F90; phini.F90; initial_sol.F90:251-299;
 * rigid_pre.F90).  Reads input_dir/{global,fluid,rigid}_par.in,
 * ycoord.dat, zcoord.dat, lmdata.in.  The state starts as inqpr leaves it. */
int fb_create(const char *input_dir, int device, fb_ctx **out);
int fb_destroy(fb_ctx *ctx);

/* One fluid time step: fluid_tsch(ns, str) (fluid_tsch.F90:4-204),
 * including checkbcs and loads_transfer_c.  Leaves press/tau for fb_rigid. */
int fb_fluid_tsch(fb_ctx *ctx, int ns);

/* rigid(ns, str, nk) (rigid.F90:4-138) on the device state; writes the
 * forcecomp.out row (8 doubles, see FB_FORCES) when forcecomp != NULL.
 * Then advances time by dt as main.F90:92 does. */
int fb_rigid(fb_ctx *ctx, int ns, double *forcecomp);

/* nsteps iterations of the reference main loop body (main.F90:85-97:
 * fluid_tsch, rigid, time += dt) starting at step index ns0, replayed from a
 * captured CUDA graph; hist (nsteps x FB_HIST_COLS, may be NULL) receives the
 * per-step history rows.  Status errors found on the device stop the call and
 * are returned after the step that raised them. */
int fb_advance(fb_ctx *ctx, int ns0, int nsteps, double *hist);

/* Marker-side coupling for a host rigid-body solver (the reference's own
 * rigid.F90 kept on the host): fb_get_loads copies press (nlm) and tau
 * (nlm x 2) to the host; fb_set_markers uploads lmcc, lmvel, lmacc, lmnor
 * (each nlm x 2, any may be NULL to keep the device copy).  fb_set_markers
 * copies the arrays into the context's pinned staging memory before it
 * returns (the caller's buffers are free again at once) and orders the
 * device copies ahead of the context's next step without waiting for them. */
int fb_get_loads(fb_ctx *ctx, double *press, double *tau);
int fb_set_markers(fb_ctx *ctx, const double *lmcc, const double *lmvel, const double *lmacc,
                   const double *lmnor);
/* The same four marker arrays back to the host (any may be NULL), with one
 * wait for all of them: the per-step read of a host that keeps its own
 * marker state (fb_get_array per array waits once per array). */
int fb_get_markers(fb_ctx *ctx, double *lmcc, double *lmvel, double *lmacc, double *lmnor);
/* No reference counterpart: one loosely coupled step of main.F90:85-97 for a
 * host that exchanges the markers every step, in one call with one wait:
 * fb_set_markers(lmcc, lmvel, lmacc, lmnor), fb_fluid_tsch(ns), fb_rigid(ns,
 * forcecomp), fb_get_markers(lmcc, lmvel, lmacc, lmnor).  The four arrays
 * (nlm x 2 each) are read and then overwritten with the updated markers;
 * forcecomp may be NULL.  Returns the step's status; unlike the separate
 * calls, the rigid update of a replayed (fixed-dt) step runs even when the
 * fluid step reported an error. */
int fb_step_markers(fb_ctx *ctx, int ns, double *lmcc, double *lmvel, double *lmacc, double *lmnor,
                    double *forcecomp);

/* Last history row written (FB_HIST_COLS doubles), for per-step callers. */
int fb_last_history(fb_ctx *ctx, double *row);
/* End-of-step diagnostics of ttime.F90 (vmaxv, vminv, cfl, divgck, kinen,
 * getintvort) into history columns 22..29 after every step; off by default. */
int fb_set_report(fb_ctx *ctx, int on);

/* ---- batches of independent cases -------------------------------------------
 * No counterpart in the reference (one case per MPI job there).  The cases
 * (contexts on one device, fixed dt, RK3) are stepped by one CUDA graph
 * launch per step.  Each context keeps its own state, history rows and
 * status; the contexts must outlive the batch and must not be stepped on
 * their own meanwhile.  fb_batch_advance returns the first non-zero case
 * status.
 *   FB_BATCH_GROUPED (fb_batch_create's mode): cases with one launch geometry
 *     (grid, marker count, helsolve tiles, options) form a group; each stage
 *     of the step is one kernel launch over the whole group; each Poisson
 *     transform is one batched DGEMM, or in the precision form one grouped
 *     3xTF32 tensor-core launch (same Poisson form and GEMM tile within a
 *     group).  Cases without the windowed helsolve run as in FB_BATCH_GRAPH
 *     inside the same graph.
 *   FB_BATCH_GRAPH: every case's own step on its own graph branch; bitwise
 *     equal to stepping the case alone. */
#define FB_BATCH_GROUPED 0
#define FB_BATCH_GRAPH 1
int fb_batch_create(fb_ctx *const *ctxs, int n, fb_batch **out);
int fb_batch_create_mode(fb_ctx *const *ctxs, int n, int mode, fb_batch **out);
int fb_batch_advance(fb_batch *b, int nsteps);
int fb_batch_last_ms(fb_batch *b, double *ms);  /* device time of the last advance */
/* info[0] groups, info[1] cases stepped on their own branch, info[2] own
 * kernel launches per step of the whole batch */
int fb_batch_info(fb_batch *b, int32_t info[3]);
int fb_batch_destroy(fb_batch *b);

/* ---- strong fluid-structure coupling and its learned predictor ------------
 * No counterpart in the reference (its coupling is explicit: FB_COUPLING_LOOSE,
 * the default).  FB_COUPLING_STRONG iterates each step on the body load
 * (Fy, Fz, M): markers placed where the load moves the body, fluid step from
 * the saved start-of-step state, Aitken relaxation towards the fluid's load,
 * until the free coordinate's load changes by <= tol * max(1, |F|); the
 * initial guess extrapolates the last two converged loads.
 * FB_COUPLING_LEARNED takes the initial guess of the free coordinate's load
 * from a trained fb_mlp (27 features: last 8 displacement increments,
 * velocities and loads as increments, Re, mass ratio, reduced velocity; 2
 * outputs: the corrections to the linear extrapolations of the displacement
 * and the load), standardised with `norm`
 * (x mean[27], x std[27], t mean[2], t std[2]).  fb_advance runs the
 * iteration; history column 30 counts the fluid solves of each step.
 * fb_coupling_samples hands out (features, targets) of converged steps for
 * training (at most cap; consumed).  Fixed dt only. */
#define FB_COUPLING_LOOSE 0
#define FB_COUPLING_STRONG 1
#define FB_COUPLING_LEARNED 2
int fb_set_coupling(fb_ctx *ctx, int mode, double tol, int max_iter);
int fb_set_predictor(fb_ctx *ctx, fb_mlp *mlp, const float *norm);
/* steps, fluid solves, steps that hit max_iter, mean relative load residual
 * of the initial guess (the predictor's error as the coupling test sees it) */
int fb_coupling_stats(fb_ctx *ctx, double out[4]);
int fb_coupling_samples(fb_ctx *ctx, float *x, float *t, int cap, int *n);

/* The perceptron (n_in -> 64 -> 64 -> n_out, tanh, FP32) with its own CUDA
 * training (Adam, deterministic block-ordered gradient sums) and inference
 * kernels.  Host arrays are row-major samples. */
int fb_mlp_create(int device, int n_in, int n_out, uint64_t seed, fb_mlp **out);
int fb_mlp_destroy(fb_mlp *m);
int fb_mlp_params(fb_mlp *m, int *n);
int fb_mlp_get(fb_mlp *m, float *params);
int fb_mlp_set(fb_mlp *m, const float *params);
int fb_mlp_predict(fb_mlp *m, const float *x, int n, float *y);
int fb_mlp_grad(fb_mlp *m, const float *x, const float *t, int n, float *grad, float *loss);
int fb_mlp_train(fb_mlp *m, const float *x, const float *t, int n, int epochs, int batch, float lr,
                 uint64_t seed, float *loss_out);

/* ---- checkpoint / restart --------------------------------------------------
 * The restart set of mpi_write_continua / writeqbns / master_rigid.dat
 * (mpi_routines.F90:532-806, iobcs.F90:114-205, ttime.F90:117-124) as raw
 * FP64 files in `dir` (rest_q2/q3/pr/ru2/ru3.bin, outflow.bin, inflow.bin,
 * master_rigid.dat), plus device_state.bin and scalars.bin with the marker,
 * boundary-increment and clock state, so that a run read back continues bit
 * for bit.  The directory must exist; the deck of the reading context must
 * have the same grid, markers and dt. */
int fb_write_restart(fb_ctx *ctx, const char *dir);
int fb_read_restart(fb_ctx *ctx, const char *dir);

/* ---- state access --------------------------------------------------------- */
/* dims: n2, n3, nlm, nsst, field pitch, Poisson pitch, pivoting flags,
 * helsolve windows of substep 1 (y | z << 8; 0 = full line scans) */
int fb_get_dims(fb_ctx *ctx, int32_t dims[8]);
int fb_get_array(fb_ctx *ctx, int id, double *host, int64_t n);
int fb_set_array(fb_ctx *ctx, int id, const double *host, int64_t n);
int fb_get_iarray(fb_ctx *ctx, int id, int32_t *host, int64_t n);
int fb_synchronize(fb_ctx *ctx);

/* ---- stage entry points (parity tests; one reference subroutine each) ---- */
int fb_set_substep(fb_ctx *ctx, int ns, int n);
int fb_stage(fb_ctx *ctx, int stage, int n);

/* ---- timing: device time of the last fb_advance, and per-kernel totals --- */
int fb_last_advance_ms(fb_ctx *ctx, double *ms);
/* Average device time (CUDA events on the context stream) of one launch of
 * a stage or of one of its kernels, over reps launches after one warm-up.
 * It overwrites the state: use a context dedicated to measurement. */
#define FB_TK_GEMM_FWD 100   /* phcalc_outflow.F90:31 eigen transform (cuBLAS DGEMM) */
#define FB_TK_POISSON_TRI 101 /* phcalc_outflow.F90:34-56 per-mode y solves */
#define FB_TK_GEMM_BWD 102   /* phcalc_outflow.F90:61 back transform */
#define FB_TK_TF32X3_GEMM 103 /* one 3xTF32 tensor-core transform (precision form) */
#define FB_TK_I8_SPLIT 104    /* digit cut of dph for the INT8 transform */
#define FB_TK_I8X8_GEMM 105   /* one INT8 digit-slice transform, hmn = dph zmmt^T */
int fb_time_stage(fb_ctx *ctx, int stage, int n, int reps, double *ms);
/* Number of this library's own kernels one captured time step launches
 * (library kernels of cuBLAS and CUB are not counted). */
int fb_kernel_count(fb_ctx *ctx, int32_t *per_step);

/* ---- forms of the Poisson eigen transforms --------------------------------
 * The reference computes phcalc's two transforms with FP64 DGEMM
 * (phcalc_outflow.F90:31,61).  A new context computes them to the same FP64
 * accuracy with this library's INT8 tensor-core kernel (FB_POISSON_INT8X8,
 * below), the default.  FB_POISSON_FP64: the transforms as cuBLAS DGEMMs,
 * kept as the comparison arm.  FB_POISSON_TF32X3: the two eigen transforms on
 * the tensor cores in split precision (TF32 high and low parts, three
 * products, FP32 accumulation), FP64 tridiagonal solves, then FP64
 * iterative-refinement sweeps on the Poisson residual (fb_set_refinement).  The forms have no
 * counterpart in the reference. */
#define FB_POISSON_FP64 0
#define FB_POISSON_TF32X3 1
/* FB_POISSON_INT8X8 (the default): the two FP64 eigen transforms computed
 * exactly in integer arithmetic on the INT8 tensor cores (rows scaled by
 * powers of two and cut into 8 signed 8-bit digits; the digit products summed
 * in FP64): FP64-level accuracy (~2e-16 of sum |a||b| at K = 1024, as DGEMM),
 * no refinement sweep; K (= n3 - 1) at most 16384. */
#define FB_POISSON_INT8X8 2
int fb_set_poisson(fb_ctx *ctx, int mode);
/* FP64 iterative-refinement sweeps of FB_POISSON_TF32X3 (1..4, default 2):
 * each sweep solves again, with the same tensor-core transforms, for the
 * FP64 residual r = dph - (A_yy + A_zz) phi and adds the correction.  No
 * counterpart in the reference. */
int fb_set_refinement(fb_ctx *ctx, int sweeps);
/* C = A * B^T with the INT8 digit-slice kernel (conventions and buffers as
 * fb_gemm_tf32x3; a test entry point). */
int fb_gemm_i8x8(int device, int M, int N, int K, const double *A, const double *B, double *C);
/* C = A * B^T with the 3xTF32 tensor-core kernel: A (M x K) and B (N x K)
 * column-major host arrays, C (M x N) column-major; allocates its own device
 * buffers on `device` (a test and calibration entry point).  bn: 64 or 128
 * (one CTA per 128 x bn tile) or 1000 + w, w = 128, 192, 256 (a CTA pair,
 * tcgen05 cta_group::2, per 256 x w tile). */
int fb_gemm_tf32x3(int device, int M, int N, int K, int bn, const double *A, const double *B, double *C);
/* Picks tile shapes for this grid size by timing the candidates on the
 * context (state preserved): the windowed helsolve's tile height and, with
 * the precision form on, the tensor-core GEMM's tile (code as fb_gemm_tf32x3's
 * bn).  Remembered per grid size for the process.  choice (may be NULL)
 * receives {height, tile code}. */
int fb_autotune(fb_ctx *ctx, int32_t choice[2]);

/* ---- host-only set-up (no GPU touched; usable on a CPU-only machine) ----- */
int fb_host_create(const char *input_dir, fb_host **out);
int fb_host_destroy(fb_host *h);
int fb_host_dims(fb_host *h, int32_t dims[8]);
int fb_host_array(fb_host *h, int id, double *out, int64_t n);
/* Symmetric-tridiagonal eigen-decomposition replacing phini's DGEEV+DGESV:
 * am/ac/ap are the z operator's sub/diag/super diagonals (n, 0-based rows);
 * writes wr (n), zmm and zmmt (n*n column-major). */
int fb_eigen_tridiag(int n, const double *am, const double *ac, const double *ap, double *wr,
                     double *zmm, double *zmmt);

/* ---- CFL number without any allocation ------------------------------------
 * No counterpart in the reference: an extra entry point for callers that
 * cannot let a library allocate device memory (their arrays live in another
 * runtime's data regions or in an arena under a hard budget).  It computes
 * what cfl.F90 computes -- out[0] = max over cells of
 * (|(v_j + v_j+1)/2 * udx2m_j| + |(w_k + w_k+1)/2 * udx3m_k|) * dt and
 * out[1] = the area-weighted mean of w -- from the caller's own device arrays:
 * q2, q3 as (j, k) at q[k*pitch + j-1], k = 0..n3; rc (n2), zz (n3),
 * udx2m (n2-1), udx3m (n3-1) 0-based; out: 2 doubles of device memory.
 * The partial results go to a fixed array inside the library (room for
 * FB_NOALLOC_MAX_ROWS rows of z cells; larger grids return FB_ERR_UNSUPPORTED).
 * The first call on a device looks up that array's address (make it before
 * any stream capture); every call shares the array, so calls whose kernels
 * overlap on the GPU race.  Asynchronous on `stream` (a cudaStream_t, or NULL).
 * A NaN or infinite velocity gives out[0] = +inf. */
#define FB_NOALLOC_MAX_ROWS 8192
int fb_cfl_noalloc(const double *q2, const double *q3, int pitch, int n2, int n3, const double *rc,
                   const double *zz, const double *udx2m, const double *udx3m, double dt, double rext2,
                   double alx3, double *out, void *stream);

const char *fb_status_string(int status);
const char *fb_version(void);

#ifdef __cplusplus
}
#endif
#endif
