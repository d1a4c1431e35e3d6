/*
 * lu_b200.h — C ABI of the B200-native dense LU solver (charmlu_b200).
 *
 * Drop-in for the factor-then-solve path of charmlu.  charmlu exposes that
 * path as a Charm++ chare API plus a command line, not as a C ABI:
 *   LUSolver(LUConfig, CkCallback)            benchmark.C:231-240, driver.ci:9-15
 *   LUBlk::startup(LUConfig, ..., callbacks)   lu.ci:467-494
 *   LUBlk::factor()                            lu.ci:31-42
 *   LUBlk::forwardSolve()/backwardSolve()      lu.ci:387-436
 *   BenchmarkLUBlk::startValidation() + LUSolver::calcScaledResidual
 *                                              benchmark.C:462-573, 385-400
 *   LUConfig {matrixSize, blockSize, pivotBatchSize, memThreshold, ...}
 *                                              luConfig.h:8-62
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions
 *  - Matrices are ROW-MAJOR with a leading dimension (the reference stores
 *    every block row-major, lu.h:151-153).  Device pointers are cudaMalloc'd
 *    memory of the current device; the caller owns them.
 *  - Pivots are LAPACK-style 0-based global rows: ipiv[k] is the row swapped
 *    with row k at step k (the reference's recordPivot(k, pivot.loc),
 *    lu.ci:329).
 *  - Every call is asynchronous on the given stream (a cudaStream_t passed
 *    as void*; NULL = legacy default stream).  A call returns LU_OK or a
 *    negative argument/launch error immediately; the numerical status
 *    (singular column, device wait timeout, non-convergence) is read with
 *    lu_status(), which synchronises the stream.  charmlu aborts instead
 *    (CkAbort at lu.ci:339-341, CkExit at benchmark.C:143-147).
 *  - A handle is not re-entrant: one call sequence at a time per handle.
 *  - Alignment: base pointers 16-byte aligned; lda even for FP64 (the row
 *    pitch must be a multiple of 16 bytes for the TMA tensor maps).
 */
#ifndef LU_B200_H
#define LU_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LU_API __attribute__((visibility("default")))
#else
#define LU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define LU_OK               0   /* >0: 1-based first column whose pivot failed the singularity test */
#define LU_ERR_ARG         -1   /* bad argument (the reference's CkExit on bad config, benchmark.C:143-147) */
#define LU_ERR_CUDA        -2   /* CUDA runtime/launch error */
#define LU_ERR_TIMEOUT     -3   /* a bounded device-side wait gave up */
#define LU_ERR_NONFINITE   -4   /* non-finite input or pivot */
#define LU_ERR_NOCONV      -5   /* iterative refinement did not reach the residual target */
#define LU_ERR_ALIGN       -6   /* pointer / leading-dimension alignment violated */
#define LU_ERR_NOMEM       -7   /* workspace allocation failed */
#define LU_ERR_UNSUPPORTED -8   /* configuration not supported by this build */

/* ---- precision of the factorisation ---------------------------------- */
#define LU_PREC_FP64   0   /* the reference's arithmetic (all FP64) */
#define LU_PREC_BF16   1   /* FP32 panel/TRSM, BF16 tensor-core trailing update, FP64 refinement */
#define LU_PREC_FP16S  2   /* as BF16 but FP16 operands with per-panel power-of-two scaling */
#define LU_PREC_FP16X3 3   /* error-compensated FP16: each FP32 operand split hi + lo (scaled FP16), the
                              update sums Lh*Uh + Lh*Ul + Ll*Uh on the tensor cores (near-FP32 factors) */

/* ---- refinement mode --------------------------------------------------- */
/* Storage of dA for lu_factor / lu_factor_solve.  LU_LAYOUT_COL
 * (column-major, as LAPACK): the matrix is transposed in place, factored,
 * and the factors transposed back, so dA ends with L\U column-major and the
 * pivots are the same as for the row-major matrix.  Other entry points take
 * row-major data; with LU_LAYOUT_COL they return LU_ERR_UNSUPPORTED
 * (lu_transpose_square converts). */
#define LU_LAYOUT_ROW  0
#define LU_LAYOUT_COL  1

#define LU_IR_CLASSIC  0   /* classical iterative refinement, GMRES-IR fallback on stagnation */
#define LU_IR_GMRES    1   /* GMRES-IR from the start */

/* Replaces LUConfig (luConfig.h:8-62).  Fields the reference uses for its
 * distributed runtime (map, PE tiles, memThreshold, mcastMgrGID) have no
 * meaning on one GPU; memThreshold is accepted by the CLI and ignored. */
typedef struct lu_config {
  int64_t n;               /* matrixSize */
  int32_t block_size;      /* blockSize: panel width b (any even value >= 2) */
  int32_t pivot_batch;     /* pivotBatchSize (default b/4, benchmark.C:98); swaps are applied per panel here */
  int32_t precision;       /* LU_PREC_* */
  int32_t lookahead;       /* 1 = overlap panel k+1 with trailing update k (two streams) */
  int32_t use_graph;       /* 1 = capture the schedule once per (n, b) as a CUDA graph and replay it */
  int32_t ir_mode;         /* LU_IR_* (mixed precision only) */
  int32_t ir_max_iter;     /* refinement iteration cap */
  int32_t layout;          /* LU_LAYOUT_ROW (default) or LU_LAYOUT_COL for lu_factor / lu_factor_solve */
  double  sing_threshold;  /* |u_jj| <= threshold sets info; the reference aborts at 100*eps (lu.ci:339) */
  double  ir_target;       /* refinement stops when r_hpl < ir_target (default 16) */
  int64_t spin_limit;      /* bounded-wait iteration cap for cross-CTA waits (0 = default) */
  int32_t gmres_restart;   /* GMRES-IR: Krylov vectors per cycle (0 = 120) */
  int32_t ir_stall;        /* refinement gives up (LU_ERR_NOCONV) after this many GMRES cycles in a row
                              that cut the scaled residual by less than 10% (0 = 3) */
  double  gmres_tol;       /* GMRES-IR: a cycle ends once ||r - op(A) d||_2 has fallen by this factor (0 = 1e-10) */
} lu_config;

typedef struct lu_handle_s* lu_handle;

/* Residual report (benchmark.C:385-400, 476-573). */
typedef struct lu_residual_info {
  double amax;     /* max |a_ij| — the reference's "|A|inf" (benchmark.C:476-483) */
  double anorm;    /* ||A||inf, max row sum */
  double bnorm;    /* ||b||inf */
  double xnorm;    /* ||x||inf */
  double rnorm;    /* ||b - Ax||inf */
  double r_ref;    /* rnorm / ((amax*xnorm + bnorm) * n * eps) — reference form, benchmark.C:390 */
  double r_hpl;    /* rnorm / ((anorm*xnorm + bnorm) * n * eps) — HPL form */
} lu_residual_info;

/* Refinement report. */
typedef struct lu_refine_info {
  int32_t iterations;        /* classical IR iterations taken */
  int32_t gmres_iterations;  /* inner GMRES iterations (0 if not used) */
  int32_t used_gmres;        /* 1 if GMRES-IR ran */
  int32_t status;            /* LU_OK or LU_ERR_NOCONV */
  double  r_hpl;             /* final scaled residual */
  double  r_hpl_initial;     /* scaled residual of the low-precision solve */
  int64_t host_bytes;        /* bytes of A copied host -> device (lu_refine_solve_host; else 0) */
  int32_t rejected;          /* refinement steps rolled back because ||b - A x||inf did not fall */
  int32_t reserved;
} lu_refine_info;

/* Fill *cfg with defaults for order n and block size b (LUConfig defaults,
 * benchmark.C:91-134). */
LU_API int lu_config_default(lu_config* cfg, int64_t n, int32_t block_size);

/* Create / destroy a solver handle on the current device; allocates the
 * handle's workspace (candidate slots, barrier counters, pivot lists).
 * Replaces LUSolver construction + LUBlk::startup (benchmark.C:258-294,
 * lu.ci:467-494). */
LU_API int lu_create(const lu_config* cfg, lu_handle* out);
LU_API int lu_destroy(lu_handle h);
/* Device workspace bytes the handle holds (precision-dependent). */
LU_API size_t lu_workspace_bytes(const lu_config* cfg);

/* Synchronise `stream` and return the numerical status of the last call
 * sequence on h: LU_OK, >0 singular column (1-based), or LU_ERR_*. */
LU_API int lu_status(lu_handle h, void* stream);

/* Clear the handle's device status word (asynchronous on stream).  The
 * factor and refine entry points clear it themselves; callers of the
 * per-block building blocks below clear it before each factorisation. */
LU_API int lu_status_clear(lu_handle h, void* stream);

/* FP64 LU with partial pivoting in place: P A = L U, L unit lower.
 * Replaces LUBlk::factor() (lu.ci:31-42) and its kernels (lu.C:26-352).
 *   dA   : n x n row-major, lda >= n, overwritten with L\U
 *   ipiv : n int32, 0-based global pivot rows
 *   rhs  : optional n-vector permuted with the rows (the reference carries
 *          b through the swaps, lu.h:66, lu.C:166-177), may be NULL */
LU_API int lu_factor(lu_handle h, double* dA, int64_t lda, int32_t* ipiv, double* rhs, void* stream);

/* Solve with stored factors.  trans = 0: A X = B (forwardSolve /
 * backwardSolve, lu.ci:387-436, applying P first); trans = 1: A^T X = B
 * (the adjoint; no reference counterpart).  B is n x nrhs row-major, ldb >=
 * nrhs, overwritten by X. */
LU_API int lu_solve(lu_handle h, const double* dLU, int64_t lda, const int32_t* ipiv,
             double* dB, int64_t ldb, int64_t nrhs, int trans, void* stream);

/* Time-to-solution entry: factor A and solve A x = b in one call, b
 * overwritten by x.  This is the span the reference times
 * (benchmark.C:243 -> 344: factor() then forwardSolve()). */
LU_API int lu_factor_solve(lu_handle h, double* dA, int64_t lda, int32_t* ipiv, double* db, void* stream);

/* Scaled residual of x against the ORIGINAL A and b (dA must hold A, not
 * its factors).  Replaces startValidation/recvXvec/sumBvec/calcResiduals/
 * calcScaledResidual (benchmark.C:462-573, 385-400).  Synchronises. */
LU_API int lu_residual(lu_handle h, const double* dA, int64_t lda, const double* dx, const double* db,
                lu_residual_info* out, void* stream);

/* Mixed-precision solve (no reference counterpart): factor a low-precision
 * working copy of A (h's precision), then refine x in FP64 against the
 * untouched FP64 A until r_hpl < cfg.ir_target (classical IR, GMRES-IR as
 * fallback).  dA is read only; db is read only; dx receives x. */
LU_API int lu_refine_solve(lu_handle h, const double* dA, int64_t lda, const double* db, double* dx,
                    lu_refine_info* info, void* stream);

/* lu_refine_solve with the FP64 matrix in host memory (no reference
 * counterpart; the out-of-core form of the mixed path, for orders whose FP64
 * matrix does not fit in HBM beside the FP32 factors).  hA (n x n,
 * row-major, lda; page-locked memory for full copy speed) is read only.
 * One pass converts it to the FP32 working copy; its leading rows stay in
 * device memory (as many as fit beside the factors, less a margin; at most
 * LU_B200_RESIDENT_BYTES bytes when that variable is set at lu_create), and
 * every later pass over A (the FP64 residual of each refinement step, each
 * GMRES product) reads those in place and streams only the other rows
 * through two staging buffers (LU_B200_STAGE_BYTES each, 256 MB default),
 * the copies overlapping the kernels.  info->host_bytes counts the bytes
 * copied.  db, dx and the result are as in lu_refine_solve (the same
 * arithmetic: the same x bit for bit).  A device pointer for hA is
 * rejected (LU_ERR_ARG). */
LU_API int lu_refine_solve_host(lu_handle h, const double* hA, int64_t lda, const double* db, double* dx,
                         lu_refine_info* info, void* stream);

/* Low-precision factorisation kept in the handle (no reference
 * counterpart): dA (read only) is converted to FP32 and factored as in
 * lu_refine_solve (cfg.precision: BF16, scaled FP16 or FP16x3 trailing
 * updates); the FP32 factors and their row permutation stay in the handle
 * for lu_refine_apply / lu_refine_adjoint until the next lu_refine_factor or
 * lu_refine_solve on it.  Asynchronous; a singular pivot is reported by the
 * next lu_refine_apply (info->status) and by lu_status. */
LU_API int lu_refine_factor(lu_handle h, const double* dA, int64_t lda, void* stream);

/* op(A) X = B with op(A) = A (trans = 0) or A^T (trans = 1) for nrhs
 * columns, by FP64 iterative refinement on the factors of the last
 * lu_refine_factor (no reference counterpart).  dA must be the matrix those
 * factors came from (FP64, even lda, 16-byte aligned): every step computes
 * the FP64 residual R = B - op(A) X and corrects X through the FP32 factors,
 * until each column's scaled residual
 *   ||r||inf / ((||op(A)||inf ||x||inf + ||b||inf) n eps)
 * is below cfg.ir_target (16 when 0) or cfg.ir_max_iter steps (50 when 0)
 * have run.  When classical steps stop contracting (or cfg.ir_mode is
 * LU_IR_GMRES), the columns still above the target get GMRES-IR cycles
 * (restart 120, FP32 factors as the preconditioner).  dB (n x nrhs, ldb) is
 * read only; dX receives X.  info reports the worst column; status
 * LU_ERR_NOCONV when a column did not converge.  Synchronises the stream
 * once per refinement step. */
LU_API int lu_refine_apply(lu_handle h, const double* dA, int64_t lda, int trans, const double* dB,
                    int64_t ldb, double* dX, int64_t ldx, int64_t nrhs, lu_refine_info* info,
                    void* stream);

/* Estimate of ||I - M^{-1} A|| for the low-precision factors M of the last
 * lu_refine_factor (no reference counterpart): iters steps of power
 * iteration on I - M^{-1} A (M^{-1} applied in FP64 arithmetic on the FP32
 * factors) from a seeded start; *est receives the last step's growth
 * factor, a lower bound on the 2-norm that approaches the spectral radius.
 * Classical refinement contracts by about *est per step and converges when
 * it is below 1.  dA: the FP64 matrix the factors came from.  Synchronises. */
LU_API int lu_refine_precond_norm(lu_handle h, const double* dA, int64_t lda, int32_t iters, double* est,
                                  void* stream);

/* Adjoint of X = A^{-1} B on low-precision factors (no reference
 * counterpart): lambda = A^{-T} W by lu_refine_apply (trans = 1) into
 * gradB, then grad_A = -lambda X^T into gradA (n x n, ldga; may be NULL).
 * Needs the factors of dA from lu_refine_factor. */
LU_API int lu_refine_adjoint(lu_handle h, const double* dA, int64_t lda, const double* dX,
                      int64_t ldx, const double* dW, int64_t ldw, int64_t nrhs, double* gradB,
                      int64_t ldgb, double* gradA, int64_t ldga, lu_refine_info* info,
                      void* stream);

/* Adjoint of X = A^{-1} B (no reference counterpart).  Given the factors
 * of A (from lu_factor), X (n x nrhs) and the upstream gradient W = dL/dX,
 * computes lambda = A^{-T} W into gradB and grad_A = -lambda X^T into gradA
 * (n x n, row-major, ldga).  gradA may be NULL. */
LU_API int lu_adjoint(lu_handle h, const double* dLU, int64_t lda, const int32_t* ipiv,
               const double* dX, int64_t ldx, const double* dW, int64_t ldw, int64_t nrhs,
               double* gradB, int64_t ldgb, double* gradA, int64_t ldga, void* stream);

/* Batched factor+solve of many independent systems of uneven order in one
 * persistent launch (no reference counterpart).  System i has order n[i]
 * (1 <= n[i] <= 1536), its matrix at dA + a_off[i] (row-major, lda = n[i])
 * and right-hand side at db + b_off[i] (overwritten by x).  precision:
 *   LU_PREC_FP64  FP64 factors in place in dA (as lu_factor);
 *   LU_PREC_FP32  FP32 factors of a copy in dWork, then FP64 refinement
 *                 against the untouched FP64 A until r_hpl < 16 (at most 10
 *                 steps; LU_ERR_NOCONV in info[i] otherwise).
 * info[i] receives each system's status (0 or 1-based singular column).
 * dWork: device scratch of lu_batched_work_bytes(...) bytes.  All pointer
 * arguments are device memory. */
#define LU_PREC_FP32   4   /* batched only: FP32 factors + FP64 refinement steps */
LU_API int lu_batched_factor_solve(int32_t count, const int32_t* n, const int64_t* a_off,
                            const int64_t* b_off, double* dA, double* db, int32_t* info,
                            int32_t precision, void* dWork, size_t work_bytes, void* stream);
/* Scratch bytes lu_batched_factor_solve needs for these orders (n_host: host array). */
LU_API size_t lu_batched_work_bytes(int32_t count, const int32_t* n_host, int32_t precision);
/* After an LU_PREC_FP32 lu_batched_factor_solve on dWork (device), once the
 * stream reaches it: hist[s] (host, 12 entries) = systems whose scaled
 * residual was below 16 after s FP64 refinement steps (s = 0 .. 10; a
 * single refinement step is s = 1), hist[11] = systems that did not get
 * there.  Synchronises.  No reference counterpart. */
LU_API int lu_batched_refine_histogram(const void* dWork, int32_t* hist, void* stream);
/* Per-size-bucket kernel parameters chosen by the autotuner: entries of
 * {n_max, panel_width, small_threshold} (host array, ascending n_max, at most
 * 16); count 0 restores the built-in defaults.  Applies to later batched
 * calls in this process. */
LU_API int lu_batched_set_tuning(int32_t entries, const int32_t* table);

/* Generators (device).  Counter-based uniform[-0.5,0.5): element (i, j)
 * of stream s is a pure function of (seed, s, i*cols + j), identical to
 * the CPU oracle's.  The reference generates A per block from Charm++'s
 * CrnDouble (benchmark.C:436-452), which is not reproducible here. */
LU_API int lu_generate_uniform(double* d, int64_t rows, int64_t cols, int64_t ld, uint64_t seed,
                        uint64_t stream_id, void* stream);
/* The reference's b generator MatGen (benchmark.C:28-74, 455-460):
 * minimal-standard LCG, seed 9934835 by default.  Host-side. */
LU_API int lu_matgen_host(double* out, int64_t count, int32_t seed, int64_t skip);

/* Profiling (no reference counterpart; the reference prints per-panel wall
 * times, lu.ci:282-286, 352-353).  lu_profile(h, 1) makes later calls on h
 * bracket every phase with CUDA events on the launching stream;
 * lu_phase_times() synchronises and returns, per phase, the summed device
 * milliseconds, the launch count and the algorithmic flops of that phase's
 * launches since the last reset (arrays of LU_NUM_PHASES entries, any may be
 * NULL), then resets.  Phases: */
#define LU_PH_PANEL   0  /* leaf getf2 launches */
#define LU_PH_LASWP   1  /* pivot compose + apply */
#define LU_PH_TRSM    2  /* TRSM leaves (U block row and panel-internal) */
#define LU_PH_GEMM    3  /* trailing-update GEMMs (one per panel step) */
#define LU_PH_GEMM_IN 4  /* GEMM halves inside the recursive panel / TRSM */
#define LU_PH_SOLVE   5  /* forward / backward substitution */
#define LU_PH_OTHER   6  /* conversions, residuals, refinement vectors */
#define LU_NUM_PHASES 7
LU_API int lu_profile(lu_handle h, int enable);
LU_API int lu_phase_times(lu_handle h, double* ms, int64_t* launches, double* flops);
/* ---- Per-block building blocks ------------------------------------------
 * For callers that distribute the matrix themselves, such as the 1D
 * block-cyclic multi-GPU driver (charmlu_b200/distributed.py), which keeps
 * each GPU's column blocks and broadcasts panels over NCCL as the
 * reference's block chares do with messages.  Each call uses the same
 * kernels as lu_factor / lu_solve on caller-supplied views: FP64,
 * row-major, even leading dimension, 16-byte aligned base, asynchronous on
 * stream.  The handle supplies workspace; its order n bounds m and w. */

/* LU with partial pivoting of the m x w panel dP (m >= w): the pivot search
 * runs over all m rows and rows are swapped across the panel's w columns.
 * d_ipiv[j] (device) = base + the 0-based panel row chosen for column j, so
 * with base = the panel's first global row it holds global rows as in
 * lu_factor.  A singular column is recorded for lu_status as base + j + 1.
 * Replaces the panel phase of LUBlk::factor: pivot search and reduction,
 * multipliers, rank-1 updates and in-panel swaps (lu.ci:256-370;
 * lu.C:197-288, 166-177). */
LU_API int lu_panel_factor(lu_handle h, double* dP, int64_t ldp, int64_t m, int32_t w, int32_t* d_ipiv,
                           int64_t base, void* stream);

/* Row interchanges d_ipiv[k0 .. k0+cnt) (device, global 0-based rows, in
 * order: row k0+i swaps with d_ipiv[k0+i]) on columns [0, ncols) of the
 * m-row matrix dA, except the columns [skip_b, skip_e) that already hold
 * them (the factored panel); db (optional, device, m entries) is permuted
 * too.  Each pivot must satisfy k0+i <= d_ipiv[k0+i] < m, as getrf's do; a
 * batch of up to 512 that does not is left unapplied and LU_ERR_ARG is
 * recorded for lu_status.  Replaces the pivot batches applied to the other
 * block columns and to b (sendPendingPivots / applySwap, lu.C:46-169;
 * pivotBatch, lu.ci:92-123). */
LU_API int lu_apply_pivots(lu_handle h, double* dA, int64_t lda, int64_t m, int32_t ncols, const int32_t* d_ipiv,
                           int64_t k0, int32_t cnt, int32_t skip_b, int32_t skip_e, double* db, void* stream);

/* dB (w x ncols) <- L^{-1} dB with L the unit lower triangle of dL (w x w).
 * Replaces LUBlk::computeU (lu.C:180-189). */
LU_API int lu_trsm_lower_unit(lu_handle h, const double* dL, int64_t ldl, int32_t w, double* dB, int64_t ldb,
                              int64_t ncols, void* stream);

/* dC (M x N) -= dA (M x K) * dB (K x N) on the FP64 tensor cores.
 * Replaces LUBlk::updateMatrix (lu.C:26-43). */
LU_API int lu_gemm_update(lu_handle h, const double* dA, int64_t lda, const double* dB, int64_t ldb, double* dC,
                          int64_t ldc, int64_t M, int64_t N, int64_t K, void* stream);

/* dx (w) <- L^{-1} dx (upper = 0, unit lower) or U^{-1} dx (upper = 1) for
 * one w x w diagonal block dT.  Replaces the diagonal solves of
 * forwardSolve / backwardSolve (lu.ci:387-436). */
LU_API int lu_trsv_block(lu_handle h, const double* dT, int64_t ldt, int32_t w, int32_t upper, double* dx,
                         void* stream);

/* dy (m) -= dA (m x k) * dx (k).  Replaces offDiagSolve's block product
 * (lu.ci:439-456). */
LU_API int lu_gemv_update(lu_handle h, const double* dA, int64_t lda, int64_t m, int32_t k, const double* dx,
                          double* dy, void* stream);

/* dA <- dA^T in place for an n x n FP64 matrix with row pitch lda (device;
 * asynchronous on stream): converts between column- and row-major
 * storage.  No reference counterpart (its blocks are row-major,
 * lu.h:151-153). */
LU_API int lu_transpose_square(double* dA, int64_t n, int64_t lda, void* stream);

/* Copy a rows x width-byte block between host and device memory (either
 * direction; pitches in bytes), asynchronous on stream.  Host memory should
 * be page-locked for the copy to overlap kernels.  Used by the out-of-core
 * FP64 driver (charmlu_b200/ooc.py) to move column panels of a row-major
 * host matrix; no reference counterpart (the reference keeps every block
 * in memory, scheduler.C:46-47 only limits how many are in flight). */
LU_API int lu_copy_2d(void* dst, int64_t dpitch, const void* src, int64_t spitch, int64_t width, int64_t rows,
                      void* stream);

/* Kernels this library has launched since it was loaded (all handles). */
LU_API int64_t lu_launch_count(void);

/* Solve without allocating (no counterpart in the reference).  For callers
 * that may not call cudaMalloc: a plugin whose host application owns the
 * device memory and grants a fixed budget, a real-time loop that cannot
 * afford an allocation's device-wide synchronisation, or a caller without a
 * handle (lu_create allocates).
 * Same result as lu_solve(h, dLU, lda, ipiv, db, 1, 1, 0, stream): x =
 * A^{-1} b from lu_factor's factors and pivots, db (device) overwritten.
 * Scratch lives in a fixed ~8 KB device array inside the library (held by
 * every GPU that loads it until exit), so n is limited to 131072; larger n
 * returns LU_ERR_ARG.  d_status (optional, device int) receives LU_OK or
 * LU_ERR_TIMEOUT.  The first call on a device resolves the array's address
 * and should come before any stream capture; the address is cached and does
 * not survive a device reset.  Calls share the array: calls that overlap on
 * the GPU race. */
LU_API int lu_solve_noalloc(const double* dLU, int64_t lda, int64_t n, const int32_t* ipiv, double* db,
                            int32_t* d_status, void* stream);

/* Message for a status code. */
LU_API const char* lu_status_string(int status);

#ifdef __cplusplus
}
#endif
#endif /* LU_B200_H */
