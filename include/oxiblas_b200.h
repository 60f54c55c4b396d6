/*
 * oxiblas_b200.h -- C ABI of the B200 (sm_100a) dense-LU engine.
 *
 * This is the drop-in boundary for OxiBLAS.jl's dense partial-pivoted LU path:
 * a Julia (`ccall`), Python (`ctypes`) or C caller hands device pointers and
 * sizes; no torch or CUDA C++ types appear in the signatures.  Matrices are
 * column-major (Julia layout) with a leading dimension; pivots are LAPACK-style
 * 1-based global row indices, exactly the `pivots` field of the reference's
 * `LUFactor` (src/lapack/factorizations.jl:5-10).
 *
 * Every entry point returns an oxi_status (0 = OXI_OK).  Calls are ordered on
 * the handle's stream.  One handle per host thread/task: a handle owns its
 * workspace (sized lazily, like the reference's GemmWorkspace,
 * src/blas/gemm.jl:45-105) and serialises its users.
 */
#ifndef OXIBLAS_B200_H
#define OXIBLAS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes and the reference exception each one maps to. */
enum oxi_status {
    OXI_OK = 0,
    OXI_EINVAL = 1,      /* ArgumentError / DimensionMismatch                        */
    OXI_ESINGULAR = 2,   /* SingularException(info): *h_info holds the first zero pivot */
    OXI_ENONFINITE = 3,  /* ArgumentError("finite mixed input required")             */
    OXI_EOVERFLOW = 4,   /* OverflowError (low-precision conversion)                 */
    OXI_ECUDA = 5,       /* CUDA runtime error                                        */
    OXI_ETIMEOUT = 6,    /* a bounded device-side wait expired                         */
    OXI_ENOMEM = 7,      /* workspace allocation failed                                */
    OXI_ENOTCONVERGED = 8, /* refinement stopped at maxiter (report still filled)     */
    OXI_ESCRATCH = 9,      /* size beyond the fixed scratch of oxi_dgetrs_noalloc       */
    OXI_ENOTPOSDEF = 10    /* PosDefException(info): *h_info holds the failing column     */
};

typedef struct oxi_handle_s *oxi_handle_t;

/* Handle life cycle.  oxi_create binds the handle to the current CUDA device. */
int oxi_create(oxi_handle_t *h);
int oxi_destroy(oxi_handle_t h);
/* cudaStream_t passed as void*; NULL = legacy default stream. */
int oxi_set_stream(oxi_handle_t h, void *stream);
const char *oxi_status_string(int status);
/* Text of the last CUDA error seen by this handle (empty if none). */
const char *oxi_last_error(oxi_handle_t h);

/* Options (the reference's keyword arguments).
 *  OXI_OPT_BLOCKSIZE   lu_factor(...; blocksize=128)     src/lapack/factorizations.jl:17
 *  OXI_OPT_GEMM        0 = tensor-core engine (default), 1 = reference summation order
 *                      (one FMA chain per dot product, as gemm.jl:286-298)
 *  OXI_OPT_TRSM_LEAF   recursive TRSM leaf size (reference default 8, level3.jl:524)
 *  OXI_OPT_LOOKAHEAD   1 (default) = overlap panel k+1 with the trailing update of
 *                      panel k on a second stream (the reference's threaded
 *                      lookahead, factorizations.jl:41-70): the mixed solve's
 *                      16-bit update as the persistent tcgen05 GEMM on whole GPCs
 *                      with one GPC left to the panel, the FP64 update as the
 *                      DMMA GEMM on a low-priority stream.  The reference-order
 *                      GEMM mode keeps the plain schedule.  Results are identical
 *                      bit for bit. */
enum oxi_option {
    OXI_OPT_BLOCKSIZE = 1,
    OXI_OPT_GEMM = 2,
    OXI_OPT_TRSM_LEAF = 3,
    OXI_OPT_LOOKAHEAD = 4,
    OXI_OPT_MIXED_BLOCKSIZE = 5, /* panel width of the mixed-precision factor (256) */
    OXI_OPT_STOP_NORMWISE = 6,   /* 1: the mixed solve stops on the normwise error  */
    OXI_OPT_GMRES_RESTART = 7,   /* GMRES-IR restart length (30)                    */
    OXI_OPT_GRAPHS = 8,          /* 1 (default): a factorization repeated with the same
                                    shape and workspace replays as a CUDA graph      */
    OXI_OPT_TOURNAMENT = 9,      /* 1: the mixed solve's FP32 factor picks each 32-column
                                    leaf's pivots by tournament (TSLU); 0 (default):
                                    partial pivoting, the reference's rule (faster on
                                    B200, see oxiblas.jl_b200/csrc/tslu.cu)           */
    OXI_OPT_WAIT_LIMIT_US = 10,  /* limit of every bounded device wait of this handle's
                                    calls, in microseconds (default 2000000 = 2 s).  The
                                    first wait that runs out sets the call's sticky abort
                                    word: every later wait and kernel of the call returns
                                    at once and the call returns OXI_ETIMEOUT.        */
    OXI_OPT_TEST_MISSING_PRODUCER = 11 /* test hook: k > 0 makes the next factorization on
                                    this handle wait, before its k-th leaf, for a flag
                                    that no kernel sets (a consumer whose producer was
                                    never launched).  One-shot; the call runs without
                                    its CUDA graph and returns OXI_ETIMEOUT after one
                                    wait limit.  No counterpart in the reference.     */
};
int oxi_set_option(oxi_handle_t h, int option, int64_t value);
int oxi_get_option(oxi_handle_t h, int option, int64_t *value);

/* ---------------------------------------------------------------------------
 * getrf: in-place partial-pivoted LU, A (m x n, column-major, lda >= m) is
 * overwritten by L (unit diagonal implicit) and U.
 * Replaces _lu_factor!/lu_factor (src/lapack/factorizations.jl:17-77), i.e. the
 * engine behind OxiBLAS.lu / OxiBLAS.lu! (src/api/linalg_api.jl:217-218).
 * d_ipiv: min(m,n) int64 on the device (1-based global rows).
 * h_info: host int64; 0, or the first zero pivot (the factorization is still
 * completed, as the reference does with check=false).  Returns OXI_ESINGULAR
 * when *h_info > 0 so that a check=true caller can raise SingularException.
 * The call synchronises the handle's stream once (to read info).
 * ------------------------------------------------------------------------- */
int oxi_dgetrf(oxi_handle_t h, int64_t m, int64_t n, double *dA, int64_t lda,
               int64_t *d_ipiv, int64_t *h_info);
int oxi_sgetrf(oxi_handle_t h, int64_t m, int64_t n, float *dA, int64_t lda,
               int64_t *d_ipiv, int64_t *h_info);

/* ---------------------------------------------------------------------------
 * getrs: solve with the factors of oxi_?getrf.  trans 'N': A X = B
 * (LinearAlgebra.ldiv!(F, B), src/api/linalg_api.jl:168-175); 'T' or 'C':
 * A^T X = B (ldiv!(transpose(F), B) / ldiv!(F', B), :176-184).  B (n x nrhs,
 * column-major) is overwritten by X.  The factors must be non-singular
 * (the caller checks info first, as _lu_dense_ready does, :163-167).
 * ------------------------------------------------------------------------- */
int oxi_dgetrs(oxi_handle_t h, char trans, int64_t n, int64_t nrhs, const double *dLU,
               int64_t lda, const int64_t *d_ipiv, double *dB, int64_t ldb);
int oxi_sgetrs(oxi_handle_t h, char trans, int64_t n, int64_t nrhs, const float *dLU,
               int64_t lda, const int64_t *d_ipiv, float *dB, int64_t ldb);

/* ---------------------------------------------------------------------------
 * oxi_dgetrs_noalloc: oxi_dgetrs that allocates nothing.  It has no counterpart
 * in the reference; it exists for callers that cannot allocate device memory
 * at solve time (a process whose device memory is held by its own pool
 * allocator, or a latency-bound loop that cudaFree's implicit device-wide
 * synchronisation would stall).  Same arguments, results and status codes as
 * oxi_dgetrs, but no handle: work runs on `stream` (cudaStream_t as void*,
 * NULL = legacy default stream) of the current device.
 * Its scratch (permutation, solve vector, control words) is one file-scope
 * device array of OXI_NOALLOC_SCRATCH_BYTES per device.  Limits:
 * n <= OXI_NOALLOC_MAX_N and n * nrhs <= OXI_NOALLOC_MAX_ELEMS, else
 * OXI_ESCRATCH (nothing is launched).  The first call on a device (and the
 * first after its context was re-created, e.g. by a device reset) resolves the
 * array's address and loads the kernels it uses; make that first call before
 * any stream capture.  Every call shares the array and leaves its
 * contents behind: calls that overlap on the GPU (two streams, two host
 * threads) race and must be serialised by the caller.  It calls no cudaMalloc,
 * cudaFree or allocating library routine.  The call synchronises `stream`.
 * ------------------------------------------------------------------------- */
#define OXI_NOALLOC_SCRATCH_BYTES (8 << 20)
#define OXI_NOALLOC_MAX_N 65536
#define OXI_NOALLOC_MAX_ELEMS 917504 /* (8 MiB - 1 MiB) / sizeof(double) */
int oxi_dgetrs_noalloc(void *stream, char trans, int64_t n, int64_t nrhs, const double *dLU,
                       int64_t lda, const int64_t *d_ipiv, double *dB, int64_t ldb);

/* ---------------------------------------------------------------------------
 * Adjoint of X = A \ B (reverse-mode rule, e.g. a ChainRulesCore rrule or a
 * torch.autograd.Function backward) with the factors of oxi_dgetrf reused:
 *   Bbar = A^-T Xbar     (the transposed solve of ldiv!(transpose(F), B),
 *                         src/api/linalg_api.jl:176-184; solve_transposed,
 *                         src/lapack/expert_refinement.jl:2-23)
 *   Abar = -Bbar X^T     (n x n, written in one pass)
 * X, Xbar, Bbar: n x nrhs column-major; Bbar may be Xbar itself (same ldb),
 * not X.  nrhs = 0 gives Abar = 0.  The reference has no differentiation rule;
 * this entry point is the one its rrule would call.
 * ------------------------------------------------------------------------- */
int oxi_dlu_adjoint(oxi_handle_t h, int64_t n, int64_t nrhs, const double *dLU, int64_t lda,
                    const int64_t *d_ipiv, const double *dX, int64_t ldx, const double *dXbar,
                    int64_t ldxbar, double *dBbar, int64_t ldbbar, double *dAbar,
                    int64_t ldabar);

/* Batched form for many independent small factorizations (orders 0..256,
 * 0..8 right-hand sides each; the factors and pivots of
 * oxi_dgetrf_batched_uneven / oxi_dgesv_batched_uneven with prec FP64), one
 * launch: per problem i, Bbar_i = A_i^-T Xbar_i and Abar_i = -Bbar_i X_i^T.  All
 * arrays are DEVICE arrays of `count` entries (d_nrhs nullable: one right-hand
 * side each); Bbar_i may be Xbar_i itself, Abar_i overlaps nothing else.
 * d_info[i]: 0, -1 for bad arguments
 * of that problem, or the first zero diagonal of its U.  Returns OXI_EINVAL /
 * OXI_ESINGULAR when any problem had that outcome.  The reference has no
 * batched factorization; its batching precedent is gemm_batched!
 * (src/blas/batched.jl:4-49), and per problem this is oxi_dlu_adjoint. */
int oxi_dlu_adjoint_batched_uneven(oxi_handle_t h, int64_t count, const int32_t *d_n,
                                   const int32_t *d_nrhs, double *const *d_LU, const int64_t *d_ldlu,
                                   int64_t *const *d_ipiv, double *const *d_X, const int64_t *d_ldx,
                                   double *const *d_Xbar, const int64_t *d_ldxbar,
                                   double *const *d_Bbar, const int64_t *d_ldbbar,
                                   double *const *d_Abar, const int64_t *d_ldabar, int32_t *d_info);

/* ---------------------------------------------------------------------------
 * Trailing-update GEMM as a standalone kernel: C <- C - A*B (column-major),
 * the gemm!(C, A, B, -1, 1) call of src/lapack/factorizations.jl:69
 * (src/blas/gemm.jl:635).
 * ------------------------------------------------------------------------- */
int oxi_dgemm_update(oxi_handle_t h, int64_t m, int64_t n, int64_t k, double *dC,
                     int64_t ldc, const double *dA, int64_t lda, const double *dB,
                     int64_t ldb);

/* ---------------------------------------------------------------------------
 * Mixed-precision solve: low-precision LU of the radix-equilibrated matrix plus
 * FP64 iterative refinement.  Replaces mixed_solve / _mixed_precision_impl
 * (src/lapack/factorizations.jl:425-427, src/lapack/extended_lapack.jl:175-226).
 *   prec    OXI_PREC_BF16 / OXI_PREC_FP16: FP32 panels, trailing updates on the
 *           tensor cores with 16-bit operands and FP32 accumulation;
 *           OXI_PREC_BF16X3 / OXI_PREC_FP16X3: the same with each operand split
 *           into two BF16 (FP16, scaled) terms and three products accumulated
 *           (one GEMM over 3K);
 *           OXI_PREC_FP32: FP32 throughout (the reference's default Low type);
 *           OXI_PREC_FP64: working-precision factor (lowtype=Float64).
 *   refine  OXI_REFINE_IR (classical, as the reference), OXI_REFINE_GMRES
 *           (GMRES-IR), OXI_REFINE_AUTO (IR, switching to GMRES-IR on stagnation).
 * A (n x n), B and X (n x nrhs, nrhs <= 16) are column-major FP64 device
 * arrays; X receives the solution.  The stop test compares the componentwise
 * backward error max_i |r_i| / (|A||x| + |b|)_i (the reference metric) with
 * rtol, or the normwise one when OXI_OPT_STOP_NORMWISE is set.  A singular low
 * factor falls back to an FP64 factor (report.fallback, reason FALLBACK).
 * Returns OXI_OK when converged, OXI_ENOTCONVERGED at maxiter (report filled),
 * OXI_ENONFINITE for non-finite input, OXI_ESINGULAR when even the FP64 factor
 * is singular, OXI_EOVERFLOW when a scaled right-hand side overflows.
 * ------------------------------------------------------------------------- */
enum oxi_precision {
    OXI_PREC_FP32 = 0,
    OXI_PREC_BF16 = 1,
    OXI_PREC_FP16 = 2,
    OXI_PREC_FP64 = 3,
    OXI_PREC_BF16X3 = 4, /* split BF16: A_hi B_hi + A_hi B_lo + A_lo B_hi, BF16 operands */
    OXI_PREC_FP16X3 = 5  /* split FP16, power-of-two scaled: the same three products with
                            FP16 operands (about 22 significant bits instead of 16) */
};
enum oxi_refinement { OXI_REFINE_IR = 0, OXI_REFINE_GMRES = 1, OXI_REFINE_AUTO = 2 };
enum oxi_reason {
    OXI_REASON_CONVERGED = 0,       /* :converged               */
    OXI_REASON_ITERATION_LIMIT = 1, /* :iteration_limit         */
    OXI_REASON_FALLBACK = 2,        /* :working_factor_fallback */
    OXI_REASON_NONFINITE = 3        /* :nonfinite_iteration     */
};
typedef struct oxi_refine_report {
    int64_t iterations;             /* outer refinement steps (reference `iterations`) */
    int64_t gmres_iterations;       /* inner GMRES iterations in total */
    double backward_error;          /* componentwise (reference `backward_error`) */
    double backward_error_normwise; /* ||b-Ax||_inf / (||A||_inf ||x||_inf + ||b||_inf) */
    double residual_norm;           /* ||B - A X||_F (reference `residual`) */
    double factor_ms;               /* equilibration + factorization time */
    double refine_ms;               /* first solve + refinement time */
    int64_t info;                   /* first zero pivot of the low-precision factor */
    int32_t converged;
    int32_t fallback;
    int32_t refine_used;            /* oxi_refinement actually used at the end */
    int32_t reason;                 /* oxi_reason */
    int32_t low_type;               /* oxi_precision of the factor */
    int32_t reserved;
} oxi_refine_report;

/* The mixed path's trailing-update kernel as a standalone call: C <- C - A*B
 * (column-major FP32) with A and B rounded to prec (OXI_PREC_BF16 / _FP16 /
 * _BF16X3 / _FP16X3, FP16
 * with power-of-two operand scaling) and FP32 accumulation on the tensor cores
 * (tcgen05); OXI_PREC_FP32 runs the FP32 CUDA-core GEMM.  The low-precision
 * counterpart of gemm!(C, A, B, -1, 1) (src/blas/gemm.jl:635). */
int oxi_sgemm_update_lowp(oxi_handle_t h, int prec, int64_t m, int64_t n, int64_t k, float *dC,
                          int64_t ldc, const float *dA, int64_t lda, const float *dB, int64_t ldb);

int oxi_dgesv_mixed(oxi_handle_t h, int prec, int refine, int64_t n, int64_t nrhs,
                    const double *dA, int64_t lda, const double *dB, int64_t ldb, double *dX,
                    int64_t ldx, int maxiter, double rtol, oxi_refine_report *out);

/* mixed_solve(A, b; factorization=:cholesky) (src/lapack/extended_lapack.jl:
 * 175-226, Cholesky family): one global scale max|a_ij| keeps the matrix
 * symmetric, the low-precision Cholesky of the lower triangle of A / scale
 * (FP32 panels, the symmetric update in prec on the tensor cores), FP64
 * refinement as oxi_dgesv_mixed.  A low factor that is not positive definite
 * falls back to the FP64 Cholesky (report fallback = 1); if that fails too:
 * OXI_ENOTPOSDEF with report->info the failing column. */
int oxi_dposv_mixed(oxi_handle_t h, int prec, int refine, int64_t n, int64_t nrhs,
                    const double *dA, int64_t lda, const double *dB, int64_t ldb, double *dX,
                    int64_t ldx, int maxiter, double rtol, oxi_refine_report *out);

/* ---------------------------------------------------------------------------
 * Expert solves and the condition estimate (FP64).
 * ------------------------------------------------------------------------- */
typedef struct oxi_solve_report {
    int64_t iterations;             /* refinement steps taken (reference `iterations`) */
    double backward_error;          /* componentwise, max_i |r_i| / (|A||x| + |b|)_i */
    double residual_norm;           /* ||B - A X||_F of the final iterate */
    double rcond_estimate;          /* refine_solve: min(1, 1 / (||A||_1 est(||A^-1||_1))) */
    double forward_error_estimate;  /* refine_solve: delta / (1 - delta), delta =
                                       est(||A^-1||_1) ||R||_1 / ||X||_1 (Inf if delta >= 1) */
    double inverse_norm_estimate;   /* refine_solve: est(||A^-1||_1) */
    int64_t info;                   /* expert_solve: first zero row or zero pivot (1-based) */
    int32_t converged;
    int32_t reserved;
} oxi_solve_report;

/* expert_solve(A, b; maxiter=8, rtol=8eps, equilibrate=true)
 * (src/lapack/advanced_factorizations.jl:591-645): rows scaled by their max
 * |a| (a zero row: OXI_ESINGULAR, info = its 1-based index), then columns by
 * theirs, FP64 partial-pivoted LU of the scaled matrix, scaled solves and
 * componentwise iterative refinement to rtol.  A (n x n), B and X (n x nrhs,
 * nrhs <= 16) column-major.  Optional outputs (NULL to skip): the row and
 * column scales (n each) and the factorization of the scaled matrix (dF, n x n,
 * leading dimension ldf; d_ipiv, n) -- the reference's `factor` field.
 * OXI_OK when converged, OXI_ENOTCONVERGED at maxiter (report filled). */
int oxi_dexpert_solve(oxi_handle_t h, int64_t n, int64_t nrhs, const double *dA, int64_t lda,
                      const double *dB, int64_t ldb, double *dX, int64_t ldx, int maxiter, double rtol,
                      int equilibrate, double *d_row_scale, double *d_col_scale, double *dF,
                      int64_t ldf, int64_t *d_ipiv, oxi_solve_report *out);
/* refine_solve(A, F, b; maxiter=8, rtol=8eps) (src/lapack/expert_refinement.jl:89-104):
 * X = F \ B, then FP64 residuals and corrections with the factors of oxi_dgetrf
 * (dLU, d_ipiv) until the componentwise backward error is <= rtol; the report
 * adds the reference's rcond and forward-error estimates. */
int oxi_drefine_solve(oxi_handle_t h, int64_t n, int64_t nrhs, const double *dA, int64_t lda,
                      const double *dLU, int64_t ldlu, const int64_t *d_ipiv, const double *dB,
                      int64_t ldb, double *dX, int64_t ldx, int maxiter, double rtol,
                      oxi_solve_report *out);
/* inverse_norm_estimate(F, T, n; maxiter=8) (src/lapack/expert_refinement.jl:45-60):
 * Hager-Higham estimate of ||A^-1||_1 from solves with the factors of oxi_dgetrf
 * and with their transpose.  An estimate, not a certified bound. */
int oxi_dinverse_norm_estimate(oxi_handle_t h, int64_t n, const double *dLU, int64_t lda,
                               const int64_t *d_ipiv, int maxiter, double *h_estimate);
/* inv(F) (src/api/linalg_api.jl:1143-1144; OxiBLAS.inv of a dense matrix,
 * native_inverse, src/lapack/dense_utilities.jl:14-32, factors first): the
 * n x n inverse from the factors of oxi_dgetrf, as the solve with the
 * identity, into dAinv (column-major, leading dimension ldainv). */
int oxi_dgetri(oxi_handle_t h, int64_t n, const double *dLU, int64_t lda, const int64_t *d_ipiv,
               double *dAinv, int64_t ldainv);

/* ---------------------------------------------------------------------------
 * Cholesky (FP64): the reference's other dense factorization on the same
 * engine (src/lapack/factorizations.jl:205-305; OxiBLAS.cholesky / cholesky!,
 * src/api/linalg_api.jl:221-290).
 * oxi_dpotrf: the lower triangle of A (n x n, column-major) is overwritten by
 * L with A = L L^T and the strict upper triangle set to zero; the upper
 * triangle is not read.  A pivot that is not finite and positive stops it:
 * *h_info = that column (1-based), OXI_ENOTPOSDEF, the upper triangle left as
 * it was.  oxi_dpotrs: B (n x nrhs) <- A^-1 B with the factor of oxi_dpotrf. */
int oxi_dpotrf(oxi_handle_t h, int64_t n, double *dA, int64_t lda, int64_t *h_info);
int oxi_dpotrs(oxi_handle_t h, int64_t n, int64_t nrhs, const double *dL, int64_t ldl, double *dB,
               int64_t ldb);

/* ---------------------------------------------------------------------------
 * Complex LU (ComplexF64, interleaved real/imaginary pairs, column-major,
 * 16-byte aligned): _lu_factor! / _lu_panel! for Complex{Float64}
 * (src/lapack/factorizations.jl:30-152; 16-column leaves, the pivot the
 * largest abs2 with abs when that square is not finite, :92-113) and
 * ldiv!(F, B) / ldiv!(transpose(F), B) / ldiv!(F', B)
 * (src/api/linalg_api.jl:168-184).  Same contracts as oxi_dgetrf /
 * oxi_dgetrs; trans 'N', 'T' or 'C'. */
int oxi_zgetrf(oxi_handle_t h, int64_t m, int64_t n, void *dA, int64_t lda, int64_t *d_ipiv,
               int64_t *h_info);
int oxi_zgetrs(oxi_handle_t h, char trans, int64_t n, int64_t nrhs, const void *dLU, int64_t lda,
               const int64_t *d_ipiv, void *dB, int64_t ldb);

/* Layout: dB (n x m, column-major, ldb) = dA^T for the m x n column-major dA
 * (lda), elements of elem_bytes = 4, 8 or 16 bytes (float, double, ComplexF64).
 * A row-major host array (Python, C) is the column-major transpose of the
 * matrix it holds: this makes the column-major copy the other entry points
 * take, on the device.  No reference counterpart (Julia arrays are already
 * column-major).  Stream-ordered; no synchronisation. */
int oxi_transpose(oxi_handle_t h, int elem_bytes, int64_t m, int64_t n, const void *dA, int64_t lda, void *dB,
                  int64_t ldb);

/* Radix equilibration, the first step of the mixed solve, as its own call:
 * equilibrate(A; radix=true) (src/lapack/dense_utilities.jl:191-213).  For the
 * m x n column-major A: d_rows[i] = 2^round(log2 max_j |A[i,j]|) (1 for a zero
 * row), then d_cols[j] = the same of column j of the row-scaled matrix, both
 * clamped to Float64's exponent range; dE (nullable, leading dimension lde)
 * receives A ./ d_rows ./ d_cols^T.  OXI_ENONFINITE for non-finite input. */
int oxi_dequilibrate(oxi_handle_t h, int64_t m, int64_t n, const double *dA, int64_t lda,
                     double *d_rows, double *d_cols, double *dE, int64_t lde);

/* ---------------------------------------------------------------------------
 * Batched LU of many independent small matrices of uneven orders (1..256), in
 * one persistent launch that takes matrices from a size-bucketed work queue
 * (replayed as a CUDA graph when the same call repeats).  The reference
 * factors one matrix per lu call (src/lapack/factorizations.jl:17-77); its
 * batching pattern is gemm_batched! (src/blas/batched.jl:4-49), an outer loop
 * over independent problems.  Per matrix the results are those of lu/ldiv!
 * (pivots with the reference's rule, factors in place, LAPACK 1-based ipiv).
 * All array arguments are DEVICE arrays of `count` entries; d_A[i] (column-
 * major, leading dimension d_lda[i] >= n) etc. point to each problem.
 * d_info[i]: 0, the first zero pivot (> 0), -1 for bad arguments of that
 * problem, -2 for non-finite input (mixed).  The call synchronises once and
 * returns OXI_EINVAL / OXI_ENONFINITE / OXI_ESINGULAR / OXI_ENOTCONVERGED if
 * any problem had that outcome (d_info tells which), else OXI_OK.
 * ------------------------------------------------------------------------- */
int oxi_dgetrf_batched_uneven(oxi_handle_t h, int64_t count, const int32_t *d_n, double *const *d_A,
                              const int64_t *d_lda, int64_t *const *d_ipiv, int32_t *d_info);
/* Factor and solve (1..8 right-hand sides each, d_nrhs[i] <= 8):
 *   prec OXI_PREC_FP64: plain FP64 LU in place (A -> factors, B -> X, as
 *        LAPACK dgesv); d_X, d_ldx, d_iters, d_berr unused (may be NULL).
 *   prec OXI_PREC_FP32: FP32 LU of the radix-equilibrated matrix plus FP64
 *        iterative refinement (mixed_solve, src/lapack/extended_lapack.jl:
 *        175-226) to componentwise backward error <= rtol or maxiter steps; A
 *        and B are left intact, X receives the solution, d_iters / d_berr
 *        (nullable) the steps and the final backward error per problem.
 * d_ipiv (nullable; entries nullable): pivots of each factor. */
int oxi_dgesv_batched_uneven(oxi_handle_t h, int prec, int64_t count, const int32_t *d_n,
                             const int32_t *d_nrhs, double *const *d_A, const int64_t *d_lda,
                             int64_t *const *d_ipiv, double *const *d_B, const int64_t *d_ldb,
                             double *const *d_X, const int64_t *d_ldx, int32_t *d_info,
                             int32_t *d_iters, double *d_berr, int maxiter, double rtol);
/* Autotuner: times candidate panel widths per size bucket (orders 32b+1..32b+32)
 * and shared-memory thresholds (orders up to n_smem keep the working matrix on
 * chip) for prec (OXI_PREC_FP64 or OXI_PREC_FP32) on synthetic matrices
 * (N(0,1) + n I) of the host-given orders h_n with nrhs right-hand sides, and
 * keeps the fastest in the handle.  *best_ms (nullable): its time. */
int oxi_batched_autotune(oxi_handle_t h, int prec, int64_t count, const int32_t *h_n, int32_t nrhs,
                         double *best_ms);
/* Current tuning (defaults when untuned) and explicit setting (a saved table). */
int oxi_batched_get_tuning(oxi_handle_t h, int prec, int32_t *n_smem, int32_t *nb /* [8] */);
int oxi_batched_set_tuning(oxi_handle_t h, int prec, int32_t n_smem, const int32_t *nb /* [8] */);

/* ---------------------------------------------------------------------------
 * Engine instrumentation (no counterpart in the reference, whose benchmarks time
 * whole calls): kernels launched per handle, and, when enabled, CUDA-event
 * timing of every launch of each kernel class on the handle's stream together
 * with its algorithmic flops and bytes.
 * ------------------------------------------------------------------------- */
enum oxi_kernel_class {
    OXI_K_LEAF = 0, OXI_K_ROWMOVES, OXI_K_TRSM_LEAF, OXI_K_GEMM_REF, OXI_K_GEMM_DMMA,
    OXI_K_GEMM_TC, OXI_K_CONVERT, OXI_K_TRSV, OXI_K_RESIDUAL, OXI_K_OTHER, OXI_K_COUNT
};
int oxi_profile_enable(oxi_handle_t h, int on);  /* also clears the records */
/* The profiled launches in issue order, 4 doubles each: kernel class, stream
 * index (order of first use), start and end in ms from the first launch's start.
 * *count = the number of records (at most max written). */
int oxi_profile_timeline(oxi_handle_t h, int64_t max, double *out, int64_t *count);
int oxi_profile_read(oxi_handle_t h, int kind, int64_t *launches, double *total_ms,
                     double *flops, double *bytes);
int oxi_launch_count(oxi_handle_t h, int64_t *count);
int oxi_launch_count_reset(oxi_handle_t h);

#ifdef __cplusplus
}
#endif

#endif /* OXIBLAS_B200_H */
