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
    OXI_ENOTCONVERGED = 8 /* refinement stopped at maxiter (report still filled)      */
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
 *  OXI_OPT_LOOKAHEAD   1 = overlap panel k+1 with the trailing update of panel k
 *                      (the reference's threaded lookahead, factorizations.jl:41-70) */
enum oxi_option {
    OXI_OPT_BLOCKSIZE = 1,
    OXI_OPT_GEMM = 2,
    OXI_OPT_TRSM_LEAF = 3,
    OXI_OPT_LOOKAHEAD = 4
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
 * Trailing-update GEMM as a standalone kernel: C <- C - A*B (column-major),
 * the gemm!(C, A, B, -1, 1) call of src/lapack/factorizations.jl:69
 * (src/blas/gemm.jl:635).
 * ------------------------------------------------------------------------- */
int oxi_dgemm_update(oxi_handle_t h, int64_t m, int64_t n, int64_t k, double *dC,
                     int64_t ldc, const double *dA, int64_t lda, const double *dB,
                     int64_t ldb);

#ifdef __cplusplus
}
#endif

#endif /* OXIBLAS_B200_H */
