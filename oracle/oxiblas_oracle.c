/*
 * oxiblas_oracle.c -- CPU restatement of OxiBLAS.jl's dense LU hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: the test suite,
 * the smoke check and the CPU-baseline leg of the benchmark load it to check
 * (or time beside) the CUDA path.  The product library never links it and
 * never falls back to it.
 *
 * Everything is column-major (Julia layout) with a leading dimension, 0-based
 * loops, and LAPACK-style 1-based global pivot indices (`ipiv`).  Each routine
 * cites the reference function it restates (paths relative to the OxiBLAS.jl
 * project root).  Arithmetic follows the reference's order where it is
 * observable: the pivot rule (largest |a|, strict '>' so the first row wins a
 * tie), division by the pivot (not a reciprocal multiply), fused multiply-add
 * in the rank-1 update, and the GEMM's "dot product first, then C - s" form.
 *
 * Built with gcc (-O3 -fopenmp -ffp-contract=off, explicit fma()) by
 * oracle/Makefile.  OpenMP parallelises the trailing GEMM, the TRSM right-hand
 * sides and the residual, the way the reference splits work across Julia
 * threads (src/blas/gemm.jl:561 worker grid, src/blas/level3.jl:383 RHS split).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <immintrin.h>

typedef int64_t i64;

/* 1 (default): the trailing-update GEMM runs register-tiled; 0: the plain
 * scalar loops.  Both give the same bits (see _gemm_tiled); the switch exists
 * so that the tests can check that. */
static int orc_gemm_tiled = 1;
void orc_set_gemm_tiled(int on) { orc_gemm_tiled = on != 0; }

/* ------------------------------------------------------------------------ */
/* Trailing-update kernel C <- C - A*B, register-tiled.                      */
/* ------------------------------------------------------------------------ */
/* Element by element this is the arithmetic of src/blas/gemm.jl:286-298
 * (_reference!): s = fma chain over p = 0..k-1 in order, from zero, then
 * C - s.  It is also the order of the reference's packed SIMD path for every
 * GEMM of the factorization (gemm.jl:414 _packed_region! -> simd.jl:151
 * _simd_micro!): the micro-kernel keeps one accumulator per element of its
 * register tile, fma-chained along p from zero over a kc-block, and stores
 * fma(beta = 1, C, alpha * acc) = C - acc; getrf's updates have k <= nb = 128,
 * below kc = 448 (Float64) / 896 (Float32), so there is one block.  The tiles
 * here (8 x 6 doubles, 16 x 6 floats: two AVX2 vectors by six broadcast
 * columns, as the reference's W = 4/8, R = 2, N = 6 tile) and the packed
 * operands (as _pack_a! / _pack_b!) only make it fast: the per-element
 * operations and their order are those of the scalar form.  Rows are blocked
 * by MC for the L2 cache; OpenMP splits row blocks x 48-column chunks (the
 * reference's worker grid, gemm.jl:561). */
#define ORC_MC 256
#define ORC_NCH 48

/* The tiles read packed operands: Ap holds MR rows of A per k step
 * (Ap[p * MR + r]), Bp six columns of B per k step (Bp[p * 6 + jj]), so both
 * stream contiguously whatever the caller's leading dimensions. */
static void d_tile_8x6(i64 k, const double *Ap, const double *Bp, double *C, i64 ldc) {
    __m256d c00 = _mm256_setzero_pd(), c01 = c00, c02 = c00, c03 = c00, c04 = c00, c05 = c00;
    __m256d c10 = c00, c11 = c00, c12 = c00, c13 = c00, c14 = c00, c15 = c00;
    for (i64 p = 0; p < k; ++p) {
        const __m256d a0 = _mm256_loadu_pd(Ap + 8 * p), a1 = _mm256_loadu_pd(Ap + 8 * p + 4);
        const double *b = Bp + 6 * p;
        __m256d bb = _mm256_broadcast_sd(b);
        c00 = _mm256_fmadd_pd(a0, bb, c00); c10 = _mm256_fmadd_pd(a1, bb, c10);
        bb = _mm256_broadcast_sd(b + 1);
        c01 = _mm256_fmadd_pd(a0, bb, c01); c11 = _mm256_fmadd_pd(a1, bb, c11);
        bb = _mm256_broadcast_sd(b + 2);
        c02 = _mm256_fmadd_pd(a0, bb, c02); c12 = _mm256_fmadd_pd(a1, bb, c12);
        bb = _mm256_broadcast_sd(b + 3);
        c03 = _mm256_fmadd_pd(a0, bb, c03); c13 = _mm256_fmadd_pd(a1, bb, c13);
        bb = _mm256_broadcast_sd(b + 4);
        c04 = _mm256_fmadd_pd(a0, bb, c04); c14 = _mm256_fmadd_pd(a1, bb, c14);
        bb = _mm256_broadcast_sd(b + 5);
        c05 = _mm256_fmadd_pd(a0, bb, c05); c15 = _mm256_fmadd_pd(a1, bb, c15);
    }
#define ORC_D_ST(j, lo, hi)                                                                   \
    _mm256_storeu_pd(C + (j) * ldc, _mm256_sub_pd(_mm256_loadu_pd(C + (j) * ldc), lo));       \
    _mm256_storeu_pd(C + (j) * ldc + 4, _mm256_sub_pd(_mm256_loadu_pd(C + (j) * ldc + 4), hi));
    ORC_D_ST(0, c00, c10) ORC_D_ST(1, c01, c11) ORC_D_ST(2, c02, c12)
    ORC_D_ST(3, c03, c13) ORC_D_ST(4, c04, c14) ORC_D_ST(5, c05, c15)
#undef ORC_D_ST
}

static void s_tile_16x6(i64 k, const float *Ap, const float *Bp, float *C, i64 ldc) {
    __m256 c00 = _mm256_setzero_ps(), c01 = c00, c02 = c00, c03 = c00, c04 = c00, c05 = c00;
    __m256 c10 = c00, c11 = c00, c12 = c00, c13 = c00, c14 = c00, c15 = c00;
    for (i64 p = 0; p < k; ++p) {
        const __m256 a0 = _mm256_loadu_ps(Ap + 16 * p), a1 = _mm256_loadu_ps(Ap + 16 * p + 8);
        const float *b = Bp + 6 * p;
        __m256 bb = _mm256_broadcast_ss(b);
        c00 = _mm256_fmadd_ps(a0, bb, c00); c10 = _mm256_fmadd_ps(a1, bb, c10);
        bb = _mm256_broadcast_ss(b + 1);
        c01 = _mm256_fmadd_ps(a0, bb, c01); c11 = _mm256_fmadd_ps(a1, bb, c11);
        bb = _mm256_broadcast_ss(b + 2);
        c02 = _mm256_fmadd_ps(a0, bb, c02); c12 = _mm256_fmadd_ps(a1, bb, c12);
        bb = _mm256_broadcast_ss(b + 3);
        c03 = _mm256_fmadd_ps(a0, bb, c03); c13 = _mm256_fmadd_ps(a1, bb, c13);
        bb = _mm256_broadcast_ss(b + 4);
        c04 = _mm256_fmadd_ps(a0, bb, c04); c14 = _mm256_fmadd_ps(a1, bb, c14);
        bb = _mm256_broadcast_ss(b + 5);
        c05 = _mm256_fmadd_ps(a0, bb, c05); c15 = _mm256_fmadd_ps(a1, bb, c15);
    }
#define ORC_S_ST(j, lo, hi)                                                                   \
    _mm256_storeu_ps(C + (j) * ldc, _mm256_sub_ps(_mm256_loadu_ps(C + (j) * ldc), lo));       \
    _mm256_storeu_ps(C + (j) * ldc + 8, _mm256_sub_ps(_mm256_loadu_ps(C + (j) * ldc + 8), hi));
    ORC_S_ST(0, c00, c10) ORC_S_ST(1, c01, c11) ORC_S_ST(2, c02, c12)
    ORC_S_ST(3, c03, c13) ORC_S_ST(4, c04, c14) ORC_S_ST(5, c05, c15)
#undef ORC_S_ST
}

#define DEFINE_GEMM_TILED(T, P, FMA, MR, TILE)                                           \
static void P##_gemm_elem(i64 k, const T *A, i64 lda, const T *B, T *c) {                \
    T s = 0;                                                                             \
    for (i64 p = 0; p < k; ++p) s = FMA(A[p * lda], B[p], s);                            \
    *c = *c - s;                                                                         \
}                                                                                        \
static void P##_gemm_tiled(i64 m, i64 n, i64 k, const T *A, i64 lda, const T *B,       \
                           i64 ldb, T *C, i64 ldc) {                                     \
    const i64 mt = m / MR * MR, nib = (mt + ORC_MC - 1) / ORC_MC;                        \
    const i64 njb = (n + ORC_NCH - 1) / ORC_NCH;                                         \
    const int par = (double)m * n * k > 2e6;                                             \
    _Pragma("omp parallel if(par)")                                                      \
    {                                                                                    \
        T *Ap = (T *)malloc(sizeof(T) * (size_t)ORC_MC * k);                             \
        T *Bp = (T *)malloc(sizeof(T) * (size_t)ORC_NCH * k);                            \
        _Pragma("omp for collapse(2) schedule(dynamic)")                                 \
        for (i64 ib = 0; ib < nib; ++ib)                                                 \
            for (i64 jb = 0; jb < njb; ++jb) {                                           \
                const i64 i0 = ib * ORC_MC, i1 = i0 + ORC_MC < mt ? i0 + ORC_MC : mt;    \
                const i64 j0 = jb * ORC_NCH, j1 = j0 + ORC_NCH < n ? j0 + ORC_NCH : n;   \
                const i64 jt = j0 + (j1 - j0) / 6 * 6;                                   \
                for (i64 i = i0; i < i1; i += MR) {                                      \
                    T *ap = Ap + (i - i0) * k;                                           \
                    for (i64 p = 0; p < k; ++p)                                          \
                        for (i64 r = 0; r < MR; ++r) ap[p * MR + r] = A[i + r + p * lda];\
                }                                                                        \
                for (i64 j = j0; j < jt; j += 6) {                                       \
                    T *bp = Bp + (j - j0) * k;                                           \
                    for (i64 p = 0; p < k; ++p)                                          \
                        for (i64 jj = 0; jj < 6; ++jj) bp[p * 6 + jj] = B[p + (j + jj) * ldb];\
                }                                                                        \
                for (i64 j = j0; j < jt; j += 6)                                         \
                    for (i64 i = i0; i < i1; i += MR)                                    \
                        TILE(k, Ap + (i - i0) * k, Bp + (j - j0) * k, C + i + j * ldc, ldc);\
                for (i64 j = jt; j < j1; ++j)                                            \
                    for (i64 i = i0; i < i1; ++i)                                        \
                        P##_gemm_elem(k, A + i, lda, B + j * ldb, C + i + j * ldc);      \
            }                                                                            \
        free(Ap);                                                                        \
        free(Bp);                                                                        \
        if (mt < m) {                                                                    \
            _Pragma("omp for schedule(static)")                                          \
            for (i64 j = 0; j < n; ++j)                                                  \
                for (i64 i = mt; i < m; ++i)                                             \
                    P##_gemm_elem(k, A + i, lda, B + j * ldb, C + i + j * ldc);          \
        }                                                                                \
    }                                                                                    \
}
DEFINE_GEMM_TILED(double, d, fma, 8, d_tile_8x6)
DEFINE_GEMM_TILED(float, s, fmaf, 16, s_tile_16x6)

/* ------------------------------------------------------------------------ */
/* Type-generic body: instantiated for double (d) and float (s).            */
/* ------------------------------------------------------------------------ */
#define DEFINE_LU(T, P, FMA, ABS)                                                        \
                                                                                         \
/* C[0:m,0:n] <- C - A[0:m,0:k] * B[0:k,0:n].                                        \
 * src/blas/gemm.jl:286-298 (_reference!): s = sum_p muladd(A[i,p], B[p,j], s), then   \
 * C = alpha*s + beta*C with alpha = -1, beta = 1 (the trailing update of             \
 * src/lapack/factorizations.jl:69).  The dot products run along p in order. */       \
static void P##_gemm_minus(i64 m, i64 n, i64 k, const T *A, i64 lda, const T *B,        \
                           i64 ldb, T *C, i64 ldc) {                                     \
    if (m <= 0 || n <= 0 || k <= 0) return;                                              \
    if (orc_gemm_tiled) { P##_gemm_tiled(m, n, k, A, lda, B, ldb, C, ldc); return; }     \
    int par = (double)m * n * k > 2e6;                                                   \
    _Pragma("omp parallel if(par)")                                                      \
    {                                                                                    \
        T *s = (T *)malloc(sizeof(T) * (size_t)m);                                       \
        _Pragma("omp for schedule(static)")                                              \
        for (i64 j = 0; j < n; ++j) {                                                    \
            for (i64 i = 0; i < m; ++i) s[i] = 0;                                        \
            for (i64 p = 0; p < k; ++p) {                                                \
                const T b = B[p + j * ldb];                                              \
                const T *a = A + p * lda;                                                \
                for (i64 i = 0; i < m; ++i) s[i] = FMA(a[i], b, s[i]);                   \
            }                                                                            \
            T *c = C + j * ldc;                                                          \
            for (i64 i = 0; i < m; ++i) c[i] = c[i] - s[i];                              \
        }                                                                                \
        free(s);                                                                         \
    }                                                                                    \
}                                                                                        \
                                                                                         \
/* Leaf of the left TRSM: src/blas/level3.jl:309-321 (_trsm_leaf_generic!, left).    \
 * Lower: rows top-down, s = B[i,j]; s = muladd(-A[i,p], B[p,j], s) for p < i;       \
 * upper: rows bottom-up over p > i; a non-unit diagonal divides. */                   \
static void P##_trsm_leaf(i64 nt, i64 nrhs, const T *A, i64 lda, T *B, i64 ldb,        \
                          int upper, int unit) {                                         \
    for (i64 j = 0; j < nrhs; ++j) {                                                     \
        T *b = B + j * ldb;                                                              \
        if (!upper) {                                                                    \
            for (i64 i = 0; i < nt; ++i) {                                               \
                T s = b[i];                                                              \
                for (i64 p = 0; p < i; ++p) s = FMA(-A[i + p * lda], b[p], s);           \
                b[i] = unit ? s : s / A[i + i * lda];                                    \
            }                                                                            \
        } else {                                                                         \
            for (i64 i = nt - 1; i >= 0; --i) {                                          \
                T s = b[i];                                                              \
                for (i64 p = i + 1; p < nt; ++p) s = FMA(-A[i + p * lda], b[p], s);      \
                b[i] = unit ? s : s / A[i + i * lda];                                    \
            }                                                                            \
        }                                                                                \
    }                                                                                    \
}                                                                                        \
                                                                                         \
/* Recursive left TRSM B <- op(A)^-1 B, src/blas/level3.jl:338-355                    \
 * (_trsm_blocks_left!): halve the triangle, solve one half, GEMM-update the other,    \
 * solve it; leaves of <= 8 (trsm! default blocksize, level3.jl:524). Only the         \
 * non-transposed form is needed here (transposed solves build op(A) explicitly). */   \
static void P##_trsm_rec(i64 nt, i64 nrhs, const T *A, i64 lda, T *B, i64 ldb,         \
                         int upper, int unit) {                                          \
    if (nt <= 8) { P##_trsm_leaf(nt, nrhs, A, lda, B, ldb, upper, unit); return; }      \
    i64 h = nt / 2;                                                                      \
    if (!upper) {                                                                        \
        P##_trsm_rec(h, nrhs, A, lda, B, ldb, upper, unit);                              \
        P##_gemm_minus(nt - h, nrhs, h, A + h, lda, B, ldb, B + h, ldb);                 \
        P##_trsm_rec(nt - h, nrhs, A + h + h * lda, lda, B + h, ldb, upper, unit);       \
    } else {                                                                             \
        P##_trsm_rec(nt - h, nrhs, A + h + h * lda, lda, B + h, ldb, upper, unit);       \
        P##_gemm_minus(h, nrhs, nt - h, A + h * lda, lda, B + h, ldb, B, ldb);           \
        P##_trsm_rec(h, nrhs, A, lda, B, ldb, upper, unit);                              \
    }                                                                                    \
}                                                                                        \
                                                                                         \
/* RHS columns split across threads, src/blas/level3.jl:383-406. */                    \
static void P##_trsm(i64 nt, i64 nrhs, const T *A, i64 lda, T *B, i64 ldb, int upper,  \
                     int unit) {                                                         \
    if (nt <= 0 || nrhs <= 0) return;                                                    \
    if (nrhs >= 64 && (double)nt * nt * nrhs > 4e6) {                                    \
        i64 chunk = 32;                                                                  \
        _Pragma("omp parallel for schedule(dynamic)")                                    \
        for (i64 j0 = 0; j0 < nrhs; j0 += chunk) {                                       \
            i64 w = nrhs - j0 < chunk ? nrhs - j0 : chunk;                               \
            P##_trsm_rec(nt, w, A, lda, B + j0 * ldb, ldb, upper, unit);                 \
        }                                                                                \
    } else {                                                                             \
        P##_trsm_rec(nt, nrhs, A, lda, B, ldb, upper, unit);                             \
    }                                                                                    \
}                                                                                        \
                                                                                         \
/* laswp: src/lapack/factorizations.jl:82-88 (_lu_swap!).  Interchanges j1..j2        \
 * (0-based pivot positions, inclusive), column by column, on columns [c0,c1).         \
 * piv holds 1-based row indices relative to row 0 of A plus `off` (global -> local). */\
static void P##_swap(T *A, i64 lda, const i64 *piv, i64 off, i64 j1, i64 j2, i64 c0,    \
                     i64 c1) {                                                           \
    _Pragma("omp parallel for schedule(static) if((c1 - c0) * (j2 - j1 + 1) > 65536)")   \
    for (i64 col = c0; col < c1; ++col) {                                                \
        T *a = A + col * lda;                                                            \
        for (i64 j = j1; j <= j2; ++j) {                                                 \
            i64 p = piv[off + j] - 1 - off;                                              \
            if (p != j) { T t = a[j]; a[j] = a[p]; a[p] = t; }                           \
        }                                                                                \
    }                                                                                    \
}                                                                                        \
                                                                                         \
/* Pivot search: src/lapack/factorizations.jl:92-107 (_lu_pivot), real branch:        \
 * first row of the largest |P[i,j]|, i >= j (strict '>'). */                          \
static i64 P##_pivot(const T *Pm, i64 ldp, i64 mp, i64 j) {                             \
    const T *c = Pm + j * ldp;                                                           \
    i64 p = j; T best = ABS(c[j]);                                                       \
    for (i64 i = j + 1; i < mp; ++i) { T v = ABS(c[i]); if (v > best) { best = v; p = i; } }\
    return p;                                                                            \
}                                                                                        \
                                                                                         \
/* Recursive panel LU (getrf2): src/lapack/factorizations.jl:114-152 (_lu_panel!).     \
 * P is mp x np with global row/column index `off` at its (0,0).  Leaves of <= 32      \
 * columns (_lu_leaf, :113) eliminate column by column.  Returns 1 when `check` and a   \
 * zero pivot was met (the reference throws SingularException there). */              \
static int P##_panel(T *Pm, i64 ldp, i64 mp, i64 np, i64 *piv, i64 off, i64 *info,     \
                     int check) {                                                        \
    if (np <= 32) {                                                                      \
        i64 q = mp < np ? mp : np;                                                       \
        for (i64 j = 0; j < q; ++j) {                                                    \
            i64 p = P##_pivot(Pm, ldp, mp, j);                                           \
            piv[off + j] = off + p + 1;                                                  \
            if (p != j)                                                                  \
                for (i64 col = 0; col < np; ++col) {                                     \
                    T t = Pm[j + col * ldp]; Pm[j + col * ldp] = Pm[p + col * ldp];      \
                    Pm[p + col * ldp] = t;                                               \
                }                                                                        \
            T d = Pm[j + j * ldp];                                                       \
            if (d == 0) {                                                                \
                if (*info == 0) *info = off + j + 1;                                     \
                if (check) return 1;                                                     \
                continue;                                                                \
            }                                                                            \
            for (i64 i = j + 1; i < mp; ++i) Pm[i + j * ldp] /= d;                       \
            _Pragma("omp parallel for schedule(static) if((mp - j) * (np - j) > 262144)")  \
            for (i64 col = j + 1; col < np; ++col) {                                     \
                T u = Pm[j + col * ldp];                                                 \
                T *pc = Pm + col * ldp; const T *pj = Pm + j * ldp;                      \
                for (i64 i = j + 1; i < mp; ++i) pc[i] = FMA(-pj[i], u, pc[i]);          \
            }                                                                            \
        }                                                                                \
        return 0;                                                                        \
    }                                                                                    \
    i64 h = np / 2;                                                                      \
    if (P##_panel(Pm, ldp, mp, h, piv, off, info, check)) return 1;                      \
    P##_swap(Pm, ldp, piv, off, 0, h - 1, h, np);                                        \
    P##_trsm(h, np - h, Pm, ldp, Pm + h * ldp, ldp, 0, 1);                               \
    if (mp > h) {                                                                        \
        P##_gemm_minus(mp - h, np - h, h, Pm + h, ldp, Pm + h * ldp, ldp,                \
                       Pm + h + h * ldp, ldp);                                           \
        if (P##_panel(Pm + h + h * ldp, ldp, mp - h, np - h, piv, off + h, info, check)) \
            return 1;                                                                    \
        i64 q = mp < np ? mp : np;                                                       \
        P##_swap(Pm, ldp, piv, off, h, q - 1, 0, h);                                     \
    }                                                                                    \
    return 0;                                                                            \
}                                                                                        \
                                                                                         \
/* Blocked right-looking getrf: src/lapack/factorizations.jl:30-77 (_lu_factor!),      \
 * sequential order (the reference's lookahead gives bit-identical factors,            \
 * test/lapack/lapack_dense.jl:32-37).  Returns 0, or 1 if `check` hit a zero pivot.   \
 * `steps` >= 0 stops after that many panels (used only to time a bounded prefix). */  \
int orc_##P##getrf_steps(i64 m, i64 n, T *A, i64 lda, i64 nb, int check, i64 *ipiv,   \
                         i64 *info, i64 steps) {                                         \
    i64 q = m < n ? m : n;                                                               \
    *info = 0;                                                                           \
    if (nb <= 0) return 2;                                                               \
    i64 done = 0;                                                                        \
    for (i64 f = 0; f < q; f += nb) {                                                    \
        if (steps >= 0 && done++ >= steps) break;                                        \
        i64 l = f + nb < q ? f + nb : q; /* exclusive */                                 \
        if (P##_panel(A + f + f * lda, lda, m - f, l - f, ipiv, f, info, check))         \
            return 1;                                                                    \
        P##_swap(A, lda, ipiv, 0, f, l - 1, 0, f);                                       \
        P##_swap(A, lda, ipiv, 0, f, l - 1, l, n);                                       \
        if (l >= n) continue;                                                            \
        P##_trsm(l - f, n - l, A + f + f * lda, lda, A + f + l * lda, lda, 0, 1);        \
        if (l >= m) continue;                                                            \
        P##_gemm_minus(m - l, n - l, l - f, A + l + f * lda, lda, A + f + l * lda, lda,  \
                       A + l + l * lda, lda);                                            \
    }                                                                                    \
    return 0;                                                                            \
}                                                                                        \
int orc_##P##getrf(i64 m, i64 n, T *A, i64 lda, i64 nb, int check, i64 *ipiv,          \
                   i64 *info) {                                                          \
    return orc_##P##getrf_steps(m, n, A, lda, nb, check, ipiv, info, -1);                \
}                                                                                        \
                                                                                         \
/* ldiv!: src/api/linalg_api.jl:168-184.  trans == 'N': laswp forward (_rowswap!,      \
 * :100-110), unit-lower solve, upper solve.  trans == 'T' (real: same as 'C'):        \
 * U^T solve, unit L^T solve, laswp in reverse.  B is n x nrhs, overwritten. */       \
int orc_##P##getrs(char trans, i64 n, i64 nrhs, const T *LU, i64 lda, const i64 *ipiv,  \
                   T *B, i64 ldb) {                                                      \
    if (n == 0 || nrhs == 0) return 0;                                                   \
    if (trans == 'N') {                                                                  \
        for (i64 c = 0; c < nrhs; ++c) {                                                 \
            T *b = B + c * ldb;                                                          \
            for (i64 j = 0; j < n; ++j) {                                                \
                i64 p = ipiv[j] - 1;                                                     \
                if (p != j) { T t = b[j]; b[j] = b[p]; b[p] = t; }                       \
            }                                                                            \
        }                                                                                \
        P##_trsm(n, nrhs, LU, lda, B, ldb, 0, 1);                                        \
        P##_trsm(n, nrhs, LU, lda, B, ldb, 1, 0);                                        \
        return 0;                                                                        \
    }                                                                                    \
    /* transposed: build U^T and L^T explicitly and reuse the lower/upper solves */     \
    T *Tt = (T *)malloc(sizeof(T) * (size_t)n * n);                                      \
    if (!Tt) return 3;                                                                   \
    for (i64 j = 0; j < n; ++j)                                                          \
        for (i64 i = 0; i < n; ++i) Tt[j + i * n] = LU[i + j * lda];                     \
    P##_trsm(n, nrhs, Tt, n, B, ldb, 0, 0);   /* U^T is lower, non-unit */               \
    P##_trsm(n, nrhs, Tt, n, B, ldb, 1, 1);   /* L^T is upper, unit */                   \
    free(Tt);                                                                            \
    for (i64 c = 0; c < nrhs; ++c) {                                                     \
        T *b = B + c * ldb;                                                              \
        for (i64 j = n - 1; j >= 0; --j) {                                               \
            i64 p = ipiv[j] - 1;                                                         \
            if (p != j) { T t = b[j]; b[j] = b[p]; b[p] = t; }                           \
        }                                                                                \
    }                                                                                    \
    return 0;                                                                            \
}

DEFINE_LU(double, d, fma, fabs)
DEFINE_LU(float, s, fmaf, fabsf)

/* gemm!(C, A, B, -1, 1) alone (the trailing update), column-major. */
void orc_dgemm_update(i64 m, i64 n, i64 k, double *C, i64 ldc, const double *A, i64 lda,
                      const double *B, i64 ldb) {
    d_gemm_minus(m, n, k, A, lda, B, ldb, C, ldc);
}
void orc_sgemm_update(i64 m, i64 n, i64 k, float *C, i64 ldc, const float *A, i64 lda,
                      const float *B, i64 ldb) {
    s_gemm_minus(m, n, k, A, lda, B, ldb, C, ldc);
}

/* ------------------------------------------------------------------------ */
/* Mixed precision pieces (FP64 only)                                        */
/* ------------------------------------------------------------------------ */

/* _refinement_residual!: src/lapack/expert_refinement.jl:67-81.  R = B - A*X in
 * FP64 (the residual work type of Float64) and the componentwise backward error
 * max_i |r_i| / (|A||x| + |b|)_i with the reference's Inf/zero conventions. */
double orc_refinement_residual(i64 n, i64 nrhs, const double *A, i64 lda, const double *X,
                               i64 ldx, const double *B, i64 ldb, double *R, i64 ldr) {
    double err = 0.0;
    for (i64 j = 0; j < nrhs; ++j) {
        double local = 0.0;
#pragma omp parallel for reduction(max : local) schedule(static) if (n >= 512)
        for (i64 i = 0; i < n; ++i) {
            double value = B[i + j * ldb], den = fabs(B[i + j * ldb]);
            for (i64 k = 0; k < n; ++k) {
                double a = A[i + k * lda], x = X[k + j * ldx];
                value -= a * x;
                den += fabs(a) * fabs(x);
            }
            R[i + j * ldr] = value;
            double rel;
            if (!isfinite(den)) rel = INFINITY;
            else if (den == 0.0) rel = (value == 0.0) ? 0.0 : INFINITY;
            else rel = fabs(value) / den;
            if (rel > local || isnan(rel)) local = rel;
        }
        if (local > err || isnan(local)) err = local;
    }
    return err;
}

/* Normwise backward error ||B - A X||_inf / (||A||_inf ||X||_inf + ||B||_inf), per RHS
 * maximum: the error measure the benchmark's 1e-14 target is stated in. */
double orc_normwise_backward_error(i64 n, i64 nrhs, const double *A, i64 lda, const double *X,
                                   i64 ldx, const double *B, i64 ldb) {
    double anorm = 0.0;
    for (i64 i = 0; i < n; ++i) {
        double s = 0.0;
        for (i64 k = 0; k < n; ++k) s += fabs(A[i + k * lda]);
        if (s > anorm) anorm = s;
    }
    double worst = 0.0;
    for (i64 j = 0; j < nrhs; ++j) {
        double rmax = 0.0, xmax = 0.0, bmax = 0.0;
#pragma omp parallel for reduction(max : rmax) schedule(static) if (n >= 512)
        for (i64 i = 0; i < n; ++i) {
            double v = B[i + j * ldb];
            for (i64 k = 0; k < n; ++k) v -= A[i + k * lda] * X[k + j * ldx];
            if (fabs(v) > rmax) rmax = fabs(v);
        }
        for (i64 i = 0; i < n; ++i) {
            if (fabs(X[i + j * ldx]) > xmax) xmax = fabs(X[i + j * ldx]);
            if (fabs(B[i + j * ldb]) > bmax) bmax = fabs(B[i + j * ldb]);
        }
        double den = anorm * xmax + bmax;
        double e = den > 0 ? rmax / den : (rmax == 0 ? 0.0 : INFINITY);
        if (e > worst) worst = e;
    }
    return worst;
}

/* 2^round(log2(v)) clamped to the exponent range of Float64: the radix scale of
 * equilibrate(A; radix=true), src/lapack/dense_utilities.jl:191-213.  Julia's
 * round is round-half-to-even (nearbyint under the default rounding mode). */
static double radix_scale(double v) {
    double e = nearbyint(log2(v));
    if (e < -1022) e = -1022;       /* exponent(floatmin(Float64)) */
    if (e > 1023) e = 1023;         /* exponent(floatmax(Float64)) */
    return ldexp(1.0, (int)e);
}

/* equilibrate(A; radix=true): rows first, then columns of the row-scaled matrix.
 * Writes the scaled matrix to E (ldE) and the scales to rows/cols. */
void orc_equilibrate_radix(i64 m, i64 n, const double *A, i64 lda, double *E, i64 lde,
                           double *rows, double *cols) {
    for (i64 j = 0; j < n; ++j)
        for (i64 i = 0; i < m; ++i) E[i + j * lde] = A[i + j * lda];
    for (i64 i = 0; i < m; ++i) {
        double v = 0.0;
        for (i64 j = 0; j < n; ++j) { double a = fabs(E[i + j * lde]); if (a > v) v = a; }
        rows[i] = 1.0;
        if (v > 0) {
            rows[i] = radix_scale(v);
            for (i64 j = 0; j < n; ++j) E[i + j * lde] /= rows[i];
        }
    }
    for (i64 j = 0; j < n; ++j) {
        double v = 0.0;
        for (i64 i = 0; i < m; ++i) { double a = fabs(E[i + j * lde]); if (a > v) v = a; }
        cols[j] = 1.0;
        if (v > 0) {
            cols[j] = radix_scale(v);
            for (i64 i = 0; i < m; ++i) E[i + j * lde] /= cols[j];
        }
    }
}

/* _mixed_extended_correction: src/lapack/extended_lapack.jl:114-131 (Low = Float32).
 * Row-scale the residual, scale by the power of two 2^exponent(max|.|), round to
 * Float32, solve with the Float32 factors, widen, multiply back, column-unscale.
 * Returns 0, or 4 when the scaled RHS overflows / is not finite. */
static int mixed_correction(i64 n, i64 nrhs, const float *LU, i64 ldlu, const i64 *ipiv,
                            const double *Rres, i64 ldr, const double *rows,
                            const double *cols, double *Cout, i64 ldc, float *work) {
    double mag = 0.0;
    for (i64 j = 0; j < nrhs; ++j)
        for (i64 i = 0; i < n; ++i) {
            double v = fabs(Rres[i + j * ldr] / rows[i]);
            if (v > mag || isnan(v)) mag = v;
        }
    if (mag == 0.0) {
        for (i64 j = 0; j < nrhs; ++j)
            for (i64 i = 0; i < n; ++i) Cout[i + j * ldc] = 0.0;
        return 0;
    }
    if (!isfinite(mag)) return 4;
    int ex; frexp(mag, &ex);         /* mag = f * 2^ex, f in [0.5,1) */
    double scale = ldexp(1.0, ex - 1); /* Julia exponent(): floor(log2(mag)) */
    for (i64 j = 0; j < nrhs; ++j)
        for (i64 i = 0; i < n; ++i) {
            float v = (float)((Rres[i + j * ldr] / rows[i]) / scale);
            if (!isfinite(v)) return 4;
            work[i + j * n] = v;
        }
    orc_sgetrs('N', n, nrhs, LU, ldlu, ipiv, work, n);
    for (i64 j = 0; j < nrhs; ++j)
        for (i64 i = 0; i < n; ++i)
            Cout[i + j * ldc] = ((double)work[i + j * n] * scale) / cols[i];
    return 0;
}

/* mixed_solve: src/lapack/factorizations.jl:425-427 -> _mixed_precision_impl,
 * src/lapack/extended_lapack.jl:175-226, LU family, Low = Float32, fallback on.
 * Outputs X (n x nrhs), the iteration count, the final componentwise backward
 * error, and whether the working-precision fallback factor was used.  The
 * fallback path (Float64 factor of the equilibrated matrix) is restated too.
 * Returns 0 on success, 1 singular (both factors), 4 overflow without fallback. */
/* Normwise backward error from a computed residual R (n x nrhs): max over the
 * right-hand sides of ||r||_inf / (anorm ||x||_inf + ||b||_inf). */
static double normwise_from_residual(i64 n, i64 nrhs, double anorm, const double *R, i64 ldr,
                                     const double *X, i64 ldx, const double *B, i64 ldb) {
    double worst = 0.0;
    for (i64 j = 0; j < nrhs; ++j) {
        double rmax = 0.0, xmax = 0.0, bmax = 0.0;
        for (i64 i = 0; i < n; ++i) {
            rmax = fmax(rmax, fabs(R[i + j * ldr]));
            xmax = fmax(xmax, fabs(X[i + j * ldx]));
            bmax = fmax(bmax, fabs(B[i + j * ldb]));
        }
        double den = anorm * xmax + bmax;
        double e = den > 0 ? rmax / den : (rmax == 0 ? 0.0 : INFINITY);
        if (!(e <= worst)) worst = e;
    }
    return worst;
}

static int mixed_solve_impl(i64 n, i64 nrhs, const double *A, i64 lda, const double *B, i64 ldb,
                            double *X, i64 ldx, i64 maxiter, double rtol, int stop_normwise,
                            i64 *iterations, double *berr, double *berr_nw, int *fallback);

/* mixed_solve with the choice of stop test: stop_normwise = 0 compares the
 * componentwise backward error with rtol (the reference's metric), 1 the
 * normwise one (the benchmark's 1e-14 target).  berr and berr_nw receive both
 * errors of the final iterate. */
int orc_mixed_solve_ex(i64 n, i64 nrhs, const double *A, i64 lda, const double *B, i64 ldb,
                       double *X, i64 ldx, i64 maxiter, double rtol, int stop_normwise,
                       i64 *iterations, double *berr, double *berr_nw, int *fallback) {
    return mixed_solve_impl(n, nrhs, A, lda, B, ldb, X, ldx, maxiter, rtol, stop_normwise, iterations,
                            berr, berr_nw, fallback);
}

int orc_mixed_solve(i64 n, i64 nrhs, const double *A, i64 lda, const double *B, i64 ldb,
                    double *X, i64 ldx, i64 maxiter, double rtol, i64 *iterations,
                    double *berr, int *fallback) {
    double nw = 0.0;
    return mixed_solve_impl(n, nrhs, A, lda, B, ldb, X, ldx, maxiter, rtol, 0, iterations, berr, &nw,
                            fallback);
}

static int mixed_solve_impl(i64 n, i64 nrhs, const double *A, i64 lda, const double *B, i64 ldb,
                            double *X, i64 ldx, i64 maxiter, double rtol, int stop_normwise,
                            i64 *iterations, double *berr, double *berr_nw, int *fallback) {
    double *E = (double *)malloc(sizeof(double) * (size_t)n * n);
    double *rows = (double *)malloc(sizeof(double) * (size_t)n);
    double *cols = (double *)malloc(sizeof(double) * (size_t)n);
    float *F = (float *)malloc(sizeof(float) * (size_t)n * n);
    double *Fd = NULL;
    i64 *ipiv = (i64 *)malloc(sizeof(i64) * (size_t)(n > 0 ? n : 1));
    double *R = (double *)malloc(sizeof(double) * (size_t)n * nrhs);
    double *Cc = (double *)malloc(sizeof(double) * (size_t)n * nrhs);
    float *work = (float *)malloc(sizeof(float) * (size_t)n * nrhs);
    int rc = 0; *fallback = 0;
    orc_equilibrate_radix(n, n, A, lda, E, n, rows, cols);
    i64 info = 0;
    int lowok = 1;
    for (i64 i = 0; i < n * n; ++i) { F[i] = (float)E[i]; if (!isfinite(F[i])) lowok = 0; }
    if (lowok) {
        if (orc_sgetrf(n, n, F, n, 128, 1, ipiv, &info) != 0) lowok = 0;
    }
    if (!lowok) {
        *fallback = 1;
        Fd = (double *)malloc(sizeof(double) * (size_t)n * n);
        memcpy(Fd, E, sizeof(double) * (size_t)n * n);
        if (orc_dgetrf(n, n, Fd, n, 128, 1, ipiv, &info) != 0) { rc = 1; goto done; }
    }
    /* first solve: correction of B itself (extended_lapack.jl:207-212) */
#define CORRECT(RES, LDRES, OUT, LDOUT)                                                    \
    do {                                                                                 \
        if (!*fallback) {                                                                \
            if (mixed_correction(n, nrhs, F, n, ipiv, RES, LDRES, rows, cols, OUT, LDOUT, \
                                 work)) { rc = 4; goto done; }                           \
        } else {                                                                         \
            for (i64 j = 0; j < nrhs; ++j)                                               \
                for (i64 i = 0; i < n; ++i) OUT[i + j * LDOUT] = RES[i + j * LDRES] / rows[i]; \
            orc_dgetrs('N', n, nrhs, Fd, n, ipiv, OUT, LDOUT);                           \
            for (i64 j = 0; j < nrhs; ++j)                                               \
                for (i64 i = 0; i < n; ++i) OUT[i + j * LDOUT] /= cols[i];               \
        }                                                                                \
    } while (0)
    CORRECT(B, ldb, X, ldx);
    double anorm = 0.0;
    if (stop_normwise) {
        double *rs = (double *)calloc((size_t)n, sizeof(double));
        for (i64 k = 0; k < n; ++k)
            for (i64 i = 0; i < n; ++i) rs[i] += fabs(A[i + k * lda]);
        for (i64 i = 0; i < n; ++i) anorm = fmax(anorm, rs[i]);
        free(rs);
    }
    double err = INFINITY, cw = INFINITY, nw = INFINITY; i64 it = 0;
    for (i64 iter = 0; iter <= maxiter; ++iter) {
        cw = orc_refinement_residual(n, nrhs, A, lda, X, ldx, B, ldb, R, n);
        nw = stop_normwise ? normwise_from_residual(n, nrhs, anorm, R, n, X, ldx, B, ldb) : NAN;
        err = stop_normwise ? nw : cw;
        it = iter;
        if (err <= rtol || iter == maxiter || !isfinite(err)) break;
        CORRECT(R, n, Cc, n);
        for (i64 j = 0; j < nrhs; ++j)
            for (i64 i = 0; i < n; ++i) X[i + j * ldx] += Cc[i + j * n];
    }
#undef CORRECT
    *iterations = it; *berr = cw; *berr_nw = nw;
done:
    free(E); free(rows); free(cols); free(F); free(Fd); free(ipiv); free(R); free(Cc);
    free(work);
    return rc;
}

/* Adjoint of x = A \ b for the loss with upstream gradient xbar:
 * lambda = A^-T xbar (transposed solve with the stored factors, the primitive
 * behind ldiv!(transpose(F), B), src/api/linalg_api.jl:176-184 and
 * solve_transposed, src/lapack/expert_refinement.jl:2-23), bbar = lambda,
 * Abar = -lambda x^T (column-major, ldabar). */
int orc_lu_adjoint(i64 n, const double *LU, i64 lda, const i64 *ipiv, const double *x,
                   const double *xbar, double *bbar, double *Abar, i64 ldabar) {
    for (i64 i = 0; i < n; ++i) bbar[i] = xbar[i];
    int rc = orc_dgetrs('T', n, 1, LU, lda, ipiv, bbar, n);
    if (rc) return rc;
    for (i64 j = 0; j < n; ++j)
        for (i64 i = 0; i < n; ++i) Abar[i + j * ldabar] = -bbar[i] * x[j];
    return 0;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_num_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

/* ------------------------------------------------------------------------ */
/* Expert solves and the condition estimate (FP64)                           */
/* ------------------------------------------------------------------------ */

/* inverse_norm_estimate(F, T, n; maxiter): src/lapack/expert_refinement.jl:45-60.
 * Hager-Higham estimate of ||A^-1||_1 from solves with the factors and with
 * their transpose (_adjoint_solve -> solve_transposed for an LU, :2-23).
 * Sums run in index order (the reference's sum(abs, y) is a pairwise
 * reduction; the estimate agrees to rounding). */
double orc_inverse_norm_estimate(i64 n, const double *LU, i64 lda, const i64 *ipiv, i64 maxiter) {
    if (n <= 0) return 0.0;
    double *x = (double *)malloc(sizeof(double) * (size_t)n);
    double *y = (double *)malloc(sizeof(double) * (size_t)n);
    double *z = (double *)malloc(sizeof(double) * (size_t)n);
    for (i64 i = 0; i < n; ++i) x[i] = 1.0 / (double)n;
    double est = 0.0;
    i64 prev = -1;
    for (i64 it = 0; it < maxiter; ++it) {
        memcpy(y, x, sizeof(double) * (size_t)n);
        orc_dgetrs('N', n, 1, LU, lda, ipiv, y, n);
        double next = 0.0;
        for (i64 i = 0; i < n; ++i) next += fabs(y[i]);
        if (next > est) est = next;
        for (i64 i = 0; i < n; ++i) z[i] = (y[i] == 0.0) ? 1.0 : y[i] / fabs(y[i]);
        orc_dgetrs('T', n, 1, LU, lda, ipiv, z, n);
        i64 idx = 0;
        for (i64 i = 1; i < n; ++i)
            if (fabs(z[i]) > fabs(z[idx])) idx = i;  /* argmax: the first maximum */
        double dot = 0.0;
        for (i64 i = 0; i < n; ++i) dot += z[i] * x[i];
        if (fabs(z[idx]) <= dot) break;
        if (idx == prev) break;
        for (i64 i = 0; i < n; ++i) x[i] = 0.0;
        x[idx] = 1.0;
        prev = idx;
    }
    const double den = (double)(n > 1 ? n - 1 : 1);
    for (i64 i = 0; i < n; ++i) x[i] = ((i % 2 == 0) ? 1.0 : -1.0) * (1.0 + (double)i / den);
    orc_dgetrs('N', n, 1, LU, lda, ipiv, x, n);
    double alt = 0.0;
    for (i64 i = 0; i < n; ++i) alt += fabs(x[i]);
    alt = 2.0 * alt / (3.0 * (double)n);
    free(x); free(y); free(z);
    return est > alt ? est : alt;
}

static double one_norm(i64 m, i64 n, const double *A, i64 lda) {
    double best = 0.0;
    for (i64 j = 0; j < n; ++j) {
        double s = 0.0;
        for (i64 i = 0; i < m; ++i) s += fabs(A[i + j * lda]);
        if (s > best) best = s;
    }
    return best;
}

/* refine_solve(A, F, b; maxiter, rtol): src/lapack/expert_refinement.jl:89-104.
 * out[0..5] = backward_error, residual_norm, rcond_estimate,
 * forward_error_estimate, inverse_norm, iterations. */
int orc_refine_solve(i64 n, i64 nrhs, const double *A, i64 lda, const double *LU, i64 ldlu, const i64 *ipiv,
                     const double *B, i64 ldb, double *X, i64 ldx, i64 maxiter, double rtol, double *out) {
    double *R = (double *)malloc(sizeof(double) * (size_t)n * nrhs);
    for (i64 j = 0; j < nrhs; ++j)
        for (i64 i = 0; i < n; ++i) X[i + j * ldx] = B[i + j * ldb];
    orc_dgetrs('N', n, nrhs, LU, ldlu, ipiv, X, ldx);
    double err = INFINITY;
    i64 it = 0;
    for (i64 iter = 0; iter <= maxiter; ++iter) {
        err = orc_refinement_residual(n, nrhs, A, lda, X, ldx, B, ldb, R, n);
        it = iter;
        if (err <= rtol || iter == maxiter) break;
        orc_dgetrs('N', n, nrhs, LU, ldlu, ipiv, R, n);  /* correction = solve(F, residual) */
        for (i64 j = 0; j < nrhs; ++j)
            for (i64 i = 0; i < n; ++i) X[i + j * ldx] += R[i + j * n];
        /* the next residual overwrites R */
    }
    const double inv_norm = orc_inverse_norm_estimate(n, LU, ldlu, ipiv, 8);
    const double anorm = one_norm(n, n, A, lda);
    const double cond = anorm * inv_norm;
    const double rcond = (cond == 0.0) ? 1.0 : fmin(1.0, 1.0 / cond);
    double r2 = 0.0;
    for (i64 e = 0; e < n * nrhs; ++e) r2 += R[e] * R[e];
    const double rnorm = sqrt(r2);
    const double xnorm = one_norm(n, nrhs, X, ldx);
    const double delta = (xnorm == 0.0) ? (rnorm == 0.0 ? 0.0 : INFINITY)
                                        : inv_norm * one_norm(n, nrhs, R, n) / xnorm;
    out[0] = err;
    out[1] = rnorm;
    out[2] = rcond;
    out[3] = delta < 1.0 ? delta / (1.0 - delta) : INFINITY;
    out[4] = inv_norm;
    out[5] = (double)it;
    free(R);
    return 0;
}

/* expert_solve(A, b; maxiter, rtol, equilibrate): src/lapack/advanced_factorizations.jl:
 * 591-645.  Row scales (max |a| of each row; a zero row is singular), then
 * column scales of the row-scaled matrix, partial-pivoted LU of the scaled
 * matrix, scaled solves and componentwise refinement in the working type.
 * F (n x n, leading dimension n) and ipiv receive the factorization.
 * out[0..1] = backward_error, iterations.  Returns 0, or 1 with *info set
 * (a zero row, or a zero pivot). */
int orc_expert_solve(i64 n, i64 nrhs, const double *A, i64 lda, const double *B, i64 ldb, double *X, i64 ldx,
                     i64 maxiter, double rtol, int equilibrate, double *rows, double *cols, double *F,
                     i64 *ipiv, i64 *info, double *out) {
    *info = 0;
    for (i64 j = 0; j < n; ++j)
        for (i64 i = 0; i < n; ++i) F[i + j * n] = A[i + j * lda];
    for (i64 i = 0; i < n; ++i) rows[i] = cols[i] = 1.0;
    if (equilibrate) {
        for (i64 i = 0; i < n; ++i) {
            double v = 0.0;
            for (i64 j = 0; j < n; ++j) v = fmax(v, fabs(F[i + j * n]));
            if (v == 0.0) { *info = i + 1; return 1; }
            rows[i] = v;
            for (i64 j = 0; j < n; ++j) F[i + j * n] /= v;
        }
        for (i64 j = 0; j < n; ++j) {
            double v = 0.0;
            for (i64 i = 0; i < n; ++i) v = fmax(v, fabs(F[i + j * n]));
            cols[j] = (v == 0.0) ? 1.0 : v;
            for (i64 i = 0; i < n; ++i) F[i + j * n] /= cols[j];
        }
    }
    if (orc_dgetrf(n, n, F, n, 128, 1, ipiv, info) != 0) return 1;
    double *R = (double *)malloc(sizeof(double) * (size_t)n * nrhs);
    for (i64 j = 0; j < nrhs; ++j)
        for (i64 i = 0; i < n; ++i) X[i + j * ldx] = B[i + j * ldb] / rows[i];
    orc_dgetrs('N', n, nrhs, F, n, ipiv, X, ldx);
    for (i64 j = 0; j < nrhs; ++j)
        for (i64 i = 0; i < n; ++i) X[i + j * ldx] /= cols[i];
    double err = INFINITY;
    i64 it = 0;
    for (i64 iter = 0; iter <= maxiter; ++iter) {
        err = 0.0;
        for (i64 j = 0; j < nrhs; ++j) {
            double local = 0.0;
#pragma omp parallel for reduction(max : local) schedule(static) if (n >= 512)
            for (i64 i = 0; i < n; ++i) {
                double s = 0.0, den = fabs(B[i + j * ldb]);
                for (i64 k = 0; k < n; ++k) {
                    s += A[i + k * lda] * X[k + j * ldx];
                    den += fabs(A[i + k * lda]) * fabs(X[k + j * ldx]);
                }
                const double r = B[i + j * ldb] - s;
                R[i + j * n] = r;
                double e;
                if (!isfinite(den)) e = INFINITY;
                else if (den == 0.0) e = (r == 0.0) ? 0.0 : INFINITY;
                else e = fabs(r) / den;
                if (e > local || isnan(e)) local = e;
            }
            if (local > err || isnan(local)) err = local;
        }
        it = iter;
        if (err <= rtol) break;
        if (iter == maxiter) break;
        for (i64 j = 0; j < nrhs; ++j)
            for (i64 i = 0; i < n; ++i) R[i + j * n] /= rows[i];
        orc_dgetrs('N', n, nrhs, F, n, ipiv, R, n);
        for (i64 j = 0; j < nrhs; ++j)
            for (i64 i = 0; i < n; ++i) X[i + j * ldx] += R[i + j * n] / cols[i];
    }
    out[0] = err;
    out[1] = (double)it;
    free(R);
    return 0;
}

/* native_inverse(A) (src/lapack/dense_utilities.jl:14-32) for the engine's
 * factors: inv(A) = U^-1 L^-1 P.  Restated as the solve with the identity
 * (the columns of the inverse are A^-1 e_j), which is what LinearAlgebra's
 * inv(F) does for an OxiBLAS factorization (src/api/linalg_api.jl:1143-1144). */
int orc_inverse(i64 n, const double *LU, i64 lda, const i64 *ipiv, double *X, i64 ldx) {
    for (i64 j = 0; j < n; ++j)
        for (i64 i = 0; i < n; ++i) X[i + j * ldx] = (i == j) ? 1.0 : 0.0;
    return orc_dgetrs('N', n, n, LU, lda, ipiv, X, ldx);
}

/* ------------------------------------------------------------------------ */
/* Cholesky (FP64)                                                           */
/* ------------------------------------------------------------------------ */

/* _cholesky_recursive!: src/lapack/factorizations.jl:263-291 (LAPACK potrf2).
 * L (n x n, column-major, lower triangle) in place; leaves of <= `leaf`
 * columns right-looking (d = sqrt(l_cc), column scaled, l_ij = fma(-l_ic, l_jc,
 * l_ij) for j > c, i >= j); above, L21 = A21 L11^-T (right solve), A22 -=
 * L21 L21^T on the lower triangle (one fma chain per element from zero, then
 * the subtraction), then L22.  Returns 0 or the global 1-based column of the
 * first pivot that is not finite and positive. */
static i64 chol_rec(double *L, i64 ld, i64 n, i64 offset, i64 leaf) {
    if (n <= leaf) {
        for (i64 c = 0; c < n; ++c) {
            double d = L[c + c * ld];
            if (!(isfinite(d) && d > 0)) return offset + c + 1;
            d = sqrt(d);
            L[c + c * ld] = d;
            for (i64 i = c + 1; i < n; ++i) L[i + c * ld] /= d;
            for (i64 j = c + 1; j < n; ++j) {
                const double cj = L[j + c * ld];
                for (i64 i = j; i < n; ++i) L[i + j * ld] = fma(-L[i + c * ld], cj, L[i + j * ld]);
            }
        }
        return 0;
    }
    const i64 h = n / 2;
    i64 info = chol_rec(L, ld, h, offset, leaf);
    if (info) return info;
    /* L21 (n-h x h) <- L21 L11^-T: row r of L21 solves x L11^T = a, i.e.
     * x_j = (a_j - sum_{p<j} x_p l_jp) / l_jj, j ascending */
    double *L21 = L + h;
#pragma omp parallel for schedule(static) if ((n - h) * h > 65536)
    for (i64 r = 0; r < n - h; ++r) {
        for (i64 j = 0; j < h; ++j) {
            double s = L21[r + j * ld];
            for (i64 p = 0; p < j; ++p) s = fma(-L21[r + p * ld], L[j + p * ld], s);
            L21[r + j * ld] = s / L[j + j * ld];
        }
    }
    /* A22 -= L21 L21^T, lower triangle */
    double *A22 = L + h + h * ld;
    const i64 m = n - h;
#pragma omp parallel for schedule(dynamic, 8) if (m * m * h > 2000000)
    for (i64 j = 0; j < m; ++j)
        for (i64 i = j; i < m; ++i) {
            double s = 0.0;
            for (i64 p = 0; p < h; ++p) s = fma(L21[i + p * ld], L21[j + p * ld], s);
            A22[i + j * ld] -= s;
        }
    return chol_rec(A22, ld, m, offset + h, leaf);
}

/* cholesky_factor(A): L from the lower triangle of A (leaf 64 for real types,
 * :212-216), strict upper triangle zeroed when it succeeds.  Returns info. */
i64 orc_dpotrf(i64 n, double *A, i64 lda) {
    const i64 info = chol_rec(A, lda, n, 0, 64);
    if (info == 0)
        for (i64 j = 0; j < n; ++j)
            for (i64 i = 0; i < j; ++i) A[i + j * lda] = 0.0;
    return info;
}

/* solve(F::CholeskyFactor, b) (:293-305): L y = b, then L^T x = y. */
void orc_dpotrs(i64 n, i64 nrhs, const double *L, i64 ldl, double *B, i64 ldb) {
    for (i64 c = 0; c < nrhs; ++c) {
        double *b = B + c * ldb;
        for (i64 i = 0; i < n; ++i) {
            double s = b[i];
            for (i64 p = 0; p < i; ++p) s = fma(-L[i + p * ldl], b[p], s);
            b[i] = s / L[i + i * ldl];
        }
        for (i64 i = n - 1; i >= 0; --i) {
            double s = b[i];
            for (i64 p = i + 1; p < n; ++p) s = fma(-L[p + i * ldl], b[p], s);
            b[i] = s / L[i + i * ldl];
        }
    }
}

/* The same recursion in Float32 (cholesky_factor of the low-precision matrix
 * inside mixed_solve, src/lapack/extended_lapack.jl:157-158). */
static i64 chol_rec_f(float *L, i64 ld, i64 n, i64 offset, i64 leaf) {
    if (n <= leaf) {
        for (i64 c = 0; c < n; ++c) {
            float d = L[c + c * ld];
            if (!(isfinite(d) && d > 0)) return offset + c + 1;
            d = sqrtf(d);
            L[c + c * ld] = d;
            for (i64 i = c + 1; i < n; ++i) L[i + c * ld] /= d;
            for (i64 j = c + 1; j < n; ++j) {
                const float cj = L[j + c * ld];
                for (i64 i = j; i < n; ++i) L[i + j * ld] = fmaf(-L[i + c * ld], cj, L[i + j * ld]);
            }
        }
        return 0;
    }
    const i64 h = n / 2;
    i64 info = chol_rec_f(L, ld, h, offset, leaf);
    if (info) return info;
    float *L21 = L + h;
#pragma omp parallel for schedule(static) if ((n - h) * h > 65536)
    for (i64 r = 0; r < n - h; ++r) {
        for (i64 j = 0; j < h; ++j) {
            float s = L21[r + j * ld];
            for (i64 p = 0; p < j; ++p) s = fmaf(-L21[r + p * ld], L[j + p * ld], s);
            L21[r + j * ld] = s / L[j + j * ld];
        }
    }
    float *A22 = L + h + h * ld;
    const i64 m = n - h;
#pragma omp parallel for schedule(dynamic, 8) if (m * m * h > 2000000)
    for (i64 j = 0; j < m; ++j)
        for (i64 i = j; i < m; ++i) {
            float s = 0.0f;
            for (i64 p = 0; p < h; ++p) s = fmaf(L21[i + p * ld], L21[j + p * ld], s);
            A22[i + j * ld] -= s;
        }
    return chol_rec_f(A22, ld, m, offset + h, leaf);
}

static void spotrs_lower(i64 n, i64 nrhs, const float *L, i64 ldl, float *B, i64 ldb) {
    for (i64 c = 0; c < nrhs; ++c) {
        float *b = B + c * ldb;
        for (i64 i = 0; i < n; ++i) {
            float s = b[i];
            for (i64 p = 0; p < i; ++p) s = fmaf(-L[i + p * ldl], b[p], s);
            b[i] = s / L[i + i * ldl];
        }
        for (i64 i = n - 1; i >= 0; --i) {
            float s = b[i];
            for (i64 p = i + 1; p < n; ++p) s = fmaf(-L[p + i * ldl], b[p], s);
            b[i] = s / L[i + i * ldl];
        }
    }
}

/* mixed_solve(A, b; factorization=:cholesky): _mixed_precision_impl,
 * src/lapack/extended_lapack.jl:175-226, Cholesky family, Low = Float32.
 * One global positive scale (max |a_ij|, one if zero) keeps the matrix
 * symmetric: E = A / scale, rows = scale, columns = 1 (:187-193); the Float32
 * Cholesky of E, or on PosDefException / an overflowing conversion the Float64
 * one (:196-202); the corrections of _mixed_extended_correction (:114-131);
 * the componentwise (or normwise) stop.  Returns 0, 1 (not positive definite
 * in working precision too; *fallback = 1), 4 overflow. */
int orc_mixed_solve_chol(i64 n, i64 nrhs, const double *A, i64 lda, const double *B, i64 ldb,
                         double *X, i64 ldx, i64 maxiter, double rtol, int stop_normwise,
                         i64 *iterations, double *berr, double *berr_nw, int *fallback, i64 *info_out) {
    double scale = 0.0;
    for (i64 j = 0; j < n; ++j)
        for (i64 i = 0; i < n; ++i) scale = fmax(scale, fabs(A[i + j * lda]));
    if (scale == 0.0) scale = 1.0;
    double *E = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n * n : 1));
    float *F = (float *)malloc(sizeof(float) * (size_t)(n > 0 ? n * n : 1));
    double *R = (double *)malloc(sizeof(double) * (size_t)(n * nrhs > 0 ? n * nrhs : 1));
    double *Cc = (double *)malloc(sizeof(double) * (size_t)(n * nrhs > 0 ? n * nrhs : 1));
    float *work = (float *)malloc(sizeof(float) * (size_t)(n * nrhs > 0 ? n * nrhs : 1));
    int rc = 0, lowok = 1;
    *fallback = 0;
    *info_out = 0;
    for (i64 j = 0; j < n; ++j)
        for (i64 i = 0; i < n; ++i) {
            E[i + j * n] = A[i + j * lda] / scale;
            F[i + j * n] = (float)E[i + j * n];
            if (!isfinite(F[i + j * n])) lowok = 0;
        }
    i64 info = lowok ? chol_rec_f(F, n, n, 0, 64) : -1;
    *info_out = info > 0 ? info : 0;
    if (info != 0) {
        *fallback = 1;
        info = chol_rec(E, n, n, 0, 64);
        if (info != 0) { *info_out = info; rc = 1; goto done; }
    }
#define CCORRECT(RES, LDRES, OUT, LDOUT)                                                   \
    do {                                                                                 \
        double mag = 0.0;                                                                \
        for (i64 j = 0; j < nrhs; ++j)                                                   \
            for (i64 i = 0; i < n; ++i) {                                                \
                double v = fabs(RES[i + j * LDRES] / scale);                             \
                if (v > mag || isnan(v)) mag = v;                                        \
            }                                                                            \
        if (mag == 0.0) {                                                                \
            for (i64 j = 0; j < nrhs; ++j)                                               \
                for (i64 i = 0; i < n; ++i) OUT[i + j * LDOUT] = 0.0;                    \
            break;                                                                       \
        }                                                                                \
        if (!isfinite(mag)) { rc = 4; goto done; }                                       \
        int ex; frexp(mag, &ex);                                                         \
        const double p2 = ldexp(1.0, ex - 1);                                            \
        if (!*fallback) {                                                                \
            for (i64 j = 0; j < nrhs; ++j)                                               \
                for (i64 i = 0; i < n; ++i) {                                            \
                    float v = (float)((RES[i + j * LDRES] / scale) / p2);                \
                    if (!isfinite(v)) { rc = 4; goto done; }                             \
                    work[i + j * n] = v;                                                 \
                }                                                                        \
            spotrs_lower(n, nrhs, F, n, work, n);                                        \
            for (i64 j = 0; j < nrhs; ++j)                                               \
                for (i64 i = 0; i < n; ++i) OUT[i + j * LDOUT] = (double)work[i + j * n] * p2; \
        } else {                                                                         \
            for (i64 j = 0; j < nrhs; ++j)                                               \
                for (i64 i = 0; i < n; ++i) OUT[i + j * LDOUT] = (RES[i + j * LDRES] / scale) / p2; \
            orc_dpotrs(n, nrhs, E, n, OUT, LDOUT);                                       \
            for (i64 j = 0; j < nrhs; ++j)                                               \
                for (i64 i = 0; i < n; ++i) OUT[i + j * LDOUT] *= p2;                    \
        }                                                                                \
    } while (0)
    CCORRECT(B, ldb, X, ldx);
    double anorm = 0.0;
    if (stop_normwise) {
        for (i64 i = 0; i < n; ++i) {
            double rsum = 0.0;
            for (i64 k = 0; k < n; ++k) rsum += fabs(A[i + k * lda]);
            anorm = fmax(anorm, rsum);
        }
    }
    double err = INFINITY, cw = INFINITY, nw = INFINITY;
    i64 it = 0;
    for (i64 iter = 0; iter <= maxiter; ++iter) {
        cw = orc_refinement_residual(n, nrhs, A, lda, X, ldx, B, ldb, R, n);
        nw = stop_normwise ? normwise_from_residual(n, nrhs, anorm, R, n, X, ldx, B, ldb) : NAN;
        err = stop_normwise ? nw : cw;
        it = iter;
        if (err <= rtol || iter == maxiter || !isfinite(err)) break;
        CCORRECT(R, n, Cc, n);
        for (i64 j = 0; j < nrhs; ++j)
            for (i64 i = 0; i < n; ++i) X[i + j * ldx] += Cc[i + j * n];
    }
#undef CCORRECT
    *iterations = it;
    *berr = cw;
    *berr_nw = nw;
done:
    free(E); free(F); free(R); free(Cc); free(work);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Complex LU (ComplexF64)                                                   */
/* ------------------------------------------------------------------------ */
#include <complex.h>
typedef double _Complex zc_t;

/* muladd(a, b, c) on complex numbers: the product, then the sum */
static inline zc_t zmuladd(zc_t a, zc_t b, zc_t c) {
    const double ar = creal(a), ai = cimag(a), br = creal(b), bi = cimag(b);
    return CMPLX(ar * br - ai * bi + creal(c), ar * bi + ai * br + cimag(c));
}
static inline double zabs2(zc_t a) { return creal(a) * creal(a) + cimag(a) * cimag(a); }
/* a / b as Julia's complex division (Smith-style scaling is not restated: the
 * test matrices keep |b| moderate) */
static inline zc_t zdiv(zc_t a, zc_t b) { return a / b; }

/* _lu_pivot, complex branch (src/lapack/factorizations.jl:92-107): abs2
 * compared with strict '>', the first row wins a tie; if the largest square
 * is not finite, the scan is redone with abs. */
static i64 z_pivot(const zc_t *c, i64 mp, i64 j) {
    i64 p = j;
    double best = zabs2(c[j]);
    for (i64 i = j + 1; i < mp; ++i) {
        const double v = zabs2(c[i]);
        if (v > best) { best = v; p = i; }
    }
    if (isfinite(best)) return p;
    p = j;
    best = cabs(c[j]);
    for (i64 i = j + 1; i < mp; ++i) {
        const double v = cabs(c[i]);
        if (v > best) { best = v; p = i; }
    }
    return p;
}

static void z_swap(zc_t *A, i64 lda, const i64 *piv, i64 off, i64 j1, i64 j2, i64 c0, i64 c1) {
    for (i64 col = c0; col < c1; ++col) {
        zc_t *a = A + col * lda;
        for (i64 j = j1; j <= j2; ++j) {
            const i64 p = piv[off + j] - 1 - off;
            if (p != j) { zc_t t = a[j]; a[j] = a[p]; a[p] = t; }
        }
    }
}

/* C - A B, one dot product per element in k order from zero, then the
 * subtraction (the reference GEMM's form) */
static void z_gemm_minus(i64 m, i64 n, i64 k, const zc_t *A, i64 lda, const zc_t *B, i64 ldb, zc_t *C,
                         i64 ldc) {
    if (m <= 0 || n <= 0 || k <= 0) return;
#pragma omp parallel for schedule(static) if ((double)m * n * k > 2e6)
    for (i64 j = 0; j < n; ++j)
        for (i64 i = 0; i < m; ++i) {
            zc_t s = 0;
            for (i64 p = 0; p < k; ++p) s = zmuladd(A[i + p * lda], B[p + j * ldb], s);
            C[i + j * ldc] -= s;
        }
}

/* unit lower (upper = 0) or non-unit upper (upper = 1) left solve by rows,
 * s = b; s = muladd(-A[i,p], b[p], s) (_trsm_leaf_generic!); conj applies the
 * conjugate transpose of A (for the 'C' solves) */
static void z_trsm(i64 nt, i64 nrhs, const zc_t *A, i64 lda, zc_t *B, i64 ldb, int upper, int unit,
                   int transposed, int conjugate) {
    for (i64 j = 0; j < nrhs; ++j) {
        zc_t *b = B + j * ldb;
        if (!upper) {
            for (i64 i = 0; i < nt; ++i) {
                zc_t s = b[i];
                for (i64 p = 0; p < i; ++p) {
                    zc_t a = transposed ? A[p + i * lda] : A[i + p * lda];
                    if (conjugate) a = conj(a);
                    s = zmuladd(-a, b[p], s);
                }
                if (!unit) { zc_t d = A[i + i * lda]; if (conjugate) d = conj(d); s = zdiv(s, d); }
                b[i] = s;
            }
        } else {
            for (i64 i = nt - 1; i >= 0; --i) {
                zc_t s = b[i];
                for (i64 p = i + 1; p < nt; ++p) {
                    zc_t a = transposed ? A[p + i * lda] : A[i + p * lda];
                    if (conjugate) a = conj(a);
                    s = zmuladd(-a, b[p], s);
                }
                if (!unit) { zc_t d = A[i + i * lda]; if (conjugate) d = conj(d); s = zdiv(s, d); }
                b[i] = s;
            }
        }
    }
}

/* _lu_panel! with the complex leaf of 16 columns (:113) */
static int z_panel(zc_t *Pm, i64 ldp, i64 mp, i64 np, i64 *piv, i64 off, i64 *info, int check) {
    if (np <= 16) {
        const i64 q = mp < np ? mp : np;
        for (i64 j = 0; j < q; ++j) {
            const i64 p = z_pivot(Pm + j * ldp, mp, j);
            piv[off + j] = off + p + 1;
            if (p != j)
                for (i64 col = 0; col < np; ++col) {
                    zc_t t = Pm[j + col * ldp]; Pm[j + col * ldp] = Pm[p + col * ldp]; Pm[p + col * ldp] = t;
                }
            const zc_t d = Pm[j + j * ldp];
            if (d == 0) {
                if (*info == 0) *info = off + j + 1;
                if (check) return 1;
                continue;
            }
            for (i64 i = j + 1; i < mp; ++i) Pm[i + j * ldp] = zdiv(Pm[i + j * ldp], d);
            for (i64 col = j + 1; col < np; ++col) {
                const zc_t u = Pm[j + col * ldp];
                for (i64 i = j + 1; i < mp; ++i) Pm[i + col * ldp] = zmuladd(-Pm[i + j * ldp], u, Pm[i + col * ldp]);
            }
        }
        return 0;
    }
    const i64 h = np / 2;
    if (z_panel(Pm, ldp, mp, h, piv, off, info, check)) return 1;
    z_swap(Pm, ldp, piv, off, 0, h - 1, h, np);
    z_trsm(h, np - h, Pm, ldp, Pm + h * ldp, ldp, 0, 1, 0, 0);
    if (mp > h) {
        z_gemm_minus(mp - h, np - h, h, Pm + h, ldp, Pm + h * ldp, ldp, Pm + h + h * ldp, ldp);
        if (z_panel(Pm + h + h * ldp, ldp, mp - h, np - h, piv, off + h, info, check)) return 1;
        const i64 q = mp < np ? mp : np;
        z_swap(Pm, ldp, piv, off, h, q - 1, 0, h);
    }
    return 0;
}

/* _lu_factor! for ComplexF64 (blocked right-looking, nb, sequential order) */
int orc_zgetrf(i64 m, i64 n, zc_t *A, i64 lda, i64 nb, int check, i64 *ipiv, i64 *info) {
    const i64 q = m < n ? m : n;
    *info = 0;
    if (nb <= 0) return 2;
    for (i64 f = 0; f < q; f += nb) {
        const i64 l = f + nb < q ? f + nb : q;
        if (z_panel(A + f + f * lda, lda, m - f, l - f, ipiv, f, info, check)) return 1;
        z_swap(A, lda, ipiv, 0, f, l - 1, 0, f);
        z_swap(A, lda, ipiv, 0, f, l - 1, l, n);
        if (l >= n) continue;
        z_trsm(l - f, n - l, A + f + f * lda, lda, A + f + l * lda, lda, 0, 1, 0, 0);
        if (l >= m) continue;
        z_gemm_minus(m - l, n - l, l - f, A + l + f * lda, lda, A + f + l * lda, lda, A + l + l * lda, lda);
    }
    return 0;
}

/* ldiv!(F, B) ('N'), ldiv!(transpose(F), B) ('T'), ldiv!(F', B) ('C') */
int orc_zgetrs(char trans, i64 n, i64 nrhs, const zc_t *LU, i64 lda, const i64 *ipiv, zc_t *B, i64 ldb) {
    if (n == 0 || nrhs == 0) return 0;
    if (trans == 'N') {
        for (i64 c = 0; c < nrhs; ++c) {
            zc_t *b = B + c * ldb;
            for (i64 j = 0; j < n; ++j) {
                const i64 p = ipiv[j] - 1;
                if (p != j) { zc_t t = b[j]; b[j] = b[p]; b[p] = t; }
            }
        }
        z_trsm(n, nrhs, LU, lda, B, ldb, 0, 1, 0, 0);
        z_trsm(n, nrhs, LU, lda, B, ldb, 1, 0, 0, 0);
        return 0;
    }
    const int cj = (trans == 'C');
    /* U^T (or U^H) is lower and non-unit, L^T (L^H) upper and unit */
    z_trsm(n, nrhs, LU, lda, B, ldb, 0, 0, 1, cj);
    z_trsm(n, nrhs, LU, lda, B, ldb, 1, 1, 1, cj);
    for (i64 c = 0; c < nrhs; ++c) {
        zc_t *b = B + c * ldb;
        for (i64 j = n - 1; j >= 0; --j) {
            const i64 p = ipiv[j] - 1;
            if (p != j) { zc_t t = b[j]; b[j] = b[p]; b[p] = t; }
        }
    }
    return 0;
}
