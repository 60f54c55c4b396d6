// Mixed-precision dense solve: low-precision LU + FP64 iterative refinement.
//
// Follows mixed_solve -> _mixed_precision_impl (src/lapack/extended_lapack.jl:
// 175-226, src/lapack/factorizations.jl:425-427), LU family:
//   1. finite input required (:182);
//   2. equilibrate(A; radix=true) -- row, then column powers of two
//      (src/lapack/dense_utilities.jl:191-213);
//   3. low-precision LU of the equilibrated matrix (FP32 panel; the trailing
//      updates on the tensor cores in BF16 or FP16, FP32 accumulation); a
//      singular low factor falls back to an FP64 factor (:199-202);
//   4. corrections by _mixed_extended_correction (:114-131): row-scale the
//      residual, scale by 2^exponent(max), round to the low type, solve, widen,
//      multiply back, column-unscale;
//   5. FP64 residual and componentwise backward error (_refinement_residual!,
//      src/lapack/expert_refinement.jl:67-81) each iteration; stop at rtol.
// Beyond the reference: the normwise backward error is reported too (and can
// drive the stop test), and GMRES-IR (left-preconditioned GMRES on A d = r with
// the low-precision LU as preconditioner, FP64 matrix-vector products) replaces
// classical IR when it stagnates or on request.
#include <algorithm>
#include <cmath>
#include <vector>
#include "oxi_internal.h"
#include "scaling.cuh"
#include "tma_util.cuh"

namespace oxi {

namespace {
constexpr int RS = 32;       // column chunks of the split residual / GEMV
constexpr int NRMAX = 4;     // right-hand sides per residual pass
constexpr int NCMAX = 16;    // right-hand sides per correction solve (one triangular-solve launch each)
inline i64 rup(i64 x, i64 a) { return (x + a - 1) / a * a; }
}  // namespace

__device__ __forceinline__ void atomic_max_nonneg(double *addr, double v) {
    // non-negative doubles order like their bit patterns; NaN is mapped to +Inf
    if (!(v == v)) v = INFINITY;
    atomicMax((unsigned long long *)addr, (unsigned long long)__double_as_longlong(v));
}

// ---------------------------------------------------------------------------
// Equilibration
// ---------------------------------------------------------------------------
// Row statistics of the m x n column-major A over column chunk blockIdx.y:
// max |a| and sum |a| per row, and a flag for non-finite entries.
__global__ void k_row_stats_part(const double *__restrict__ A, i64 lda, int m, int n, int chunk,
                                 double *__restrict__ pmax, double *__restrict__ psum,
                                 int *__restrict__ nonfinite) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (i >= m) return;
    const int j0 = s * chunk, j1 = min(n, j0 + chunk);
    double mx = 0.0, sm = 0.0;
    bool bad = false;
    const double *a = A + i;
#pragma unroll 8
    for (int j = j0; j < j1; ++j) {
        const double v = fabs(a[(i64)j * lda]);
        bad |= !isfinite(v);
        mx = fmax(mx, v);
        sm += v;
    }
    pmax[(i64)s * m + i] = mx;
    psum[(i64)s * m + i] = sm;
    if (bad) atomicExch(nonfinite, 1);
}

// Row scales: radix = 1 (mixed_solve): the power of two nearest each row's
// max |a|, 1 for a zero row; radix = 0 (expert_solve): the max itself, and a
// zero row recorded in *zero_row (the smallest 1-based index; the reference
// throws SingularException for it).
__global__ void k_row_stats_final(const double *__restrict__ pmax, const double *__restrict__ psum,
                                  int n, int parts, double *__restrict__ rows,
                                  double *__restrict__ anorm, int radix = 1, int *__restrict__ zero_row = nullptr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double mx = 0.0, sm = 0.0;
    for (int s = 0; s < parts; ++s) {
        mx = fmax(mx, pmax[(i64)s * n + i]);
        sm += psum[(i64)s * n + i];
    }
    if (radix) rows[i] = mx > 0.0 ? radix_scale(mx) : 1.0;
    else rows[i] = mx > 0.0 ? mx : 1.0;
    if (!(mx > 0.0) && zero_row) atomicMin(zero_row, i + 1);
    atomic_max_nonneg(anorm, sm);
}

__global__ void k_col_scale(const double *__restrict__ A, i64 lda, int m,
                            const double *__restrict__ rows, double *__restrict__ cols, int radix = 1) {
    const int j = blockIdx.x;
    double mx = 0.0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) mx = fmax(mx, fabs(A[i + (i64)j * lda]) / rows[i]);
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        mx = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        if (threadIdx.x == 0) cols[j] = mx > 0.0 ? (radix ? radix_scale(mx) : mx) : 1.0;
    }
}

// W[i][j] = T(A[i,j] / rows[i] / cols[j]): the equilibrated matrix, rounded to
// the factor type, in the engine's row-major layout.
template <typename T>
__global__ void k_equilibrated_rm(const double *__restrict__ A, i64 lda, T *__restrict__ W, i64 ldw,
                                  int n, const double *__restrict__ rows,
                                  const double *__restrict__ cols) {
    __shared__ T tile[32][33];
    const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {
        const int i = i0 + tx, j = j0 + r;
        if (i < n && j < n) tile[r][tx] = (T)((A[i + (i64)j * lda] / rows[i]) / cols[j]);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int i = i0 + r, j = j0 + tx;
        if (i < n && j < n) W[(i64)i * ldw + j] = tile[tx][r];
    }
}

// E = A ./ rows ./ cols (column-major m x n): the matrix of equilibrate(A).
__global__ void k_equilibrated_cm(const double *__restrict__ A, i64 lda, double *__restrict__ E, i64 lde,
                                  int m, int n, const double *__restrict__ rows,
                                  const double *__restrict__ cols) {
    const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (i64)m * n) return;
    const int i = (int)(idx % m), j = (int)(idx / m);
    E[i + (i64)j * lde] = (A[i + (i64)j * lda] / rows[i]) / cols[j];
}

// column j of the n x n identity (grid: row blocks x columns)
__global__ void k_identity(double *__restrict__ X, i64 ldx, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i < n) X[i + (i64)j * ldx] = (i == j) ? 1.0 : 0.0;
}

// Cholesky family of mixed_solve (src/lapack/extended_lapack.jl:187-193): one
// global positive scale, max |a_ij| over the whole matrix (1 if zero), from the
// row-statistics partials; rows = scale, columns = 1; perm = identity.
__global__ void __launch_bounds__(1024) k_global_scale(const double *__restrict__ pmax, i64 count,
                                                       double *__restrict__ out) {
    double mx = 0.0;
    for (i64 e = threadIdx.x; e < count; e += blockDim.x) mx = fmax(mx, pmax[e]);
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    __shared__ double red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, red[w]);
        *out = (t == 0.0) ? 1.0 : t;
    }
}
__global__ void k_chol_scales(const double *__restrict__ scale, double *__restrict__ rows,
                              double *__restrict__ cols, int64_t *__restrict__ perm, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rows[i] = *scale;
    cols[i] = 1.0;
    perm[i] = i;
}
// W (column-major, ldw) = T(A / scale): the matrix the low-precision Cholesky
// factors (its lower triangle)
template <typename T>
__global__ void k_scaled_copy(const double *__restrict__ A, i64 lda, T *__restrict__ W, i64 ldw, int n,
                              const double *__restrict__ scale) {
    const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (i64)n * n) return;
    const i64 j = idx / n, i = idx - j * n;
    W[i + j * ldw] = (T)(A[i + j * lda] / *scale);
}

__global__ void k_fill(double *__restrict__ v, int n, double x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = x;
}

__global__ void k_check_finite(const double *__restrict__ B, i64 ldb, int n, int nrhs, int *flag) {
    const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (i64)n * nrhs) return;
    const int i = (int)(idx % n), k = (int)(idx / n);
    if (!isfinite(B[i + (i64)k * ldb])) atomicExch(flag, 1);
}

// ---------------------------------------------------------------------------
// FP64 residual R = B - A X (or product Y = A X) with the componentwise error
// ---------------------------------------------------------------------------
// Each thread owns two adjacent rows (one 16-byte load per column when the
// column base is 16-byte aligned); columns split into RS chunks.  NR is the
// accumulator count (a single right-hand side keeps fewer registers, so more
// warps hide the loads' latency); partial sums are laid out NRMAX apart.
template <int NR>
__global__ void k_resid_part(const double *__restrict__ A, i64 lda, int n, const double *__restrict__ X,
                             i64 ldx, int nr, double *__restrict__ pax, double *__restrict__ pden) {
    const int i = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    const int s = blockIdx.y;
    if (i >= n) return;
    const int chunk = (n + RS - 1) / RS;
    const int j0 = s * chunk, j1 = min(n, j0 + chunk);
    const bool two = i + 1 < n;
    const bool vec = two && ((lda & 1) == 0) && ((((uintptr_t)(A + i)) & 15) == 0);
    double ax[2][NR], den[2][NR];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int k = 0; k < NR; ++k) { ax[h][k] = 0.0; den[h][k] = 0.0; }
    const double *a = A + i;
#pragma unroll 8
    for (int j = j0; j < j1; ++j) {
        double2 v;
        if (vec) v = __ldcs((const double2 *)(a + (i64)j * lda));
        else { v.x = a[(i64)j * lda]; v.y = two ? a[(i64)j * lda + 1] : 0.0; }
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            if (k < nr) {
                const double x = __ldg(&X[j + (i64)k * ldx]);
                ax[0][k] = fma(v.x, x, ax[0][k]);
                ax[1][k] = fma(v.y, x, ax[1][k]);
                den[0][k] = fma(fabs(v.x), fabs(x), den[0][k]);
                den[1][k] = fma(fabs(v.y), fabs(x), den[1][k]);
            }
        }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        if (h == 1 && !two) break;
#pragma unroll
        for (int k = 0; k < NR; ++k)
            if (k < nr) {
                pax[((i64)s * NRMAX + k) * n + i + h] = ax[h][k];
                if (pden) pden[((i64)s * NRMAX + k) * n + i + h] = den[h][k];
            }
    }
}

// mode 0: R = B - sum(pax), errors into scal[k*4 + {0 cw, 1 rmax, 2 xmax, 3 bmax}], scal[64+k] += r^2
// mode 1: Y = sum(pax)
__global__ void k_resid_final(const double *__restrict__ B, i64 ldb, double *__restrict__ R, i64 ldr,
                              const double *__restrict__ X, i64 ldx, int n, int nr, int k0,
                              const double *__restrict__ pax, const double *__restrict__ pden, int mode,
                              double *__restrict__ scal) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = blockIdx.y;
    if (k >= nr) return;
    double cw = 0.0, rabs = 0.0, xabs = 0.0, babs = 0.0, r2 = 0.0;
    if (i < n) {
        double ax = 0.0, den = 0.0;
        for (int s = 0; s < RS; ++s) {
            ax += pax[((i64)s * NRMAX + k) * n + i];
            if (mode == 0) den += pden[((i64)s * NRMAX + k) * n + i];
        }
        if (mode == 1) {
            R[i + (i64)k * ldr] = ax;
            return;
        }
        const double b = B[i + (i64)k * ldb];
        const double r = b - ax;
        den += fabs(b);
        R[i + (i64)k * ldr] = r;
        if (!isfinite(den)) cw = INFINITY;
        else if (den == 0.0) cw = (r == 0.0) ? 0.0 : INFINITY;
        else cw = fabs(r) / den;
        rabs = fabs(r);
        xabs = fabs(X[i + (i64)k * ldx]);
        babs = fabs(b);
        r2 = r * r;
    }
    if (mode == 1) return;
    // block reductions
    __shared__ double red[5][8];
    double v[5] = {cw, rabs, xabs, babs, r2};
#pragma unroll
    for (int q = 0; q < 4; ++q)
        for (int off = 16; off > 0; off >>= 1) v[q] = fmax(v[q], __shfl_xor_sync(0xffffffffu, v[q], off));
    for (int off = 16; off > 0; off >>= 1) v[4] += __shfl_xor_sync(0xffffffffu, v[4], off);
    if ((threadIdx.x & 31) == 0)
        for (int q = 0; q < 5; ++q) red[q][threadIdx.x >> 5] = v[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int q = 0; q < 5; ++q) {
            double acc = red[q][0];
            for (int w = 1; w < nw; ++w) acc = (q < 4) ? fmax(acc, red[q][w]) : acc + red[q][w];
            if (q < 4) atomic_max_nonneg(&scal[(k0 + k) * 4 + q], acc);
            else atomicAdd(&scal[64 + k0 + k], acc);
        }
    }
}

// ---------------------------------------------------------------------------
// Corrections (_mixed_extended_correction)
// ---------------------------------------------------------------------------
__global__ void k_scaled_absmax(const double *__restrict__ R, i64 ldr, int n, int nr,
                                const double *__restrict__ rows, double *__restrict__ mag) {
    const int k = blockIdx.y;
    double mx = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        mx = fmax(mx, fabs(R[i + (i64)k * ldr] / rows[i]));
    if (!isfinite(mx)) mx = INFINITY;
    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&mag[k], mx);
}

// low[i, k] = T((R[perm[i], k] / rows[perm[i]]) / mag_k): scale, round, permute
template <typename T>
__global__ void k_to_low(const double *__restrict__ R, i64 ldr, int n, int nr,
                         const double *__restrict__ rows, const int64_t *__restrict__ perm,
                         const double *__restrict__ mag, T *__restrict__ low, int *__restrict__ err) {
    const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (i64)n * nr) return;
    const int i = (int)(idx % n), k = (int)(idx / n);
    const double m = mag[k];
    if (!isfinite(m)) { atomicExch(err, 4); low[idx] = T(0); return; }
    const double sc = binary_scale(m);
    const int64_t p = perm[i];
    const T v = sc == 0.0 ? T(0) : (T)((R[p + (i64)k * ldr] / rows[p]) / sc);
    if (!isfinite((double)v)) atomicExch(err, 4);
    low[idx] = v;
}

// X (+)= T-result * mag / cols
template <typename T>
__global__ void k_apply_corr(double *__restrict__ X, i64 ldx, int n, int nr, const T *__restrict__ low,
                             const double *__restrict__ mag, const double *__restrict__ cols, int add) {
    const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (i64)n * nr) return;
    const int i = (int)(idx % n), k = (int)(idx / n);
    const double sc = binary_scale(mag[k]);
    const double c = ((double)low[idx] * sc) / cols[i];
    if (add) X[i + (i64)k * ldx] += c;
    else X[i + (i64)k * ldx] = c;
}

// ---------------------------------------------------------------------------
// GMRES helpers: dots h_l = V[:,l] . w (l < cnt), w -= V h, norms
// ---------------------------------------------------------------------------
constexpr int GM_MAXV = 64;
__global__ void k_dots_part(const double *__restrict__ V, i64 ldv, int cnt, const double *__restrict__ w,
                            int n, double *__restrict__ part) {
    __shared__ double red[8][GM_MAXV];
    double acc[GM_MAXV];
    for (int l = 0; l < GM_MAXV; ++l) acc[l] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double wi = w[i];
        for (int l = 0; l < cnt; ++l) acc[l] = fma(V[i + (i64)l * ldv], wi, acc[l]);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int l = 0; l < cnt; ++l) {
        double v = acc[l];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[warp][l] = v;
    }
    __syncthreads();
    for (int l = threadIdx.x; l < cnt; l += blockDim.x) {
        double v = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) v += red[q][l];
        part[(i64)blockIdx.x * GM_MAXV + l] = v;
    }
}
__global__ void k_dots_final(const double *__restrict__ part, int blocks, int cnt, double *__restrict__ h) {
    const int l = threadIdx.x;
    if (l >= cnt) return;
    double v = 0.0;
    for (int b = 0; b < blocks; ++b) v += part[(i64)b * GM_MAXV + l];
    h[l] = v;
}
__global__ void k_sub_vh(const double *__restrict__ V, i64 ldv, int cnt, const double *__restrict__ h,
                         double *__restrict__ w, int n, double scale_out, double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = w[i];
    for (int l = 0; l < cnt; ++l) v = fma(-V[i + (i64)l * ldv], h[l], v);
    w[i] = v;
    if (out) out[i] = v * scale_out;
}
__global__ void k_axpy_vy(const double *__restrict__ V, i64 ldv, int cnt, const double *__restrict__ y,
                          double *__restrict__ x, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = x[i];
    for (int l = 0; l < cnt; ++l) v = fma(V[i + (i64)l * ldv], y[l], v);
    x[i] = v;
}
__global__ void k_scale_copy(const double *__restrict__ src, double *__restrict__ dst, int n, const double *__restrict__ nrm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double s = *nrm > 0 ? 1.0 / sqrt(*nrm) : 0.0;
    dst[i] = src[i] * s;
}

__global__ void k_add_to(double *__restrict__ x, const double *__restrict__ y, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += y[i];
}
__global__ void k_sub(double *__restrict__ out, const double *__restrict__ a, const double *__restrict__ b, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] - b[i];
}

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------
struct MixedRun {
    oxi_handle_s *h;
    cudaStream_t s;
    i64 n, nrhs;
    const double *A;
    i64 lda;
    const double *B;
    i64 ldb;
    double *X;
    i64 ldx;
    // device workspace
    double *rows, *cols, *pmax, *psum, *pax, *pden, *R, *C, *mag;
    float *low32;
    double *low64;
    int64_t *perm, *ipiv;
    void *W;  // float (low) or double (fallback) row-major factors
    i64 ldw;
    void *dinvL, *dinvU;  // inverses of the 64 x 64 diagonal blocks of L and U
    bool fallback = false;
    bool chol = false;  // Cholesky family: W holds the column-major lower factor L
    double *scal;  // device scalars (cw/rmax/xmax/bmax per rhs, r^2)
    int *err;      // device error word
    double anorm = 0.0;
    // pinned host staging (sized once per call: no reallocation while in use)
    int64_t *hpiv;  // n + 8 entries
    double *hsc;    // 512 doubles of scalars
    // GMRES
    double *V, *gw, *gt, *gpart, *gh, *gz;
    int restart;
};

static inline unsigned blocks_for(i64 n, int t = 256) { return (unsigned)((n + t - 1) / t); }

static void residual(MixedRun &M, const double *Xin, double *Rout, std::vector<double> &cw,
                     std::vector<double> &nw, double &r2) {
    cudaStream_t s = M.s;
    const int n = (int)M.n, nrhs = (int)M.nrhs;
    OXI_CUDA(cudaMemsetAsync(M.scal, 0, sizeof(double) * 128, s));
    ProfScope ps(KC_RESIDUAL, s, 2.0 * (double)n * n * nrhs, 8.0 * (double)n * n);
    for (int k0 = 0; k0 < nrhs; k0 += NRMAX) {
        const int nr = std::min(NRMAX, nrhs - k0);
        dim3 g1(blocks_for((n + 1) / 2, 128), RS);
        if (nr == 1)
            k_resid_part<1><<<g1, 128, 0, s>>>(M.A, M.lda, n, Xin + (i64)k0 * M.ldx, M.ldx, nr, M.pax, M.pden);
        else
            k_resid_part<NRMAX><<<g1, 128, 0, s>>>(M.A, M.lda, n, Xin + (i64)k0 * M.ldx, M.ldx, nr, M.pax, M.pden);
        OXI_LAUNCH_CHECK();
        dim3 g2(blocks_for(n), nr);
        k_resid_final<<<g2, 256, 0, s>>>(M.B + (i64)k0 * M.ldb, M.ldb, Rout + (i64)k0 * M.n, M.n,
                                          Xin + (i64)k0 * M.ldx, M.ldx, n, nr, k0, M.pax, M.pden, 0,
                                          M.scal);
        OXI_LAUNCH_CHECK();
    }
    double *hs = M.hsc;
    OXI_CUDA(cudaMemcpyAsync(hs, M.scal, sizeof(double) * 128, cudaMemcpyDeviceToHost, s));
    OXI_CUDA(cudaStreamSynchronize(s));
    cw.assign(nrhs, 0.0);
    nw.assign(nrhs, 0.0);
    r2 = 0.0;
    for (int k = 0; k < nrhs; ++k) {
        cw[k] = hs[k * 4 + 0];
        const double rmax = hs[k * 4 + 1], xmax = hs[k * 4 + 2], bmax = hs[k * 4 + 3];
        const double den = M.anorm * xmax + bmax;
        nw[k] = den > 0 ? rmax / den : (rmax == 0 ? 0.0 : INFINITY);
        if (!std::isfinite(den)) nw[k] = INFINITY;
        r2 += hs[64 + k];
    }
}

// y = A x (FP64)
static void matvec(MixedRun &M, const double *x, double *y) {
    cudaStream_t s = M.s;
    const int n = (int)M.n;
    dim3 g1(blocks_for((n + 1) / 2, 128), RS);
    k_resid_part<1><<<g1, 128, 0, s>>>(M.A, M.lda, n, x, n, 1, M.pax, nullptr);
    OXI_LAUNCH_CHECK();
    k_resid_final<<<dim3(blocks_for(n), 1), 256, 0, s>>>(nullptr, 0, y, n, nullptr, 0, n, 1, 0, M.pax,
                                                         nullptr, 1, nullptr);
    OXI_LAUNCH_CHECK();
}

// Z = M^-1 R through the low-precision factors (_mixed_extended_correction).
static void precond(MixedRun &M, const double *Rin, i64 ldr, double *Z, i64 ldz, int nr) {
    cudaStream_t s = M.s;
    const int n = (int)M.n;
    OXI_CUDA(cudaMemsetAsync(M.mag, 0, sizeof(double) * nr, s));
    k_scaled_absmax<<<dim3(64, nr), 256, 0, s>>>(Rin, ldr, n, nr, M.rows, M.mag);
    OXI_LAUNCH_CHECK();
    const unsigned gb = blocks_for((i64)n * nr);
    if (!M.fallback) {
        k_to_low<float><<<gb, 256, 0, s>>>(Rin, ldr, n, nr, M.rows, M.perm, M.mag, M.low32, M.err);
        OXI_LAUNCH_CHECK();
        if (M.chol)
            chol_solve_ops<float>(M.h, (const float *)M.W, M.ldw, n, M.low32, n, nr, M.err,
                                  (const float *)M.dinvL, (const float *)M.dinvU);
        else
            lu_solve_rowmajor<float>(M.h, (const float *)M.W, M.ldw, n, M.low32, n, nr, M.err,
                                     (const float *)M.dinvL, (const float *)M.dinvU);
        k_apply_corr<float><<<gb, 256, 0, s>>>(Z, ldz, n, nr, M.low32, M.mag, M.cols, 0);
    } else {
        k_to_low<double><<<gb, 256, 0, s>>>(Rin, ldr, n, nr, M.rows, M.perm, M.mag, M.low64, M.err);
        OXI_LAUNCH_CHECK();
        if (M.chol)
            chol_solve_ops<double>(M.h, (const double *)M.W, M.ldw, n, M.low64, n, nr, M.err,
                                   (const double *)M.dinvL, (const double *)M.dinvU);
        else
            lu_solve_rowmajor<double>(M.h, (const double *)M.W, M.ldw, n, M.low64, n, nr, M.err,
                                      (const double *)M.dinvL, (const double *)M.dinvU);
        k_apply_corr<double><<<gb, 256, 0, s>>>(Z, ldz, n, nr, M.low64, M.mag, M.cols, 0);
    }
    OXI_LAUNCH_CHECK();
}

static void dots(MixedRun &M, const double *V, int cnt, const double *w, double *h_dev) {
    const int blocks = 120;
    k_dots_part<<<blocks, 256, 0, M.s>>>(V, M.n, cnt, w, (int)M.n, M.gpart);
    OXI_LAUNCH_CHECK();
    k_dots_final<<<1, GM_MAXV, 0, M.s>>>(M.gpart, blocks, cnt, h_dev);
    OXI_LAUNCH_CHECK();
}

static double fetch_scalar(MixedRun &M, const double *dptr) {
    OXI_CUDA(cudaMemcpyAsync(M.hsc + 256, dptr, sizeof(double), cudaMemcpyDeviceToHost, M.s));
    OXI_CUDA(cudaStreamSynchronize(M.s));
    return M.hsc[256];
}

// One GMRES-IR correction for a right-hand side: solve A d = r with
// left-preconditioned restarted GMRES (classical Gram-Schmidt applied twice),
// then x += d.  Returns the number of inner iterations.
static int gmres_correction(MixedRun &M, const double *r, double *x, double tol, int max_inner) {
    cudaStream_t s = M.s;
    const int n = (int)M.n, m = M.restart;
    const unsigned gb = blocks_for(n);
    int iters = 0;
    OXI_CUDA(cudaMemsetAsync(M.gz, 0, sizeof(double) * n, s));  // d = 0
    double beta0 = -1.0;
    for (int cycle = 0; cycle < 8 && iters < max_inner; ++cycle) {
        if (cycle == 0) {
            OXI_CUDA(cudaMemcpyAsync(M.gt, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        } else {  // t = r - A d
            matvec(M, M.gz, M.gw);
            k_sub<<<gb, 256, 0, s>>>(M.gt, r, M.gw, n);
            OXI_LAUNCH_CHECK();
        }
        precond(M, M.gt, n, M.gw, n, 1);  // v0 = M^-1 t
        dots(M, M.gw, 1, M.gw, M.gh);
        const double beta = std::sqrt(fetch_scalar(M, M.gh));
        if (beta0 < 0) beta0 = beta;
        if (!(beta > 0) || !std::isfinite(beta)) break;
        if (cycle > 0 && beta <= tol * beta0) break;
        k_scale_copy<<<gb, 256, 0, s>>>(M.gw, M.V, n, M.gh);
        OXI_LAUNCH_CHECK();
        std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1, 0.0);
        g[0] = beta;
        int j = 0;
        bool done = false;
        for (; j < m && iters < max_inner; ++j) {
            ++iters;
            double *vj = M.V + (i64)j * n, *vn = M.V + (i64)(j + 1) * n;
            matvec(M, vj, M.gt);
            precond(M, M.gt, n, vn, n, 1);
            std::vector<double> hcol(j + 2, 0.0);
            for (int pass = 0; pass < 2; ++pass) {
                dots(M, M.V, j + 1, vn, M.gh);
                k_sub_vh<<<gb, 256, 0, s>>>(M.V, n, j + 1, M.gh, vn, n, 0.0, nullptr);
                OXI_LAUNCH_CHECK();
                OXI_CUDA(cudaMemcpyAsync(M.hsc, M.gh, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, s));
                OXI_CUDA(cudaStreamSynchronize(s));
                for (int l = 0; l <= j; ++l) hcol[l] += M.hsc[l];
            }
            dots(M, vn, 1, vn, M.gh);
            const double nrm2 = fetch_scalar(M, M.gh);
            hcol[j + 1] = std::sqrt(nrm2);
            if (nrm2 > 0) {
                k_scale_copy<<<gb, 256, 0, s>>>(vn, vn, n, M.gh);
                OXI_LAUNCH_CHECK();
            }
            for (int l = 0; l < j; ++l) {  // earlier Givens rotations
                const double a = hcol[l], b = hcol[l + 1];
                hcol[l] = cs[l] * a + sn[l] * b;
                hcol[l + 1] = -sn[l] * a + cs[l] * b;
            }
            const double a = hcol[j], b = hcol[j + 1];
            const double rr = std::hypot(a, b);
            cs[j] = rr > 0 ? a / rr : 1.0;
            sn[j] = rr > 0 ? b / rr : 0.0;
            hcol[j] = rr;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            for (int l = 0; l <= j; ++l) H[(size_t)l * m + j] = hcol[l];
            if (std::fabs(g[j + 1]) <= tol * beta0 || !(nrm2 > 0)) { ++j; done = true; break; }
        }
        const int kk = j;  // least squares: H y = g (upper triangular)
        std::vector<double> y(kk, 0.0);
        for (int l = kk - 1; l >= 0; --l) {
            double v = g[l];
            for (int q = l + 1; q < kk; ++q) v -= H[(size_t)l * m + q] * y[q];
            y[l] = H[(size_t)l * m + l] != 0 ? v / H[(size_t)l * m + l] : 0.0;
        }
        if (kk > 0) {
            std::copy(y.begin(), y.end(), M.hsc);
            OXI_CUDA(cudaMemcpyAsync(M.gh, M.hsc, sizeof(double) * kk, cudaMemcpyHostToDevice, s));
            k_axpy_vy<<<gb, 256, 0, s>>>(M.V, n, kk, M.gh, M.gz, n);  // d += V y
            OXI_LAUNCH_CHECK();
            OXI_CUDA(cudaStreamSynchronize(s));
        }
        if (done) break;
    }
    k_add_to<<<gb, 256, 0, s>>>(x, M.gz, n);  // x += d
    OXI_LAUNCH_CHECK();
    return iters;
}

// expert_solve's differences from mixed_solve (src/lapack/advanced_factorizations.jl:
// 591-645): scales are the row and column maxima themselves (not powers of two),
// a zero row is singular, the factor is FP64, the stop test componentwise, and
// the scales and the factorization go back to the caller.
struct ExpertOpts {
    int equilibrate = 1;
    double *rows_out = nullptr, *cols_out = nullptr;  // device, n each (nullable)
    double *F_out = nullptr;                           // device, column-major n x n (nullable)
    i64 ldf = 0;
    int64_t *ipiv_out = nullptr;                       // device, n (nullable)
    int64_t zero_row = 0;                              // out: first zero row (1-based), 0 if none
};

static int dgesv_mixed(oxi_handle_s *h, int prec, int refine, i64 n, i64 nrhs, const double *dA,
                       i64 lda, const double *dB, i64 ldb, double *dX, i64 ldx, int maxiter, double rtol,
                       oxi_refine_report *out, ExpertOpts *xo = nullptr, bool chol = false) {
    if (xo) {
        prec = OXI_PREC_FP64;
        refine = OXI_REFINE_IR;
    }
    cudaStream_t s = h->stream;
    MixedRun M;
    M.h = h; M.s = s; M.n = n; M.nrhs = nrhs; M.A = dA; M.lda = lda; M.B = dB; M.ldb = ldb;
    M.X = dX; M.ldx = ldx;
    M.chol = chol;
    M.restart = std::max(2, std::min(h->opt.gmres_restart, GM_MAXV - 2));
    cudaEvent_t e0, e1, e2;
    OXI_CUDA(cudaEventCreate(&e0));
    OXI_CUDA(cudaEventCreate(&e1));
    OXI_CUDA(cudaEventCreate(&e2));
    struct EvGuard {
        cudaEvent_t a, b, c;
        ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); cudaEventDestroy(c); }
    } evg{e0, e1, e2};
    OXI_CUDA(cudaEventRecord(e0, s));

    // ---- workspace ----
    const i64 ldw = rup(n, 32);
    M.ldw = ldw;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
    const size_t o_rows = take(8 * n), o_cols = take(8 * n), o_pmax = take(8 * n * RS),
                 o_psum = take(8 * n * RS), o_pax = take(8 * n * RS * NRMAX),
                 o_pden = take(8 * n * RS * NRMAX), o_R = take(8 * n * nrhs), o_C = take(8 * n * nrhs),
                 o_mag = take(8 * 64), o_low32 = take(4 * n * nrhs), o_low64 = take(8 * n * nrhs),
                 o_perm = take(8 * n), o_ipiv = take(8 * n), o_V = take(8 * n * GM_MAXV),
                 o_gw = take(8 * n), o_gt = take(8 * n), o_gpart = take(8 * 120 * GM_MAXV),
                 o_gh = take(8 * GM_MAXV), o_gz = take(8 * n),
                 o_dinv = take(2 * 8 * (size_t)lu_block_inverse_elems(n)),
                 o_pwork = chol ? take(8 * potrf_work_elems(n)) : take(0);
    char *ws = (char *)h->mixed_ws.get(off);
    M.rows = (double *)(ws + o_rows); M.cols = (double *)(ws + o_cols);
    M.pmax = (double *)(ws + o_pmax); M.psum = (double *)(ws + o_psum);
    M.pax = (double *)(ws + o_pax); M.pden = (double *)(ws + o_pden);
    M.R = (double *)(ws + o_R); M.C = (double *)(ws + o_C); M.mag = (double *)(ws + o_mag);
    M.low32 = (float *)(ws + o_low32); M.low64 = (double *)(ws + o_low64);
    M.perm = (int64_t *)(ws + o_perm); M.ipiv = (int64_t *)(ws + o_ipiv);
    M.V = (double *)(ws + o_V); M.gw = (double *)(ws + o_gw); M.gt = (double *)(ws + o_gt);
    M.gpart = (double *)(ws + o_gpart); M.gh = (double *)(ws + o_gh); M.gz = (double *)(ws + o_gz);
    const i64 inv_elems = lu_block_inverse_elems(n);
    char *sc = (char *)h->scratch.get(kScratchBytes);
    M.err = (int *)(sc + kScratchErrOff);
    int *nonfinite = M.err + 1;
    int64_t *d_info = (int64_t *)sc;
    int *d_nmoves = (int *)(sc + 64);
    int *d_moves = (int *)(sc + 128);
    M.scal = (double *)(sc + kScratchScalOff);
    char *hb = (char *)h->host_ws.get(sizeof(int64_t) * (n + 16) + sizeof(double) * 512);
    M.hpiv = (int64_t *)hb;
    M.hsc = (double *)(hb + sizeof(int64_t) * (n + 16));
    // M.err (the call's abort word, also set to 4 by an overflowing conversion)
    // and the non-finite flag were cleared by the entry point's AbortScope

    // ---- 1-2. finiteness + equilibration ----
    {
        const int chunk = (int)((n + RS - 1) / RS);
        dim3 g(blocks_for(n, 128), RS);
        k_row_stats_part<<<g, 128, 0, s>>>(dA, lda, (int)n, (int)n, chunk, M.pmax, M.psum, nonfinite);
        OXI_LAUNCH_CHECK();
        k_check_finite<<<blocks_for(n * nrhs), 256, 0, s>>>(dB, ldb, (int)n, (int)nrhs, nonfinite);
        OXI_LAUNCH_CHECK();
        OXI_CUDA(cudaMemsetAsync(M.scal, 0, sizeof(double) * 128, s));
        const int radix = xo ? 0 : 1;
        int *zrow = (int *)(M.scal + 120);
        if (xo) {
            const int big = 0x7fffffff;
            OXI_CUDA(cudaMemcpyAsync(zrow, &big, sizeof(int), cudaMemcpyHostToDevice, s));
        }
        k_row_stats_final<<<blocks_for(n), 256, 0, s>>>(M.pmax, M.psum, (int)n, RS, M.rows, M.scal, radix,
                                                         xo ? zrow : nullptr);
        OXI_LAUNCH_CHECK();
        if (chol) {
            k_global_scale<<<1, 1024, 0, s>>>(M.pmax, (i64)n * RS, M.scal + 100);
            OXI_LAUNCH_CHECK();
            k_chol_scales<<<blocks_for(n), 256, 0, s>>>(M.scal + 100, M.rows, M.cols, M.perm, (int)n);
        } else {
            k_col_scale<<<(unsigned)n, 256, 0, s>>>(dA, lda, (int)n, M.rows, M.cols, radix);
        }
        OXI_LAUNCH_CHECK();
        int *hflag = (int *)(M.hsc + 300);
        OXI_CUDA(cudaMemcpyAsync(hflag, nonfinite, sizeof(int), cudaMemcpyDeviceToHost, s));
        OXI_CUDA(cudaMemcpyAsync(M.hsc + 301, M.scal, sizeof(double), cudaMemcpyDeviceToHost, s));
        if (xo) OXI_CUDA(cudaMemcpyAsync(hflag + 1, zrow, sizeof(int), cudaMemcpyDeviceToHost, s));
        OXI_CUDA(cudaStreamSynchronize(s));
        if (hflag[0]) return OXI_ENONFINITE;
        M.anorm = M.hsc[301];
        if (xo) {
            if (xo->equilibrate && hflag[1] != 0x7fffffff) {  // a zero row: SingularException(i)
                xo->zero_row = hflag[1];
                if (out) out->info = hflag[1];
                return OXI_ESINGULAR;
            }
            if (!xo->equilibrate) {  // unscaled: both scale vectors are ones
                k_fill<<<blocks_for(n), 256, 0, s>>>(M.rows, (int)n, 1.0);
                OXI_LAUNCH_CHECK();
                k_fill<<<blocks_for(n), 256, 0, s>>>(M.cols, (int)n, 1.0);
                OXI_LAUNCH_CHECK();
            }
        }
    }

    // ---- 3. low-precision factorization ----
    int64_t info = 0;
    auto factor_chol = [&](bool fp64) {
        // the Cholesky family: T(A / scale), its lower triangle factored in place
        OXI_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int64_t), s));
        const unsigned gb = blocks_for((i64)n * n);
        M.dinvL = ws + o_dinv;
        if (!fp64) {
            float *W = (float *)h->work.get((size_t)n * ldw * sizeof(float));
            M.W = W;
            k_scaled_copy<float><<<gb, 256, 0, s>>>(dA, lda, W, ldw, (int)n, M.scal + 100);
            OXI_LAUNCH_CHECK();
            const int saved_tr = h->trailing;
            h->trailing = prec;
            try {
                potrf_rowmajor<float>(h, W, ldw, n, d_info, (float *)(ws + o_pwork));
            } catch (...) {
                h->trailing = saved_tr;
                throw;
            }
            h->trailing = saved_tr;
            M.dinvU = (float *)M.dinvL + inv_elems;
            chol_block_ops<float>(h, W, ldw, n, (float *)M.dinvL, (float *)M.dinvU);
        } else {
            double *W = (double *)h->work.get((size_t)n * ldw * sizeof(double));
            M.W = W;
            k_scaled_copy<double><<<gb, 256, 0, s>>>(dA, lda, W, ldw, (int)n, M.scal + 100);
            OXI_LAUNCH_CHECK();
            potrf_rowmajor<double>(h, W, ldw, n, d_info, (double *)(ws + o_pwork));
            M.dinvU = (double *)M.dinvL + inv_elems;
            chol_block_ops<double>(h, W, ldw, n, (double *)M.dinvL, (double *)M.dinvU);
        }
        OXI_CUDA(cudaMemcpyAsync(M.hpiv, d_info, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        OXI_CUDA(cudaStreamSynchronize(s));
        info = M.hpiv[0];
    };
    auto factor = [&](bool fp64) {
        if (M.chol) {
            factor_chol(fp64);
            return;
        }
        OXI_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int64_t), s));
        dim3 g((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32));
        if (!fp64) {
            float *W = (float *)h->work.get((size_t)n * ldw * sizeof(float));
            M.W = W;
            k_equilibrated_rm<float><<<g, dim3(32, 8), 0, s>>>(dA, lda, W, ldw, (int)n, M.rows, M.cols);
            OXI_LAUNCH_CHECK();
            const i64 saved_bs = h->opt.blocksize;
            const int saved_tr = h->trailing;
            h->opt.blocksize = h->opt.mixed_blocksize;
            h->trailing = prec;
            h->tslu = h->opt.tournament;
            try {
                getrf_rowmajor_cached<float>(h, W, ldw, n, n, M.ipiv, d_info, d_moves, d_nmoves);
            } catch (...) {
                h->opt.blocksize = saved_bs;
                h->trailing = saved_tr;
                h->tslu = 0;
                throw;
            }
            h->opt.blocksize = saved_bs;
            h->trailing = saved_tr;
            h->tslu = 0;
        } else {
            double *W = (double *)h->work.get((size_t)n * ldw * sizeof(double));
            M.W = W;
            k_equilibrated_rm<double><<<g, dim3(32, 8), 0, s>>>(dA, lda, W, ldw, (int)n, M.rows, M.cols);
            OXI_LAUNCH_CHECK();
            getrf_rowmajor_cached<double>(h, W, ldw, n, n, M.ipiv, d_info, d_moves, d_nmoves);
        }
        if (!fp64) {
            M.dinvL = ws + o_dinv;
            M.dinvU = (float *)M.dinvL + inv_elems;
            lu_block_inverses_rowmajor<float>(h, (const float *)M.W, ldw, n, (float *)M.dinvL, (float *)M.dinvU);
        } else {
            M.dinvL = ws + o_dinv;
            M.dinvU = (double *)M.dinvL + inv_elems;
            lu_block_inverses_rowmajor<double>(h, (const double *)M.W, ldw, n, (double *)M.dinvL, (double *)M.dinvU);
        }
        OXI_CUDA(cudaMemcpyAsync(M.hpiv, d_info, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        OXI_CUDA(cudaMemcpyAsync(M.hpiv + 8, M.ipiv, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, s));
        OXI_CUDA(cudaStreamSynchronize(s));
        info = M.hpiv[0];
        if (info == 0) {
            std::vector<int64_t> perm(n);
            perm_from_ipiv(M.hpiv + 8, n, n, perm.data());
            std::copy(perm.begin(), perm.end(), M.hpiv + 8);
            OXI_CUDA(cudaMemcpyAsync(M.perm, M.hpiv + 8, sizeof(int64_t) * n, cudaMemcpyHostToDevice, s));
            OXI_CUDA(cudaStreamSynchronize(s));
        }
    };
    M.fallback = (prec == OXI_PREC_FP64);
    factor(M.fallback);
    const int64_t low_info = info;
    bool used_fallback = false;
    if (info != 0 && !M.fallback) {  // SingularException of the low factor: working-precision factor
        M.fallback = true;
        used_fallback = true;
        factor(true);
    }
    if (out) out->info = M.chol && info != 0 ? info : low_info;
    if (info != 0) return M.chol ? OXI_ENOTPOSDEF : OXI_ESINGULAR;
    if (xo) {  // the scales and the factorization of the scaled matrix
        if (xo->rows_out)
            OXI_CUDA(cudaMemcpyAsync(xo->rows_out, M.rows, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        if (xo->cols_out)
            OXI_CUDA(cudaMemcpyAsync(xo->cols_out, M.cols, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        if (xo->ipiv_out)
            OXI_CUDA(cudaMemcpyAsync(xo->ipiv_out, M.ipiv, sizeof(int64_t) * n, cudaMemcpyDeviceToDevice, s));
        if (xo->F_out) launch_rm_to_cm<double, double>((const double *)M.W, ldw, xo->F_out, xo->ldf, n, n, s);
    }
    OXI_CUDA(cudaEventRecord(e1, s));

    // ---- 4-5. first solve and refinement ----
    const int nr_i = (int)nrhs;
    auto correct_all = [&](const double *Rin, i64 ldr, int add) {
        for (int k0 = 0; k0 < nr_i; k0 += NCMAX) {
            const int nr = std::min(NCMAX, nr_i - k0);
            if (!add) {
                precond(M, Rin + (i64)k0 * ldr, ldr, dX + (i64)k0 * ldx, ldx, nr);
            } else {
                precond(M, Rin + (i64)k0 * ldr, ldr, M.C, n, nr);
                for (int k = 0; k < nr; ++k) {
                    k_add_to<<<blocks_for(n), 256, 0, s>>>(dX + (i64)(k0 + k) * ldx, M.C + (i64)k * n, (int)n);
                    OXI_LAUNCH_CHECK();
                }
            }
        }
    };
    correct_all(dB, ldb, 0);
    std::vector<double> cw, nw;
    double r2 = 0.0, err_prev = INFINITY, err = INFINITY;
    int it = 0;
    i64 gm_total = 0;
    bool use_gmres = (refine == OXI_REFINE_GMRES);
    int refine_used = use_gmres ? OXI_REFINE_GMRES : OXI_REFINE_IR;
    const bool stop_nw = h->opt.stop_normwise != 0 && !xo;
    for (int iter = 0; iter <= maxiter; ++iter) {
        residual(M, dX, M.R, cw, nw, r2);
        double ecw = 0, enw = 0;
        for (int k = 0; k < nr_i; ++k) { ecw = std::max(ecw, cw[k]); enw = std::max(enw, nw[k]); }
        err = stop_nw ? enw : ecw;
        it = iter;
        if (out) {
            out->backward_error = ecw;
            out->backward_error_normwise = enw;
            out->residual_norm = std::sqrt(r2);
        }
        if (err <= rtol || iter == maxiter || !std::isfinite(err)) break;
        if (refine == OXI_REFINE_AUTO && !use_gmres && iter > 0 && err > 0.5 * err_prev) {
            use_gmres = true;  // classical refinement stagnates: GMRES-IR from here on
            refine_used = OXI_REFINE_GMRES;
        }
        err_prev = err;
        if (!use_gmres) {
            correct_all(M.R, n, 1);
        } else {
            for (int k = 0; k < nr_i; ++k)
                gm_total += gmres_correction(M, M.R + (i64)k * n, dX + (i64)k * ldx, h->opt.gmres_tol, 400);
        }
        int *herr = (int *)(M.hsc + 310);
        OXI_CUDA(cudaMemcpyAsync(herr, M.err, sizeof(int), cudaMemcpyDeviceToHost, s));
        OXI_CUDA(cudaStreamSynchronize(s));
        if (*herr == 4) return OXI_EOVERFLOW;
        if (*herr) return OXI_ETIMEOUT;
    }
    OXI_CUDA(cudaEventRecord(e2, s));
    OXI_CUDA(cudaEventSynchronize(e2));
    const bool finite = std::isfinite(err);
    const bool conv = err <= rtol;
    if (out) {
        float f1 = 0, f2 = 0;
        cudaEventElapsedTime(&f1, e0, e1);
        cudaEventElapsedTime(&f2, e1, e2);
        out->iterations = it;
        out->gmres_iterations = gm_total;
        out->converged = conv ? 1 : 0;
        out->fallback = used_fallback ? 1 : 0;
        out->refine_used = refine_used;
        out->low_type = prec;
        out->factor_ms = f1;
        out->refine_ms = f2;
        out->reason = !finite ? OXI_REASON_NONFINITE
                              : used_fallback ? OXI_REASON_FALLBACK
                                              : conv ? OXI_REASON_CONVERGED : OXI_REASON_ITERATION_LIMIT;
    }
    return conv ? OXI_OK : OXI_ENOTCONVERGED;
}

}  // namespace oxi

extern "C" int oxi_dgesv_mixed(oxi_handle_t h, int prec, int refine, int64_t n, int64_t nrhs,
                               const double *dA, int64_t lda, const double *dB, int64_t ldb,
                               double *dX, int64_t ldx, int maxiter, double rtol,
                               oxi_refine_report *out) {
    if (!h) return OXI_EINVAL;
    if (out) *out = oxi_refine_report{};
    if (n < 0 || nrhs < 0 || maxiter < 0 || !(rtol >= 0) || !std::isfinite(rtol)) return OXI_EINVAL;
    if (prec < OXI_PREC_FP32 || prec > OXI_PREC_FP16X3 || refine < 0 || refine > OXI_REFINE_AUTO)
        return OXI_EINVAL;
    if (n == 0 || nrhs == 0) return OXI_OK;
    if (!dA || !dB || !dX || lda < n || ldb < n || ldx < n || nrhs > 16) return OXI_EINVAL;
    if (oxi::leaf_width_for<float>(n) == 0 || n >= (1ll << 31)) return OXI_EINVAL;
    try {
        oxi::ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        oxi::AbortScope ab(h);
        const int st = oxi::dgesv_mixed(h, prec, refine, n, nrhs, dA, lda, dB, ldb, dX, ldx, maxiter, rtol, out);
        h->stall_at = 0;  // the test hook is one-shot
        if (st == OXI_EOVERFLOW) return st;  // the conversion's code in the abort word
        int *he = (int *)h->host_ws.get(64);
        oxi::queue_abort_read(h, he);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        const int we = oxi::check_abort(h, he);
        return we != OXI_OK ? we : st;
    } catch (const oxi::CudaError &e) {
        h->stall_at = 0;
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

// mixed_solve(A, b; factorization=:cholesky): the same driver with the
// Cholesky family's scaling and factor (src/lapack/extended_lapack.jl:175-226).
extern "C" int oxi_dposv_mixed(oxi_handle_t h, int prec, int refine, int64_t n, int64_t nrhs,
                               const double *dA, int64_t lda, const double *dB, int64_t ldb,
                               double *dX, int64_t ldx, int maxiter, double rtol,
                               oxi_refine_report *out) {
    if (!h) return OXI_EINVAL;
    if (out) *out = oxi_refine_report{};
    if (n < 0 || nrhs < 0 || maxiter < 0 || !(rtol >= 0) || !std::isfinite(rtol)) return OXI_EINVAL;
    if (prec < OXI_PREC_FP32 || prec > OXI_PREC_FP16X3 || refine < 0 || refine > OXI_REFINE_AUTO)
        return OXI_EINVAL;
    if (n == 0 || nrhs == 0) return OXI_OK;
    if (!dA || !dB || !dX || lda < n || ldb < n || ldx < n || nrhs > 16 || n >= (1ll << 31)) return OXI_EINVAL;
    try {
        oxi::ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        oxi::AbortScope ab(h);
        const int st = oxi::dgesv_mixed(h, prec, refine, n, nrhs, dA, lda, dB, ldb, dX, ldx, maxiter, rtol, out,
                                        nullptr, /*chol=*/true);
        if (st == OXI_EOVERFLOW) return st;
        int *he = (int *)h->host_ws.get(64);
        oxi::queue_abort_read(h, he);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        const int we = oxi::check_abort(h, he);
        return we != OXI_OK ? we : st;
    } catch (const oxi::CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

// ---------------------------------------------------------------------------
// equilibrate(A; radix=true) alone (src/lapack/dense_utilities.jl:191-213): the
// row scales (powers of two nearest each row's max |a|), then the column scales
// of the row-scaled matrix, and optionally the equilibrated matrix itself.
extern "C" int oxi_dequilibrate(oxi_handle_t h, int64_t m, int64_t n, const double *dA, int64_t lda,
                                double *d_rows, double *d_cols, double *dE, int64_t lde) {
    using namespace oxi;
    if (!h || m < 0 || n < 0 || lda < std::max<int64_t>(1, m)) return OXI_EINVAL;
    if (dE && lde < std::max<int64_t>(1, m)) return OXI_EINVAL;
    if (m >= (1ll << 31) || n >= (1ll << 31)) return OXI_EINVAL;
    if (m == 0 && n == 0) return OXI_OK;
    if ((m > 0 && !d_rows) || (n > 0 && !d_cols) || (m > 0 && n > 0 && !dA)) return OXI_EINVAL;
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        AbortScope ab(h);
        cudaStream_t s = h->stream;
        int *nonfinite = ab.word + 1;  // cleared by the scope
        if (m == 0) {  // no rows: every column scale is one
            std::vector<double> one((size_t)n, 1.0);
            OXI_CUDA(cudaMemcpyAsync(d_cols, one.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
            OXI_CUDA(cudaStreamSynchronize(s));
            return OXI_OK;
        }
        const int parts = (int)std::min<int64_t>(RS, std::max<int64_t>(1, n));
        const int chunk = (int)((std::max<int64_t>(n, 1) + parts - 1) / parts);
        double *ws = (double *)h->mixed_ws.get(sizeof(double) * (2 * (size_t)parts * m + 8));
        double *pmax = ws, *psum = ws + (size_t)parts * m, *anorm = psum + (size_t)parts * m;
        OXI_CUDA(cudaMemsetAsync(anorm, 0, sizeof(double), s));
        dim3 g(blocks_for(m, 128), parts);
        k_row_stats_part<<<g, 128, 0, s>>>(dA, lda, (int)m, (int)n, chunk, pmax, psum, nonfinite);
        OXI_LAUNCH_CHECK();
        k_row_stats_final<<<blocks_for(m), 256, 0, s>>>(pmax, psum, (int)m, parts, d_rows, anorm);
        OXI_LAUNCH_CHECK();
        if (n > 0) {
            k_col_scale<<<(unsigned)n, 256, 0, s>>>(dA, lda, (int)m, d_rows, d_cols);
            OXI_LAUNCH_CHECK();
            if (dE) {
                k_equilibrated_cm<<<blocks_for(m * n), 256, 0, s>>>(dA, lda, dE, lde, (int)m, (int)n, d_rows,
                                                                     d_cols);
                OXI_LAUNCH_CHECK();
            }
        }
        int *hflag = (int *)h->host_ws.get(64);
        OXI_CUDA(cudaMemcpyAsync(hflag, nonfinite, sizeof(int), cudaMemcpyDeviceToHost, s));
        OXI_CUDA(cudaStreamSynchronize(s));
        return hflag[0] ? OXI_ENONFINITE : OXI_OK;
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

// ---------------------------------------------------------------------------
// expert_solve, refine_solve, inverse_norm_estimate and the inverse
// ---------------------------------------------------------------------------
namespace oxi {

// One CTA: out[0] = sum |v|, out[1] = max |v|, out[2] = its first index,
// out[3] = v . x (x nullable).
__global__ void __launch_bounds__(1024) k_vec_stats(const double *__restrict__ v, const double *__restrict__ x,
                                                    int n, double *__restrict__ out) {
    __shared__ double s_sum[32], s_dot[32], s_max[32];
    __shared__ int s_idx[32];
    double sm = 0.0, dt = 0.0, mx = -1.0;
    int ix = 0x7fffffff;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double a = fabs(v[i]);
        sm += a;
        if (x) dt += v[i] * x[i];
        if (a > mx) { mx = a; ix = i; }  // i ascends per thread: the first maximum
    }
    for (int off = 16; off > 0; off >>= 1) {
        sm += __shfl_xor_sync(0xffffffffu, sm, off);
        dt += __shfl_xor_sync(0xffffffffu, dt, off);
        const double om = __shfl_xor_sync(0xffffffffu, mx, off);
        const int oi = __shfl_xor_sync(0xffffffffu, ix, off);
        if (om > mx || (om == mx && oi < ix)) { mx = om; ix = oi; }
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { s_sum[w] = sm; s_dot[w] = dt; s_max[w] = mx; s_idx[w] = ix; }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        sm = lane < nw ? s_sum[lane] : 0.0;
        dt = lane < nw ? s_dot[lane] : 0.0;
        mx = lane < nw ? s_max[lane] : -1.0;
        ix = lane < nw ? s_idx[lane] : 0x7fffffff;
        for (int off = 16; off > 0; off >>= 1) {
            sm += __shfl_xor_sync(0xffffffffu, sm, off);
            dt += __shfl_xor_sync(0xffffffffu, dt, off);
            const double om = __shfl_xor_sync(0xffffffffu, mx, off);
            const int oi = __shfl_xor_sync(0xffffffffu, ix, off);
            if (om > mx || (om == mx && oi < ix)) { mx = om; ix = oi; }
        }
        if (lane == 0) { out[0] = sm; out[1] = mx; out[2] = (double)ix; out[3] = dt; }
    }
}

// z = sign(y) with sign(0) = 1 (value / abs(value), the reference's signs)
__global__ void k_signs(const double *__restrict__ y, double *__restrict__ z, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) z[i] = (y[i] == 0.0) ? 1.0 : y[i] / fabs(y[i]);
}
// x = e_idx
__global__ void k_unit(double *__restrict__ x, int n, int idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = (i == idx) ? 1.0 : 0.0;
}
// x_i = (-1)^i (1 + i / max(1, n - 1)), 0-based i: the final probe vector
__global__ void k_alt_probe(double *__restrict__ x, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = ((i & 1) ? -1.0 : 1.0) * (1.0 + (double)i / (double)(n > 1 ? n - 1 : 1));
}
// max_j sum_i |A[i, j]| (column-major m x n), one CTA per column
__global__ void __launch_bounds__(256) k_one_norm(const double *__restrict__ A, i64 lda, int m,
                                                  double *__restrict__ out) {
    const int j = blockIdx.x;
    double sm = 0.0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) sm += fabs(A[i + (i64)j * lda]);
    __shared__ double red[8];
    for (int off = 16; off > 0; off >>= 1) sm += __shfl_xor_sync(0xffffffffu, sm, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[w];
        atomic_max_nonneg(out, t);
    }
}

// 0-based permutation of the factors' ipiv, uploaded into the handle's perm
// workspace (validating every entry): OXI_OK or OXI_EINVAL.
static int upload_perm(oxi_handle_s *h, i64 n, const int64_t *d_ipiv, int64_t **dperm_out) {
    std::vector<int64_t> ip(n), perm(n);
    OXI_CUDA(cudaMemcpyAsync(ip.data(), d_ipiv, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, h->stream));
    OXI_CUDA(cudaStreamSynchronize(h->stream));
    for (i64 j = 0; j < n; ++j)
        if (ip[j] < 1 || ip[j] > n) return OXI_EINVAL;
    perm_from_ipiv(ip.data(), n, n, perm.data());
    int64_t *dperm = (int64_t *)h->perm_ws.get(sizeof(int64_t) * n);
    int64_t *hperm = (int64_t *)h->host_ws.get(sizeof(int64_t) * (n + 64));
    std::copy(perm.begin(), perm.end(), hperm);
    OXI_CUDA(cudaMemcpyAsync(dperm, hperm, sizeof(int64_t) * n, cudaMemcpyHostToDevice, h->stream));
    OXI_CUDA(cudaStreamSynchronize(h->stream));
    *dperm_out = dperm;
    return OXI_OK;
}

// inverse_norm_estimate (src/lapack/expert_refinement.jl:45-60): Hager-Higham
// with solves by the factors (trans 'N') and their transpose ('T'); the
// decisions (stop tests, next unit vector) are taken on the host from one
// reduction per solve.  ws: 3n + 8 doubles of device memory.
static double inverse_norm_est(oxi_handle_s *h, i64 n, const double *LU, i64 lda, const int64_t *dperm,
                               int maxiter, double *ws, int *ab) {
    cudaStream_t s = h->stream;
    double *x = ws, *y = ws + n, *z = ws + 2 * n, *st = ws + 3 * n;
    double *hs = (double *)h->host_ws.get(sizeof(double) * 64) + 32;
    const unsigned gb = blocks_for(n);
    k_fill<<<gb, 256, 0, s>>>(x, (int)n, 1.0 / (double)n);
    OXI_LAUNCH_CHECK();
    double est = 0.0;
    long prev = -1;
    for (int it = 0; it < maxiter; ++it) {
        OXI_CUDA(cudaMemcpyAsync(y, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        getrs_perm<double>(h, 'N', n, 1, LU, lda, dperm, y, n, ab);
        k_signs<<<gb, 256, 0, s>>>(y, z, (int)n);
        OXI_LAUNCH_CHECK();
        k_vec_stats<<<1, 1024, 0, s>>>(y, nullptr, (int)n, st);
        OXI_LAUNCH_CHECK();
        getrs_perm<double>(h, 'T', n, 1, LU, lda, dperm, z, n, ab);
        k_vec_stats<<<1, 1024, 0, s>>>(z, x, (int)n, st + 4);
        OXI_LAUNCH_CHECK();
        OXI_CUDA(cudaMemcpyAsync(hs, st, sizeof(double) * 8, cudaMemcpyDeviceToHost, s));
        OXI_CUDA(cudaStreamSynchronize(s));
        est = std::max(est, hs[0]);
        const long idx = (long)hs[6];
        if (hs[5] <= hs[7]) break;  // |z[idx]| <= z . x
        if (idx == prev) break;
        k_unit<<<gb, 256, 0, s>>>(x, (int)n, (int)idx);
        OXI_LAUNCH_CHECK();
        prev = idx;
    }
    k_alt_probe<<<gb, 256, 0, s>>>(x, (int)n);
    OXI_LAUNCH_CHECK();
    getrs_perm<double>(h, 'N', n, 1, LU, lda, dperm, x, n, ab);
    k_vec_stats<<<1, 1024, 0, s>>>(x, nullptr, (int)n, st);
    OXI_LAUNCH_CHECK();
    OXI_CUDA(cudaMemcpyAsync(hs, st, sizeof(double), cudaMemcpyDeviceToHost, s));
    OXI_CUDA(cudaStreamSynchronize(s));
    return std::max(est, 2.0 * hs[0] / (3.0 * (double)n));
}

}  // namespace oxi

extern "C" int oxi_dinverse_norm_estimate(oxi_handle_t h, int64_t n, const double *dLU, int64_t lda,
                                          const int64_t *d_ipiv, int maxiter, double *h_estimate) {
    using namespace oxi;
    if (!h || !h_estimate || n < 0 || maxiter < 1 || lda < std::max<int64_t>(1, n)) return OXI_EINVAL;
    *h_estimate = 0.0;
    if (n == 0) return OXI_OK;
    if (!dLU || !d_ipiv || n >= (1ll << 31)) return OXI_EINVAL;
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        AbortScope ab(h);
        int64_t *dperm = nullptr;
        if (upload_perm(h, n, d_ipiv, &dperm) != OXI_OK) return OXI_EINVAL;
        double *ws = (double *)h->mixed_ws.get(sizeof(double) * (3 * (size_t)n + 8));
        const double est = inverse_norm_est(h, n, dLU, lda, dperm, maxiter, ws, ab.word);
        int *he = (int *)h->host_ws.get(64);
        queue_abort_read(h, he);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        const int st = check_abort(h, he);
        if (st == OXI_OK) *h_estimate = est;
        return st;
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

// refine_solve(A, F, b; maxiter, rtol) (src/lapack/expert_refinement.jl:89-104)
// with the factors of oxi_dgetrf.
extern "C" int oxi_drefine_solve(oxi_handle_t h, int64_t n, int64_t nrhs, const double *dA, int64_t lda,
                                 const double *dLU, int64_t ldlu, const int64_t *d_ipiv, const double *dB,
                                 int64_t ldb, double *dX, int64_t ldx, int maxiter, double rtol,
                                 oxi_solve_report *out) {
    using namespace oxi;
    if (!h) return OXI_EINVAL;
    if (out) *out = oxi_solve_report{};
    const int64_t mn = std::max<int64_t>(1, n);
    if (n < 0 || nrhs < 0 || maxiter < 0 || !(rtol >= 0) || lda < mn || ldlu < mn || ldb < mn || ldx < mn)
        return OXI_EINVAL;
    if (n == 0 || nrhs == 0) {
        if (out) { out->converged = 1; out->rcond_estimate = 1.0; }
        return OXI_OK;
    }
    if (!dA || !dLU || !d_ipiv || !dB || !dX || n >= (1ll << 31)) return OXI_EINVAL;
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        AbortScope ab(h);
        cudaStream_t s = h->stream;
        int64_t *dperm = nullptr;
        if (upload_perm(h, n, d_ipiv, &dperm) != OXI_OK) return OXI_EINVAL;
        // workspace: residual partials, R (n x nrhs), the estimator's vectors
        size_t off = 0;
        auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
        const size_t o_pax = take(8 * n * RS * NRMAX), o_pden = take(8 * n * RS * NRMAX),
                     o_R = take(8 * n * nrhs), o_est = take(8 * (3 * n + 8)), o_nrm = take(8 * 8);
        char *ws = (char *)h->mixed_ws.get(off);
        MixedRun M;
        M.h = h; M.s = s; M.n = n; M.nrhs = nrhs; M.A = dA; M.lda = lda; M.B = dB; M.ldb = ldb;
        M.X = dX; M.ldx = ldx;
        M.pax = (double *)(ws + o_pax); M.pden = (double *)(ws + o_pden);
        M.R = (double *)(ws + o_R);
        M.scal = (double *)((char *)h->scratch.get(kScratchBytes) + kScratchScalOff);
        M.hsc = (double *)h->host_ws.get(sizeof(double) * 512);
        M.anorm = 0.0;
        double *nrm = (double *)(ws + o_nrm);
        // X = solve(F, B)
        OXI_CUDA(cudaMemcpy2DAsync(dX, ldx * 8, dB, ldb * 8, n * 8, nrhs, cudaMemcpyDeviceToDevice, s));
        getrs_perm<double>(h, 'N', n, nrhs, dLU, ldlu, dperm, dX, ldx, ab.word);
        std::vector<double> cw, nw;
        double r2 = 0.0, err = INFINITY;
        int it = 0;
        for (int iter = 0; iter <= maxiter; ++iter) {
            residual(M, dX, M.R, cw, nw, r2);
            err = 0.0;
            for (double e : cw) err = (e > err || std::isnan(e)) ? e : err;
            it = iter;
            if (err <= rtol || iter == maxiter) break;
            // correction = solve(F, residual): in place in R, then X += R (R is
            // recomputed at the next step)
            getrs_perm<double>(h, 'N', n, nrhs, dLU, ldlu, dperm, M.R, n, ab.word);
            for (i64 k = 0; k < nrhs; ++k) {
                k_add_to<<<blocks_for(n), 256, 0, s>>>(dX + k * ldx, M.R + k * n, (int)n);
                OXI_LAUNCH_CHECK();
            }
        }
        // the final residual stays in R; the estimates of the reference's tuple
        const double inv_norm = inverse_norm_est(h, n, dLU, ldlu, dperm, 8, (double *)(ws + o_est), ab.word);
        OXI_CUDA(cudaMemsetAsync(nrm, 0, sizeof(double) * 3, s));
        k_one_norm<<<(unsigned)n, 256, 0, s>>>(dA, lda, (int)n, nrm);
        OXI_LAUNCH_CHECK();
        k_one_norm<<<(unsigned)nrhs, 256, 0, s>>>(dX, ldx, (int)n, nrm + 1);
        OXI_LAUNCH_CHECK();
        k_one_norm<<<(unsigned)nrhs, 256, 0, s>>>(M.R, n, (int)n, nrm + 2);
        OXI_LAUNCH_CHECK();
        double *hn = M.hsc + 400;
        OXI_CUDA(cudaMemcpyAsync(hn, nrm, sizeof(double) * 3, cudaMemcpyDeviceToHost, s));
        int *he = (int *)(M.hsc + 408);
        queue_abort_read(h, he);
        OXI_CUDA(cudaStreamSynchronize(s));
        const int st = check_abort(h, he);
        if (st != OXI_OK) return st;
        const double anorm = hn[0], xnorm = hn[1], rnorm1 = hn[2];
        const double cond = anorm * inv_norm;
        const double rnorm = std::sqrt(r2);
        const double delta = xnorm == 0.0 ? (rnorm == 0.0 ? 0.0 : INFINITY) : inv_norm * rnorm1 / xnorm;
        if (out) {
            out->iterations = it;
            out->backward_error = err;
            out->residual_norm = rnorm;
            out->rcond_estimate = cond == 0.0 ? 1.0 : std::min(1.0, 1.0 / cond);
            out->forward_error_estimate = delta < 1.0 ? delta / (1.0 - delta) : INFINITY;
            out->inverse_norm_estimate = inv_norm;
            out->converged = err <= rtol ? 1 : 0;
        }
        return err <= rtol ? OXI_OK : OXI_ENOTCONVERGED;
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

// expert_solve(A, b; maxiter, rtol, equilibrate) (src/lapack/advanced_factorizations.jl:591-645).
extern "C" int oxi_dexpert_solve(oxi_handle_t h, int64_t n, int64_t nrhs, const double *dA, int64_t lda,
                                 const double *dB, int64_t ldb, double *dX, int64_t ldx, int maxiter, double rtol,
                                 int equilibrate, double *d_row_scale, double *d_col_scale, double *dF,
                                 int64_t ldf, int64_t *d_ipiv, oxi_solve_report *out) {
    using namespace oxi;
    if (!h) return OXI_EINVAL;
    if (out) *out = oxi_solve_report{};
    const int64_t mn = std::max<int64_t>(1, n);
    if (n < 0 || nrhs < 0 || maxiter < 0 || !(rtol >= 0) || !std::isfinite(rtol) || lda < mn || ldb < mn ||
        ldx < mn || (dF && ldf < mn))
        return OXI_EINVAL;
    if (n == 0 || nrhs == 0) {
        if (out) out->converged = 1;
        return OXI_OK;
    }
    if (!dA || !dB || !dX || nrhs > 16) return OXI_EINVAL;
    if (leaf_width_for<double>(n) == 0 || n >= (1ll << 31)) return OXI_EINVAL;
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        AbortScope ab(h);
        ExpertOpts xo;
        xo.equilibrate = equilibrate != 0;
        xo.rows_out = d_row_scale;
        xo.cols_out = d_col_scale;
        xo.F_out = dF;
        xo.ldf = ldf;
        xo.ipiv_out = d_ipiv;
        oxi_refine_report rep{};
        const int st = dgesv_mixed(h, OXI_PREC_FP64, OXI_REFINE_IR, n, nrhs, dA, lda, dB, ldb, dX, ldx, maxiter,
                                   rtol, &rep, &xo);
        h->stall_at = 0;
        if (out) {
            out->iterations = rep.iterations;
            out->backward_error = rep.backward_error;
            out->residual_norm = rep.residual_norm;
            out->rcond_estimate = NAN;
            out->forward_error_estimate = NAN;
            out->inverse_norm_estimate = NAN;
            out->info = rep.info;
            out->converged = rep.converged;
        }
        if (st == OXI_EOVERFLOW || st == OXI_ESINGULAR || st == OXI_ENONFINITE) return st;
        int *he = (int *)h->host_ws.get(64);
        queue_abort_read(h, he);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        const int we = check_abort(h, he);
        return we != OXI_OK ? we : st;
    } catch (const CudaError &e) {
        h->stall_at = 0;
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

// inv(F) for the factors of oxi_dgetrf: the solve with the identity, the
// columns of A^-1 (LinearAlgebra's inv over ldiv!, src/api/linalg_api.jl:1143-1144).
extern "C" int oxi_dgetri(oxi_handle_t h, int64_t n, const double *dLU, int64_t lda, const int64_t *d_ipiv,
                          double *dAinv, int64_t ldainv) {
    using namespace oxi;
    if (!h || n < 0 || lda < std::max<int64_t>(1, n) || ldainv < std::max<int64_t>(1, n)) return OXI_EINVAL;
    if (n == 0) return OXI_OK;
    if (!dLU || !d_ipiv || !dAinv || n >= (1ll << 31)) return OXI_EINVAL;
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        AbortScope ab(h);
        int64_t *dperm = nullptr;
        if (upload_perm(h, n, d_ipiv, &dperm) != OXI_OK) return OXI_EINVAL;
        k_identity<<<dim3((unsigned)((n + 255) / 256), (unsigned)n), 256, 0, h->stream>>>(dAinv, ldainv, (int)n);
        OXI_LAUNCH_CHECK();
        getrs_perm<double>(h, 'N', n, n, dLU, lda, dperm, dAinv, ldainv, ab.word);
        int *he = (int *)h->host_ws.get(64);
        queue_abort_read(h, he);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        return check_abort(h, he);
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}
