// Batched LU of many small matrices of uneven orders (1..256) in ONE persistent
// launch: factor, solve and (mixed mode) FP64 iterative refinement of each
// matrix run inside one CTA, which takes the next matrix from a work queue
// ordered by size bucket, largest bucket first (the longest items start first,
// the short ones fill the tail).
//
// The reference factors one matrix per call (src/lapack/factorizations.jl:
// 17-77) and batches only its GEMM (gemm_batched!, src/blas/batched.jl:4-49:
// an outer loop over independent problems, no nested parallelism).  Per matrix
// the algorithm is the same right-looking partial-pivoted LU:
//   panel (jb columns) factored unblocked with the reference's pivot rule
//   (largest |a|, first index on ties; a zero pivot records info and skips the
//   interchange and the elimination; full panels with each thread's row in
//   registers), its interchanges applied to the other
//   columns, U12 = L11^-1 A12, A22 -= L21 U12 (product accumulated from zero,
//   then subtracted, as gemm!(C, A, B, -1, 1)).
// Where the working matrix lives is a tuning choice: orders up to n_smem keep
// it in shared memory; larger ones work in place in global memory (the plain
// FP64 mode: the caller's matrix; the mixed mode: a per-CTA FP32 workspace),
// which mostly stays in L2, with the panel and U12 staged in shared memory so
// the trailing update reads them on chip.  The panel width per size bucket and
// n_smem are picked by oxi_batched_autotune.
//
// Mixed mode follows mixed_solve (src/lapack/extended_lapack.jl:175-226) per
// matrix: radix equilibration, FP32 factor of the scaled matrix, corrections
// by _mixed_extended_correction (:114-131), FP64 residual and componentwise
// backward error (src/lapack/expert_refinement.jl:67-81), stop at rtol.
#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>
#include "oxi_internal.h"
#include "scaling.cuh"

namespace oxi {

namespace bt {
constexpr int NT = 256, NW = NT / 32;
constexpr int NMAX = 256;      // largest order
constexpr int NQ = NMAX / 32;  // rows per lane in the warp solves
constexpr int NBMAX = 32;      // largest panel width
constexpr int MAXRHS = 8;
constexpr int NBUCKET = 8;     // bucket b holds orders 32b+1 .. 32b+32
constexpr int MODE_GETRF = 0, MODE_GESV = 1, MODE_MIXED = 2;
}  // namespace bt

struct BatchDesc {
    int count;
    int mode;
    const int32_t *n;
    double *const *A;
    const int64_t *lda;
    int64_t *const *ipiv;  // nullable (and entries nullable): pivots not returned
    int32_t *info;         // per matrix: 0, first zero pivot, -1 bad arguments, -2 non-finite
    const int32_t *nrhs;
    double *const *B;
    const int64_t *ldb;
    double *const *X;
    const int64_t *ldx;
    int32_t *iters;  // nullable
    double *berr;    // nullable
    const int32_t *order;
    int32_t *head;
    int32_t *status;  // [0] singular, [1] bad arguments, [2] non-finite, [3] not converged
    float *wsp;       // mixed: NMAX*NMAX floats per CTA
    int maxiter;
    double rtol;
    int n_smem;
    int nbmax;
    int nb[bt::NBUCKET];
    int off_p, off_u, off_x, off_r, off_w;  // shared-memory carve (bytes)
};

// Shared-memory bytes of the batched kernel for the element size, mode and tuning.
static int batch_smem_layout(int esize, int mode, int n_smem, int nbmax, BatchDesc *d) {
    using namespace bt;
    int off = 0;
    auto take = [&](int bytes) { const int o = off; off += (bytes + 15) & ~15; return o; };
    const bool global_mode = n_smem < NMAX;
    const int op = take(global_mode ? NMAX * nbmax * esize : 0);
    const int ou = take(global_mode ? nbmax * NMAX * esize : 0);
    const int ox = take(mode == MODE_MIXED ? NMAX * MAXRHS * 8 : 0);
    const int orr = take(mode == MODE_MIXED ? NMAX * MAXRHS * 8 : 0);
    const int ow = take(n_smem * n_smem * esize);
    if (d) {
        d->off_p = op;
        d->off_u = ou;
        d->off_x = ox;
        d->off_r = orr;
        d->off_w = ow;
    }
    return off;
}

namespace {


struct Misc {
    double red_v[2][bt::NW], red_x[2][bt::NW];
    int red_i[2][bt::NW];
    double red_m[bt::NW][bt::MAXRHS];
    int piv[bt::NMAX];   // pivot row (0-based, within the matrix) of each column
    int rowat[bt::NMAX]; // a panel's net permutation: position p holds row rowat[p]
    int mvpos[2 * bt::NBMAX];
    int nmv;
    int perm[bt::NMAX];  // net permutation: row i of L U is row perm[i] of A
    // reciprocals of the radix row and column scales: powers of two in
    // [2^-1023, 2^1022], so x * rrow[i] is exactly x / (row scale i)
    double rrow[bt::NMAX], rcol[bt::NMAX];
    double prow[2][bt::NBMAX];  // register panel: the pivot row and the old row j
    double vjv[2];
    int item, info, bad;
};

// Rows [0, m) of a column from global memory into dst (m <= NMAX, one warp):
// every lane issues its loads before its stores, so the round trips overlap.
template <typename T, typename U>
__device__ __forceinline__ void load_col(T *dst, const U *src, int m, int lane) {
    T v[bt::NQ];
#pragma unroll
    for (int q = 0; q < bt::NQ; ++q) {
        const int r = lane + 32 * q;
        v[q] = r < m ? (T)src[r] : T(0);
    }
#pragma unroll
    for (int q = 0; q < bt::NQ; ++q) {
        const int r = lane + 32 * q;
        if (r < m) dst[r] = v[q];
    }
}

// The pivot candidates of column j (all threads): the row of the largest
// |col[i]|, i in (j, m), first index on ties (INT_MAX when none compares), its
// value, and col[j] -- every value read before the barrier, so no thread can
// see a row the interchange that follows has already moved.
template <typename T>
__device__ int block_argmax(const T *col, int j, int m, Misc &S, int par, double &best, double &val,
                            double &vj) {
    using namespace bt;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    vj = (double)col[j];
    double bv = -1.0, bx = 0.0;
    int bi = INT_MAX;
    for (int i = j + 1 + threadIdx.x; i < m; i += NT) {
        const double x = (double)col[i], v = fabs(x);
        if (v > bv) {
            bv = v;
            bi = i;
            bx = x;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
        const double ox = __shfl_xor_sync(0xffffffffu, bx, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (ov > bv || (ov == bv && oi < bi)) {
            bv = ov;
            bi = oi;
            bx = ox;
        }
    }
    if (lane == 0) {
        S.red_v[par][warp] = bv;
        S.red_i[par][warp] = bi;
        S.red_x[par][warp] = bx;
    }
    __syncthreads();
    bv = S.red_v[par][0];
    bi = S.red_i[par][0];
    bx = S.red_x[par][0];
#pragma unroll
    for (int w = 1; w < NW; ++w) {
        const double ov = S.red_v[par][w];
        const int oi = S.red_i[par][w];
        if (ov > bv || (ov == bv && oi < bi)) {
            bv = ov;
            bi = oi;
            bx = S.red_x[par][w];
        }
    }
    best = bv;
    val = bx;
    return bi;
}

// Unblocked LU of the panel P (m x jb, column-major, ldp) holding columns
// k..k+jb of rows k..n; records S.piv[k + j] and the first zero pivot.
template <typename T>
__device__ void panel_lu(T *P, int ldp, int m, int jb, int k, Misc &S) {
    using namespace bt;
    for (int j = 0; j < jb; ++j) {
        T *colj = P + (i64)j * ldp;
        // _lu_pivot (src/lapack/factorizations.jl:92-107): start from row j with
        // strict '>' -- the first maximum; a NaN at row j keeps row j, a NaN
        // below never wins
        double bv, bx, vj;
        const int pb = block_argmax(colj, j, m, S, j & 1, bv, bx, vj);
        const bool below = pb != INT_MAX && bv > fabs(vj);
        const int p = below ? pb : j;
        const T d = (T)(below ? bx : vj);
        if (threadIdx.x == 0) S.piv[k + j] = k + p;
        if (d == T(0)) {  // zero column: info, no interchange, no elimination
            if (threadIdx.x == 0 && S.info == 0) S.info = k + j + 1;
            continue;
        }
        if (p != j) {
            for (int c = threadIdx.x; c < jb; c += NT) {
                const T t = P[j + (i64)c * ldp];
                P[j + (i64)c * ldp] = P[p + (i64)c * ldp];
                P[p + (i64)c * ldp] = t;
            }
        }
        __syncthreads();
        for (int i = j + 1 + threadIdx.x; i < m; i += NT) {
            const T l = P[i + (i64)j * ldp] / d;
            P[i + (i64)j * ldp] = l;
            for (int c = j + 1; c < jb; ++c) P[i + (i64)c * ldp] = fma(-l, P[j + (i64)c * ldp], P[i + (i64)c * ldp]);
        }
        __syncthreads();
    }
    __syncthreads();  // S.piv / S.info of a final zero column are visible to all
}

// One column of U12 = L11^-1 A12 (unit lower L11 in P, ldp): rows k..k+jb of
// column wc, forward substitution in registers; the result back to wc and,
// when su is given, to su[i NMAX] (the staged U12 the update reads).  JB is
// the panel width at compile time (JB = jb), or NBMAX with jb <= JB checked
// per step for a narrower last panel.
template <typename T, int JB>
__device__ __forceinline__ void u12_column(T *wc, int k, int jb, const T *P, int ldp, T *su) {
    T x[JB];
#pragma unroll
    for (int i = 0; i < JB; ++i) x[i] = (i < jb) ? wc[k + i] : T(0);
#pragma unroll
    for (int i = 1; i < JB; ++i) {
        if (i < jb) {
            T s = x[i];
#pragma unroll
            for (int q = 0; q < i; ++q) s = fma(-P[i + (i64)q * ldp], x[q], s);
            x[i] = s;
        }
    }
#pragma unroll
    for (int i = 0; i < JB; ++i) {
        if (i < jb) {
            wc[k + i] = x[i];
            if (su) su[i * bt::NMAX] = x[i];
        }
    }
}

// C (m2 x m2, column-major, ldc) -= A B, A m2 x jb (column-major, lda), B jb x m2
// with element (kk, c) at B[kk bsk + c bsc]: each product accumulated from zero
// in kk order, then subtracted (gemm!(C, A, B, -1, 1)).  One warp, columns
// c0..c0+3 of rows r0..r0+32 NU: lane l holds rows r0 + l + 32 u, so every A
// load and C access covers 32 consecutive rows (no shared-memory bank
// conflicts, whole sectors in global memory), and two columns' C elements
// are loaded before any of them is stored.
template <typename T, int NU>
__device__ __forceinline__ void update_tile(const T *Ap, int lda, const T *Bp, int bsk, int bsc, T *Cp,
                                            int ldc, int m2, int jb, int r0, int c0, int lane) {
    T acc[NU][4];
#pragma unroll
    for (int u = 0; u < NU; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = T(0);
    const int r = r0 + lane;
    for (int kk = 0; kk < jb; ++kk) {
        T a[NU], b[4];
#pragma unroll
        for (int u = 0; u < NU; ++u) a[u] = (r + 32 * u < m2) ? Ap[(r + 32 * u) + (i64)kk * lda] : T(0);
#pragma unroll
        for (int v = 0; v < 4; ++v) b[v] = (c0 + v < m2) ? Bp[(i64)kk * bsk + (i64)(c0 + v) * bsc] : T(0);
#pragma unroll
        for (int u = 0; u < NU; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
#pragma unroll
    for (int h = 0; h < 4; h += 2) {  // two columns' C elements loaded before any is stored
        T cv[NU][2];
#pragma unroll
        for (int v = 0; v < 2; ++v)
#pragma unroll
            for (int u = 0; u < NU; ++u)
                cv[u][v] = (r + 32 * u < m2 && c0 + h + v < m2) ? Cp[(r + 32 * u) + (i64)(c0 + h + v) * ldc] : T(0);
#pragma unroll
        for (int v = 0; v < 2; ++v)
#pragma unroll
            for (int u = 0; u < NU; ++u)
                if (r + 32 * u < m2 && c0 + h + v < m2)
                    Cp[(r + 32 * u) + (i64)(c0 + h + v) * ldc] = cv[u][v] - acc[u][h + v];
    }
}

// Unblocked LU of a full panel of JB columns (m <= NT rows, P column-major,
// ldp) with thread i holding row i in registers: per column one reduction for
// the pivot (the reference's rule, as panel_lu), the pivot row and the old
// row j exchanged through shared memory, the rank-1 update on registers -- two
// barriers a column instead of three and no shared-memory round trip per
// updated element.  Same operations in the same order as panel_lu.
template <typename T, int JB>
__device__ void panel_lu_reg(T *P, int ldp, int m, int k, Misc &S) {
    using namespace bt;
    const int i = threadIdx.x, lane = i & 31, warp = i >> 5;
    const bool own = i < m;
    T row[JB];
#pragma unroll
    for (int c = 0; c < JB; ++c) row[c] = own ? P[i + (i64)c * ldp] : T(0);
#pragma unroll
    for (int j = 0; j < JB; ++j) {
        const int par = j & 1;
        // candidates: rows below j (a NaN never becomes one: NaN > -1 is false)
        const double ax = fabs((double)row[j]);
        const bool cand = own && i > j && ax > -1.0;
        double bv = cand ? ax : -1.0, bx = cand ? (double)row[j] : 0.0;
        int bi = cand ? i : INT_MAX;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
            const double ox = __shfl_xor_sync(0xffffffffu, bx, off);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
            if (ov > bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
                bx = ox;
            }
        }
        if (lane == 0) {
            S.red_v[par][warp] = bv;
            S.red_i[par][warp] = bi;
            S.red_x[par][warp] = bx;
        }
        if (i == j) S.vjv[par] = (double)row[j];
        __syncthreads();
        bv = S.red_v[par][0];
        bi = S.red_i[par][0];
        bx = S.red_x[par][0];
#pragma unroll
        for (int w = 1; w < NW; ++w) {
            const double ov = S.red_v[par][w];
            const int oi = S.red_i[par][w];
            if (ov > bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
                bx = S.red_x[par][w];
            }
        }
        const double vj = S.vjv[par];
        const bool below = bi != INT_MAX && bv > fabs(vj);
        const int p = below ? bi : j;
        const T d = (T)(below ? bx : vj);
        if (i == 0) S.piv[k + j] = k + p;
        if (d == T(0)) {  // zero column: info, no interchange, no elimination
            if (i == 0 && S.info == 0) S.info = k + j + 1;
            continue;
        }
        double *pa = S.prow[0], *pj = S.prow[1];
        if (i == p) {
#pragma unroll
            for (int c = 0; c < JB; ++c) pa[c] = (double)row[c];
        }
        if (p != j && i == j) {
#pragma unroll
            for (int c = 0; c < JB; ++c) pj[c] = (double)row[c];
        }
        __syncthreads();
        if (i == j) {
#pragma unroll
            for (int c = 0; c < JB; ++c) row[c] = (T)pa[c];
        } else if (p != j && i == p) {
#pragma unroll
            for (int c = 0; c < JB; ++c) row[c] = (T)pj[c];
        }
        if (own && i > j) {
            const T l = row[j] / d;
            row[j] = l;
#pragma unroll
            for (int c = j + 1; c < JB; ++c) row[c] = fma(-l, (T)pa[c], row[c]);
        }
    }
    if (own) {
#pragma unroll
        for (int c = 0; c < JB; ++c) P[i + (i64)c * ldp] = row[c];
    }
    __syncthreads();  // the panel, S.piv and S.info visible to all
}

// Right-looking blocked LU of W (n x n, column-major, ldw; shared or global).
template <typename T>
__device__ void lu_blocked(T *W, int ldw, int n, int nb, bool in_smem, T *sP, T *sU, Misc &S) {
    using namespace bt;
    for (int k = 0; k < n; k += nb) {
        const int jb = min(nb, n - k), m = n - k;
        T *P;
        int ldp;
        if (in_smem) {
            P = W + k + (i64)k * ldw;
            ldp = ldw;
        } else {
            P = sP;
            ldp = m;
            // a warp per column, its lanes down the rows (coalesced, no index division)
            for (int c = (int)(threadIdx.x >> 5); c < jb; c += NW)
                load_col(sP + c * ldp, W + k + (i64)(k + c) * ldw, m, (int)(threadIdx.x & 31));
            __syncthreads();
        }
        if (jb == 16) panel_lu_reg<T, 16>(P, ldp, m, k, S);
        else if (jb == 8) panel_lu_reg<T, 8>(P, ldp, m, k, S);
        else if (jb == 32) panel_lu_reg<T, 32>(P, ldp, m, k, S);
        else panel_lu(P, ldp, m, jb, k, S);
        if (!in_smem) {
            for (int c = (int)(threadIdx.x >> 5); c < jb; c += NW)
                for (int r = (int)(threadIdx.x & 31); r < m; r += 32) W[(k + r) + (i64)(k + c) * ldw] = sP[r + c * ldp];
        }
        // interchanges on the other columns, then U12 = L11^-1 A12
        const int c2 = k + jb;
        if (!in_smem) {
            // global working matrix: the panel's net permutation once, every moved
            // row of the other columns staged in shared memory (sU), then written
            // back -- one round trip instead of jb dependent swaps per column
            for (int p = k + threadIdx.x; p < n; p += NT) S.rowat[p] = p;
            if (threadIdx.x == 0) S.nmv = 0;
            __syncthreads();
            if (threadIdx.x == 0)
                for (int j = 0; j < jb; ++j) {
                    const int a = k + j, b = S.piv[k + j];
                    const int t = S.rowat[a];
                    S.rowat[a] = S.rowat[b];
                    S.rowat[b] = t;
                }
            __syncthreads();
            for (int p = k + threadIdx.x; p < n; p += NT)
                if (S.rowat[p] != p) S.mvpos[atomicAdd(&S.nmv, 1)] = p;
            __syncthreads();
            const int nmv = S.nmv;  // <= 2 jb
            if (nmv > 0) {
                const int ccap = (nb * NMAX) / nmv;  // columns per pass (>= 128)
                for (int cb = 0; cb < n; cb += ccap) {
                    const int cn = min(ccap, n - cb);
                    // a warp per moved row, its lanes across the columns
                    // cn <= n <= 32 NQ: a lane's columns of a moved row in one batch of loads
                    for (int mv = (int)(threadIdx.x >> 5); mv < nmv; mv += NW) {
                        const int src = S.rowat[S.mvpos[mv]];
                        T v[NQ];
#pragma unroll
                        for (int q = 0; q < NQ; ++q) {
                            const int cc = (int)(threadIdx.x & 31) + 32 * q, c = cb + cc;
                            v[q] = (cc < cn && !(c >= k && c < c2)) ? W[src + (i64)c * ldw] : T(0);
                        }
#pragma unroll
                        for (int q = 0; q < NQ; ++q) {
                            const int cc = (int)(threadIdx.x & 31) + 32 * q, c = cb + cc;
                            if (cc < cn && !(c >= k && c < c2)) sU[mv * ccap + cc] = v[q];
                        }
                    }
                    __syncthreads();
                    for (int mv = (int)(threadIdx.x >> 5); mv < nmv; mv += NW) {
                        const int dst = S.mvpos[mv];
                        for (int cc = (int)(threadIdx.x & 31); cc < cn; cc += 32) {
                            const int c = cb + cc;
                            if (c >= k && c < c2) continue;
                            W[dst + (i64)c * ldw] = sU[mv * ccap + cc];
                        }
                    }
                    __syncthreads();
                }
            }
        }
        for (int c = threadIdx.x; c < n; c += NT) {
            if (c >= k && c < c2) continue;
            T *wc = W + (i64)c * ldw;
            if (in_smem) {
                for (int j = 0; j < jb; ++j) {
                    const int p = S.piv[k + j];
                    if (p != k + j) {
                        const T t = wc[k + j];
                        wc[k + j] = wc[p];
                        wc[p] = t;
                    }
                }
            }
            if (c >= c2) {  // full panels at a compile-time width: no predicated steps
                T *su = in_smem ? nullptr : sU + (c - c2);
                if (jb == 16) u12_column<T, 16>(wc, k, 16, P, ldp, su);
                else if (jb == 8) u12_column<T, 8>(wc, k, 8, P, ldp, su);
                else if (jb == 32) u12_column<T, 32>(wc, k, 32, P, ldp, su);
                else u12_column<T, NBMAX>(wc, k, jb, P, ldp, su);
            }
        }
        __syncthreads();
        // A22 -= L21 U12: a warp takes up to 128 rows x 4 columns (update_tile)
        const int m2 = n - c2;
        if (m2 > 0) {
            const T *Ap = P + jb;
            T *Cp = W + c2 + (i64)c2 * ldw;
            const T *Bp = in_smem ? W + k + (i64)c2 * ldw : sU;
            const int bsk = in_smem ? 1 : NMAX;
            const int bsc = in_smem ? ldw : 1;
            const int RB = (m2 + 127) >> 7, tasks = RB * ((m2 + 3) >> 2);
            const int lane = (int)(threadIdx.x & 31);
            for (int t = (int)(threadIdx.x >> 5); t < tasks; t += NW) {
                const int r0 = (t % RB) * 128, c0 = (t / RB) * 4;
                const int nu = min(4, (m2 - r0 + 31) >> 5);  // warp-uniform
                if (nu == 4) update_tile<T, 4>(Ap, ldp, Bp, bsk, bsc, Cp, ldw, m2, jb, r0, c0, lane);
                else if (nu == 3) update_tile<T, 3>(Ap, ldp, Bp, bsk, bsc, Cp, ldw, m2, jb, r0, c0, lane);
                else if (nu == 2) update_tile<T, 2>(Ap, ldp, Bp, bsk, bsc, Cp, ldw, m2, jb, r0, c0, lane);
                else update_tile<T, 1>(Ap, ldp, Bp, bsk, bsc, Cp, ldw, m2, jb, r0, c0, lane);
            }
        }
        __syncthreads();
    }
}

// One warp solves L U y = z (unit L) with z, y distributed as y[q] = row lane + 32 q.
template <typename T>
__device__ void warp_lu_solve(const T *W, int ldw, int n, T (&y)[bt::NQ]) {
    using namespace bt;
    const int lane = threadIdx.x & 31;
#pragma unroll 2
    for (int j = 0; j < n; ++j) {
        const int qj = j >> 5, lj = j & 31;
        T src = y[0];
#pragma unroll
        for (int q = 1; q < NQ; ++q)
            if (q == qj) src = y[q];
        const T yj = __shfl_sync(0xffffffffu, src, lj);
        const T *col = W + (i64)j * ldw;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int i = lane + 32 * q;
            if (i > j && i < n) y[q] = fma(-col[i], yj, y[q]);
        }
    }
#pragma unroll 2
    for (int j = n - 1; j >= 0; --j) {
        const int qj = j >> 5, lj = j & 31;
        T src = y[0];
#pragma unroll
        for (int q = 1; q < NQ; ++q)
            if (q == qj) src = y[q];
        const T *col = W + (i64)j * ldw;
        const T xj = __shfl_sync(0xffffffffu, src, lj) / col[j];
        if (lane == lj) {
#pragma unroll
            for (int q = 0; q < NQ; ++q)
                if (q == qj) y[q] = xj;
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int i = lane + 32 * q;
            if (i < j) y[q] = fma(-col[i], xj, y[q]);
        }
    }
}

// The whole CTA solves L U y = z for the right-hand sides held by its active
// warps (y distributed as in warp_lu_solve), the factor read from global
// memory in chunks of cs columns staged in shared memory (two buffers of cs
// columns in stage, which holds cap columns of NMAX): while the active warps
// run the dependent steps of one chunk, every warp's loads of the next chunk
// are in flight (two columns a warp), so each step reads shared memory and the
// L2 round trips overlap the steps.  Every thread calls it.
template <typename T>
__device__ void block_lu_solve(const T *W, int ldw, int n, T *stage, int cap, bool active, T (&y)[bt::NQ]) {
    using namespace bt;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cs = min(2 * NW, cap / 2);
    T pv[2][NQ];
    auto fetch = [&](int a, int b) {  // columns a + warp, a + warp + NW of [a, b)
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const int jj = warp + NW * t, j = a + jj;
            const bool mine = jj < cs && j < b;
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const int r = lane + 32 * q;
                pv[t][q] = (mine && r < n) ? W[r + (i64)j * ldw] : T(0);
            }
        }
    };
    auto put = [&](T *buf, int a, int b) {
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const int jj = warp + NW * t;
            if (jj < cs && a + jj < b) {
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const int r = lane + 32 * q;
                    if (r < n) buf[r + jj * NMAX] = pv[t][q];
                }
            }
        }
    };
    T *cur = stage, *nxt = stage + cs * NMAX;
    __syncthreads();  // the stage's previous use is over
    fetch(0, min(cs, n));
    put(cur, 0, min(cs, n));
    __syncthreads();
    for (int j0 = 0; j0 < n; j0 += cs) {  // forward, unit lower
        const int j1 = min(j0 + cs, n);
        const bool more = j1 < n;
        if (more) fetch(j1, min(j1 + cs, n));
        if (active) {
            for (int j = j0; j < j1; ++j) {
                const int qj = j >> 5, lj = j & 31;
                T src = y[0];
#pragma unroll
                for (int q = 1; q < NQ; ++q)
                    if (q == qj) src = y[q];
                const T yj = __shfl_sync(0xffffffffu, src, lj);
                const T *col = cur + (j - j0) * NMAX;
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const int i = lane + 32 * q;
                    if (i > j && i < n) y[q] = fma(-col[i], yj, y[q]);
                }
            }
        }
        if (more) put(nxt, j1, min(j1 + cs, n));
        __syncthreads();
        T *t = cur;
        cur = nxt;
        nxt = t;
    }
    {
        const int a0 = max(0, n - cs);
        fetch(a0, n);
        put(cur, a0, n);
        __syncthreads();
    }
    for (int b = n; b > 0; b -= cs) {  // backward, upper
        const int a = max(0, b - cs), na = max(0, a - cs);
        const bool more = a > 0;
        if (more) fetch(na, a);
        if (active) {
            for (int j = b - 1; j >= a; --j) {
                const int qj = j >> 5, lj = j & 31;
                T src = y[0];
#pragma unroll
                for (int q = 1; q < NQ; ++q)
                    if (q == qj) src = y[q];
                const T *col = cur + (j - a) * NMAX;
                const T xj = __shfl_sync(0xffffffffu, src, lj) / col[j];
                if (lane == lj) {
#pragma unroll
                    for (int q = 0; q < NQ; ++q)
                        if (q == qj) y[q] = xj;
                }
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const int i = lane + 32 * q;
                    if (i < j) y[q] = fma(-col[i], xj, y[q]);
                }
            }
        }
        if (more) put(nxt, na, a);
        __syncthreads();
        T *t = cur;
        cur = nxt;
        nxt = t;
    }
}

__device__ __forceinline__ int bucket_of(int n) { return (n - 1) >> 5; }

}  // namespace

// Work queue: item order by size bucket, largest bucket first; orders outside
// 1..NMAX (empty or invalid) last.
__global__ void __launch_bounds__(1024) k_batch_order(const int32_t *__restrict__ n, int count,
                                                      int32_t *__restrict__ order, int32_t *__restrict__ head,
                                                      int32_t *__restrict__ status) {
    using namespace bt;
    __shared__ int cnt[NBUCKET + 1], base[NBUCKET + 1];
    if (threadIdx.x <= NBUCKET) cnt[threadIdx.x] = 0;
    if (threadIdx.x == 0) *head = 0;
    if (threadIdx.x < 4) status[threadIdx.x] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const int ni = n[i];
        atomicAdd(&cnt[(ni >= 1 && ni <= NMAX) ? bucket_of(ni) : NBUCKET], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int pos = 0;
        for (int b = NBUCKET - 1; b >= 0; --b) {
            base[b] = pos;
            pos += cnt[b];
        }
        base[NBUCKET] = pos;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const int ni = n[i];
        const int b = (ni >= 1 && ni <= NMAX) ? bucket_of(ni) : NBUCKET;
        order[atomicAdd(&base[b], 1)] = i;
    }
}

template <typename T>
__global__ void __launch_bounds__(bt::NT, 2) k_lu_batched(const __grid_constant__ BatchDesc d) {
    using namespace bt;
    extern __shared__ __align__(16) unsigned char bsm[];
    __shared__ Misc S;
    T *sP = (T *)(bsm + d.off_p);
    T *sU = (T *)(bsm + d.off_u);
    double *sX = (double *)(bsm + d.off_x);
    double *sR = (double *)(bsm + d.off_r);
    T *sW = (T *)(bsm + d.off_w);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        if (tid == 0) S.item = atomicAdd(d.head, 1);
        __syncthreads();
        const int it = S.item;
        if (it >= d.count) break;
        const int mi = d.order[it];
        const int n = d.n[mi];
        double *A = (n > 0) ? d.A[mi] : nullptr;
        const i64 lda = d.lda[mi];
        const int nr = (d.mode != MODE_GETRF) ? d.nrhs[mi] : 0;
        double *B = (nr > 0) ? d.B[mi] : nullptr;
        const i64 ldb = (d.mode != MODE_GETRF) ? d.ldb[mi] : 1;
        double *Xo = (d.mode == MODE_MIXED && nr > 0) ? d.X[mi] : nullptr;
        const i64 ldxo = (d.mode == MODE_MIXED) ? d.ldx[mi] : 1;
        bool bad = n < 0 || n > NMAX || lda < max(1, n) || (n > 0 && !A);
        if (d.mode != MODE_GETRF) bad |= nr < 0 || nr > MAXRHS || ldb < max(1, n) || (nr > 0 && n > 0 && !B);
        if (d.mode == MODE_MIXED) bad |= ldxo < max(1, n) || (nr > 0 && n > 0 && !Xo);
        if (bad) {
            if (tid == 0) {
                d.info[mi] = -1;
                atomicAdd(&d.status[1], 1);
            }
            __syncthreads();
            continue;
        }
        if (n == 0) {
            if (tid == 0) {
                d.info[mi] = 0;
                if (d.iters) d.iters[mi] = 0;
                if (d.berr) d.berr[mi] = 0.0;
            }
            __syncthreads();
            continue;
        }
        const int nb = d.nb[bucket_of(n)];
        const bool in_smem = n <= d.n_smem;
        if (tid == 0) {
            S.info = 0;
            S.bad = 0;
        }
        T *W;
        int ldw;
        if constexpr (sizeof(T) == 8) {
            // plain FP64: the caller's matrix is the working matrix (in place)
            if (in_smem) {
                W = sW;
                ldw = n;
                for (int c = warp; c < n; c += NW) load_col(W + c * ldw, A + (i64)c * lda, n, lane);
            } else {
                W = (T *)A;
                ldw = (int)lda;
            }
            __syncthreads();
        } else {
            // mixed: radix equilibration, then the scaled matrix in FP32
            W = in_smem ? sW : (T *)(d.wsp + (size_t)blockIdx.x * NMAX * NMAX);
            ldw = n;
            for (int i = tid; i < n; i += NT) {
                double mx = 0.0;
                bool nf = false;
                for (int j0 = 0; j0 < n; j0 += 8) {  // eight loads in flight
                    double v[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) v[u] = (j0 + u < n) ? fabs(A[i + (i64)(j0 + u) * lda]) : 0.0;
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        nf |= !isfinite(v[u]);
                        mx = fmax(mx, v[u]);
                    }
                }
                S.rrow[i] = mx > 0.0 ? 1.0 / radix_scale(mx) : 1.0;
                if (nf) S.bad = 1;
            }
            __syncthreads();
            if (S.bad) {
                if (tid == 0) {
                    d.info[mi] = -2;
                    atomicAdd(&d.status[2], 1);
                    if (d.iters) d.iters[mi] = 0;
                    if (d.berr) d.berr[mi] = INFINITY;
                }
                __syncthreads();
                continue;
            }
            // column scales and the scaled FP32 copy in one pass: a warp per column,
            // the column's values (times the row scales) kept in registers
            for (int j = warp; j < n; j += NW) {
                double v[NQ];
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const int i = lane + 32 * q;
                    v[q] = i < n ? A[i + (i64)j * lda] * S.rrow[i] : 0.0;
                }
                double mx = fabs(v[0]);
#pragma unroll
                for (int q = 1; q < NQ; ++q) mx = fmax(mx, fabs(v[q]));
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
                const double rc = mx > 0.0 ? 1.0 / radix_scale(mx) : 1.0;
                if (lane == 0) S.rcol[j] = rc;
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const int i = lane + 32 * q;
                    if (i < n) W[i + j * ldw] = (T)(v[q] * rc);
                }
            }
            __syncthreads();
        }

        lu_blocked<T>(W, ldw, n, nb, in_smem, sP, sU, S);

        const int info = S.info;
        if (tid == 0) {
            d.info[mi] = info;
            if (info) atomicAdd(&d.status[0], 1);
        }
        int64_t *ip = d.ipiv ? d.ipiv[mi] : nullptr;
        if (ip)
            for (int j = tid; j < n; j += NT) ip[j] = S.piv[j] + 1;
        if constexpr (sizeof(T) == 8) {
            if (in_smem)
                for (int c = warp; c < n; c += NW)
                    for (int r = lane; r < n; r += 32) A[r + (i64)c * lda] = W[r + c * ldw];
        }
        if (d.mode == MODE_GETRF || info != 0 || nr == 0) {
            if (d.mode == MODE_MIXED && tid == 0) {
                if (d.iters) d.iters[mi] = 0;
                if (d.berr) d.berr[mi] = info ? INFINITY : 0.0;
            }
            __syncthreads();
            continue;
        }
        if (tid == 0) {
            for (int i = 0; i < n; ++i) S.perm[i] = i;
            for (int j = 0; j < n; ++j) {
                const int p = S.piv[j];
                const int t = S.perm[j];
                S.perm[j] = S.perm[p];
                S.perm[p] = t;
            }
        }
        __syncthreads();

        if constexpr (sizeof(T) == 8) {
            // plain solve in place in B: warp r takes right-hand side r (nr <= 8 warps)
            {
                const bool active = warp < nr;
                double *b = active ? B + (i64)warp * ldb : nullptr;
                T y[NQ];
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const int i = lane + 32 * q;
                    y[q] = (active && i < n) ? (T)b[S.perm[i]] : T(0);
                }
                __syncwarp();
                if (in_smem) {
                    if (active) warp_lu_solve<T>(W, ldw, n, y);
                } else {
                    block_lu_solve<T>(W, ldw, n, sP, 2 * d.nbmax, active, y);
                }
                if (active) {
#pragma unroll
                    for (int q = 0; q < NQ; ++q) {
                        const int i = lane + 32 * q;
                        if (i < n) b[i] = y[q];
                    }
                }
            }
            __syncthreads();
        } else {
            // correction of each right-hand side by its warp: sX (+)= C (LU)^-1 P (R^-1 r / s) s
            auto correct = [&](bool add) {
                const bool active = warp < nr;  // warp r takes right-hand side r
                double sc = 0.0;
                T y[NQ];
#pragma unroll
                for (int q = 0; q < NQ; ++q) y[q] = T(0);
                if (active) {
                    const double *rr = sR + warp * NMAX;
                    double mx = 0.0;
                    for (int i = lane; i < n; i += 32) mx = fmax(mx, fabs(rr[i] * S.rrow[i]));
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
                    sc = isfinite(mx) ? binary_scale(mx) : 0.0;
#pragma unroll
                    for (int q = 0; q < NQ; ++q) {
                        const int i = lane + 32 * q;
                        if (i < n && sc != 0.0) {
                            const int p = S.perm[i];
                            y[q] = (T)((rr[p] * S.rrow[p]) / sc);
                        }
                    }
                }
                if (in_smem) {
                    if (active) warp_lu_solve<T>(W, ldw, n, y);
                } else {
                    block_lu_solve<T>(W, ldw, n, sP, 2 * d.nbmax, active, y);
                }
                if (active) {
                    double *xx = sX + warp * NMAX;
#pragma unroll
                    for (int q = 0; q < NQ; ++q) {
                        const int i = lane + 32 * q;
                        if (i < n) {
                            const double c = ((double)y[q] * sc) * S.rcol[i];
                            xx[i] = add ? xx[i] + c : c;
                        }
                    }
                }
                __syncthreads();
            };
            for (int r = warp; r < nr; r += NW)
                for (int i = lane; i < n; i += 32) sR[r * NMAX + i] = B[i + (i64)r * ldb];
            __syncthreads();
            correct(false);
            double err = INFINITY;
            int iter = 0;
            for (;; ++iter) {
                // r = b - A x and the componentwise backward error, FP64
                double cw[MAXRHS];
#pragma unroll
                for (int r = 0; r < MAXRHS; ++r) cw[r] = 0.0;
                for (int i = tid; i < n; i += NT) {
                    double ax[MAXRHS], den[MAXRHS];
#pragma unroll
                    for (int r = 0; r < MAXRHS; ++r) {
                        ax[r] = 0.0;
                        den[r] = 0.0;
                    }
                    for (int j0 = 0; j0 < n; j0 += 8) {  // eight loads in flight, then the
                        double av[8];                    // sums in column order
#pragma unroll
                        for (int u = 0; u < 8; ++u) av[u] = (j0 + u < n) ? A[i + (i64)(j0 + u) * lda] : 0.0;
#pragma unroll
                        for (int u = 0; u < 8; ++u) {
                            if (j0 + u >= n) break;
                            const double a = av[u];
#pragma unroll
                            for (int r = 0; r < MAXRHS; ++r) {
                                if (r < nr) {
                                    const double x = sX[r * NMAX + j0 + u];
                                    ax[r] = fma(a, x, ax[r]);
                                    den[r] = fma(fabs(a), fabs(x), den[r]);
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int r = 0; r < MAXRHS; ++r) {
                        if (r < nr) {
                            const double b = B[i + (i64)r * ldb];
                            const double res = b - ax[r];
                            const double dn = den[r] + fabs(b);
                            sR[r * NMAX + i] = res;
                            double q;
                            if (!isfinite(dn)) q = INFINITY;
                            else if (dn == 0.0) q = (res == 0.0) ? 0.0 : INFINITY;
                            else q = fabs(res) / dn;
                            if (!(q == q)) q = INFINITY;
                            cw[r] = fmax(cw[r], q);
                        }
                    }
                }
#pragma unroll
                for (int r = 0; r < MAXRHS; ++r) {
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) cw[r] = fmax(cw[r], __shfl_xor_sync(0xffffffffu, cw[r], off));
                    if (lane == 0) S.red_m[warp][r] = cw[r];
                }
                __syncthreads();
                err = 0.0;
                for (int w = 0; w < NW; ++w)
                    for (int r = 0; r < nr; ++r) err = fmax(err, S.red_m[w][r]);
                if (err <= d.rtol || iter >= d.maxiter || !isfinite(err)) break;
                correct(true);
            }
            for (int r = warp; r < nr; r += NW)
                for (int i = lane; i < n; i += 32) Xo[i + (i64)r * ldxo] = sX[r * NMAX + i];
            if (tid == 0) {
                if (d.iters) d.iters[mi] = iter;
                if (d.berr) d.berr[mi] = err;
                if (!(err <= d.rtol)) atomicAdd(&d.status[3], 1);
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------
// Host side: launch, graph replay, autotuner
// ---------------------------------------------------------------------------
static int pick_tune(oxi_handle_s *h, int mode, BatchDesc &d) {
    using namespace bt;
    auto &tn = h->btune[mode == MODE_MIXED ? 1 : 0];
    if (!tn.tuned) {  // untuned defaults
        tn.n_smem = (mode == MODE_MIXED) ? 96 : 64;
        for (int b = 0; b < NBUCKET; ++b) tn.nb[b] = (b < 2) ? 8 : 16;
    }
    d.n_smem = tn.n_smem;
    d.nbmax = 8;
    for (int b = 0; b < NBUCKET; ++b) {
        d.nb[b] = tn.nb[b];
        d.nbmax = std::max(d.nbmax, tn.nb[b]);
    }
    return batch_smem_layout(mode == MODE_MIXED ? 4 : 8, mode, d.n_smem, d.nbmax, &d);
}

// Persistent grid: as many CTAs as fit on the SMs at this shared-memory size.
static int batch_grid(oxi_handle_s *h, int mode, int smem, int count) {
    using namespace bt;
    const void *kern = (mode == MODE_MIXED) ? (const void *)k_lu_batched<float> : (const void *)k_lu_batched<double>;
    int optin = 0;
    OXI_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    cudaFuncAttributes fa;
    OXI_CUDA(cudaFuncGetAttributes(&fa, kern));
    const int limit = optin - (int)fa.sharedSizeBytes;  // the kernel's own static shared memory
    if (smem > limit) throw CudaError{cudaErrorInvalidValue, "batched tuning exceeds shared memory"};
    set_max_dyn_smem(kern, limit);
    int per_sm = 0;
    OXI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
    if (per_sm < 1) throw CudaError{cudaErrorInvalidConfiguration, "batched LU does not fit an SM"};
    return std::max(1, std::min(count, per_sm * h->sm_count));
}

static void launch_batched(oxi_handle_s *h, const BatchDesc &d, int smem, int grid) {
    using namespace bt;
    cudaStream_t s = h->stream;
    const bool mixed = d.mode == MODE_MIXED;
    k_batch_order<<<1, 1024, 0, s>>>(d.n, d.count, (int32_t *)d.order, d.head, d.status);
    OXI_LAUNCH_CHECK();
    ProfScope ps(KC_OTHER, s, 0.0, 0.0);
    if (mixed) k_lu_batched<float><<<grid, NT, smem, s>>>(d);
    else k_lu_batched<double><<<grid, NT, smem, s>>>(d);
    OXI_LAUNCH_CHECK();
}

// Direct launch, or replay of the captured graph when the same call repeats.
static void run_batched(oxi_handle_s *h, const BatchDesc &d, int smem, int grid) {
    auto &gc = h->bgraph;
    std::vector<uint64_t> key((sizeof(BatchDesc) + 7) / 8 + 4, 0);
    std::memcpy(key.data(), &d, sizeof(BatchDesc));
    key[key.size() - 4] = (uint64_t)smem | ((uint64_t)grid << 32);
    key[key.size() - 3] = (uint64_t)(uintptr_t)h->stream;
    key[key.size() - 2] = (uint64_t)(uintptr_t)h->batch_wsp.ptr;
    key[key.size() - 1] = (uint64_t)(uintptr_t)h->batch_ctl.ptr;
    const bool usable = h->opt.graphs && !h->prof.enabled && h->stream != nullptr;
    const bool same = gc.seen > 0 && gc.key == key;
    if (usable && same && gc.exec) {
        OXI_CUDA(cudaGraphLaunch(gc.exec, h->stream));
        if (t_prof) t_prof->launches += gc.nlaunch;  // the replay's kernels count as launched
        return;
    }
    if (usable && same) {
        cudaStreamCaptureStatus st;
        OXI_CUDA(cudaStreamIsCapturing(h->stream, &st));
        if (st == cudaStreamCaptureStatusNone) {
            OXI_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
            const uint64_t before = t_prof ? t_prof->launches : 0;
            try {
                launch_batched(h, d, smem, grid);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(h->stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            OXI_CUDA(cudaStreamEndCapture(h->stream, &gc.graph));
            gc.nlaunch = (t_prof ? t_prof->launches : 0) - before;
            OXI_CUDA(cudaGraphInstantiate(&gc.exec, gc.graph, 0));
            gc.seen = 2;
            OXI_CUDA(cudaGraphLaunch(gc.exec, h->stream));
            return;
        }
    }
    if (!same) {
        gc.reset();
        gc.key = key;
    }
    gc.seen = std::max(gc.seen, 1);
    launch_batched(h, d, smem, grid);
}

static int finish_batched(oxi_handle_s *h, int32_t *d_status) {
    int32_t *hs = (int32_t *)h->host_ws.get(64);
    OXI_CUDA(cudaMemcpyAsync(hs, d_status, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    OXI_CUDA(cudaStreamSynchronize(h->stream));
    if (hs[1]) return OXI_EINVAL;
    if (hs[2]) return OXI_ENONFINITE;
    if (hs[0]) return OXI_ESINGULAR;
    if (hs[3]) return OXI_ENOTCONVERGED;
    return OXI_OK;
}

static int batched_entry(oxi_handle_s *h, int mode, int64_t count, const int32_t *d_n, const int32_t *d_nrhs,
                         double *const *d_A, const int64_t *d_lda, int64_t *const *d_ipiv, double *const *d_B,
                         const int64_t *d_ldb, double *const *d_X, const int64_t *d_ldx, int32_t *d_info,
                         int32_t *d_iters, double *d_berr, int maxiter, double rtol) {
    using namespace bt;
    if (!h || count < 0 || count > INT32_MAX) return OXI_EINVAL;
    if (count == 0) return OXI_OK;
    if (!d_n || !d_A || !d_lda || !d_info) return OXI_EINVAL;
    if (mode != MODE_GETRF && (!d_nrhs || !d_B || !d_ldb)) return OXI_EINVAL;
    if (mode == MODE_MIXED && (!d_X || !d_ldx || maxiter < 0 || !(rtol >= 0.0))) return OXI_EINVAL;
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        BatchDesc d;
        std::memset(&d, 0, sizeof(d));  // the bytes form the graph key
        d.count = (int)count;
        d.mode = mode;
        d.n = d_n;
        d.A = d_A;
        d.lda = d_lda;
        d.ipiv = d_ipiv;
        d.info = d_info;
        d.nrhs = d_nrhs;
        d.B = d_B;
        d.ldb = d_ldb;
        d.X = d_X;
        d.ldx = d_ldx;
        d.iters = d_iters;
        d.berr = d_berr;
        d.maxiter = maxiter;
        d.rtol = rtol;
        char *ctl = (char *)h->batch_ctl.get(sizeof(int32_t) * ((size_t)count + 64));
        d.head = (int32_t *)ctl;
        d.status = d.head + 16;
        d.order = d.head + 64;
        const int smem = pick_tune(h, mode, d);
        const int grid = batch_grid(h, mode, smem, d.count);
        if (mode == MODE_MIXED)  // one FP32 working matrix per CTA, sized before the graph key
            d.wsp = (float *)h->batch_wsp.get(sizeof(float) * (size_t)NMAX * NMAX * grid);
        run_batched(h, d, smem, grid);
        return finish_batched(h, d.status);
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

// ---------------------------------------------------------------------------
// Autotuner: times candidate panel widths per size bucket and shared-memory
// thresholds on synthetic matrices (N(0,1) entries + n I) of the caller's
// orders, keeps the fastest in the handle.
// ---------------------------------------------------------------------------
__global__ void k_fill_randn(double *A, i64 rows, i64 cols, i64 lda, double shift, uint64_t seed) {
    const i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * cols) return;
    const i64 r = e % rows, c = e / rows;
    // splitmix64 -> two uniforms in (0, 1) -> Box-Muller
    auto mix = [](uint64_t x) {
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        return x ^ (x >> 31);
    };
    const uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(e + 1);
    const double u1 = ((mix(z) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    const double u2 = ((mix(z ^ 0xD1B54A32D192ED03ull) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    double g = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    if (r == c) g += shift;
    A[r + c * lda] = g;
}

}  // namespace oxi

using oxi::bt::MODE_GESV;
using oxi::bt::MODE_GETRF;
using oxi::bt::MODE_MIXED;

extern "C" int oxi_dgetrf_batched_uneven(oxi_handle_t h, int64_t count, const int32_t *d_n, double *const *d_A,
                                         const int64_t *d_lda, int64_t *const *d_ipiv, int32_t *d_info) {
    return oxi::batched_entry(h, MODE_GETRF, count, d_n, nullptr, d_A, d_lda, d_ipiv, nullptr, nullptr, nullptr,
                              nullptr, d_info, nullptr, nullptr, 0, 0.0);
}

extern "C" int oxi_dgesv_batched_uneven(oxi_handle_t h, int prec, int64_t count, const int32_t *d_n,
                                        const int32_t *d_nrhs, double *const *d_A, const int64_t *d_lda,
                                        int64_t *const *d_ipiv, double *const *d_B, const int64_t *d_ldb,
                                        double *const *d_X, const int64_t *d_ldx, int32_t *d_info,
                                        int32_t *d_iters, double *d_berr, int maxiter, double rtol) {
    if (prec == OXI_PREC_FP64)
        return oxi::batched_entry(h, MODE_GESV, count, d_n, d_nrhs, d_A, d_lda, d_ipiv, d_B, d_ldb, nullptr,
                                  nullptr, d_info, nullptr, nullptr, 0, 0.0);
    if (prec == OXI_PREC_FP32)
        return oxi::batched_entry(h, MODE_MIXED, count, d_n, d_nrhs, d_A, d_lda, d_ipiv, d_B, d_ldb, d_X, d_ldx,
                                  d_info, d_iters, d_berr, maxiter, rtol);
    return OXI_EINVAL;
}

namespace oxi {

// Time one configuration of the tuning on the synthetic batch (best of reps).
static float time_batched(oxi_handle_s *h, BatchDesc d, const int (&nb)[bt::NBUCKET], int n_smem,
                          const std::vector<std::pair<void *, const void *>> &restore,
                          const std::vector<size_t> &restore_bytes, int reps) {
    using namespace bt;
    d.n_smem = n_smem;
    d.nbmax = 8;
    for (int b = 0; b < NBUCKET; ++b) {
        d.nb[b] = nb[b];
        d.nbmax = std::max(d.nbmax, nb[b]);
    }
    const int smem = batch_smem_layout(d.mode == MODE_MIXED ? 4 : 8, d.mode, n_smem, d.nbmax, &d);
    int optin = 0;
    OXI_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    if (smem + (int)sizeof(Misc) + 256 > optin) return INFINITY;  // static part: Misc plus alignment
    const int grid = batch_grid(h, d.mode, smem, d.count);
    if (d.mode == MODE_MIXED) d.wsp = (float *)h->batch_wsp.get(sizeof(float) * (size_t)NMAX * NMAX * grid);
    cudaEvent_t e0, e1;
    OXI_CUDA(cudaEventCreate(&e0));
    OXI_CUDA(cudaEventCreate(&e1));
    float best = INFINITY;
    for (int r = 0; r < reps; ++r) {
        for (size_t i = 0; i < restore.size(); ++i)
            OXI_CUDA(cudaMemcpyAsync(restore[i].first, restore[i].second, restore_bytes[i], cudaMemcpyDeviceToDevice,
                                     h->stream));
        OXI_CUDA(cudaEventRecord(e0, h->stream));
        launch_batched(h, d, smem, grid);
        OXI_CUDA(cudaEventRecord(e1, h->stream));
        OXI_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        OXI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

static int batched_autotune(oxi_handle_s *h, int prec, int64_t count, const int32_t *h_n, int nrhs,
                            double *best_ms) {
    using namespace bt;
    if (!h || !h_n || count <= 0 || count > INT32_MAX || nrhs < 1 || nrhs > MAXRHS) return OXI_EINVAL;
    if (prec != OXI_PREC_FP64 && prec != OXI_PREC_FP32) return OXI_EINVAL;
    for (int64_t i = 0; i < count; ++i)
        if (h_n[i] < 1 || h_n[i] > NMAX) return OXI_EINVAL;
    const int mode = prec == OXI_PREC_FP64 ? MODE_GESV : MODE_MIXED;
    std::vector<void *> allocs;
    auto dalloc = [&](size_t bytes) {
        void *p = nullptr;
        OXI_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 256)));
        allocs.push_back(p);
        return p;
    };
    int rc = OXI_OK;
    try {
        OXI_CUDA(cudaSetDevice(h->device));
        h->bgraph.reset();
        const int cnt = (int)count;
        std::vector<size_t> offA(cnt), offB(cnt);
        size_t totA = 0, totB = 0;
        for (int i = 0; i < cnt; ++i) {
            offA[i] = totA;
            offB[i] = totB;
            totA += (size_t)h_n[i] * h_n[i];
            totB += (size_t)h_n[i] * nrhs;
        }
        double *A0 = (double *)dalloc(8 * totA), *A = (double *)dalloc(8 * totA);
        double *B0 = (double *)dalloc(8 * totB), *Bw = (double *)dalloc(8 * totB), *X = (double *)dalloc(8 * totB);
        std::vector<double *> pa(cnt), pb(cnt), px(cnt);
        std::vector<int64_t> ld(cnt);
        std::vector<int32_t> nr(cnt, nrhs);
        for (int i = 0; i < cnt; ++i) {
            pa[i] = A + offA[i];
            pb[i] = Bw + offB[i];
            px[i] = X + offB[i];
            ld[i] = h_n[i];
            const i64 e = (i64)h_n[i] * h_n[i];
            k_fill_randn<<<(unsigned)((e + 255) / 256), 256, 0, h->stream>>>(A0 + offA[i], h_n[i], h_n[i], h_n[i],
                                                                            (double)h_n[i], 0x5EEDull * (i + 1));
            OXI_LAUNCH_CHECK();
        }
        k_fill_randn<<<(unsigned)((totB + 255) / 256), 256, 0, h->stream>>>(B0, (i64)totB, 1, (i64)totB, 0.0,
                                                                           0xB0B0ull);
        OXI_LAUNCH_CHECK();
        int32_t *dn = (int32_t *)dalloc(4 * cnt), *dnr = (int32_t *)dalloc(4 * cnt), *dinfo = (int32_t *)dalloc(4 * cnt);
        int32_t *dit = (int32_t *)dalloc(4 * cnt);
        double *dbe = (double *)dalloc(8 * cnt);
        int64_t *dld = (int64_t *)dalloc(8 * cnt);
        double **dpa = (double **)dalloc(8 * cnt), **dpb = (double **)dalloc(8 * cnt), **dpx = (double **)dalloc(8 * cnt);
        OXI_CUDA(cudaMemcpy(dn, h_n, 4 * cnt, cudaMemcpyHostToDevice));
        OXI_CUDA(cudaMemcpy(dnr, nr.data(), 4 * cnt, cudaMemcpyHostToDevice));
        OXI_CUDA(cudaMemcpy(dld, ld.data(), 8 * cnt, cudaMemcpyHostToDevice));
        OXI_CUDA(cudaMemcpy(dpa, pa.data(), 8 * cnt, cudaMemcpyHostToDevice));
        OXI_CUDA(cudaMemcpy(dpb, pb.data(), 8 * cnt, cudaMemcpyHostToDevice));
        OXI_CUDA(cudaMemcpy(dpx, px.data(), 8 * cnt, cudaMemcpyHostToDevice));
        BatchDesc d;
        std::memset(&d, 0, sizeof(d));
        d.count = cnt;
        d.mode = mode;
        d.n = dn;
        d.A = dpa;
        d.lda = dld;
        d.info = dinfo;
        d.nrhs = dnr;
        d.B = dpb;
        d.ldb = dld;
        d.X = dpx;
        d.ldx = dld;
        d.iters = dit;
        d.berr = dbe;
        d.maxiter = 10;
        d.rtol = 1e-13;
        char *ctl = (char *)h->batch_ctl.get(sizeof(int32_t) * ((size_t)cnt + 64));
        d.head = (int32_t *)ctl;
        d.status = d.head + 16;
        d.order = d.head + 64;
        std::vector<std::pair<void *, const void *>> restore = {{A, A0}, {Bw, B0}};
        std::vector<size_t> restore_bytes = {8 * totA, 8 * totB};
        bool present[NBUCKET] = {};
        for (int i = 0; i < cnt; ++i) present[(h_n[i] - 1) >> 5] = true;
        const int smem_cands[5] = {0, 64, 96, 128, mode == MODE_MIXED ? 160 : 112};
        const int nb_cands[3] = {8, 16, 32};
        int nb[NBUCKET];
        for (int b = 0; b < NBUCKET; ++b) nb[b] = 16;
        int best_smem = 0;
        float best = INFINITY;
        auto sweep_smem = [&]() {
            for (int sm : smem_cands) {
                const float t = time_batched(h, d, nb, sm, restore, restore_bytes, 2);
                if (t < best) {
                    best = t;
                    best_smem = sm;
                }
            }
        };
        sweep_smem();
        for (int b = 0; b < NBUCKET; ++b) {
            if (!present[b]) continue;
            int keep = nb[b];
            for (int c : nb_cands) {
                if (c == keep) continue;
                nb[b] = c;
                const float t = time_batched(h, d, nb, best_smem, restore, restore_bytes, 2);
                if (t < best) {
                    best = t;
                    keep = c;
                }
            }
            nb[b] = keep;
        }
        sweep_smem();
        auto &tn = h->btune[mode == MODE_MIXED ? 1 : 0];
        tn.tuned = true;
        tn.n_smem = best_smem;
        for (int b = 0; b < NBUCKET; ++b) tn.nb[b] = nb[b];
        if (best_ms) *best_ms = best;
        OXI_CUDA(cudaStreamSynchronize(h->stream));
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        rc = OXI_ECUDA;
    }
    cudaStreamSynchronize(h->stream);
    for (void *p : allocs) cudaFree(p);
    return rc;
}

}  // namespace oxi

extern "C" int oxi_batched_autotune(oxi_handle_t h, int prec, int64_t count, const int32_t *h_n, int32_t nrhs,
                                    double *best_ms) {
    return oxi::batched_autotune(h, prec, count, h_n, nrhs, best_ms);
}

extern "C" int oxi_batched_get_tuning(oxi_handle_t h, int prec, int32_t *n_smem, int32_t *nb) {
    if (!h || !n_smem || !nb || (prec != OXI_PREC_FP64 && prec != OXI_PREC_FP32)) return OXI_EINVAL;
    oxi::BatchDesc d;
    std::memset(&d, 0, sizeof(d));
    oxi::pick_tune(h, prec == OXI_PREC_FP64 ? MODE_GESV : MODE_MIXED, d);
    *n_smem = d.n_smem;
    for (int b = 0; b < oxi::bt::NBUCKET; ++b) nb[b] = d.nb[b];
    return OXI_OK;
}

extern "C" int oxi_batched_set_tuning(oxi_handle_t h, int prec, int32_t n_smem, const int32_t *nb) {
    if (!h || !nb || (prec != OXI_PREC_FP64 && prec != OXI_PREC_FP32)) return OXI_EINVAL;
    if (n_smem < 0 || n_smem > oxi::bt::NMAX) return OXI_EINVAL;
    for (int b = 0; b < oxi::bt::NBUCKET; ++b)
        if (nb[b] != 8 && nb[b] != 16 && nb[b] != 32) return OXI_EINVAL;
    const int esize = prec == OXI_PREC_FP64 ? 8 : 4;
    int nbmax = 8;
    for (int b = 0; b < oxi::bt::NBUCKET; ++b) nbmax = std::max(nbmax, (int)nb[b]);
    const int smem = oxi::batch_smem_layout(esize, prec == OXI_PREC_FP64 ? MODE_GESV : MODE_MIXED, n_smem, nbmax,
                                            nullptr);
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device) != cudaSuccess)
        return OXI_ECUDA;
    if (smem + (int)sizeof(oxi::Misc) + 256 > optin) return OXI_EINVAL;
    auto &tn = h->btune[prec == OXI_PREC_FP64 ? 0 : 1];
    tn.tuned = true;
    tn.n_smem = n_smem;
    for (int b = 0; b < oxi::bt::NBUCKET; ++b) tn.nb[b] = nb[b];
    h->bgraph.reset();
    return OXI_OK;
}
