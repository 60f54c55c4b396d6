// Adjoint (reverse-mode rule) of X = A \ B with stored LU factors.
//
// For a loss L(X) with upstream gradient Xbar = dL/dX:
//   Bbar   = A^-T Xbar      -- the transposed solve with the factors already
//                             computed, the primitive behind ldiv!(transpose(F), B)
//                             (src/api/linalg_api.jl:176-184) and solve_transposed
//                             (src/lapack/expert_refinement.jl:2-23);
//   Abar   = -Bbar X^T      -- a rank-nrhs outer product written once.
// The reference has no differentiation rule of its own; this is the rule a
// ChainRulesCore rrule for x = A \ b returns, with the factorization reused.
//
// Abar is n^2 doubles and nothing else in the rule is larger, so its write
// bounds the kernel: one pass, 16-byte streaming stores, the small operands
// (Bbar rows in registers, X rows broadcast from shared memory) read once per
// CTA.
#include <algorithm>
#include "oxi_internal.h"

namespace oxi {

namespace {
constexpr int ADJ_NT = 256;   // threads per CTA: 2 rows each
constexpr int ADJ_ROWS = 2 * ADJ_NT;
constexpr int ADJ_COLS = 32;  // columns of Abar per CTA
constexpr int ADJ_KMAX = 16;  // right-hand sides per pass
}  // namespace

// Abar[i, j] (+)= -sum_k L[i, k] X[j, k], column-major, for k in [0, kc).
template <int KC, bool VEC>
__global__ void __launch_bounds__(ADJ_NT)
k_neg_outer(const double *__restrict__ L, i64 ldl, const double *__restrict__ X, i64 ldx, int n,
            double *__restrict__ Abar, i64 ldab, int accumulate) {
    __shared__ double sx[ADJ_COLS][KC];
    const int i = blockIdx.x * ADJ_ROWS + 2 * threadIdx.x;
    const int j0 = blockIdx.y * ADJ_COLS;
    const int cols = min(ADJ_COLS, n - j0);
    for (int e = threadIdx.x; e < ADJ_COLS * KC; e += ADJ_NT) {
        const int jj = e / KC, k = e % KC;
        sx[jj][k] = (jj < cols) ? X[(i64)(j0 + jj) + (i64)k * ldx] : 0.0;
    }
    __syncthreads();
    if (i >= n) return;
    const bool two = i + 1 < n;
    double l0[KC], l1[KC];
#pragma unroll
    for (int k = 0; k < KC; ++k) {
        l0[k] = L[i + (i64)k * ldl];
        l1[k] = two ? L[i + 1 + (i64)k * ldl] : 0.0;
    }
    for (int jj = 0; jj < cols; ++jj) {
        double v0 = 0.0, v1 = 0.0;
#pragma unroll
        for (int k = 0; k < KC; ++k) {
            v0 = fma(l0[k], sx[jj][k], v0);
            v1 = fma(l1[k], sx[jj][k], v1);
        }
        double *col = Abar + (i64)(j0 + jj) * ldab + i;
        if (VEC && two) {
            double2 w;
            if (accumulate) {
                const double2 o = __ldcs((const double2 *)col);
                w.x = o.x - v0;
                w.y = o.y - v1;
            } else {
                w.x = -v0;
                w.y = -v1;
            }
            __stcs((double2 *)col, w);
        } else {
            col[0] = accumulate ? col[0] - v0 : -v0;
            if (two) col[1] = accumulate ? col[1] - v1 : -v1;
        }
    }
}

template <int KC>
static void neg_outer_launch(const double *L, i64 ldl, const double *X, i64 ldx, i64 n, double *Abar,
                             i64 ldab, int accumulate, cudaStream_t s) {
    const bool vec = ((ldab & 1) == 0) && (((uintptr_t)Abar & 15) == 0);
    dim3 grid((unsigned)((n + ADJ_ROWS - 1) / ADJ_ROWS), (unsigned)((n + ADJ_COLS - 1) / ADJ_COLS));
    ProfScope ps(KC_OTHER, s, 2.0 * n * n * KC, 8.0 * n * n * (accumulate ? 2 : 1));
    if (vec)
        k_neg_outer<KC, true><<<grid, ADJ_NT, 0, s>>>(L, ldl, X, ldx, (int)n, Abar, ldab, accumulate);
    else
        k_neg_outer<KC, false><<<grid, ADJ_NT, 0, s>>>(L, ldl, X, ldx, (int)n, Abar, ldab, accumulate);
    OXI_LAUNCH_CHECK();
}

// Abar = -L X^T over right-hand-side chunks of at most ADJ_KMAX.
static void neg_outer(const double *L, i64 ldl, const double *X, i64 ldx, i64 n, i64 nrhs, double *Abar,
                      i64 ldab, cudaStream_t s) {
    for (i64 k0 = 0; k0 < nrhs; k0 += ADJ_KMAX) {
        const i64 kc = std::min<i64>(ADJ_KMAX, nrhs - k0);
        const double *Lk = L + k0 * ldl, *Xk = X + k0 * ldx;
        const int acc = k0 > 0;
        switch (kc) {
#define OXI_ADJ_CASE(K) \
    case K: neg_outer_launch<K>(Lk, ldl, Xk, ldx, n, Abar, ldab, acc, s); break;
            OXI_ADJ_CASE(1) OXI_ADJ_CASE(2) OXI_ADJ_CASE(3) OXI_ADJ_CASE(4)
            OXI_ADJ_CASE(5) OXI_ADJ_CASE(6) OXI_ADJ_CASE(7) OXI_ADJ_CASE(8)
            OXI_ADJ_CASE(9) OXI_ADJ_CASE(10) OXI_ADJ_CASE(11) OXI_ADJ_CASE(12)
            OXI_ADJ_CASE(13) OXI_ADJ_CASE(14) OXI_ADJ_CASE(15) OXI_ADJ_CASE(16)
#undef OXI_ADJ_CASE
            default: throw CudaError{cudaErrorInvalidValue, "adjoint chunk"};
        }
    }
}

}  // namespace oxi

extern "C" int oxi_dlu_adjoint(oxi_handle_t h, int64_t n, int64_t nrhs, const double *dLU, int64_t lda,
                               const int64_t *d_ipiv, const double *dX, int64_t ldx, const double *dXbar,
                               int64_t ldxbar, double *dBbar, int64_t ldbbar, double *dAbar,
                               int64_t ldabar) {
    using oxi::i64;
    if (!h || n < 0 || nrhs < 0) return OXI_EINVAL;
    const i64 mn = std::max<i64>(1, n);
    if (lda < mn || ldx < mn || ldxbar < mn || ldbbar < mn || ldabar < mn) return OXI_EINVAL;
    if (n == 0) return OXI_OK;
    if (!dLU || !d_ipiv || !dAbar || (nrhs > 0 && (!dX || !dXbar || !dBbar))) return OXI_EINVAL;
    if (dBbar == dXbar && ldbbar != ldxbar) return OXI_EINVAL;
    if (nrhs == 0) {  // no right-hand side: the gradient of A is zero
        try {
            OXI_CUDA(cudaSetDevice(h->device));
            OXI_CUDA(cudaMemset2DAsync(dAbar, ldabar * sizeof(double), 0, n * sizeof(double), n, h->stream));
            OXI_CUDA(cudaStreamSynchronize(h->stream));
            return OXI_OK;
        } catch (const oxi::CudaError &e) {
            h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
            return OXI_ECUDA;
        }
    }
    try {
        OXI_CUDA(cudaSetDevice(h->device));
        if (dBbar != dXbar)
            OXI_CUDA(cudaMemcpy2DAsync(dBbar, ldbbar * sizeof(double), dXbar, ldxbar * sizeof(double),
                                       n * sizeof(double), nrhs, cudaMemcpyDeviceToDevice, h->stream));
    } catch (const oxi::CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
    // Bbar = A^-T Xbar through the stored factors (synchronises once)
    const int st = oxi_dgetrs(h, 'T', n, nrhs, dLU, lda, d_ipiv, dBbar, ldbbar);
    if (st != OXI_OK) return st;
    try {
        oxi::ProfGuard pg(&h->prof);
        oxi::neg_outer(dBbar, ldbbar, dX, ldx, n, nrhs, dAbar, ldabar, h->stream);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        return OXI_OK;
    } catch (const oxi::CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

// ---------------------------------------------------------------------------
// Batched adjoint: the same rule for many independent small factorizations
// (the stored factors of oxi_dgetrf_batched_uneven / oxi_dgesv_batched_uneven),
// one CTA per problem.  Per problem i (order n <= 256, k <= 8 right-hand sides):
//   Bbar = A^-T Xbar  -- U^T W = Xbar (forward), L^T V = W (backward, unit
//                        diagonal), Bbar = the interchanges undone in reverse
//                        order (as ldiv!(transpose(F), B), src/api/linalg_api.jl:
//                        176-184);
//   Abar = -Bbar X^T  -- n x n, written once, coalesced down the columns.
// Each right-hand side's two substitutions run on one warp: step i requests
// all of the lane's rows of the contiguous column i of the factors at once
// (coalesced, with U[i,i]), reduces them against the solved entries across
// the warp, and lane 0 finishes the step.
// ---------------------------------------------------------------------------
namespace oxi {
namespace {
constexpr int BADJ_NT = 256, BADJ_NMAX = 256, BADJ_KMAX = 8;
}

struct BatchAdjDesc {
    int count;
    const int32_t *n, *nrhs;
    double *const *LU;
    const int64_t *ldlu;
    int64_t *const *ipiv;
    double *const *X;
    const int64_t *ldx;
    double *const *Xbar;
    const int64_t *ldxbar;
    double *const *Bbar;
    const int64_t *ldbbar;
    double *const *Abar;
    const int64_t *ldabar;
    int32_t *info;
    int *status;  // [0] invalid problems, [1] singular ones
};

__device__ __forceinline__ double warp_sum(double v) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

__global__ void __launch_bounds__(BADJ_NT, 8) k_lu_adjoint_batched(const __grid_constant__ BatchAdjDesc d) {
    __shared__ double s_w[BADJ_KMAX][BADJ_NMAX];  // Xbar -> W -> V -> Bbar, per right-hand side
    __shared__ int s_ip[BADJ_NMAX];               // the interchanges, 0-based
    __shared__ int s_bad;
    const int pi = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = d.n[pi], k = d.nrhs ? d.nrhs[pi] : 1;
    const double *LU = d.LU[pi];
    const i64 ld = d.ldlu[pi], ldx = d.ldx[pi], ldxb = d.ldxbar[pi], ldbb = d.ldbbar[pi], ldab = d.ldabar[pi];
    const bool bad = n < 0 || n > BADJ_NMAX || k < 0 || k > BADJ_KMAX || (n > 0 && (!LU || !d.ipiv[pi] || !d.Abar[pi])) ||
                     (n > 0 && k > 0 && (!d.X[pi] || !d.Xbar[pi] || !d.Bbar[pi])) || (n > 0 && (ld < n || ldab < n)) ||
                     (n > 0 && k > 0 && (ldx < n || ldxb < n || ldbb < n));
    if (bad) {
        if (tid == 0) {
            d.info[pi] = -1;
            atomicAdd(&d.status[0], 1);
        }
        return;
    }
    if (tid == 0) s_bad = 0;
    if (n == 0) {
        if (tid == 0) d.info[pi] = 0;
        return;
    }
    const double *Xb = d.Xbar[pi], *X = d.X[pi];
    for (int e = tid; e < n * k; e += BADJ_NT) {
        const int i = e % n, r = e / n;
        s_w[r][i] = Xb[i + (i64)r * ldxb];
    }
    for (int j = tid; j < n; j += BADJ_NT) s_ip[j] = (int)d.ipiv[pi][j] - 1;
    __syncthreads();
    if (warp < k) {
        double *w = s_w[warp];
        // U^T W = Xbar: w_i = (xbar_i - sum_{p<i} U[p,i] w_p) / U[i,i]
        for (int i = 0; i < n; ++i) {
            const double *col = LU + (i64)i * ld;
            const double u = lane == 0 ? col[i] : 0.0;  // requested with the column
            double cv[BADJ_NMAX / 32];  // the lane's rows, all requested together
#pragma unroll
            for (int q = 0; q < BADJ_NMAX / 32; ++q) cv[q] = (lane + 32 * q < i) ? col[lane + 32 * q] : 0.0;
            double acc = 0.0;
#pragma unroll
            for (int q = 0; q < BADJ_NMAX / 32; ++q)
                if (lane + 32 * q < i) acc = fma(cv[q], w[lane + 32 * q], acc);
            acc = warp_sum(acc);
            if (lane == 0) {
                if (u == 0.0) s_bad = i + 1;
                w[i] = (w[i] - acc) / u;
            }
            __syncwarp();
        }
        // L^T V = W (unit): v_i = w_i - sum_{p>i} L[p,i] v_p
        for (int i = n - 1; i >= 0; --i) {
            const double *col = LU + (i64)i * ld;
            double cv[BADJ_NMAX / 32];
#pragma unroll
            for (int q = 0; q < BADJ_NMAX / 32; ++q) {
                const int p = i + 1 + lane + 32 * q;
                cv[q] = p < n ? col[p] : 0.0;
            }
            double acc = 0.0;
#pragma unroll
            for (int q = 0; q < BADJ_NMAX / 32; ++q) {
                const int p = i + 1 + lane + 32 * q;
                if (p < n) acc = fma(cv[q], w[p], acc);
            }
            acc = warp_sum(acc);
            if (lane == 0) w[i] -= acc;
            __syncwarp();
        }
        // the interchanges undone in reverse order
        if (lane == 0) {
            for (int j = n - 1; j >= 0; --j) {
                const int q = s_ip[j];
                if (q != j && q >= 0 && q < n) {
                    const double t = w[j];
                    w[j] = w[q];
                    w[q] = t;
                }
            }
        }
    }
    __syncthreads();
    double *Bb = d.Bbar[pi];
    for (int e = tid; e < n * k; e += BADJ_NT) {
        const int i = e % n, r = e / n;
        Bb[i + (i64)r * ldbb] = s_w[r][i];
    }
    double *Ab = d.Abar[pi];
    for (int e = tid; e < n * n; e += BADJ_NT) {
        const int i = e % n, j = e / n;
        double v = 0.0;
        for (int r = 0; r < k; ++r) v = fma(s_w[r][i], X[j + (i64)r * ldx], v);  // X[j, r]: one address a warp
        Ab[i + (i64)j * ldab] = -v;
    }
    if (tid == 0) {
        d.info[pi] = s_bad;
        if (s_bad) atomicAdd(&d.status[1], 1);
    }
}

}  // namespace oxi

extern "C" int oxi_dlu_adjoint_batched_uneven(oxi_handle_t h, int64_t count, const int32_t *d_n,
                                              const int32_t *d_nrhs, double *const *d_LU, const int64_t *d_ldlu,
                                              int64_t *const *d_ipiv, double *const *d_X, const int64_t *d_ldx,
                                              double *const *d_Xbar, const int64_t *d_ldxbar,
                                              double *const *d_Bbar, const int64_t *d_ldbbar,
                                              double *const *d_Abar, const int64_t *d_ldabar, int32_t *d_info) {
    using namespace oxi;
    if (!h || count < 0 || count >= (1ll << 31)) return OXI_EINVAL;
    if (count == 0) return OXI_OK;
    if (!d_n || !d_LU || !d_ldlu || !d_ipiv || !d_X || !d_ldx || !d_Xbar || !d_ldxbar || !d_Bbar || !d_ldbbar ||
        !d_Abar || !d_ldabar || !d_info)
        return OXI_EINVAL;
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        AbortScope ab(h);
        int *status = (int *)((char *)h->scratch.get(kScratchBytes) + kScratchErrOff + 64);
        OXI_CUDA(cudaMemsetAsync(status, 0, 2 * sizeof(int), h->stream));
        BatchAdjDesc d{(int)count, d_n, d_nrhs, d_LU, d_ldlu, d_ipiv, d_X, d_ldx, d_Xbar, d_ldxbar,
                       d_Bbar, d_ldbbar, d_Abar, d_ldabar, d_info, status};
        {
            ProfScope ps(KC_OTHER, h->stream, 0.0, 0.0);
            k_lu_adjoint_batched<<<(unsigned)count, BADJ_NT, 0, h->stream>>>(d);
            OXI_LAUNCH_CHECK();
        }
        int *hs = (int *)h->host_ws.get(64);
        OXI_CUDA(cudaMemcpyAsync(hs, status, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        queue_abort_read(h, hs + 4);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        const int we = check_abort(h, hs + 4);
        if (we != OXI_OK) return we;
        if (hs[0]) return OXI_EINVAL;
        return hs[1] ? OXI_ESINGULAR : OXI_OK;
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}
