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
