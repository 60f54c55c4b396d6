// Triangular solves with the LU factors (ldiv!), column-major factors as the
// caller holds them.
//
// N: X = B[p, :], then L (unit lower) and U solves   (src/api/linalg_api.jl:168-175)
// T: U^T then L^T solves, then X[p, :] = X            (src/api/linalg_api.jl:176-184)
//
// Each triangular solve is ONE launch of k_trsv: a CTA takes the next 64-row
// block from an atomic ticket (so every block it waits on is already running,
// which rules out deadlock), accumulates the products with the solved blocks as
// their "done" flags appear (bounded spin; a timeout sets an error word and the
// kernel returns), solves its 64 x 64 diagonal block with warp shuffles, and
// publishes its rows.  The factor is read once, coalesced: threads run along
// the contiguous dimension of the factor (rows for L/U, columns for L^T/U^T).
#include <vector>
#include "oxi_internal.h"
#include "tma_util.cuh"

namespace oxi {

constexpr int SB = 64;        // rows per block
constexpr int SOLVE_NT = 256; // threads per CTA

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// M is the effective triangle: M(r, j) = TRANS ? A[j + r*lda] : A[r + j*lda].
// LOWER (of M) = (UPPER_A == TRANS).
template <typename T, bool UPPER_A, bool UNIT, bool TRANS, int NR>
__global__ void __launch_bounds__(SOLVE_NT)
k_trsv(const T *__restrict__ A, i64 lda, T *__restrict__ X, i64 ldx, int n, int *__restrict__ ticket,
       int *__restrict__ flags, int *__restrict__ err) {
    constexpr bool LOWER = (UPPER_A == TRANS);
    __shared__ int s_blk;
    __shared__ T sx[SB][NR];
    __shared__ T sD[SB][SB + 1];
    __shared__ T sred[4][SB][NR];
    __shared__ int s_abort;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nb = (n + SB - 1) / SB;
    if (t == 0) { s_blk = atomicAdd(ticket, 1); s_abort = 0; }
    __syncthreads();
    const int bi = s_blk;
    if (bi >= nb) return;
    const int b = LOWER ? bi : nb - 1 - bi;
    const int r0 = b * SB;
    const int rows = min(SB, n - r0);
    auto Mv = [&](int r, int j) -> T { return TRANS ? A[(i64)j + (i64)r * lda] : A[(i64)r + (i64)j * lda]; };

    // ---- products with the already-solved blocks ----
    // !TRANS: thread owns row rr = t % 64 and a quarter of each block's columns.
    // TRANS : lane owns columns (lane, lane+32) of each block, warp owns 8 rows.
    T acc[TRANS ? 8 : 1][NR];
#pragma unroll
    for (int a = 0; a < (TRANS ? 8 : 1); ++a)
#pragma unroll
        for (int k = 0; k < NR; ++k) acc[a][k] = T(0);

    for (int step = 0; step < bi; ++step) {
        const int c = LOWER ? step : nb - 1 - step;
        if (t == 0 && ld_acquire(&flags[c]) == 0) {
            const uint64_t t0 = global_ns();
            uint32_t it = 0;
            while (ld_acquire(&flags[c]) == 0) {
                if ((++it & 255) == 0 && global_ns() - t0 > kWaitLimitNs) {
                    atomicExch(err, 3);
                    s_abort = 1;
                    break;
                }
            }
        }
        __syncthreads();
        if (s_abort) return;
        const int c0 = c * SB;
        const int cols = min(SB, n - c0);
        for (int e = t; e < SB * NR; e += SOLVE_NT) {
            const int jj = e % SB, k = e / SB;
            sx[jj][k] = (jj < cols) ? __ldcg(&X[(i64)(c0 + jj) + (i64)k * ldx]) : T(0);
        }
        __syncthreads();
        if (!TRANS) {
            const int rr = t % SB, jg = t / SB;
            if (rr < rows) {
#pragma unroll 4
                for (int q = 0; q < SB / 4; ++q) {
                    const int jj = jg * (SB / 4) + q;
                    if (jj < cols) {
                        const T a = Mv(r0 + rr, c0 + jj);
#pragma unroll
                        for (int k = 0; k < NR; ++k) acc[0][k] = fma(a, sx[jj][k], acc[0][k]);
                    }
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int rr = warp + 8 * i;
                if (rr < rows) {
#pragma unroll
                    for (int hh = 0; hh < 2; ++hh) {
                        const int jj = lane + 32 * hh;
                        if (jj < cols) {
                            const T a = Mv(r0 + rr, c0 + jj);
#pragma unroll
                            for (int k = 0; k < NR; ++k) acc[i][k] = fma(a, sx[jj][k], acc[i][k]);
                        }
                    }
                }
            }
        }
        __syncthreads();
    }

    // ---- right-hand side of the diagonal block: y = b - acc ----
    if (!TRANS) {
        const int rr = t % SB, jg = t / SB;
#pragma unroll
        for (int k = 0; k < NR; ++k) sred[jg][rr][k] = acc[0][k];
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int k = 0; k < NR; ++k) {
                T v = acc[i][k];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
                if (lane == 0) sred[0][warp + 8 * i][k] = v;
            }
    }
    // diagonal block of M into shared memory
    for (int e = t; e < SB * SB; e += SOLVE_NT) {
        int r, j;
        if (!TRANS) { r = e % SB; j = e / SB; } else { j = e % SB; r = e / SB; }
        sD[r][j] = (r < rows && j < rows) ? Mv(r0 + r, r0 + j) : T(0);
    }
    __syncthreads();

    // ---- diagonal solve: warp k handles right-hand side k ----
    for (int k = warp; k < NR; k += SOLVE_NT / 32) {
        T y[2];
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            const int r = lane + 32 * hh;
            T s = T(0);
            if (!TRANS) s = sred[0][r][k] + sred[1][r][k] + sred[2][r][k] + sred[3][r][k];
            else s = sred[0][r][k];
            y[hh] = (r < rows) ? (X[(i64)(r0 + r) + (i64)k * ldx] - s) : T(0);
        }
        for (int step = 0; step < rows; ++step) {
            const int p = LOWER ? step : rows - 1 - step;
            const int hp = p >> 5, lp = p & 31;
            T yp = __shfl_sync(0xffffffffu, hp ? y[1] : y[0], lp);
            const T xp = UNIT ? yp : yp / sD[p][p];
            if (lane == lp) { if (hp) y[1] = xp; else y[0] = xp; }
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
                const int r = lane + 32 * hh;
                const bool below = LOWER ? (r > p) : (r < p);
                if (below && r < rows) y[hh] = fma(-sD[r][p], xp, y[hh]);
            }
        }
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            const int r = lane + 32 * hh;
            if (r < rows) X[(i64)(r0 + r) + (i64)k * ldx] = y[hh];
        }
    }
    __threadfence();
    __syncthreads();
    if (t == 0) st_release(&flags[b], 1);
}

template <typename T>
__global__ void k_gather_rows(const T *__restrict__ B, i64 ldb, const int64_t *__restrict__ perm,
                              T *__restrict__ X, i64 ldx, int n, int nrhs, int scatter) {
    const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (i64)n * nrhs) return;
    const int i = (int)(idx % n), k = (int)(idx / n);
    if (!scatter) X[i + (i64)k * ldx] = B[perm[i] + (i64)k * ldb];
    else X[perm[i] + (i64)k * ldx] = B[i + (i64)k * ldb];
}

template <typename T, bool UPPER_A, bool UNIT, bool TRANS>
static void trsv_launch(const T *A, i64 lda, T *X, i64 ldx, int n, int nrhs, int *ctl, int *err,
                        cudaStream_t s) {
    const int nb = (n + SB - 1) / SB;
    ProfScope ps(KC_TRSV, s, (double)n * n * nrhs, (double)n * n * sizeof(T) / 2);
    for (int k0 = 0; k0 < nrhs;) {
        const int left = nrhs - k0;
        OXI_CUDA(cudaMemsetAsync(ctl, 0, sizeof(int) * (nb + 1), s));
        int *ticket = ctl, *flags = ctl + 1;
        T *Xk = X + (i64)k0 * ldx;
        if (left >= 4) {
            k_trsv<T, UPPER_A, UNIT, TRANS, 4><<<nb, SOLVE_NT, 0, s>>>(A, lda, Xk, ldx, n, ticket, flags, err);
            k0 += 4;
        } else if (left >= 2) {
            k_trsv<T, UPPER_A, UNIT, TRANS, 2><<<nb, SOLVE_NT, 0, s>>>(A, lda, Xk, ldx, n, ticket, flags, err);
            k0 += 2;
        } else {
            k_trsv<T, UPPER_A, UNIT, TRANS, 1><<<nb, SOLVE_NT, 0, s>>>(A, lda, Xk, ldx, n, ticket, flags, err);
            k0 += 1;
        }
        OXI_LAUNCH_CHECK();
    }
}

// Solve with device-resident permutation `perm` (0-based, A[perm,:] = L U).
template <typename T>
void getrs_perm(oxi_handle_s *h, char trans, i64 n, i64 nrhs, const T *LU, i64 lda,
                const int64_t *d_perm, T *B, i64 ldb, int *d_err) {
    cudaStream_t s = h->stream;
    const i64 nb = (n + SB - 1) / SB;
    char *ws = (char *)h->solve_ws.get(sizeof(T) * (size_t)n * nrhs + sizeof(int) * (nb + 8) + 256);
    T *X = (T *)ws;
    int *ctl = (int *)(ws + ((sizeof(T) * (size_t)n * nrhs + 255) & ~size_t(255)));
    const i64 tot = n * nrhs;
    const int nt = 256;
    if (trans == 'N') {
        k_gather_rows<T><<<(unsigned)((tot + nt - 1) / nt), nt, 0, s>>>(B, ldb, d_perm, X, n, (int)n, (int)nrhs, 0);
        OXI_LAUNCH_CHECK();
        trsv_launch<T, false, true, false>(LU, lda, X, n, (int)n, (int)nrhs, ctl, d_err, s);
        trsv_launch<T, true, false, false>(LU, lda, X, n, (int)n, (int)nrhs, ctl, d_err, s);
        OXI_CUDA(cudaMemcpy2DAsync(B, ldb * sizeof(T), X, n * sizeof(T), n * sizeof(T), nrhs,
                                   cudaMemcpyDeviceToDevice, s));
    } else {
        OXI_CUDA(cudaMemcpy2DAsync(X, n * sizeof(T), B, ldb * sizeof(T), n * sizeof(T), nrhs,
                                   cudaMemcpyDeviceToDevice, s));
        trsv_launch<T, true, false, true>(LU, lda, X, n, (int)n, (int)nrhs, ctl, d_err, s);
        trsv_launch<T, false, true, true>(LU, lda, X, n, (int)n, (int)nrhs, ctl, d_err, s);
        k_gather_rows<T><<<(unsigned)((tot + nt - 1) / nt), nt, 0, s>>>(X, n, d_perm, B, ldb, (int)n, (int)nrhs, 1);
        OXI_LAUNCH_CHECK();
    }
}
template void getrs_perm<double>(oxi_handle_s *, char, i64, i64, const double *, i64, const int64_t *, double *, i64, int *);
template void getrs_perm<float>(oxi_handle_s *, char, i64, i64, const float *, i64, const int64_t *, float *, i64, int *);

// Row-major factors W are the column-major matrix W^T: L (lower) is then an
// upper-stored triangle read transposed, U likewise.
template <typename T>
void lu_solve_rowmajor(oxi_handle_s *h, const T *W, i64 ld, i64 n, T *X, i64 ldx, i64 nrhs,
                       int *d_err) {
    const i64 nb = (n + SB - 1) / SB;
    if (nb + 1 > kTrsvCtlInts) throw CudaError{cudaErrorInvalidValue, "system too large for the solve control block"};
    int *ctl = (int *)((char *)h->scratch.get(kScratchBytes) + kScratchTrsvOff);
    trsv_launch<T, true, true, true>(W, ld, X, ldx, (int)n, (int)nrhs, ctl, d_err, h->stream);
    trsv_launch<T, false, false, true>(W, ld, X, ldx, (int)n, (int)nrhs, ctl, d_err, h->stream);
}
template void lu_solve_rowmajor<float>(oxi_handle_s *, const float *, i64, i64, float *, i64, i64, int *);
template void lu_solve_rowmajor<double>(oxi_handle_s *, const double *, i64, i64, double *, i64, i64, int *);

// LUFactor.p from the interchange sequence (src/lapack/factorizations.jl:72-75).
void perm_from_ipiv(const int64_t *ipiv, i64 q, i64 m, int64_t *perm) {
    for (i64 i = 0; i < m; ++i) perm[i] = i;
    for (i64 j = 0; j < q; ++j) {
        const i64 p = ipiv[j] - 1;
        const int64_t t = perm[j];
        perm[j] = perm[p];
        perm[p] = t;
    }
}

template <typename T>
static int getrs_entry(oxi_handle_s *h, char trans, i64 n, i64 nrhs, const T *dLU, i64 lda,
                       const int64_t *d_ipiv, T *dB, i64 ldb) {
    if (!h) return OXI_EINVAL;
    if (trans == 'C') trans = 'T';
    if (trans != 'N' && trans != 'T') return OXI_EINVAL;
    if (n < 0 || nrhs < 0 || lda < std::max<i64>(1, n) || ldb < std::max<i64>(1, n)) return OXI_EINVAL;
    if (n == 0 || nrhs == 0) return OXI_OK;
    if (!dLU || !d_ipiv || !dB || n >= (1ll << 31)) return OXI_EINVAL;
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        // The interchange sequence is inherently sequential: fold it into the
        // permutation once on the host (n int64 each way).
        std::vector<int64_t> ip(n), perm(n);
        OXI_CUDA(cudaMemcpyAsync(ip.data(), d_ipiv, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, h->stream));
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        for (i64 j = 0; j < n; ++j)
            if (ip[j] < 1 || ip[j] > n) return OXI_EINVAL;
        perm_from_ipiv(ip.data(), n, n, perm.data());
        char *sc = (char *)h->scratch.get(kScratchBytes);
        int *d_err = (int *)(sc + kScratchErrOff);
        int64_t *dperm = (int64_t *)h->perm_ws.get(sizeof(int64_t) * n);
        int64_t *hperm = (int64_t *)h->host_ws.get(sizeof(int64_t) * (n + 8));
        std::copy(perm.begin(), perm.end(), hperm);
        OXI_CUDA(cudaMemcpyAsync(dperm, hperm, sizeof(int64_t) * n, cudaMemcpyHostToDevice, h->stream));
        OXI_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), h->stream));
        getrs_perm<T>(h, trans, n, nrhs, dLU, lda, dperm, dB, ldb, d_err);
        int *herr = (int *)(hperm + n);
        OXI_CUDA(cudaMemcpyAsync(herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        return *herr ? OXI_ETIMEOUT : OXI_OK;
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

}  // namespace oxi

extern "C" int oxi_dgetrs(oxi_handle_t h, char trans, int64_t n, int64_t nrhs, const double *dLU,
                          int64_t lda, const int64_t *d_ipiv, double *dB, int64_t ldb) {
    return oxi::getrs_entry<double>(h, trans, n, nrhs, dLU, lda, d_ipiv, dB, ldb);
}
extern "C" int oxi_sgetrs(oxi_handle_t h, char trans, int64_t n, int64_t nrhs, const float *dLU,
                          int64_t lda, const int64_t *d_ipiv, float *dB, int64_t ldb) {
    return oxi::getrs_entry<float>(h, trans, n, nrhs, dLU, lda, d_ipiv, dB, ldb);
}
