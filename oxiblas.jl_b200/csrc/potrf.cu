// Dense Cholesky factorization A = L L^T (FP64) and its solve.
//
// Replaces cholesky_factor / _cholesky_factor! (src/lapack/factorizations.jl:
// 205-291, LAPACK potrf2 recursion with 64-column leaves) and the solve of a
// CholeskyFactor (:293-305) behind OxiBLAS.cholesky / cholesky! and
// ldiv!(F::Cholesky, B) (src/api/linalg_api.jl:221-290).
//
// Layout: the lower triangle of the caller's column-major A, read with the
// same leading dimension as a ROW-major matrix, is the upper triangle of that
// matrix, and L (column-major, lower) is U = L^T (row-major, upper) in the same
// memory.  So the factorization runs in place, row-oriented, with no copy:
// blocks of NB rows of U, each
//   1. U_kk = chol(A_kk) and W = U_kk^-1, one CTA, the block in shared memory;
//   2. U_k,right = W^T A_k,right on the FP64 tensor cores (the block-row solve
//      as a product with the inverted diagonal block, into a scratch block row
//      X, then copied into place);
//   3. A_right,right -= X^T X on the FP64 tensor cores, upper triangle only
//      (tiles wholly below the diagonal skipped, crossing tiles write only on
//      and above it), its left operand a transposed copy of X so that both
//      operands are K-contiguous.
// The reference solves the block row by substitution (trsm!); the product with
// the inverted 128 x 128 block is the same solve with another association of
// the sums (the diagonal blocks of a positive definite matrix's factor are
// well conditioned: cond(U_kk)^2 <= cond(A)).
// A pivot that is not finite and positive stops the factorization there: info
// is its 1-based column (PosDefException(info)); the inverse of that block and
// of every later one is written as zero, so the later products change nothing,
// and the block rows are not copied back.
#include <algorithm>
#include <cmath>
#include "oxi_internal.h"
#include "tma_util.cuh"

namespace oxi {

namespace {
constexpr int PO_NB = 128;          // block rows per step
constexpr int PO_NT = 512;          // threads of the diagonal-block kernel (4 per column of the inverse)
}  // namespace

// Cholesky of the t x t diagonal block (row-major upper, ld) in shared memory:
// for each row c, d = sqrt(a_cc), the row scaled by d, then the rank-1 update
// of the upper triangle below it, a_ij = fma(-u_ci, u_cj, a_ij) for c < i <= j
// (the reference leaf's column updates, src/lapack/factorizations.jl:266-282,
// read through the transposition).  Then W = U^-1 by 32 x 32 diagonal blocks
// and the off-diagonal blocks of the 64 and 128 levels, W^T kept in the
// block's unused strict lower triangle, and
// Wneg = -W^T (t x t, row-major, lower) written for the block-row product.
template <typename T>
__global__ void __launch_bounds__(PO_NT) k_potrf_diag(T *__restrict__ U, i64 ld, int t, i64 g0,
                                                      int64_t *__restrict__ info, T *__restrict__ Wneg) {
    extern __shared__ __align__(16) unsigned char po_smem_raw[];
    const int lp = t + 1;
    T *S = (T *)po_smem_raw;
    T *s_inv = S + (size_t)t * lp;  // 1 / u_ii
    __shared__ int s_fail;
    const int tid = threadIdx.x;
    if (tid == 0) s_fail = (*(volatile int64_t *)info != 0) ? 1 : 0;
    __syncthreads();
    if (s_fail) {  // an earlier block failed: later products change nothing
        for (int e = tid; e < t * t; e += PO_NT) Wneg[e] = T(0);
        return;
    }
    for (int e = tid; e < t * t; e += PO_NT) {
        const int i = e / t, j = e - i * t;
        S[i * lp + j] = (j >= i) ? U[(i64)i * ld + j] : T(0);
    }
    __syncthreads();
    for (int c = 0; c < t; ++c) {
        T d = S[c * lp + c];
        if (!(d > T(0)) || !isfinite(d)) {  // not positive definite at global column g0 + c + 1
            if (tid == 0) {
                s_fail = 1;
                if (*info == 0) *info = g0 + c + 1;
            }
            break;
        }
        d = sqrt(d);
        // the row right of the pivot (the pivot itself is written after the
        // barrier: every thread has read it by then)
        for (int j = c + 1 + tid; j < t; j += PO_NT) S[c * lp + j] = S[c * lp + j] / d;
        __syncthreads();
        if (tid == 0) S[c * lp + c] = d;
        // rows i below c, columns j >= i: 16 row groups x 32 columns of threads
        const int tx = tid & 31, ty = tid >> 5;
        for (int i = c + 1 + ty; i < t; i += PO_NT / 32) {
            const T ui = S[c * lp + i];
            for (int j = i + tx; j < t; j += 32) S[i * lp + j] = fma(-ui, S[c * lp + j], S[i * lp + j]);
        }
        __syncthreads();
    }
    __syncthreads();
    for (int e = tid; e < t * t; e += PO_NT) {
        const int i = e / t, j = e - i * t;
        if (j >= i) U[(i64)i * ld + j] = S[i * lp + j];
    }
    if (s_fail) {
        for (int e = tid; e < t * t; e += PO_NT) Wneg[e] = T(0);
        return;
    }
    // W = U^-1 by blocks (only the full 128-row blocks have a block row to the
    // right; a shorter last block needs no inverse): the four 32 x 32 diagonal
    // blocks column by column (a thread per column, the columns independent),
    // then the off-diagonal block of each 64 x 64 and of the 128 x 128 level,
    //   W[A, C] = -W[A, A] (U[A, C] W[C, C]),
    // as two products in shared memory.  W (upper) is kept transposed in the
    // strict lower part of S (w_rc at S[c * lp + r], r < c), its diagonal in s_inv.
    if (t != PO_NB) {
        for (int e = tid; e < t * t; e += PO_NT) Wneg[e] = T(0);
        return;
    }
    for (int i = tid; i < t; i += PO_NT) s_inv[i] = T(1) / S[i * lp + i];
    __syncthreads();
    if (tid < t) {
        const int c = tid, b0 = c & ~31;
        for (int i = c - 1; i >= b0; --i) {
            T part = T(0);
            for (int p = i + 1; p <= c; ++p) part = fma(S[i * lp + p], (p == c) ? s_inv[c] : S[c * lp + p], part);
            S[c * lp + i] = -part * s_inv[i];
        }
    }
    __syncthreads();
    T *Tm = s_inv + t;  // (t / 2h) blocks of h x h: U[A, C] W[C, C]
    for (int hh = 32; hh < t; hh *= 2) {
        const int nel = (t / (2 * hh)) * hh * hh;
        for (int e = tid; e < nel; e += PO_NT) {
            const int blk = e / (hh * hh), rc = e - blk * hh * hh, r = rc / hh, c = rc - r * hh;
            const int a0 = blk * 2 * hh, c0 = a0 + hh;
            T acc = T(0);
            for (int p = 0; p <= c; ++p)
                acc = fma(S[(a0 + r) * lp + c0 + p], (p == c) ? s_inv[c0 + c] : S[(c0 + c) * lp + c0 + p], acc);
            Tm[e] = acc;
        }
        __syncthreads();
        for (int e = tid; e < nel; e += PO_NT) {
            const int blk = e / (hh * hh), rc = e - blk * hh * hh, r = rc / hh, c = rc - r * hh;
            const int a0 = blk * 2 * hh, c0 = a0 + hh;
            const T *tcol = Tm + blk * hh * hh + c;
            T acc = T(0);
            for (int q = r; q < hh; ++q) acc = fma((q == r) ? s_inv[a0 + r] : S[(a0 + q) * lp + a0 + r], tcol[q * hh], acc);
            S[(c0 + c) * lp + a0 + r] = -acc;
        }
        __syncthreads();
    }
    // Wneg = -W^T: row i holds -w_pi for p <= i
    for (int e = tid; e < t * t; e += PO_NT) {
        const int i = e / t, p = e - i * t;
        Wneg[e] = (p < i) ? -S[i * lp + p] : (p == i ? -s_inv[i] : T(0));
    }
}

// The solved block row back into place (row-major t x N), unless the
// factorization failed.
template <typename T>
__global__ void k_copy_block_row(const T *__restrict__ X, i64 ldx, T *__restrict__ B, i64 ldb, int t,
                                 i64 N, const int64_t *__restrict__ info) {
    if (*(volatile const int64_t *)info != 0) return;
    const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (i64)t * N) return;
    const i64 i = idx / N, c = idx - i * N;
    B[i * ldb + c] = X[i * ldx + c];
}

// The strict lower triangle of the row-major view (the strict upper triangle
// of the caller's column-major matrix) set to zero, as the reference does.
template <typename T>
__global__ void k_zero_strict_lower(T *__restrict__ U, i64 ld, int n, const int64_t *__restrict__ info) {
    if (*info != 0) return;  // as the reference: a failed factorization keeps its other triangle
    const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (i64)n * n) return;
    const int i = (int)(idx / n), j = (int)(idx - (i64)i * n);
    if (j < i) U[(i64)i * ld + j] = T(0);
}

// Workspace of one factorization, in elements: T (n x NB) and X (NB x ldx),
// two of each (the lookahead's update of block k reads them while block k + 1
// writes the other pair), Bc (NB x ldx), Wneg (NB x NB).
size_t potrf_work_elems(i64 n) {
    const i64 ldx = (n + 3) / 4 * 4;
    return 2 * (size_t)n * PO_NB + 3 * (size_t)PO_NB * ldx + (size_t)PO_NB * PO_NB + 64;
}

// X (t x N) = 0 - Wneg B and the symmetric update A22 -= T X (T = X^T), upper
// triangle of the row-major view: FP64 on the DMMA tensor-core GEMM; FP32 (the
// mixed solve's low-precision factor, a private copy) with the product on the
// CUDA cores and the update in the handle's trailing precision (tcgen05 for the
// 16-bit kinds; the whole square, the other triangle being scratch there).
static void po_block_row(oxi_handle_s *h, double *X, i64 ldx, const double *Wneg, int t, const double *B, i64 ldb,
                         i64 N, cudaStream_t s) {
    launch_gemm_dmma(X, ldx, Wneg, t, B, ldb, t, N, t, s);
}
static void po_block_row(oxi_handle_s *, float *X, i64 ldx, const float *Wneg, int t, const float *B, i64 ldb,
                         i64 N, cudaStream_t s) {
    launch_gemm_simt<float>(X, ldx, Wneg, t, B, ldb, t, N, t, s);
}
// rows x N block of the symmetric update whose (0, 0) is on the diagonal
// (M <= N): FP64 only on and above the diagonal
static void po_sym_update(oxi_handle_s *, double *A22, i64 ld, const double *T, int t, const double *X, i64 ldx,
                          i64 M, i64 N, cudaStream_t s) {
    launch_gemm_dmma(A22, ld, T, t, X, ldx, M, N, t, s, /*upper_only=*/true);
}
static void po_sym_update(oxi_handle_s *h, float *A22, i64 ld, const float *T, int t, const float *X, i64 ldx,
                          i64 M, i64 N, cudaStream_t s) {
    if (h->trailing == TRAIL_NATIVE) launch_gemm_simt<float>(A22, ld, T, t, X, ldx, M, N, t, s);
    else gemm_trailing_f32(h, A22, ld, T, t, X, ldx, M, N, t);
}

// One factorization: U in place (row-major view), *d_info set on failure.
// With the lookahead (OXI_OPT_LOOKAHEAD, the reference GEMM mode excluded)
// block k's symmetric update is split: the next block's rows first, on the
// panel stream (they are what block k + 1 needs), the rest on the low-priority
// stream beside block k + 1's diagonal factor and block-row product; the
// next block's rows wait for that rest of block k - 1's update.  Every element
// is updated by the same products in the same order: the factor is the same.
template <typename T>
void potrf_rowmajor(oxi_handle_s *h, T *U, i64 ld, i64 n, int64_t *d_info, T *work) {
    const cudaStream_t caller = h->stream;
    const bool la = h->opt.lookahead && h->opt.gemm == 0 && n > 2 * PO_NB;
    const i64 ldx = (n + 3) / 4 * 4;  // 16-byte rows for the TMA-fed GEMMs
    T *Tt2[2] = {work, work + (size_t)n * PO_NB};
    T *X2[2] = {work + 2 * (size_t)n * PO_NB, work + 2 * (size_t)n * PO_NB + (size_t)PO_NB * ldx};
    T *Bc = X2[1] + (size_t)PO_NB * ldx;
    T *Wneg = Bc + (size_t)PO_NB * ldx;
    if (la) {
        ensure_lookahead_streams(h);
        OXI_CUDA(cudaEventRecord(h->la_in, caller));
        OXI_CUDA(cudaStreamWaitEvent(h->la_main, h->la_in, 0));
        h->stream = h->la_main;
    }
    const cudaStream_t s = h->stream;
    bool b_pending = false;
    try {
        for (i64 k0 = 0, kb = 0; k0 < n; k0 += PO_NB, ++kb) {
            const int t = (int)std::min<i64>(PO_NB, n - k0);
            T *Ukk = U + k0 * ld + k0;
            T *Tt = Tt2[kb & 1], *X = X2[kb & 1];
            {
                // the block, 1 / u_ii, and the inverse's product scratch (h x h at the top level)
                const size_t smem = sizeof(T) * ((size_t)t * (t + 1) + t + (size_t)(PO_NB / 2) * (PO_NB / 2));
                set_max_dyn_smem((const void *)k_potrf_diag<T>,
                                 (int)(sizeof(T) * (PO_NB * (PO_NB + 1) + PO_NB + (PO_NB / 2) * (PO_NB / 2))));
                ProfScope ps(KC_LEAF, s, (double)t * t * t * (2.0 / 3.0), 2.0 * sizeof(T) * t * t);
                k_potrf_diag<T><<<1, PO_NT, smem, s>>>(Ukk, ld, t, k0, d_info, Wneg);
                OXI_LAUNCH_CHECK();
            }
            const i64 right = n - k0 - t;
            if (right <= 0) break;
            T *Bk = Ukk + t;  // rows k0..k0+t, columns k0+t..n
            // the tensor-core GEMM reads its operands through TMA (16-byte aligned
            // rows); a block row at an odd offset or pitch is copied first
            const T *Bop = Bk;
            i64 ldb_op = ld;
            if ((uintptr_t)Bk % 16 != 0 || (ld * (i64)sizeof(T)) % 16 != 0) {
                OXI_CUDA(cudaMemcpy2DAsync(Bc, sizeof(T) * ldx, Bk, sizeof(T) * ld, sizeof(T) * right, (size_t)t,
                                           cudaMemcpyDeviceToDevice, s));
                Bop = Bc;
                ldb_op = ldx;
            }
            // X = 0 - (-W^T) A_k,right = U_kk^-T A_k,right
            OXI_CUDA(cudaMemsetAsync(X, 0, sizeof(T) * (size_t)t * ldx, s));
            po_block_row(h, X, ldx, Wneg, t, Bop, ldb_op, right, s);
            k_copy_block_row<T><<<(unsigned)(((i64)t * right + 255) / 256), 256, 0, s>>>(X, ldx, Bk, ld, t, right,
                                                                                        d_info);
            OXI_LAUNCH_CHECK();
            // Tt = X^T (right x t, row-major): X read as a column-major right x t matrix
            launch_cm_to_rm<T, T>(X, ldx, Tt, t, right, t, s);
            T *A22 = U + (k0 + t) * ld + (k0 + t);
            if (!la) {
                po_sym_update(h, A22, ld, Tt, t, X, ldx, right, right, s);
                continue;
            }
            // the next block's rows, after the rest of the previous update
            if (b_pending) {
                OXI_CUDA(cudaStreamWaitEvent(s, h->la_join, 0));
                b_pending = false;
            }
            const i64 t2 = std::min<i64>(PO_NB, right);
            po_sym_update(h, A22, ld, Tt, t, X, ldx, t2, right, s);
            if (right > t2) {  // the rest on the low-priority stream
                OXI_CUDA(cudaEventRecord(h->la_fork, s));
                OXI_CUDA(cudaStreamWaitEvent(h->la_stream, h->la_fork, 0));
                h->stream = h->la_stream;
                h->tc_slot = 1;
                // tcgen05: persistent clusters on every GPC but one, which stays free for
                // the next block's diagonal factor and block-row product
                if constexpr (sizeof(T) == 4) h->gemm_ctas = -64;
                po_sym_update(h, A22 + t2 * ld + t2, ld, Tt + t2 * t, t, X + t2, ldx, right - t2, right - t2,
                              h->la_stream);
                h->stream = s;
                h->tc_slot = 0;
                h->gemm_ctas = 0;
                OXI_CUDA(cudaEventRecord(h->la_join, h->la_stream));
                b_pending = true;
            }
        }
        if (b_pending) OXI_CUDA(cudaStreamWaitEvent(s, h->la_join, 0));
        const i64 tot = n * n;
        k_zero_strict_lower<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(U, ld, (int)n, d_info);
        OXI_LAUNCH_CHECK();
        if (la) {
            OXI_CUDA(cudaEventRecord(h->la_out, s));
            OXI_CUDA(cudaStreamWaitEvent(caller, h->la_out, 0));
        }
        h->stream = caller;
    } catch (...) {
        h->stream = caller;
        h->tc_slot = 0;
        h->gemm_ctas = 0;
        throw;
    }
}
template void potrf_rowmajor<double>(oxi_handle_s *, double *, i64, i64, int64_t *, double *);
template void potrf_rowmajor<float>(oxi_handle_s *, float *, i64, i64, int64_t *, float *);

// ---------------------------------------------------------------------------
// Solves with the factor: L y = b, then L^T x = y (the reference's two
// triangular solves, src/lapack/factorizations.jl:293-305).  L is the caller's
// column-major lower factor: the non-unit lower block-operator solve and its
// transpose (solve.cu).
// ---------------------------------------------------------------------------
template <typename T>
void potrs_colmajor(oxi_handle_s *h, i64 n, i64 nrhs, const T *L, i64 ldl, T *B, i64 ldb, int *d_err);

}  // namespace oxi

extern "C" int oxi_dpotrf(oxi_handle_t h, int64_t n, double *dA, int64_t lda, int64_t *h_info) {
    using namespace oxi;
    if (!h || !h_info || n < 0 || lda < std::max<int64_t>(1, n)) return OXI_EINVAL;
    *h_info = 0;
    if (n == 0) return OXI_OK;
    if (!dA || n >= (1ll << 31)) return OXI_EINVAL;
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        AbortScope ab(h);
        char *sc = (char *)h->scratch.get(kScratchBytes);
        int64_t *d_info = (int64_t *)sc;
        OXI_CUDA(cudaMemsetAsync(d_info, 0, sizeof(int64_t), h->stream));
        // T (the transposed block row, n x NB) and room for an aligned copy of the block row
        double *work = (double *)h->work.get(sizeof(double) * potrf_work_elems(n));
        potrf_rowmajor<double>(h, dA, lda, n, d_info, work);
        int64_t *hi = (int64_t *)h->host_ws.get(64);
        OXI_CUDA(cudaMemcpyAsync(hi, d_info, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream));
        queue_abort_read(h, (int *)(hi + 2));
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        *h_info = hi[0];
        const int we = check_abort(h, (const int *)(hi + 2));
        if (we != OXI_OK) return we;
        return hi[0] > 0 ? OXI_ENOTPOSDEF : OXI_OK;
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

extern "C" int oxi_dpotrs(oxi_handle_t h, int64_t n, int64_t nrhs, const double *dL, int64_t ldl, double *dB,
                          int64_t ldb) {
    using namespace oxi;
    if (!h || n < 0 || nrhs < 0 || ldl < std::max<int64_t>(1, n) || ldb < std::max<int64_t>(1, n))
        return OXI_EINVAL;
    if (n == 0 || nrhs == 0) return OXI_OK;
    if (!dL || !dB || n >= (1ll << 31)) return OXI_EINVAL;
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        AbortScope ab(h);
        potrs_colmajor<double>(h, n, nrhs, dL, ldl, dB, ldb, ab.word);
        int *he = (int *)h->host_ws.get(64);
        queue_abort_read(h, he);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        return check_abort(h, he);
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}
