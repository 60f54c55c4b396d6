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
#include <atomic>
#include <mutex>
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

// M is the effective triangle: ROWACC ? M(r, j) = A[r*lda + j] : M(r, j) = A[r + j*lda].
// A CTA owns a row block (ticket order); its 8 warps take the solved column
// blocks round-robin, each lane accumulating two rows, so the off-diagonal
// products of one block run with 8-way memory parallelism and no cross-lane
// reductions.  The diagonal block is solved by substitution.  The handle's
// solves use the block-operator kernel below (k_trsv3); this one needs no
// workspace beyond its flags and serves the no-allocation entry point.
constexpr int TRSV_WARPS = SOLVE_NT / 32;

template <typename T, int NR>
struct TrsvSmem {
    T x[TRSV_WARPS][SB][NR];     // per-warp staging of solved blocks
    T acc[TRSV_WARPS][SB][NR];   // per-warp partial sums
    T y[SB][NR];                 // right-hand side of the diagonal block
    T x0[SB][NR];                // the critical block's solution
    T part[SOLVE_NT / SB][SB][NR];
    T tile[SB][SB + 1];          // the critical off-diagonal tile, prefetched
    T diag[SB][SB + 1];          // the diagonal block
};

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Wait for the tagged word of the current epoch and return its float value.
__device__ __forceinline__ float tagged_get(const unsigned long long *p, uint32_t epoch, int *err) {
    unsigned long long w = ld_volatile_u64(p);
    if ((uint32_t)(w >> 32) != epoch) {
        const uint64_t t0 = global_ns();
        uint32_t it = 0;
        while ((uint32_t)((w = ld_volatile_u64(p)) >> 32) != epoch) {
            if (spin_give_up<256>(it, t0, err, 3)) break;
        }
    }
    return __uint_as_float((uint32_t)w);
}

// A solved block is published through its flag (release after the rows are
// stored; consumers acquire it before reading the rows).
template <typename T, bool LOWER, bool UNIT, bool ROWACC, int NR>
__global__ void __launch_bounds__(SOLVE_NT)
k_trsv2(const T *__restrict__ A, i64 lda, T *__restrict__ X, i64 ldx, int n, int *__restrict__ ticket,
        int *__restrict__ flags, int *__restrict__ err) {
    extern __shared__ __align__(16) unsigned char trsv_smem[];
    TrsvSmem<T, NR> &S = *reinterpret_cast<TrsvSmem<T, NR> *>(trsv_smem);
    __shared__ int s_blk;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nb = (n + SB - 1) / SB;
    if (t == 0) s_blk = aborted(err) ? nb : atomicAdd(ticket, 1);  // an aborted call: no block
    __syncthreads();
    const int bi = s_blk;
    if (bi >= nb) return;
    const int b = LOWER ? bi : nb - 1 - bi;
    const int r0 = b * SB;
    const int rows = min(SB, n - r0);
    auto Mv = [&](int r, int j) -> T {
        return ROWACC ? A[(i64)r * lda + j] : A[(i64)r + (i64)j * lda];
    };

    // ---- prefetch (no dependency on other blocks): diagonal block and critical tile ----
    const bool has_crit = bi > 0;
    const int cc = LOWER ? b - 1 : b + 1;  // the last block solved before this one
    const int cc0 = cc * SB, ccols = has_crit ? min(SB, n - cc0) : 0;
    for (int e = t; e < SB * SB; e += SOLVE_NT) {
        // threads run along the contiguous index of the stored factor
        int r, j;
        if (ROWACC) { r = e / SB; j = e % SB; } else { r = e % SB; j = e / SB; }
        S.diag[r][j] = (r < rows && j < rows) ? Mv(r0 + r, r0 + j) : T(0);
        if (has_crit) S.tile[r][j] = (r < rows && j < ccols) ? Mv(r0 + r, cc0 + j) : T(0);
    }

    // ---- products with the other solved blocks (warps round-robin) ----
    // 16-byte row loads only when every row start is 16-byte aligned (the
    // caller's lda need not be even).
    const bool vec_rows = ROWACC && ((lda * (i64)sizeof(T)) % 16 == 0) && ((((uintptr_t)A) & 15) == 0);
    T acc[2][NR];
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int k = 0; k < NR; ++k) acc[q][k] = T(0);
    for (int step = warp; step < bi - 1; step += TRSV_WARPS) {
        const int c = LOWER ? step : nb - 1 - step;
        const int c0 = c * SB;
        const int cols = min(SB, n - c0);
        if (lane == 0 && ld_acquire(&flags[c]) == 0) {
            const uint64_t t0 = global_ns();
            uint32_t it = 0;
            while (ld_acquire(&flags[c]) == 0) {
                if (spin_give_up<256>(it, t0, err, 3)) break;
            }
        }
        __syncwarp();
        for (int e = lane; e < SB * NR; e += 32) {
            const int jj = e % SB, k = e / SB;
            S.x[warp][jj][k] = (jj < cols) ? __ldcg(&X[(i64)(c0 + jj) + (i64)k * ldx]) : T(0);
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int r = lane + 32 * q;
            if (r >= rows) continue;
            if (ROWACC) {
                const T *arow = A + (i64)(r0 + r) * lda + c0;
                if (cols == SB && vec_rows) {
#pragma unroll 16
                    for (int jj = 0; jj < SB; jj += 16 / (int)sizeof(T)) {
                        T av[16 / sizeof(T)];
                        *(int4 *)av = *(const int4 *)(arow + jj);
#pragma unroll
                        for (int u = 0; u < (int)(16 / sizeof(T)); ++u)
#pragma unroll
                            for (int k = 0; k < NR; ++k) acc[q][k] = fma(av[u], S.x[warp][jj + u][k], acc[q][k]);
                    }
                } else {
                    for (int jj = 0; jj < cols; ++jj)
#pragma unroll
                        for (int k = 0; k < NR; ++k) acc[q][k] = fma(arow[jj], S.x[warp][jj][k], acc[q][k]);
                }
            } else {
                const T *acol = A + (i64)(r0 + r) + (i64)c0 * lda;
#pragma unroll 16
                for (int jj = 0; jj < cols; ++jj) {
                    const T a = acol[(i64)jj * lda];
#pragma unroll
                    for (int k = 0; k < NR; ++k) acc[q][k] = fma(a, S.x[warp][jj][k], acc[q][k]);
                }
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int k = 0; k < NR; ++k) S.acc[warp][lane + 32 * q][k] = acc[q][k];
    __syncthreads();
    for (int e = t; e < SB * NR; e += SOLVE_NT) {
        const int r = e % SB, k = e / SB;
        T v = T(0);
#pragma unroll
        for (int w = 0; w < TRSV_WARPS; ++w) v += S.acc[w][r][k];
        S.y[r][k] = (r < rows) ? (X[(i64)(r0 + r) + (i64)k * ldx] - v) : T(0);
    }

    // ---- critical path: the block solved just before, then the diagonal ----
    constexpr int SEG = SOLVE_NT / SB, SEGW = SB / SEG;
    const int pr = t % SB, ps = t / SB;
    if (has_crit) {
        if (t == 0 && ld_acquire(&flags[cc]) == 0) {
            const uint64_t t0 = global_ns();
            uint32_t it = 0;
            while (ld_acquire(&flags[cc]) == 0) {
                if (spin_give_up<256>(it, t0, err, 3)) break;
            }
        }
        __syncthreads();
        for (int e = t; e < SB * NR; e += SOLVE_NT) {
            const int jj = e % SB, k = e / SB;
            S.x0[jj][k] = (jj < ccols) ? __ldcg(&X[(i64)(cc0 + jj) + (i64)k * ldx]) : T(0);
        }
        __syncthreads();
        T pv[NR];
#pragma unroll
        for (int k = 0; k < NR; ++k) pv[k] = T(0);
#pragma unroll
        for (int jj = 0; jj < SEGW; ++jj) {
            const T a = S.tile[pr][ps * SEGW + jj];
#pragma unroll
            for (int k = 0; k < NR; ++k) pv[k] = fma(a, S.x0[ps * SEGW + jj][k], pv[k]);
        }
#pragma unroll
        for (int k = 0; k < NR; ++k) S.part[ps][pr][k] = pv[k];
        __syncthreads();
        for (int e = t; e < SB * NR; e += SOLVE_NT) {
            const int r = e % SB, k = e / SB;
            T v = T(0);
#pragma unroll
            for (int q = 0; q < SEG; ++q) v += S.part[q][r][k];
            S.y[r][k] -= v;
        }
    }
    __syncthreads();

    // substitution on the diagonal block: warp k takes right-hand side k
    for (int k = warp; k < NR; k += TRSV_WARPS) {
        T y[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) y[q] = S.y[lane + 32 * q][k];
        for (int st = 0; st < rows; ++st) {
            const int p = LOWER ? st : rows - 1 - st;
            const int hp = p >> 5, lp = p & 31;
            const T yp = __shfl_sync(0xffffffffu, hp ? y[1] : y[0], lp);
            const T xp = UNIT ? yp : yp / S.diag[p][p];
            if (lane == lp) { if (hp) y[1] = xp; else y[0] = xp; }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int r = lane + 32 * q;
                const bool below = LOWER ? (r > p) : (r < p);
                if (below && r < rows) y[q] = fma(-S.diag[r][p], xp, y[q]);
            }
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int r = lane + 32 * q;
            if (r < rows) X[(i64)(r0 + r) + (i64)k * ldx] = y[q];
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

// ---------------------------------------------------------------------------
// Block-operator triangular solve.  For block b of the effective triangle M in
// solve order, with p1, p2, p3 the blocks solved one, two and three steps
// before it,
//   x_b = Dinv_b (r_b - sum_{older c} M(b,c) x_c) - sum_q Q_q,b x_pq,
//   Dinv_b = M(b,b)^-1,  Q_q,b = Dinv_b M(b,p_q)  (q = 1..TRSV_WIN),
// the operators precomputed per factor (k_trsv_prep).  The older products and
// Dinv run while the previous blocks are still being solved (they need no
// block solved less than TRSV_WIN + 1 steps before), so the dependency chain
// from block to block is one warp-local 64 x 64 matrix-vector product: each
// warp owns 8 rows, four lanes per row, and reads x_p1 straight from the
// tagged words, with no CTA barrier on the chain.
// Solved values travel as tagged 64-bit words (value bits | epoch << 32; FP64
// as two such halves), so a consumer spins on the data itself.
// ---------------------------------------------------------------------------
template <typename T> struct TagWords { static constexpr int n = (int)sizeof(T) / 4; };

__device__ __forceinline__ void tag_put(unsigned long long *w, float v, uint32_t epoch) {
    *(volatile unsigned long long *)w = ((unsigned long long)epoch << 32) | __float_as_uint(v);
}
__device__ __forceinline__ void tag_put(unsigned long long *w, double v, uint32_t epoch) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    const unsigned long long e = (unsigned long long)epoch << 32;
    *(volatile unsigned long long *)w = e | (b & 0xffffffffull);
    *(volatile unsigned long long *)(w + 1) = e | (b >> 32);
}
template <typename T>
__device__ __forceinline__ T tag_get(const unsigned long long *w, uint32_t epoch, int *err);
template <>
__device__ __forceinline__ float tag_get<float>(const unsigned long long *w, uint32_t epoch, int *err) {
    return tagged_get(w, epoch, err);
}
template <>
__device__ __forceinline__ double tag_get<double>(const unsigned long long *w, uint32_t epoch, int *err) {
    unsigned long long lo = ld_volatile_u64(w), hi = ld_volatile_u64(w + 1);
    if ((uint32_t)(lo >> 32) != epoch || (uint32_t)(hi >> 32) != epoch) {
        const uint64_t t0 = global_ns();
        uint32_t it = 0;
        for (;;) {
            lo = ld_volatile_u64(w);
            hi = ld_volatile_u64(w + 1);
            if ((uint32_t)(lo >> 32) == epoch && (uint32_t)(hi >> 32) == epoch) break;
            if (spin_give_up<256>(it, t0, err, 3)) break;
        }
    }
    return __longlong_as_double((long long)((hi << 32) | (lo & 0xffffffffull)));
}

constexpr int TRSV_WIN = 3;                       // blocks coupled on the chain
constexpr int TRSV_OPS = (1 + TRSV_WIN) * SB * SB;  // operator elements per block: Dinv, Q1..Q3

__device__ __forceinline__ float tag_decode(const unsigned long long (&w)[1]) { return __uint_as_float((uint32_t)w[0]); }
__device__ __forceinline__ double tag_decode(const unsigned long long (&w)[2]) {
    return __longlong_as_double((long long)((w[1] << 32) | (w[0] & 0xffffffffull)));
}

// One warp stages the solution of a 64-row block (rows row0.., `cols` of them,
// NR right-hand sides) from the tagged words into xs[64][NR]: every word's load
// is in flight at once, and the words still of an older epoch are polled again
// together, one round trip per pass however many there are.
template <typename T, int NR>
__device__ __forceinline__ void stage_block(T (*xs)[NR], const unsigned long long *__restrict__ xtag, int row0,
                                            int cols, uint32_t epoch, int *err, int lane) {
    constexpr int TW = TagWords<T>::n;
    constexpr int PL = SB * NR / 32;
    unsigned long long w[PL][TW];
    bool rdy[PL];
    auto word = [&](int v) {
        const int e = lane + 32 * v, jj = e % SB, k = e / SB;
        return xtag + ((i64)(row0 + jj) * NR + k) * TW;
    };
#pragma unroll
    for (int v = 0; v < PL; ++v) {
        const int jj = (lane + 32 * v) % SB;
        rdy[v] = jj >= cols;
#pragma unroll
        for (int h = 0; h < TW; ++h) w[v][h] = rdy[v] ? 0ull : ld_volatile_u64(word(v) + h);
    }
    bool all = true;
#pragma unroll
    for (int v = 0; v < PL; ++v) {
        if (!rdy[v]) {
            bool ok = true;
#pragma unroll
            for (int h = 0; h < TW; ++h) ok = ok && (uint32_t)(w[v][h] >> 32) == epoch;
            rdy[v] = ok;
        }
        all = all && rdy[v];
    }
    if (!all) {
        const uint64_t t0 = global_ns();
        uint32_t it = 0;
        for (;;) {
#pragma unroll
            for (int v = 0; v < PL; ++v)
                if (!rdy[v]) {
#pragma unroll
                    for (int h = 0; h < TW; ++h) w[v][h] = ld_volatile_u64(word(v) + h);
                }
            all = true;
#pragma unroll
            for (int v = 0; v < PL; ++v) {
                if (!rdy[v]) {
                    bool ok = true;
#pragma unroll
                    for (int h = 0; h < TW; ++h) ok = ok && (uint32_t)(w[v][h] >> 32) == epoch;
                    rdy[v] = ok;
                }
                all = all && rdy[v];
            }
            if (all) break;
            if (spin_give_up<64>(it, t0, err, 3)) break;
        }
    }
#pragma unroll
    for (int v = 0; v < PL; ++v) {
        const int e = lane + 32 * v, jj = e % SB, k = e / SB;
        xs[jj][k] = (jj < cols) ? (T)tag_decode(w[v]) : T(0);
    }
}

// One CTA per block: the inverse of the diagonal block by substitution (64
// threads, one column each), then the coupling operators as 64 x 64 x 64
// products.  Rows and columns past n are padded with the identity (Dinv) and
// zeros (Q).
template <typename T, bool LOWER, bool UNIT, bool ROWACC>
__global__ void __launch_bounds__(SOLVE_NT) k_trsv_prep(const T *__restrict__ A, i64 lda, int n,
                                                       T *__restrict__ P) {
    extern __shared__ __align__(16) unsigned char prep_smem[];
    T(*sM)[SB + 1] = reinterpret_cast<T(*)[SB + 1]>(prep_smem);
    T(*sX)[SB + 1] = reinterpret_cast<T(*)[SB + 1]>(prep_smem + sizeof(T) * SB * (SB + 1));
    const int nb = (n + SB - 1) / SB;
    const int bi = blockIdx.x;
    const int b = LOWER ? bi : nb - 1 - bi;
    const int r0 = b * SB, rows = min(SB, n - r0);
    const int t = threadIdx.x;
    auto Mv = [&](int r, int j) -> T { return ROWACC ? A[(i64)r * lda + j] : A[(i64)r + (i64)j * lda]; };
    for (int e = t; e < SB * SB; e += SOLVE_NT) {
        int r, j;
        if (ROWACC) { r = e / SB; j = e % SB; } else { r = e % SB; j = e / SB; }
        T v = (r == j) ? T(1) : T(0);
        if (r < rows && j < rows && !(UNIT && r == j)) v = Mv(r0 + r, r0 + j);
        sM[r][j] = v;
    }
    __syncthreads();
    if (t < SB) {
        const int j = t;
        for (int st = 0; st < SB; ++st) {
            const int i = LOWER ? st : SB - 1 - st;
            T s = (i == j) ? T(1) : T(0);
            if (LOWER) {
                for (int p = 0; p < i; ++p) s = fma(-sM[i][p], sX[p][j], s);
            } else {
                for (int p = i + 1; p < SB; ++p) s = fma(-sM[i][p], sX[p][j], s);
            }
            sX[i][j] = UNIT ? s : s / sM[i][i];
        }
    }
    __syncthreads();
    T *Pb = P + (i64)bi * TRSV_OPS;
    for (int e = t; e < SB * SB; e += SOLVE_NT) Pb[e] = sX[e / SB][e % SB];
    for (int q = 1; q <= TRSV_WIN; ++q) {
        if (bi - q < 0) break;
        const int pb = LOWER ? b - q : b + q;
        const int c0 = pb * SB, cols = min(SB, n - c0);
        __syncthreads();
        for (int e = t; e < SB * SB; e += SOLVE_NT) {
            int r, j;
            if (ROWACC) { r = e / SB; j = e % SB; } else { r = e % SB; j = e / SB; }
            sM[r][j] = (r < rows && j < cols) ? Mv(r0 + r, c0 + j) : T(0);
        }
        __syncthreads();
        const int r = t >> 2, j0 = (t & 3) * 16;
        T o[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) o[u] = T(0);
        for (int p = 0; p < SB; ++p) {
            const T xv = sX[r][p];
#pragma unroll
            for (int u = 0; u < 16; ++u) o[u] = fma(xv, sM[p][j0 + u], o[u]);
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) Pb[q * SB * SB + r * SB + j0 + u] = o[u];
    }
}

template <typename T, int NR>
struct Trsv3Smem {
    T xs[TRSV_WARPS][SB][NR];  // per-warp staging of solved blocks
    T acc[TRSV_WARPS][SB][NR];
    T y[SB][NR];
    T z[SB][NR];
    T part[SOLVE_NT / SB][SB][NR];
    T op[1 + TRSV_WIN][SB][SB + 1];  // Dinv, Q1..Q3 of this block
};

template <typename T, bool LOWER, bool ROWACC, int NR>
__global__ void __launch_bounds__(SOLVE_NT)
k_trsv3(const T *__restrict__ A, i64 lda, const T *__restrict__ P, T *__restrict__ X, i64 ldx, int n,
        int *__restrict__ ticket, int *__restrict__ err, unsigned long long *__restrict__ xtag, uint32_t epoch) {
    constexpr int TW = TagWords<T>::n;
    extern __shared__ __align__(16) unsigned char trsv3_smem[];
    Trsv3Smem<T, NR> &S = *reinterpret_cast<Trsv3Smem<T, NR> *>(trsv3_smem);
    __shared__ int s_blk;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nb = (n + SB - 1) / SB;
    if (t == 0) s_blk = aborted(err) ? nb : atomicAdd(ticket, 1);  // an aborted call: no block
    __syncthreads();
    const int bi = s_blk;
    if (bi >= nb) return;
    const int b = LOWER ? bi : nb - 1 - bi;
    const int r0 = b * SB;
    const int rows = min(SB, n - r0);
    auto xw = [&](int row, int k) { return xtag + ((i64)row * NR + k) * TW; };

    // ---- this block's operators (no dependency on other blocks) ----
    const T *Pb = P + (i64)bi * TRSV_OPS;
    const int nops = min(bi, TRSV_WIN) + 1;
    for (int e = t; e < nops * SB * SB; e += SOLVE_NT) {
        const int o = e / (SB * SB), rr = (e / SB) % SB, jj = e % SB;
        S.op[o][rr][jj] = Pb[e];
    }

    // right-hand side of this block, read before anything waits
    for (int e = t; e < SB * NR; e += SOLVE_NT) {
        const int r = e % SB, k = e / SB;
        S.y[r][k] = (r < rows) ? X[(i64)(r0 + r) + (i64)k * ldx] : T(0);
    }

    // ---- products with the blocks solved TRSV_WIN + 1 or more steps before ----
    // Blocks in solve order; within each, warp w takes tile columns [8w, 8w+8)
    // and each lane two rows.  The next block's tile and solution words are
    // loaded before the current block's products, so the loads' latency is
    // hidden and the loop runs at issue rate behind the chain.
    {
        const int jw = warp * 8;
        const bool vec8 = ROWACC && ((lda * (i64)sizeof(T)) % 16 == 0) && ((((uintptr_t)A) & 15) == 0);
        auto load_tile = [&](int step, T (&a)[2][8]) {
            const int c = LOWER ? step : nb - 1 - step;
            const int c0 = c * SB;
            const int cols = min(SB, n - c0);
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int rr = lane + 32 * q;
                if (ROWACC) {
                    const T *arow = A + (i64)(r0 + rr) * lda + c0 + jw;
                    if (rr < rows && vec8 && jw + 8 <= cols) {
#pragma unroll
                        for (int u = 0; u < 8; u += 16 / (int)sizeof(T)) *(int4 *)&a[q][u] = *(const int4 *)(arow + u);
                    } else {
#pragma unroll
                        for (int u = 0; u < 8; ++u) a[q][u] = (rr < rows && jw + u < cols) ? arow[u] : T(0);
                    }
                } else {
                    const T *acol = A + (i64)(r0 + rr) + (i64)(c0 + jw) * lda;
#pragma unroll
                    for (int u = 0; u < 8; ++u) a[q][u] = (rr < rows && jw + u < cols) ? acol[(i64)u * lda] : T(0);
                }
            }
        };
        // solution words of the warp's 8 columns: lane e < 8 NR holds (column e % 8, rhs e / 8)
        constexpr int XPL = (8 * NR + 31) / 32;  // words per lane
        auto xidx = [&](int step, int v, int &row, int &k, bool &ok) {
            const int c = LOWER ? step : nb - 1 - step;
            const int e = lane + 32 * v;
            row = c * SB + jw + (e & 7);
            k = e >> 3;
            ok = (e < 8 * NR) && (row < n);
        };
        T acc[2][NR];
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int k = 0; k < NR; ++k) acc[q][k] = T(0);
        const int nsteps = bi - TRSV_WIN;
        // the next step's tile and raw solution words are loaded one step ahead
        // (all in flight at once); a word of an older epoch is polled again only
        // when its step comes
        T an[2][8];
        unsigned long long xr[XPL][TW];
        auto issue_x = [&](int step) {
#pragma unroll
            for (int v = 0; v < XPL; ++v) {
                int row, k; bool ok;
                xidx(step, v, row, k, ok);
#pragma unroll
                for (int hw = 0; hw < TW; ++hw)
                    xr[v][hw] = ok ? ld_volatile_u64(xw(row, k) + hw) : ((unsigned long long)epoch << 32);
            }
        };
        if (nsteps > 0) {
            load_tile(0, an);
            issue_x(0);
        }
        for (int step = 0; step < nsteps; ++step) {
            T a[2][8];
#pragma unroll
            for (int q = 0; q < 2; ++q)
#pragma unroll
                for (int u = 0; u < 8; ++u) a[q][u] = an[q][u];
            T *xsw = &S.xs[warp][0][0];  // [rhs k][column u] at k * 8 + u
#pragma unroll
            for (int v = 0; v < XPL; ++v) {
                int row, k; bool ok;
                xidx(step, v, row, k, ok);
                bool ready = true;
#pragma unroll
                for (int hw = 0; hw < TW; ++hw) ready = ready && (uint32_t)(xr[v][hw] >> 32) == epoch;
                if (!ready) {
                    const uint64_t t0 = global_ns();
                    uint32_t it = 0;
                    for (;;) {
                        ready = true;
#pragma unroll
                        for (int hw = 0; hw < TW; ++hw) {
                            xr[v][hw] = ld_volatile_u64(xw(row, k) + hw);
                            ready = ready && (uint32_t)(xr[v][hw] >> 32) == epoch;
                        }
                        if (ready) break;
                        if (spin_give_up<256>(it, t0, err, 3)) break;
                    }
                }
                if (lane + 32 * v < 8 * NR) xsw[lane + 32 * v] = ok ? (T)tag_decode(xr[v]) : T(0);
            }
            if (step + 1 < nsteps) {
                load_tile(step + 1, an);
                issue_x(step + 1);
            }
            __syncwarp();
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int k = 0; k < NR; ++k) {
                    const T xv = xsw[k * 8 + u];
#pragma unroll
                    for (int q = 0; q < 2; ++q) acc[q][k] = fma(a[q][u], xv, acc[q][k]);
                }
            __syncwarp();
        }
#pragma unroll
        for (int q = 0; q < 2; ++q)
#pragma unroll
            for (int k = 0; k < NR; ++k) S.acc[warp][lane + 32 * q][k] = acc[q][k];
    }
    __syncthreads();
    for (int e = t; e < SB * NR; e += SOLVE_NT) {
        const int r = e % SB, k = e / SB;
        T v = T(0);
#pragma unroll
        for (int w = 0; w < TRSV_WARPS; ++w) v += S.acc[w][r][k];
        S.y[r][k] -= v;
    }
    __syncthreads();

    // ---- the chain's operands: 8 rows per warp, 4 lanes per row (16 columns each) ----
    const int r = warp * 8 + (lane >> 2), sg = lane & 3;
    T s[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) s[k] = T(0);
    auto couple = [&](int q) {  // s += Q_q x_(block solved q steps before)
        const int pb = LOWER ? b - q : b + q;
        const int c0 = pb * SB;
        stage_block<T, NR>(S.xs[warp], xtag, c0, min(SB, n - c0), epoch, err, lane);
        __syncwarp();
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) {
            const T a = S.op[q][r][sg * 16 + jj];
#pragma unroll
            for (int k = 0; k < NR; ++k) s[k] = fma(a, S.xs[warp][sg * 16 + jj][k], s[k]);
        }
        __syncwarp();
    };
    // ---- z = Dinv y, over SEG column segments ----
    constexpr int SEG = SOLVE_NT / SB, SEGW = SB / SEG;
    {
        const int pr = t % SB, ps = t / SB;
        T pv[NR];
#pragma unroll
        for (int k = 0; k < NR; ++k) pv[k] = T(0);
#pragma unroll
        for (int jj = 0; jj < SEGW; ++jj) {
            const T a = S.op[0][pr][ps * SEGW + jj];
#pragma unroll
            for (int k = 0; k < NR; ++k) pv[k] = fma(a, S.y[ps * SEGW + jj][k], pv[k]);
        }
#pragma unroll
        for (int k = 0; k < NR; ++k) S.part[ps][pr][k] = pv[k];
    }
    __syncthreads();
    for (int e = t; e < SB * NR; e += SOLVE_NT) {
        const int rr = e % SB, k = e / SB;
        T v = T(0);
#pragma unroll
        for (int q = 0; q < SEG; ++q) v += S.part[q][rr][k];
        S.z[rr][k] = v;
    }
    __syncthreads();

    // ---- the chain: x_b = z - sum_q Q_q x_pq, warp-local; only x_p1 is fresh ----
#pragma unroll
    for (int q = TRSV_WIN; q >= 1; --q)
        if (bi >= q) couple(q);
#pragma unroll
    for (int k = 0; k < NR; ++k) {
        s[k] += __shfl_xor_sync(0xffffffffu, s[k], 1);
        s[k] += __shfl_xor_sync(0xffffffffu, s[k], 2);
    }
    if (r < rows) {
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            if ((k & 3) != sg) continue;
            const T x = S.z[r][k] - s[k];
            X[(i64)(r0 + r) + (i64)k * ldx] = x;
            tag_put(xw(r0 + r, k), x, epoch);
        }
    }
}

// UPPER_A / TRANS describe the stored factor as in LAPACK (column-major A,
// op(A) = A or A^T); ROWACC access of the same memory is the transposed view.
static std::atomic<uint32_t> g_trsv_epoch{0};  // tags of the exchange words, one per launch
// The next launch's tag; 0 is skipped on wrap-around, since zeroed (fresh)
// words carry it.
static uint32_t next_trsv_epoch() {
    uint32_t e = ++g_trsv_epoch;
    if (e == 0) e = ++g_trsv_epoch;
    return e;
}

template <typename T, bool UPPER_A, bool UNIT, bool TRANS>
static void trsv_launch(const T *A, i64 lda, T *X, i64 ldx, int n, int nrhs, int *ctl, int *err,
                        cudaStream_t s) {
    constexpr bool LOWER = (UPPER_A == TRANS);
    const int nb = (n + SB - 1) / SB;
    ProfScope ps(KC_TRSV, s, (double)n * n * nrhs, (double)n * n * sizeof(T) / 2);
    for (int k0 = 0; k0 < nrhs;) {
        const int left = nrhs - k0;
        OXI_CUDA(cudaMemsetAsync(ctl, 0, sizeof(int) * (nb + 1), s));
        int *ticket = ctl, *flags = ctl + 1;
        T *Xk = X + (i64)k0 * ldx;
#define OXI_TRSV_GO(NRV)                                                                              \
    do {                                                                                             \
        const int smem = (int)sizeof(TrsvSmem<T, NRV>);                                             \
        auto kern = k_trsv2<T, LOWER, UNIT, TRANS, NRV>;                                             \
        OXI_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));     \
        kern<<<nb, SOLVE_NT, smem, s>>>(A, lda, Xk, ldx, n, ticket, flags, err);                      \
        k0 += NRV;                                                                                   \
    } while (0)
        if (left >= 8) OXI_TRSV_GO(8);
        else if (left >= 4) OXI_TRSV_GO(4);
        else if (left >= 2) OXI_TRSV_GO(2);
        else OXI_TRSV_GO(1);
#undef OXI_TRSV_GO
        OXI_LAUNCH_CHECK();
    }
}

template <typename T, bool UPPER_A, bool UNIT, bool TRANS>
static void trsv_prep_launch(const T *A, i64 lda, int n, T *P, cudaStream_t s) {
    constexpr bool LOWER = (UPPER_A == TRANS);
    const int nb = (n + SB - 1) / SB;
    const int smem = 2 * (int)sizeof(T) * SB * (SB + 1);
    set_max_dyn_smem((const void *)k_trsv_prep<T, LOWER, UNIT, TRANS>, smem);
    ProfScope ps(KC_TRSV, s, 2.0 * SB * SB * (double)n * 3, 3.0 * (double)n * SB * sizeof(T));
    k_trsv_prep<T, LOWER, UNIT, TRANS><<<nb, SOLVE_NT, smem, s>>>(A, lda, n, P);
    OXI_LAUNCH_CHECK();
}

template <typename T, bool UPPER_A, bool TRANS>
static void trsv3_launch(const T *A, i64 lda, T *X, i64 ldx, int n, int nrhs, int *ctl, int *err,
                         cudaStream_t s, const T *P, unsigned long long *xtag) {
    constexpr bool LOWER = (UPPER_A == TRANS);
    const int nb = (n + SB - 1) / SB;
    ProfScope ps(KC_TRSV, s, (double)n * n * nrhs, (double)n * n * sizeof(T) / 2);
    for (int k0 = 0; k0 < nrhs;) {
        const int left = nrhs - k0;
        OXI_CUDA(cudaMemsetAsync(ctl, 0, sizeof(int), s));
        T *Xk = X + (i64)k0 * ldx;
#define OXI_TRSV3_GO(NRV)                                                                            \
    do {                                                                                             \
        const int smem = (int)sizeof(Trsv3Smem<T, NRV>);                                            \
        const uint32_t ep = next_trsv_epoch();                                                       \
        auto kern = k_trsv3<T, LOWER, TRANS, NRV>;                                                   \
        set_max_dyn_smem((const void *)kern, smem);                                                  \
        kern<<<nb, SOLVE_NT, smem, s>>>(A, lda, P, Xk, ldx, n, ctl, err, xtag, ep);                 \
        k0 += NRV;                                                                                   \
    } while (0)
        bool wide = false;
        if constexpr (sizeof(T) == 4) {
            if (left >= 16) {
                OXI_TRSV3_GO(16);
                wide = true;
            }
        }
        if (wide) {
        } else if (left >= 8) OXI_TRSV3_GO(8);
        else if (left >= 4) OXI_TRSV3_GO(4);
        else if (left >= 2) OXI_TRSV3_GO(2);
        else OXI_TRSV3_GO(1);
#undef OXI_TRSV3_GO
        OXI_LAUNCH_CHECK();
    }
}

// Tagged solution words for the triangular solves: n rows x 16 words (FP32 up
// to 16 right-hand sides, FP64 up to 8 at two words each).  A fresh or grown
// buffer is zeroed: epoch 0 never matches a launch.
static unsigned long long *xtag_words(oxi_handle_s *h, i64 n) {
    const size_t need = sizeof(unsigned long long) * (size_t)n * 16;
    if (h->xtag_ws.bytes < need) {
        void *p = h->xtag_ws.get(need);
        OXI_CUDA(cudaMemsetAsync(p, 0, h->xtag_ws.bytes, h->stream));
    }
    return (unsigned long long *)h->xtag_ws.get(need);
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
    // the two triangles' block operators (inverse and coupling blocks), then the solves
    T *P1 = (T *)h->trsv_ws.get(2 * sizeof(T) * (size_t)nb * TRSV_OPS);
    T *P2 = P1 + (size_t)nb * TRSV_OPS;
    unsigned long long *xtag = xtag_words(h, n);
    if (trans == 'N') {
        k_gather_rows<T><<<(unsigned)((tot + nt - 1) / nt), nt, 0, s>>>(B, ldb, d_perm, X, n, (int)n, (int)nrhs, 0);
        OXI_LAUNCH_CHECK();
        trsv_prep_launch<T, false, true, false>(LU, lda, (int)n, P1, s);
        trsv_prep_launch<T, true, false, false>(LU, lda, (int)n, P2, s);
        trsv3_launch<T, false, false>(LU, lda, X, n, (int)n, (int)nrhs, ctl, d_err, s, P1, xtag);
        trsv3_launch<T, true, false>(LU, lda, X, n, (int)n, (int)nrhs, ctl, d_err, s, P2, xtag);
        OXI_CUDA(cudaMemcpy2DAsync(B, ldb * sizeof(T), X, n * sizeof(T), n * sizeof(T), nrhs,
                                   cudaMemcpyDeviceToDevice, s));
    } else {
        OXI_CUDA(cudaMemcpy2DAsync(X, n * sizeof(T), B, ldb * sizeof(T), n * sizeof(T), nrhs,
                                   cudaMemcpyDeviceToDevice, s));
        trsv_prep_launch<T, true, false, true>(LU, lda, (int)n, P1, s);
        trsv_prep_launch<T, false, true, true>(LU, lda, (int)n, P2, s);
        trsv3_launch<T, true, true>(LU, lda, X, n, (int)n, (int)nrhs, ctl, d_err, s, P1, xtag);
        trsv3_launch<T, false, true>(LU, lda, X, n, (int)n, (int)nrhs, ctl, d_err, s, P2, xtag);
        k_gather_rows<T><<<(unsigned)((tot + nt - 1) / nt), nt, 0, s>>>(X, n, d_perm, B, ldb, (int)n, (int)nrhs, 1);
        OXI_LAUNCH_CHECK();
    }
}
// Cholesky solve with the column-major lower factor L: L Y = B (non-unit lower),
// then L^T X = Y (its transpose, upper); B overwritten.
template <typename T>
void potrs_colmajor(oxi_handle_s *h, i64 n, i64 nrhs, const T *L, i64 ldl, T *B, i64 ldb, int *d_err) {
    cudaStream_t s = h->stream;
    const i64 nb = (n + SB - 1) / SB;
    char *ws = (char *)h->solve_ws.get(sizeof(T) * (size_t)n * nrhs + sizeof(int) * (nb + 8) + 256);
    T *X = (T *)ws;
    int *ctl = (int *)(ws + ((sizeof(T) * (size_t)n * nrhs + 255) & ~size_t(255)));
    T *P1 = (T *)h->trsv_ws.get(2 * sizeof(T) * (size_t)nb * TRSV_OPS);
    T *P2 = P1 + (size_t)nb * TRSV_OPS;
    unsigned long long *xtag = xtag_words(h, n);
    OXI_CUDA(cudaMemcpy2DAsync(X, n * sizeof(T), B, ldb * sizeof(T), n * sizeof(T), nrhs,
                               cudaMemcpyDeviceToDevice, s));
    trsv_prep_launch<T, false, false, false>(L, ldl, (int)n, P1, s);
    trsv_prep_launch<T, false, false, true>(L, ldl, (int)n, P2, s);
    trsv3_launch<T, false, false>(L, ldl, X, n, (int)n, (int)nrhs, ctl, d_err, s, P1, xtag);
    trsv3_launch<T, false, true>(L, ldl, X, n, (int)n, (int)nrhs, ctl, d_err, s, P2, xtag);
    OXI_CUDA(cudaMemcpy2DAsync(B, ldb * sizeof(T), X, n * sizeof(T), n * sizeof(T), nrhs,
                               cudaMemcpyDeviceToDevice, s));
}
template void potrs_colmajor<double>(oxi_handle_s *, i64, i64, const double *, i64, double *, i64, int *);

template void getrs_perm<double>(oxi_handle_s *, char, i64, i64, const double *, i64, const int64_t *, double *, i64, int *);
template void getrs_perm<float>(oxi_handle_s *, char, i64, i64, const float *, i64, const int64_t *, float *, i64, int *);

// Row-major factors W are the column-major matrix W^T: L (lower) is then an
// upper-stored triangle read transposed, U likewise.  DinvL / DinvU (optional):
// the per-block operators of L and of U (diagonal-block inverse and coupling
// blocks) from lu_block_inverses_rowmajor; without them the substitution
// kernel runs.
template <typename T>
void lu_solve_rowmajor(oxi_handle_s *h, const T *W, i64 ld, i64 n, T *X, i64 ldx, i64 nrhs,
                       int *d_err, const T *DinvL, const T *DinvU) {
    const i64 nb = (n + SB - 1) / SB;
    if (nb + 1 > kTrsvCtlInts) throw CudaError{cudaErrorInvalidValue, "system too large for the solve control block"};
    int *ctl = (int *)((char *)h->scratch.get(kScratchBytes) + kScratchTrsvOff);
    if (DinvL && DinvU) {  // block operators from lu_block_inverses_rowmajor
        unsigned long long *xtag = xtag_words(h, n);
        trsv3_launch<T, true, true>(W, ld, X, ldx, (int)n, (int)nrhs, ctl, d_err, h->stream, DinvL, xtag);
        trsv3_launch<T, false, true>(W, ld, X, ldx, (int)n, (int)nrhs, ctl, d_err, h->stream, DinvU, xtag);
        return;
    }
    trsv_launch<T, true, true, true>(W, ld, X, ldx, (int)n, (int)nrhs, ctl, d_err, h->stream);
    trsv_launch<T, false, false, true>(W, ld, X, ldx, (int)n, (int)nrhs, ctl, d_err, h->stream);
}
template void lu_solve_rowmajor<float>(oxi_handle_s *, const float *, i64, i64, float *, i64, i64, int *, const float *, const float *);
template void lu_solve_rowmajor<double>(oxi_handle_s *, const double *, i64, i64, double *, i64, i64, int *, const double *, const double *);

template <typename T>
void lu_block_inverses_rowmajor(oxi_handle_s *h, const T *W, i64 ld, i64 n, T *DinvL, T *DinvU) {
    trsv_prep_launch<T, true, true, true>(W, ld, (int)n, DinvL, h->stream);
    trsv_prep_launch<T, false, false, true>(W, ld, (int)n, DinvU, h->stream);
}
template void lu_block_inverses_rowmajor<float>(oxi_handle_s *, const float *, i64, i64, float *, float *);
template void lu_block_inverses_rowmajor<double>(oxi_handle_s *, const double *, i64, i64, double *, double *);
i64 lu_block_inverse_elems(i64 n) { return ((n + SB - 1) / SB) * (i64)TRSV_OPS; }

template <typename T>
void chol_block_ops(oxi_handle_s *h, const T *L, i64 ldl, i64 n, T *P1, T *P2) {
    trsv_prep_launch<T, false, false, false>(L, ldl, (int)n, P1, h->stream);
    trsv_prep_launch<T, false, false, true>(L, ldl, (int)n, P2, h->stream);
}
template void chol_block_ops<float>(oxi_handle_s *, const float *, i64, i64, float *, float *);
template void chol_block_ops<double>(oxi_handle_s *, const double *, i64, i64, double *, double *);

template <typename T>
void chol_solve_ops(oxi_handle_s *h, const T *L, i64 ldl, i64 n, T *X, i64 ldx, i64 nrhs, int *d_err,
                    const T *P1, const T *P2) {
    const i64 nb = (n + SB - 1) / SB;
    if (nb + 1 > kTrsvCtlInts) throw CudaError{cudaErrorInvalidValue, "system too large for the solve control block"};
    int *ctl = (int *)((char *)h->scratch.get(kScratchBytes) + kScratchTrsvOff);
    unsigned long long *xtag = xtag_words(h, n);
    trsv3_launch<T, false, false>(L, ldl, X, ldx, (int)n, (int)nrhs, ctl, d_err, h->stream, P1, xtag);
    trsv3_launch<T, false, true>(L, ldl, X, ldx, (int)n, (int)nrhs, ctl, d_err, h->stream, P2, xtag);
}
template void chol_solve_ops<float>(oxi_handle_s *, const float *, i64, i64, float *, i64, i64, int *, const float *,
                                    const float *);
template void chol_solve_ops<double>(oxi_handle_s *, const double *, i64, i64, double *, i64, i64, int *,
                                     const double *, const double *);

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
        AbortScope ab(h);
        int64_t *dperm = (int64_t *)h->perm_ws.get(sizeof(int64_t) * n);
        int64_t *hperm = (int64_t *)h->host_ws.get(sizeof(int64_t) * (n + 8));
        std::copy(perm.begin(), perm.end(), hperm);
        OXI_CUDA(cudaMemcpyAsync(dperm, hperm, sizeof(int64_t) * n, cudaMemcpyHostToDevice, h->stream));
        getrs_perm<T>(h, trans, n, nrhs, dLU, lda, dperm, dB, ldb, ab.word);
        int *herr = (int *)(hperm + n);
        queue_abort_read(h, herr);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        return check_abort(h, herr);
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

// ---------------------------------------------------------------------------
// No-allocation FP64 getrs.  Its scratch is one file-scope device array:
//   [0, 4)        abort word of the triangular solves (cleared every call)
//   [4, 8)        invalid-pivot flag (cleared every call)
//   [8, 16)       wait limit of the solves' bounded waits: never written, so
//                 zero (the default, 2 s) from the module's load
//   [256, 4356)   tickets + per-block flags of k_trsv2 (cleared per launch)
//   [8 KiB, +8n)  0-based permutation, int64 (written whole every call)
//   [1 MiB, 8 MiB) the solve vector X, n x nrhs (written before it is read)
constexpr i64 kNaScratchBytes = OXI_NOALLOC_SCRATCH_BYTES;
constexpr i64 kNaCtlOff = 256, kNaPermOff = 8192, kNaXOff = 1 << 20;
constexpr i64 kNaMaxN = OXI_NOALLOC_MAX_N;
constexpr i64 kNaMaxElems = OXI_NOALLOC_MAX_ELEMS;
static_assert(kNaMaxElems * (i64)sizeof(double) == kNaScratchBytes - kNaXOff, "X region");
static_assert(kNaPermOff + 8 * kNaMaxN <= kNaXOff, "permutation region");
static_assert(kNaCtlOff + 4 * (kNaMaxN / SB + 1) <= kNaPermOff, "control region");
constexpr int kNaMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaScratchBytes];

// The interchange sequence folded into a permutation (as perm_from_ipiv) on the
// device: all threads check the pivots and seed the identity, then one thread
// applies the n swaps in shared memory (16-bit rows, n <= 65536), eight pivots
// fetched ahead at a time.  An out-of-range pivot sets *bad and writes nothing.
__global__ void __launch_bounds__(1024) k_perm_from_ipiv_na(const int64_t *__restrict__ ipiv, int n,
                                                            int64_t *__restrict__ perm, int *__restrict__ bad) {
    extern __shared__ uint16_t s_perm[];
    int badl = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int64_t p = ipiv[i];
        badl |= (p < 1 || p > n);
        s_perm[i] = (uint16_t)i;
    }
    if (__syncthreads_or(badl)) {
        if (threadIdx.x == 0) *bad = 1;
        return;
    }
    if (threadIdx.x == 0) {
        for (int j0 = 0; j0 < n; j0 += 8) {
            int p[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) p[u] = (j0 + u < n) ? (int)ipiv[j0 + u] - 1 : j0 + u;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                if (j0 + u >= n) break;
                const uint16_t a = s_perm[j0 + u], b = s_perm[p[u]];
                s_perm[j0 + u] = b;
                s_perm[p[u]] = a;
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = s_perm[i];
}

template <bool UPPER_A, bool UNIT, bool TRANS>
static void na_load_trsv(cudaFuncAttributes *fa) {
    constexpr bool LOWER = (UPPER_A == TRANS);
    OXI_CUDA(cudaFuncGetAttributes(fa, k_trsv2<double, LOWER, UNIT, TRANS, 1>));
    OXI_CUDA(cudaFuncGetAttributes(fa, k_trsv2<double, LOWER, UNIT, TRANS, 2>));
    OXI_CUDA(cudaFuncGetAttributes(fa, k_trsv2<double, LOWER, UNIT, TRANS, 4>));
    OXI_CUDA(cudaFuncGetAttributes(fa, k_trsv2<double, LOWER, UNIT, TRANS, 8>));
}

// Identity of the current context (cuCtxGetCurrent + cuCtxGetId through the
// runtime's driver entry points): the array's address belongs to the context
// that resolved it.
static unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void *p1 = nullptr, *p2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        OXI_CUDA(cudaGetDriverEntryPoint("cuCtxGetCurrent", &p1, cudaEnableDefault, &q1));
        OXI_CUDA(cudaGetDriverEntryPoint("cuCtxGetId", &p2, cudaEnableDefault, &q2));
        if (!p1 || !p2 || q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess)
            throw CudaError{cudaErrorNotSupported, "cuCtxGetCurrent / cuCtxGetId unavailable"};
        get_current = (GetCurrent)p1;
        get_id = (GetId)p2;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) {
        // this host thread has not used the runtime yet: a symbol query makes
        // the device's primary context current (it allocates nothing)
        void *sym = nullptr;
        OXI_CUDA(cudaGetSymbolAddress(&sym, g_noalloc_scratch));
        if (get_current(&ctx) != CUDA_SUCCESS || !ctx) throw CudaError{cudaErrorInvalidResourceHandle, "no current context"};
    }
    if (get_id(ctx, &id) != CUDA_SUCCESS) throw CudaError{cudaErrorInvalidResourceHandle, "cuCtxGetId"};
    return id;
}

// Once per device and context, with that device current: the array's address,
// and the kernels of this path loaded (so no later call loads a module).  A
// device reset or a re-created primary context gives a new context id, and the
// address is resolved again.
static char *noalloc_scratch(int dev) {
    struct Slot {
        std::atomic<char *> ptr{nullptr};
        std::atomic<unsigned long long> ctx{0};
    };
    static Slot slots[kNaMaxDevices];
    static std::mutex mu;
    const unsigned long long ctx = current_context_id();
    Slot &sl = slots[dev];
    char *p = sl.ptr.load(std::memory_order_acquire);
    if (p && sl.ctx.load(std::memory_order_acquire) == ctx) return p;
    std::lock_guard<std::mutex> lk(mu);
    p = sl.ptr.load(std::memory_order_acquire);
    if (p && sl.ctx.load(std::memory_order_acquire) == ctx) return p;
    void *sym = nullptr;
    OXI_CUDA(cudaGetSymbolAddress(&sym, g_noalloc_scratch));
    OXI_CUDA(cudaFuncSetAttribute(k_perm_from_ipiv_na, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(uint16_t) * kNaMaxN)));
    cudaFuncAttributes fa;
    OXI_CUDA(cudaFuncGetAttributes(&fa, k_gather_rows<double>));
    na_load_trsv<false, true, false>(&fa);
    na_load_trsv<true, false, false>(&fa);
    na_load_trsv<true, false, true>(&fa);
    na_load_trsv<false, true, true>(&fa);
    p = (char *)sym;
    sl.ctx.store(ctx, std::memory_order_release);
    sl.ptr.store(p, std::memory_order_release);
    return p;
}

static int getrs_noalloc(cudaStream_t s, char trans, i64 n, i64 nrhs, const double *dLU, i64 lda,
                         const int64_t *d_ipiv, double *dB, i64 ldb) {
    if (trans == 'C') trans = 'T';
    if (trans != 'N' && trans != 'T') return OXI_EINVAL;
    if (n < 0 || nrhs < 0 || lda < std::max<i64>(1, n) || ldb < std::max<i64>(1, n)) return OXI_EINVAL;
    if (n == 0 || nrhs == 0) return OXI_OK;
    if (!dLU || !d_ipiv || !dB) return OXI_EINVAL;
    if (n > kNaMaxN || nrhs > kNaMaxElems || n * nrhs > kNaMaxElems) return OXI_ESCRATCH;
    try {
        int dev = 0;
        OXI_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kNaMaxDevices) return OXI_EINVAL;
        char *sc = noalloc_scratch(dev);
        int *err = (int *)sc, *bad = err + 1, *ctl = (int *)(sc + kNaCtlOff);
        int64_t *perm = (int64_t *)(sc + kNaPermOff);
        double *X = (double *)(sc + kNaXOff);
        int hflags[2] = {0, 0};
        OXI_CUDA(cudaMemsetAsync(sc, 0, sizeof(hflags), s));
        k_perm_from_ipiv_na<<<1, 1024, sizeof(uint16_t) * n, s>>>(d_ipiv, (int)n, perm, bad);
        OXI_LAUNCH_CHECK();
        OXI_CUDA(cudaMemcpyAsync(hflags, sc, sizeof(hflags), cudaMemcpyDeviceToHost, s));
        OXI_CUDA(cudaStreamSynchronize(s));
        if (hflags[1]) return OXI_EINVAL;  // B untouched, as oxi_dgetrs
        const i64 tot = n * nrhs;
        const int nt = 256;
        const unsigned gb = (unsigned)((tot + nt - 1) / nt);
        if (trans == 'N') {
            k_gather_rows<double><<<gb, nt, 0, s>>>(dB, ldb, perm, X, n, (int)n, (int)nrhs, 0);
            OXI_LAUNCH_CHECK();
            trsv_launch<double, false, true, false>(dLU, lda, X, n, (int)n, (int)nrhs, ctl, err, s);
            trsv_launch<double, true, false, false>(dLU, lda, X, n, (int)n, (int)nrhs, ctl, err, s);
            OXI_CUDA(cudaMemcpy2DAsync(dB, ldb * sizeof(double), X, n * sizeof(double), n * sizeof(double),
                                       nrhs, cudaMemcpyDeviceToDevice, s));
        } else {
            OXI_CUDA(cudaMemcpy2DAsync(X, n * sizeof(double), dB, ldb * sizeof(double), n * sizeof(double),
                                       nrhs, cudaMemcpyDeviceToDevice, s));
            trsv_launch<double, true, false, true>(dLU, lda, X, n, (int)n, (int)nrhs, ctl, err, s);
            trsv_launch<double, false, true, true>(dLU, lda, X, n, (int)n, (int)nrhs, ctl, err, s);
            k_gather_rows<double><<<gb, nt, 0, s>>>(X, n, perm, dB, ldb, (int)n, (int)nrhs, 1);
            OXI_LAUNCH_CHECK();
        }
        OXI_CUDA(cudaMemcpyAsync(hflags, sc, sizeof(int), cudaMemcpyDeviceToHost, s));
        OXI_CUDA(cudaStreamSynchronize(s));
        return hflags[0] ? OXI_ETIMEOUT : OXI_OK;
    } catch (const CudaError &) {
        return OXI_ECUDA;
    }
}

}  // namespace oxi

extern "C" int oxi_dgetrs_noalloc(void *stream, char trans, int64_t n, int64_t nrhs, const double *dLU,
                                  int64_t lda, const int64_t *d_ipiv, double *dB, int64_t ldb) {
    return oxi::getrs_noalloc((cudaStream_t)stream, trans, n, nrhs, dLU, lda, d_ipiv, dB, ldb);
}

extern "C" int oxi_dgetrs(oxi_handle_t h, char trans, int64_t n, int64_t nrhs, const double *dLU,
                          int64_t lda, const int64_t *d_ipiv, double *dB, int64_t ldb) {
    return oxi::getrs_entry<double>(h, trans, n, nrhs, dLU, lda, d_ipiv, dB, ldb);
}
extern "C" int oxi_sgetrs(oxi_handle_t h, char trans, int64_t n, int64_t nrhs, const float *dLU,
                          int64_t lda, const int64_t *d_ipiv, float *dB, int64_t ldb) {
    return oxi::getrs_entry<float>(h, trans, n, nrhs, dLU, lda, d_ipiv, dB, ldb);
}
