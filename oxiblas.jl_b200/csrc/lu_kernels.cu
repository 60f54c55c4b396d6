// Panel-level kernels of the dense LU: layout conversion, the cluster leaf LU,
// row interchanges, the TRSM leaf and the reference-order GEMM.
//
// Storage inside the engine is ROW-major (row i of an m x n matrix is n
// contiguous elements, leading dimension ld).  Row interchanges -- the laswp of
// src/lapack/factorizations.jl:82-88 -- then move contiguous row segments, and
// a panel row (w elements) is one contiguous load.  The C ABI converts from and
// to the caller's column-major layout at entry and exit.
#include <cooperative_groups.h>
#include <algorithm>
#include <climits>
#include <type_traits>
#include "oxi_internal.h"
#include "tma_util.cuh"

namespace cg = cooperative_groups;

namespace oxi {

// ---------------------------------------------------------------------------
// Layout conversion (32 x 32 tiles through shared memory, conflict-free).
// ---------------------------------------------------------------------------
template <typename TS, typename TD>
__global__ void k_cm_to_rm(const TS *__restrict__ A, i64 lda, TD *__restrict__ W, i64 ldw,
                           i64 m, i64 n) {
    __shared__ TD tile[32][33];
    const i64 i0 = (i64)blockIdx.x * 32, j0 = (i64)blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int r = ty; r < 32; r += 8) {             // read column j0+r, rows i0+tx
        i64 i = i0 + tx, j = j0 + r;
        if (i < m && j < n) tile[r][tx] = (TD)A[i + j * lda];
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {  // write row i0+r, columns j0+tx
        i64 i = i0 + r, j = j0 + tx;
        if (i < m && j < n) W[i * ldw + j] = tile[tx][r];
    }
}

template <typename TS, typename TD>
__global__ void k_rm_to_cm(const TS *__restrict__ W, i64 ldw, TD *__restrict__ A, i64 lda,
                           i64 m, i64 n) {
    __shared__ TD tile[32][33];
    const i64 i0 = (i64)blockIdx.x * 32, j0 = (i64)blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {  // read row i0+r, columns j0+tx
        i64 i = i0 + r, j = j0 + tx;
        if (i < m && j < n) tile[r][tx] = (TD)W[i * ldw + j];
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {  // write column j0+r, rows i0+tx
        i64 i = i0 + tx, j = j0 + r;
        if (i < m && j < n) A[i + j * lda] = tile[tx][r];
    }
}

template <typename TS, typename TD>
void launch_cm_to_rm(const TS *A, i64 lda, TD *W, i64 ldw, i64 m, i64 n, cudaStream_t s) {
    if (m <= 0 || n <= 0) return;
    dim3 grid((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32));
    k_cm_to_rm<TS, TD><<<grid, dim3(32, 8), 0, s>>>(A, lda, W, ldw, m, n);
    OXI_LAUNCH_CHECK();
}
template <typename TS, typename TD>
void launch_rm_to_cm(const TS *W, i64 ldw, TD *A, i64 lda, i64 m, i64 n, cudaStream_t s) {
    if (m <= 0 || n <= 0) return;
    dim3 grid((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32));
    k_rm_to_cm<TS, TD><<<grid, dim3(32, 8), 0, s>>>(W, ldw, A, lda, m, n);
    OXI_LAUNCH_CHECK();
}
template void launch_cm_to_rm<double, double>(const double *, i64, double *, i64, i64, i64, cudaStream_t);
template void launch_cm_to_rm<float, float>(const float *, i64, float *, i64, i64, i64, cudaStream_t);
template void launch_cm_to_rm<double, float>(const double *, i64, float *, i64, i64, i64, cudaStream_t);
template void launch_cm_to_rm<double2, double2>(const double2 *, i64, double2 *, i64, i64, i64, cudaStream_t);
template void launch_rm_to_cm<double, double>(const double *, i64, double *, i64, i64, i64, cudaStream_t);
template void launch_rm_to_cm<float, float>(const float *, i64, float *, i64, i64, i64, cudaStream_t);
template void launch_rm_to_cm<float, double>(const float *, i64, double *, i64, i64, i64, cudaStream_t);

// ---------------------------------------------------------------------------
// Leaf LU: one thread-block cluster (1..16 CTAs of NT = 256 or 512 threads) holds the
// m x W leaf in REGISTERS, R rows per thread (row position i lives in thread
// g = i mod G, slot k = i / G, G = cluster threads).  Column by column, as the
// leaf loop of _lu_panel! (src/lapack/factorizations.jl:116-139):
//   pivot = first row of the largest |a_ij|, i >= j (_lu_pivot, :92-107);
//   swap rows j and p over the leaf's W columns;
//   zero pivot -> info (first one), skip the column;
//   l_ij = a_ij / a_jj (a true division, as the reference);
//   a_ic = muladd(-l_ij, a_jc, a_ic) for c > j.
// Per column each CTA reduces its candidate in registers/shared memory and
// PUSHES it (|value|, position, the whole candidate row) into every CTA's
// shared memory with st.async, one 16-byte store per thread, each completing
// its bytes on the receiver's mbarrier; a CTA waits on its own barrier until
// all candidates have landed and picks the same winner as every other CTA.
// The CTA that owns position j also pushes row j, so the two swapped rows
// never need a second exchange.  Slots are double-buffered by column parity,
// which is what makes one exchange per column sufficient.  Each row carries
// the index of the row it started as; at the end a position whose row changed
// emits a (dst, src) move.  The net permutation reaches the other columns by
// k_rowmoves, or, inside a composed panel, through the leaf itself after a
// cluster barrier (one warp per moved row).
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Warp arg-max for the pivot search with redux.sync: |v| >= 0 orders like its
// bit pattern, so the warp maximum is an integer max (FP64: high word, then
// low word), and the first row among equal maxima is an integer min of the
// positions -- the reference's "largest |a|, first row on ties".  NaN maps to
// the smallest key, as a NaN never wins the reference's strict '>' comparison.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t redux_max_u32(uint32_t v) {
    uint32_t r;
    asm volatile("redux.sync.max.u32 %0, %1, 0xffffffff;" : "=r"(r) : "r"(v));
    return r;
}
__device__ __forceinline__ uint32_t redux_min_u32(uint32_t v) {
    uint32_t r;
    asm volatile("redux.sync.min.u32 %0, %1, 0xffffffff;" : "=r"(r) : "r"(v));
    return r;
}
__device__ __forceinline__ uint64_t pivot_key(float a) {
    return (a == a) ? (uint64_t)__float_as_uint(fabsf(a)) : 0ull;
}
__device__ __forceinline__ uint64_t pivot_key(double a) {
    return (a == a) ? (uint64_t)__double_as_longlong(fabs(a)) : 0ull;
}
// (key, pos) of the warp winner, identical in every lane; pos = INT_MAX when no lane has one.
template <typename T>
__device__ __forceinline__ void warp_argmax(uint64_t &key, int &pos) {
    const uint32_t p = (uint32_t)pos;
    if constexpr (sizeof(T) == 4) {
        const uint32_t k = (uint32_t)key;
        const uint32_t mk = redux_max_u32(p == (uint32_t)INT_MAX ? 0u : k);
        const uint32_t mp = redux_min_u32(k == mk ? p : (uint32_t)INT_MAX);
        key = mk;
        pos = (int)mp;
    } else {
        const uint32_t hi = (uint32_t)(key >> 32), lo = (uint32_t)key;
        const bool valid = p != (uint32_t)INT_MAX;
        const uint32_t mh = redux_max_u32(valid ? hi : 0u);
        const uint32_t ml = redux_max_u32(valid && hi == mh ? lo : 0u);
        const uint32_t mp = redux_min_u32(hi == mh && lo == ml ? p : (uint32_t)INT_MAX);
        key = ((uint64_t)mh << 32) | ml;
        pos = (int)mp;
    }
}

// A row of W elements between registers and 16-byte-aligned shared memory.
template <typename T, int W>
__device__ __forceinline__ void store_row(T *dst, const T (&v)[W]) {
    constexpr int VEC = 16 / sizeof(T);
#pragma unroll
    for (int c = 0; c < W; c += VEC) {
        int4 x;
        T *xx = (T *)&x;
#pragma unroll
        for (int e = 0; e < VEC; ++e) xx[e] = v[c + e];
        *(int4 *)(dst + c) = x;
    }
}
template <typename T, int W>
__device__ __forceinline__ void load_row(T (&v)[W], const T *src) {
    constexpr int VEC = 16 / sizeof(T);
#pragma unroll
    for (int c = 0; c < W; c += VEC) {
        const int4 x = *(const int4 *)(src + c);
        const T *xx = (const T *)&x;
#pragma unroll
        for (int e = 0; e < VEC; ++e) v[c + e] = xx[e];
    }
}

constexpr int LEAF_NT = 512;
constexpr int LEAF_MAX_CS = 16;


template <typename T, int W, int R, int NT>
__global__ void __launch_bounds__(NT, 1)
k_leaf_lu(T *__restrict__ P, i64 ld, int m, int wact, i64 gofs, int64_t *__restrict__ ipiv,
          int64_t *__restrict__ info, int *__restrict__ moves, int *__restrict__ nmoves,
          LeafPanel pn) {
    cg::cluster_group cl = cg::this_cluster();
    const int CS = (int)cl.num_blocks();
    const int cr = (int)cl.block_rank();
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    constexpr int NW = NT / 32;
    // in-leaf row moves: at most 2W moved rows, over at least 8 warps; at most
    // LEAF_MAX_OTHER other panel columns, in 32-column chunks
    constexpr int MOVE_PW = (2 * W + NW - 1) / NW;
    constexpr int MOVE_CH = LEAF_MAX_OTHER / 32;
    constexpr int VEC = 16 / sizeof(T);  // elements per 16-byte vector
    const int G = CS * NT;  // a power of two: positions split by shift and mask
    const int lgG = __ffs(G) - 1;
    const int g = cr * NT + t;
    constexpr int LG_NT = (NT == 512) ? 9 : (NT == 256 ? 8 : 10);
    static_assert((1 << LG_NT) == NT, "NT must be 256 or 512");

    __shared__ __align__(16) uint4 s_cmeta[2][LEAF_MAX_CS];  // per CTA: {key lo, key hi, position, row id}
    __shared__ __align__(16) T s_crow[2][LEAF_MAX_CS][W];
    __shared__ __align__(16) T s_jslot[2][W];
    __shared__ __align__(16) uint4 s_jmeta[2];               // {row id of position j, 0, 0, 0}
    __shared__ __align__(8) uint64_t s_xbar[2];              // exchange barriers, by column parity
    __shared__ uint64_t s_wkey[NW];
    __shared__ int s_wpos[NW];
    __shared__ __align__(16) T s_myrow[W];
    __shared__ int s_myid;
    __shared__ __align__(16) T s_jrow[W];
    __shared__ int s_jid;
    __shared__ int s_piv[W];   // pivots and info stay on chip until the end: no global
    __shared__ int s_info;     // store ahead of the per-column exchange
    __shared__ int s_skip;     // the call was aborted before this launch
    if (t == 0) {
        s_info = 0;
        s_skip = aborted(pn.abort) ? 1 : 0;
        mbar_init(&s_xbar[0], 1);
        mbar_init(&s_xbar[1], 1);
        fence_barrier_init();
    }
    // every CTA's exchange barriers exist before any CTA pushes into them
    if (CS > 1) cl.sync();
    else __syncthreads();
    // CTA 0's reading of the abort word decides for the whole cluster (the
    // word may change between the CTAs' own readings)
    const int skip = (CS > 1) ? *cl.map_shared_rank(&s_skip, 0) : s_skip;
    if (skip) {
        if (CS > 1) cl.sync();  // CTA 0's shared memory stays alive until every CTA read it
        return;
    }
    // An exchange wait that gave up (timeout or the call aborted elsewhere):
    // the CTA leaves the column loop together (at its next barrier), stores
    // nothing and emits no moves, but still meets every cluster barrier.
    bool dead = false;

    // a block the previous launch left in a buffer (see LeafPanel): rows above the leaf
    if (pn.u_rows > 0) {
        const T *us = (const T *)pn.u_src;
        T *ud = (T *)pn.u_dst;
        for (int e = g; e < pn.u_rows * pn.u_cols; e += G) ud[(i64)(e / pn.u_cols) * ld + e % pn.u_cols] = us[e];
    }

    // ---- load: rows of W elements, 16-byte vectors when the row is whole and aligned ----
    T r[R][W];
    int id[R];
    const bool vec_ok = (wact == W) && ((ld * (i64)sizeof(T)) % 16 == 0) && (((uintptr_t)P) % 16 == 0);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int i = k * G + g;
        id[k] = i;
#pragma unroll
        for (int c = 0; c < W; ++c) r[k][c] = T(0);
        if (i < m) {
            const T *src = P + (i64)i * ld;
            if (vec_ok) {
#pragma unroll
                for (int c = 0; c < W; c += VEC) {
                    const int4 v = *(const int4 *)(src + c);
                    const T *vv = (const T *)&v;
#pragma unroll
                    for (int u = 0; u < VEC; ++u) r[k][c + u] = vv[u];
                }
            } else {
#pragma unroll
                for (int c = 0; c < W; ++c)
                    if (c < wact) r[k][c] = src[c];
            }
        }
    }
    const int q = m < wact ? m : wact;

    // The column loop is kept rolled (one copy of the code, resident in the
    // instruction cache).  Each row's registers ROTATE by one slot per column:
    // at step j the active column sits in slot 0, the unfinished columns
    // j+1..W-1 in slots 1..W-1-j and the finished ones behind them, so every
    // register index is static and the update is W-1 independent predicated
    // FMAs.  After W steps the rotation has returned the row to its order.
#pragma unroll 1
    for (int j = 0; j < q; ++j) {
        const int par = j & 1;
        // (a) this thread's best candidate in column j (slot 0)
        uint64_t bk = 0;
        int bp = INT_MAX;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int i = k * G + g;
            // _lu_pivot starts from row j with strict '>': a NaN at row j keeps
            // row j (the largest key), a NaN below never wins (key 0)
            const T v = r[k][0];
            const uint64_t key = (i == j && v != v) ? ~0ull : pivot_key(v);
            if (i >= j && i < m && (bp == INT_MAX || key > bk)) { bk = key; bp = i; }  // slots ascend in i
        }
        // (b) warp winner
        warp_argmax<T>(bk, bp);
        if (lane == 0) { s_wkey[warp] = bk; s_wpos[warp] = bp; }
        __syncthreads();
        // (c) CTA winner: every warp reduces the NW warp results
        uint64_t ck = lane < NW ? s_wkey[lane] : 0ull;
        int cp = lane < NW ? s_wpos[lane] : INT_MAX;
        warp_argmax<T>(ck, cp);
        if (cp != INT_MAX && (cp & (G - 1)) == g) {
            const int kk = cp >> lgG;
#pragma unroll
            for (int k = 0; k < R; ++k)
                if (k == kk) {
                    if (CS == 1) {  // a single CTA stages straight into the slots it reads
                        store_row<T, W>(&s_crow[par][0][0], r[k]);
                        s_cmeta[par][0] = make_uint4((uint32_t)ck, (uint32_t)(ck >> 32), (uint32_t)cp, (uint32_t)id[k]);
                    } else {
                        store_row<T, W>(s_myrow, r[k]);
                        s_myid = id[k];
                    }
                }
        }
        if (CS == 1 && t == 0 && cp == INT_MAX) s_cmeta[par][0] = make_uint4(0u, 0u, (uint32_t)INT_MAX, 0u);
        const bool own_j = (g == j);  // position j: slot 0 of thread j of CTA 0
        if (own_j) {
            if (CS == 1) {
                store_row<T, W>(&s_jslot[par][0], r[0]);
                s_jmeta[par] = make_uint4((uint32_t)id[0], 0u, 0u, 0u);
            } else {
                store_row<T, W>(s_jrow, r[0]);
                s_jid = id[0];
            }
        }
        __syncthreads();
        // (d) every CTA's candidate and, from CTA 0, row j into every CTA's slots
        // of this parity.  Across CTAs each 16-byte store completes its bytes on
        // the receiver's exchange barrier (st.async), and each CTA waits only on
        // its own barrier: no cluster-wide barrier per column.  A slot is
        // rewritten two columns later, after its receiver has pushed the column in
        // between, i.e. after it finished reading the slot.
        if (CS > 1 && !dead) {
            constexpr int PER = 1 + W * (int)sizeof(T) / 16;  // stores per row: meta + 16-byte chunks
            const int npush = CS * PER;                          // this CTA's candidate, to every CTA
            if (t == 0) mbar_arrive_expect_tx(&s_xbar[par], (uint32_t)((CS + 1) * 16 * PER));
            // One 16-byte store per thread, spread over the CTA's warps so that no
            // warp issues more than one round: the candidate on threads
            // 0..npush-1 and, in CTA 0, row j on the next npush.
            const int nall = (cr == 0) ? 2 * npush : npush;
            for (int e = t; e < nall; e += NT) {
                const bool jr = e >= npush;
                const int ee = jr ? e - npush : e;
                const int dst = ee / PER, qq = ee - dst * PER;
                uint4 v;
                uint32_t raddr;
                if (!jr) {
                    if (qq == 0) {
                        v = make_uint4((uint32_t)ck, (uint32_t)(ck >> 32), (uint32_t)cp, (uint32_t)s_myid);
                        raddr = cluster_map_u32(&s_cmeta[par][cr], dst);
                    } else {
                        v = reinterpret_cast<const uint4 *>(s_myrow)[qq - 1];
                        raddr = cluster_map_u32(&s_crow[par][cr][0], dst) + 16u * (qq - 1);
                    }
                } else {
                    if (qq == 0) {
                        v = make_uint4((uint32_t)s_jid, 0u, 0u, 0u);
                        raddr = cluster_map_u32(&s_jmeta[par], dst);
                    } else {
                        v = reinterpret_cast<const uint4 *>(s_jrow)[qq - 1];
                        raddr = cluster_map_u32(&s_jslot[par][0], dst) + 16u * (qq - 1);
                    }
                }
                st_async_v4(raddr, v, cluster_map_u32(&s_xbar[par], dst));
            }
            if (!mbar_wait(&s_xbar[par], (uint32_t)((j >> 1) & 1), pn.abort, 1)) dead = true;
        }
        // (e) winner, identical in every CTA: lanes 0..CS-1 hold one candidate each;
        // the winning row sits in the slot of the CTA that owns its position
        uint64_t wk = 0ull;
        int wp = INT_MAX;
        if (lane < CS) {
            const uint4 mv = s_cmeta[par][lane];
            wk = ((uint64_t)mv.y << 32) | mv.x;
            wp = (int)mv.z;
        }
        warp_argmax<T>(wk, wp);
        const int wq = (wp == INT_MAX) ? 0 : ((wp & (G - 1)) >> LG_NT);
        const T *prow = (wp == INT_MAX) ? &s_jslot[par][0] : &s_crow[par][wq][0];
        const int pid = (wp == INT_MAX) ? (int)s_jmeta[par].x : (int)s_cmeta[par][wq].w;
        if (wp == INT_MAX) wp = j;  // no comparable candidate (all NaN): keep row j
        if (t == 0) s_piv[j] = wp;
        const T d = prow[0];
        if (d == T(0)) {
            // zero pivot: info, no interchange, no elimination (the column is all zero)
            if (t == 0 && s_info == 0) s_info = j + 1;
        } else {
            const int live = W - j;  // slots 1..live-1 hold the unfinished columns
            // (f) the interchange lands in the two owner threads' registers
            if (wp != j) {
                if (own_j) {
#pragma unroll
                    for (int c = 0; c < W; ++c) r[0][c] = prow[c];
                    id[0] = pid;
                }
                if ((wp & (G - 1)) == g) {
                    const int kk = wp >> lgG;
#pragma unroll
                    for (int k = 0; k < R; ++k)
                        if (k == kk) {
                            load_row<T, W>(r[k], &s_jslot[par][0]);
                            id[k] = (int)s_jmeta[par].x;
                        }
                }
            }
            // (g) scale the column and apply the rank-1 update below the pivot to
            // the unfinished slots (the compare is uniform across the warp).  FP32
            // multiplies finished slots by a zero instead of skipping them
            // (fma(-l, 0, a) == a for finite l), FP64 predicates each slot: the
            // faster form measured for each
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int i = k * G + g;
                if (i > j && i < m) {
                    const T l = r[k][0] / d;
                    r[k][0] = l;
                    if constexpr (sizeof(T) == 4) {
#pragma unroll
                        for (int c = 1; c < W; ++c) r[k][c] = fma(-l, (c < live) ? prow[c] : T(0), r[k][c]);
                    } else {
#pragma unroll
                        for (int c = 1; c < W; ++c)
                            if (c < live) r[k][c] = fma(-l, prow[c], r[k][c]);
                    }
                }
            }
        }
        // (h) rotate: the finished column moves behind the unfinished ones
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const T t0 = r[k][0];
#pragma unroll
            for (int c = 0; c < W - 1; ++c) r[k][c] = r[k][c + 1];
            r[k][W - 1] = t0;
        }
    }
    // pivots and info, written once
    dead = __syncthreads_or(dead);
    if (!dead && cr == 0 && t < q) ipiv[gofs + t] = gofs + s_piv[t] + 1;
    if (!dead && cr == 0 && t == 0 && s_info != 0 && *info == 0) *info = gofs + s_info;
    // undo the rotation left by q < W steps (slot s holds column (s + q) mod W)
    const int rot = q % W;

    // store the leaf and emit the moves of the net permutation
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int i = k * G + g;
        if (i < m && !dead) {
            T *dst = P + (i64)i * ld;
            if (vec_ok && rot == 0) {
#pragma unroll
                for (int c = 0; c < W; c += VEC) {
                    int4 v;
                    T *vv = (T *)&v;
#pragma unroll
                    for (int u = 0; u < VEC; ++u) vv[u] = r[k][c + u];
                    *(int4 *)(dst + c) = v;
                }
            } else {
#pragma unroll
                for (int s = 0; s < W; ++s) {
                    int c = s + rot;
                    if (c >= W) c -= W;
                    if (c < wact) dst[c] = r[k][s];
                }
            }
            if (id[k] != i) {
                const int slot = atomicAdd(nmoves, 1);
                moves[2 * slot] = i;
                moves[2 * slot + 1] = id[k];
            }
        }
    }
    if (pn.nother > 0 || pn.map) {
        // The leaf's row interchanges on the panel's other columns, and on the
        // panel row map, done here rather than by separate launches: read every
        // moved row segment, meet at a cluster barrier, write.
        __threadfence();
        if (CS > 1) cl.sync(); else __syncthreads();
        const int cnt = min(*(volatile int *)nmoves, 2 * W);
        // One warp per moved row (warps of the whole cluster, in turn), one lane
        // per column of each 32-column chunk: no division, and the leaf's rows are
        // stored, so their registers are free for the staged values.
        const int gw = cr * NW + warp, nwc = CS * NW;
        const int nother = pn.nother;
        T vals[MOVE_PW][MOVE_CH];
        int dsts[MOVE_PW];
        int mapv[R];
#pragma unroll
        for (int mi = 0; mi < MOVE_PW; ++mi) {
            const int mv = gw + mi * nwc;
            dsts[mi] = -1;
            if (mv < cnt) {
                const int src = __ldcg(&moves[2 * mv + 1]);
                dsts[mi] = __ldcg(&moves[2 * mv]);
                const T *srow = P + (i64)src * ld - pn.leaf_c0;
#pragma unroll
                for (int ci = 0; ci < MOVE_CH; ++ci) {
                    const int oc = ci * 32 + lane;
                    if (oc < nother) vals[mi][ci] = srow[oc < pn.left_n ? pn.pc_lo + oc : pn.right_lo + (oc - pn.left_n)];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int i = k * G + g;
            mapv[k] = (!dead && pn.map && i < m && id[k] != i) ? pn.map[pn.map_off + id[k]] : 0;
        }
        if (CS > 1) cl.sync(); else __syncthreads();
#pragma unroll
        for (int mi = 0; mi < MOVE_PW; ++mi) {
            if (dsts[mi] >= 0) {
                T *drow = P + (i64)dsts[mi] * ld - pn.leaf_c0;
#pragma unroll
                for (int ci = 0; ci < MOVE_CH; ++ci) {
                    const int oc = ci * 32 + lane;
                    if (oc < nother) drow[oc < pn.left_n ? pn.pc_lo + oc : pn.right_lo + (oc - pn.left_n)] = vals[mi][ci];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int i = k * G + g;
            if (!dead && pn.map && i < m && id[k] != i) pn.map[pn.map_off + i] = mapv[k];
        }
    }
    // keep every CTA's shared memory alive until all remote pushes have landed
    if (CS > 1) cl.sync();
    // the move counter back to zero for the next leaf, once every CTA has read it
    if (pn.reset_nmoves) {
        if (CS == 1) __syncthreads();
        if (cr == 0 && t == 0) *nmoves = 0;
    }
}


template <typename T> int leaf_width_for(i64 m);
template <> int leaf_width_for<double>(i64 m) {
    const i64 cap = (i64)LEAF_MAX_CS * LEAF_NT;  // rows per slot
    if (m <= cap * 1) return 32;
    if (m <= cap * 2) return 16;
    if (m <= cap * 4) return 8;
    if (m <= cap * 8) return 4;
    return 0;
}
template <> int leaf_width_for<float>(i64 m) {
    const i64 cap = (i64)LEAF_MAX_CS * LEAF_NT;
    if (m <= cap * 2) return 32;
    if (m <= cap * 4) return 16;
    if (m <= cap * 8) return 8;
    return 0;
}

template <typename T, int W, int R, int NT = LEAF_NT>
static void launch_leaf_wr(T *P, i64 ld, i64 m, int w, i64 gofs, int64_t *ipiv, int64_t *info,
                           int *moves, int *nmoves, cudaStream_t s, LeafPanel pn) {
    const i64 per_cta = (i64)NT * R;
    int need = (int)((m + per_cta - 1) / per_cta);
    int cs = 1;  // cluster sizes kept to powers of two
    while (cs < need) cs <<= 1;
    auto kern = k_leaf_lu<T, W, R, NT>;
    if (cs > 8) OXI_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (pn.nother > LEAF_MAX_OTHER)
        throw CudaError{cudaErrorInvalidValue, "panel too wide for the in-leaf row moves"};
    pn.abort = cur_abort();
    ProfScope ps(KC_LEAF, s, 0.0, 2.0 * (double)m * w * sizeof(T));
    OXI_CUDA(cudaLaunchKernelEx(&cfg, kern, P, ld, (int)m, w, gofs, ipiv, info, moves, nmoves, pn));
    count_launch();
}

template <typename T>
void launch_leaf(T *P, i64 ld, i64 m, int w, i64 gofs, int64_t *ipiv, int64_t *info, int *moves,
                 int *nmoves, int leafw, cudaStream_t s, LeafPanel pn) {
    const i64 cap = (i64)LEAF_MAX_CS * LEAF_NT;
    // FP32 32-wide leaves up to 8192 rows: 256 threads x 2 rows (about 15% faster per
    // column than 512 x 1: half the warps repeat the per-column work); FP64 keeps
    // 512 x 1 (its 2-row variant needs 254 registers and measured slower)
    if constexpr (sizeof(T) == 8) {
        if (leafw == 32) launch_leaf_wr<T, 32, 1>(P, ld, m, w, gofs, ipiv, info, moves, nmoves, s, pn);
        else if (leafw == 16) launch_leaf_wr<T, 16, 2>(P, ld, m, w, gofs, ipiv, info, moves, nmoves, s, pn);
        else if (leafw == 8) launch_leaf_wr<T, 8, 4>(P, ld, m, w, gofs, ipiv, info, moves, nmoves, s, pn);
        else launch_leaf_wr<T, 4, 8>(P, ld, m, w, gofs, ipiv, info, moves, nmoves, s, pn);
    } else {
        if (leafw == 32) {
            if (m <= cap) launch_leaf_wr<T, 32, 2, 256>(P, ld, m, w, gofs, ipiv, info, moves, nmoves, s, pn);
            else launch_leaf_wr<T, 32, 2>(P, ld, m, w, gofs, ipiv, info, moves, nmoves, s, pn);
        } else if (leafw == 16) {
            launch_leaf_wr<T, 16, 4>(P, ld, m, w, gofs, ipiv, info, moves, nmoves, s, pn);
        } else {
            launch_leaf_wr<T, 8, 8>(P, ld, m, w, gofs, ipiv, info, moves, nmoves, s, pn);
        }
    }
}
template void launch_leaf<double>(double *, i64, i64, int, i64, int64_t *, int64_t *, int *, int *, int, cudaStream_t, LeafPanel);
template void launch_leaf<float>(float *, i64, i64, int, i64, int64_t *, int64_t *, int *, int *, int, cudaStream_t, LeafPanel);

// ---------------------------------------------------------------------------
// Row moves: W[r0 + dst][c] <- W[r0 + src][c] for every move, all sources read
// before any destination is written.  One thread per column: the moves of a
// column are private to its thread, so no synchronisation is needed, and a warp
// touches 32 contiguous elements of each row (coalesced).
// ---------------------------------------------------------------------------
constexpr int MAX_MOVES = 64;
constexpr int MAX_MOVES_LEAF = 64;  // a leaf of <= 32 columns moves at most 64 rows

template <typename T>
__global__ void k_rowmoves(T *__restrict__ W, i64 ld, i64 r0, const int *__restrict__ moves,
                           const int *__restrict__ nmoves, i64 c_lo, i64 c_hi, i64 skip_lo,
                           i64 skip_hi) {
    const i64 c = c_lo + (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= c_hi || (c >= skip_lo && c < skip_hi)) return;
    const int cnt = min(*nmoves, MAX_MOVES);
    T tmp[MAX_MOVES];
    T *base = W + r0 * ld + c;
#pragma unroll
    for (int e = 0; e < MAX_MOVES; ++e)
        if (e < cnt) tmp[e] = base[(i64)moves[2 * e + 1] * ld];
#pragma unroll
    for (int e = 0; e < MAX_MOVES; ++e)
        if (e < cnt) base[(i64)moves[2 * e] * ld] = tmp[e];
}

template <typename T>
void launch_rowmoves(T *W, i64 ld, i64 r0, const int *moves, const int *nmoves, i64 c_lo, i64 c_hi,
                     i64 skip_lo, i64 skip_hi, cudaStream_t s) {
    if (c_hi <= c_lo) return;
    const int nt = 128;
    const i64 cols = c_hi - c_lo;
    ProfScope ps(KC_ROWMOVES, s, 0.0, 0.0);
    k_rowmoves<T><<<(unsigned)((cols + nt - 1) / nt), nt, 0, s>>>(W, ld, r0, moves, nmoves, c_lo, c_hi,
                                                                   skip_lo, skip_hi);
    OXI_LAUNCH_CHECK();
}
template void launch_rowmoves<double>(double *, i64, i64, const int *, const int *, i64, i64, i64, i64, cudaStream_t);
template void launch_rowmoves<float>(float *, i64, i64, const int *, const int *, i64, i64, i64, i64, cudaStream_t);

// ---------------------------------------------------------------------------
// Panel-level composition of the leaves' row permutations.  map[p] = the row
// (relative to the panel's first row) whose data sits at position p; each
// leaf's moves compose into it, and at the end of the panel the positions with
// map[p] != p form one move list for all the columns outside the panel.
// ---------------------------------------------------------------------------
// identity row map of a panel; also zeroes the panel's move counter and its
// move-list count (no separate memsets on the panel's critical path)
__global__ void k_rowmap_init(int *__restrict__ map, int len, int *__restrict__ zero0, int *__restrict__ zero1) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < len) map[p] = p;
    if (p == 0) {
        if (zero0) *zero0 = 0;
        if (zero1) *zero1 = 0;
    }
}
__global__ void k_rowmap_apply(int *__restrict__ map, int offset, const int *__restrict__ moves,
                               const int *__restrict__ nmoves) {
    const int e = threadIdx.x;
    const int cnt = min(*nmoves, MAX_MOVES_LEAF);
    int v = 0;
    if (e < cnt) v = map[offset + moves[2 * e + 1]];
    __syncthreads();
    if (e < cnt) map[offset + moves[2 * e]] = v;
}
__global__ void k_rowmap_extract(const int *__restrict__ map, int len, int *__restrict__ list,
                                 int *__restrict__ cnt) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= len) return;
    const int src = map[p];
    if (src != p) {
        const int slot = atomicAdd(cnt, 1);
        list[2 * slot] = p;
        list[2 * slot + 1] = src;
    }
}

// All sources of a CTA's column slab are staged in shared memory before any
// destination is written, so cycles of the permutation are safe.  Each thread
// owns one 16-byte vector column of the slab and walks the move list with a
// stride, 8 independent loads in flight.
template <typename T, bool VEC>
__global__ void __launch_bounds__(256) k_rowmoves_big(T *__restrict__ W, i64 ld, i64 r0,
                                                      const int *__restrict__ list,
                                                      const int *__restrict__ cnt_ptr, int maxcnt,
                                                      i64 c_lo, i64 c_hi, int cpc) {
    extern __shared__ __align__(16) unsigned char rm_smem[];
    constexpr int V = VEC ? 16 / (int)sizeof(T) : 1;
    using VT = typename std::conditional<VEC, int4, T>::type;
    VT *buf = reinterpret_cast<VT *>(rm_smem);
    const int cnt = min(*cnt_ptr, maxcnt);
    const i64 cbase = c_lo + (i64)blockIdx.x * cpc;
    const int cols = (int)((c_hi - cbase) < (i64)cpc ? (c_hi - cbase) : (i64)cpc);
    if (cols <= 0 || cnt == 0) return;
    const int nv = cpc / V;                 // vector columns per slab
    const int v = threadIdx.x % nv, g = threadIdx.x / nv, G = blockDim.x / nv;
    const bool full = (v + 1) * V <= cols;  // this thread's vector lies inside the slab
    const bool part = !full && v * V < cols;
    T *base = W + r0 * ld + cbase + (i64)v * V;
#pragma unroll 8
    for (int e = g; e < cnt; e += G) {
        const T *src = base + (i64)list[2 * e + 1] * ld;
        if (full) {
            buf[(i64)e * nv + v] = *reinterpret_cast<const VT *>(src);
        } else if (part) {
            T tmp[V];
            for (int u = 0; u < V; ++u) tmp[u] = (v * V + u < cols) ? src[u] : T(0);
            buf[(i64)e * nv + v] = *reinterpret_cast<VT *>(tmp);
        }
    }
    __syncthreads();
#pragma unroll 8
    for (int e = g; e < cnt; e += G) {
        T *dst = base + (i64)list[2 * e] * ld;
        if (full) {
            *reinterpret_cast<VT *>(dst) = buf[(i64)e * nv + v];
        } else if (part) {
            const VT val = buf[(i64)e * nv + v];
            const T *tv = reinterpret_cast<const T *>(&val);
            for (int u = 0; u < V; ++u)
                if (v * V + u < cols) dst[u] = tv[u];
        }
    }
}

void launch_rowmap_init(int *map, i64 len, int *zero0, int *zero1, cudaStream_t s) {
    if (len <= 0) return;
    k_rowmap_init<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(map, (int)len, zero0, zero1);
    OXI_LAUNCH_CHECK();
}
void launch_rowmap_apply(int *map, i64 offset, const int *moves, const int *nmoves, cudaStream_t s) {
    k_rowmap_apply<<<1, MAX_MOVES_LEAF, 0, s>>>(map, (int)offset, moves, nmoves);
    OXI_LAUNCH_CHECK();
}
void launch_rowmap_extract(const int *map, i64 len, int *list, int *cnt, cudaStream_t s) {
    if (len <= 0) return;
    k_rowmap_extract<<<(unsigned)((len + 255) / 256), 256, 0, s>>>(map, (int)len, list, cnt);
    OXI_LAUNCH_CHECK();
}
template <typename T>
void launch_rowmoves_big(T *W, i64 ld, i64 r0, const int *list, const int *cnt, int maxcnt, i64 c_lo,
                         i64 c_hi, cudaStream_t s) {
    if (c_hi <= c_lo || maxcnt <= 0) return;
    const int V = 16 / (int)sizeof(T);
    const bool vec = ((uintptr_t)W % 16 == 0) && ((ld * (i64)sizeof(T)) % 16 == 0) && (c_lo % V == 0);
    // slab of 64 columns (FP32) / 32 (FP64): 16 or 8 threads per row, 16 or 32 rows at once
    int cpc = vec ? 16 * V : 64;
    while (cpc > V && (size_t)maxcnt * cpc * sizeof(T) > 160 * 1024) cpc /= 2;
    const size_t smem = (size_t)maxcnt * cpc * sizeof(T);
    constexpr int kMaxSmem = 200 * 1024;  // the kernel's one limit (see set_max_dyn_smem)
    if (smem > (size_t)kMaxSmem) throw CudaError{cudaErrorInvalidValue, "panel too wide for the row moves"};
    ProfScope ps(KC_ROWMOVES, s, 0.0, 2.0 * maxcnt * (double)(c_hi - c_lo) * sizeof(T));
    const i64 blocks = (c_hi - c_lo + cpc - 1) / cpc;
    if (vec) {
        set_max_dyn_smem((const void *)k_rowmoves_big<T, true>, kMaxSmem);
        k_rowmoves_big<T, true><<<(unsigned)blocks, 256, smem, s>>>(W, ld, r0, list, cnt, maxcnt, c_lo, c_hi, cpc);
    } else {
        set_max_dyn_smem((const void *)k_rowmoves_big<T, false>, kMaxSmem);
        k_rowmoves_big<T, false><<<(unsigned)blocks, 256, smem, s>>>(W, ld, r0, list, cnt, maxcnt, c_lo, c_hi, cpc);
    }
    OXI_LAUNCH_CHECK();
}
template void launch_rowmoves_big<double>(double *, i64, i64, const int *, const int *, int, i64, i64, cudaStream_t);
template void launch_rowmoves_big<float>(float *, i64, i64, const int *, const int *, int, i64, i64, cudaStream_t);

// ---------------------------------------------------------------------------
// TRSM leaf: B (t x N) <- L^-1 B with L unit lower (t <= 32), row-major.  One
// thread per right-hand-side column, L staged in shared memory; the order is
// the reference leaf's (src/blas/level3.jl:309-321): s = b_i, then
// s = muladd(-L_ip, b_p, s) for p = 1..i-1.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_trsm_leaf(const T *__restrict__ L, i64 ldl, T *__restrict__ B, i64 ldb, int t,
                            i64 N) {
    __shared__ T sL[32][33];
    for (int e = threadIdx.x; e < t * t; e += blockDim.x) {
        const int i = e / t, p = e - i * t;
        sL[i][p] = L[(i64)i * ldl + p];
    }
    __syncthreads();
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    T x[32];
#pragma unroll
    for (int i = 0; i < 32; ++i)
        if (i < t) x[i] = B[(i64)i * ldb + c];
#pragma unroll
    for (int i = 1; i < 32; ++i) {
        if (i < t) {
            T s = x[i];
#pragma unroll
            for (int p = 0; p < i; ++p) s = fma(-sL[i][p], x[p], s);
            x[i] = s;
        }
    }
#pragma unroll
    for (int i = 1; i < 32; ++i)
        if (i < t) B[(i64)i * ldb + c] = x[i];
}

// Column-oriented (right-looking) leaf for the tensor-core engine: once x_p is
// final, x_i -= L_ip x_p for all i > p -- t-p independent FMAs per step instead
// of one dependent chain per row.  One right-hand-side column per thread.
template <typename T>
__global__ void k_trsm_leaf_col(const T *__restrict__ L, i64 ldl, T *__restrict__ B, i64 ldb, int t,
                                i64 N) {
    __shared__ T sL[32][33];
    for (int e = threadIdx.x; e < t * t; e += blockDim.x) {
        const int i = e / t, p = e - i * t;
        sL[i][p] = L[(i64)i * ldl + p];
    }
    __syncthreads();
    const i64 c = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    T x[32];
#pragma unroll
    for (int i = 0; i < 32; ++i)
        if (i < t) x[i] = B[(i64)i * ldb + c];
#pragma unroll
    for (int p = 0; p < 31; ++p) {
        if (p + 1 < t) {
            const T xp = x[p];
#pragma unroll
            for (int i = p + 1; i < 32; ++i)
                if (i < t) x[i] = fma(-sL[i][p], xp, x[i]);
        }
    }
#pragma unroll
    for (int i = 1; i < 32; ++i)
        if (i < t) B[(i64)i * ldb + c] = x[i];
}

template <typename T>
void launch_trsm_leaf(const T *L, i64 ldl, T *B, i64 ldb, int t, i64 N, cudaStream_t s,
                      bool ref_order) {
    if (t <= 1 || N <= 0) return;  // a unit 1x1 triangle is the identity
    const int nt = 128;
    ProfScope ps(KC_TRSM_LEAF, s, (double)t * t * N, 2.0 * (double)t * N * sizeof(T));
    if (ref_order) {
        k_trsm_leaf<T><<<(unsigned)((N + nt - 1) / nt), nt, 0, s>>>(L, ldl, B, ldb, t, N);
    } else {
        k_trsm_leaf_col<T><<<(unsigned)((N + nt - 1) / nt), nt, 0, s>>>(L, ldl, B, ldb, t, N);
    }
    OXI_LAUNCH_CHECK();
}
// ---------------------------------------------------------------------------
// Fused blocked TRSM (tensor-core engine): B (t x N) <- L^-1 B for a unit lower
// L with t <= 256, one CTA per 32-column strip of B kept in shared memory for
// the whole solve.  Block row I: X_I -= sum_{J<I} L_IJ X_J (L blocks staged
// through shared memory), then the 32 x 32 diagonal block by warp-shuffle
// substitution (lane = row, one warp per 4 columns).  One launch replaces the
// recursive halving's leaves and GEMMs.
// ---------------------------------------------------------------------------
constexpr int TF_TB = 32, TF_TMAX = 256;

// Right-looking: for each 32-row block J, solve its 32 x 32 diagonal block by
// warp-shuffle substitution (lane = row, one warp per CW/8 columns), then update
// all rows below with that block's solution in one pass (L column block staged in
// shared memory, four columns per thread).  CW = 32 columns per CTA for wide
// right-hand sides, 8 for narrow ones (a panel's U12): four times the CTAs, a
// quarter of the dependent chain per CTA.
template <typename T, int CW>
__global__ void __launch_bounds__(256) k_trsm_fused(const T *__restrict__ L, i64 ldl, T *__restrict__ B,
                                                    i64 ldb, int t, i64 N) {
    constexpr int NG = CW / 4, RG = 256 / NG;                 // column groups of 4, row groups
    constexpr int QMAX = (TF_TMAX - TF_TB + RG - 1) / RG;     // rows per thread below a block
    constexpr int CPW = CW / 8;                               // chain columns per warp
    extern __shared__ __align__(16) unsigned char tf_smem[];
    T(*X)[CW + 1] = reinterpret_cast<T(*)[CW + 1]>(tf_smem);
    T(*Lc)[TF_TB + 1] = reinterpret_cast<T(*)[TF_TB + 1]>(tf_smem + sizeof(T) * TF_TMAX * (CW + 1));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const i64 c0 = (i64)blockIdx.x * CW;
    const int cols = (int)((N - c0) < CW ? (N - c0) : CW);
    for (int e = tid; e < t * CW; e += 256) {
        const int i = e / CW, c = e % CW;
        X[i][c] = (c < cols) ? B[(i64)i * ldb + c0 + c] : T(0);
    }
    const int nblk = (t + TF_TB - 1) / TF_TB;
    const int cq = (tid % NG) * 4, rq = tid / NG;  // update mapping: rows rq + RG q, columns cq..cq+3
    for (int J = 0; J < nblk; ++J) {
        const int j0 = J * TF_TB, jrows = min(TF_TB, t - j0);
        const int rb = j0 + jrows, nrem = t - rb;  // rows below the block
        // stage L[j0.., j0..j0+31] (diagonal block first, then the rows below)
        for (int e = tid; e < (t - j0) * TF_TB; e += 256) {
            const int rr = e / TF_TB, pp = e % TF_TB;
            Lc[rr][pp] = (pp < jrows) ? L[(i64)(j0 + rr) * ldl + j0 + pp] : T(0);
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < CPW; ++q) {
            const int c = warp * CPW + q;
            T x = (lane < jrows) ? X[j0 + lane][c] : T(0);
            for (int p = 0; p < jrows - 1; ++p) {
                const T xp = __shfl_sync(0xffffffffu, x, p);
                if (lane > p) x = fma(-Lc[lane][p], xp, x);
            }
            if (lane < jrows) X[j0 + lane][c] = x;
        }
        __syncthreads();
        if (nrem > 0) {
            T acc[QMAX][4];
#pragma unroll
            for (int q = 0; q < QMAX; ++q)
#pragma unroll
                for (int u = 0; u < 4; ++u) acc[q][u] = T(0);
#pragma unroll 4
            for (int p = 0; p < jrows; ++p) {
                const T x0 = X[j0 + p][cq], x1 = X[j0 + p][cq + 1], x2 = X[j0 + p][cq + 2], x3 = X[j0 + p][cq + 3];
#pragma unroll
                for (int q = 0; q < QMAX; ++q) {
                    const int r = rq + RG * q;
                    if (r < nrem) {
                        const T l = Lc[TF_TB + r][p];
                        acc[q][0] = fma(l, x0, acc[q][0]);
                        acc[q][1] = fma(l, x1, acc[q][1]);
                        acc[q][2] = fma(l, x2, acc[q][2]);
                        acc[q][3] = fma(l, x3, acc[q][3]);
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < QMAX; ++q) {
                const int r = rq + RG * q;
                if (r < nrem) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) X[rb + r][cq + u] -= acc[q][u];
                }
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < t * CW; e += 256) {
        const int i = e / CW, c = e % CW;
        if (c < cols) B[(i64)i * ldb + c0 + c] = X[i][c];
    }
}

template <typename T>
void launch_trsm_fused(const T *L, i64 ldl, T *B, i64 ldb, int t, i64 N, cudaStream_t s) {
    if (t <= 1 || N <= 0) return;
    ProfScope ps(KC_TRSM_LEAF, s, (double)t * t * N, 2.0 * (double)t * N * sizeof(T));
    if (N <= 2048) {
        constexpr int CW = 8;
        const size_t smem = sizeof(T) * ((size_t)TF_TMAX * (CW + 1) + (size_t)TF_TMAX * (TF_TB + 1));
        set_max_dyn_smem((const void *)k_trsm_fused<T, CW>, (int)smem);
        k_trsm_fused<T, CW><<<(unsigned)((N + CW - 1) / CW), 256, smem, s>>>(L, ldl, B, ldb, t, N);
    } else {
        constexpr int CW = 32;
        const size_t smem = sizeof(T) * ((size_t)TF_TMAX * (CW + 1) + (size_t)TF_TMAX * (TF_TB + 1));
        set_max_dyn_smem((const void *)k_trsm_fused<T, CW>, (int)smem);
        k_trsm_fused<T, CW><<<(unsigned)((N + CW - 1) / CW), 256, smem, s>>>(L, ldl, B, ldb, t, N);
    }
    OXI_LAUNCH_CHECK();
}
// ---------------------------------------------------------------------------
// Reference-order TRSM (FP64, t <= 128): B (t x N) <- L^-1 B for a unit lower
// L, performing element by element the operations of the reference's
// recursive solve (src/blas/level3.jl:338-355, _trsm_blocks_left!): halve the
// triangle (h = t / 2), solve the top half, update the bottom half with one
// fma chain from zero per element followed by a subtraction (the GEMM of
// src/blas/gemm.jl:286-298 / simd.jl:151 for k <= kc), solve the bottom half;
// leaves of <= 8 rows by substitution, s = b; s = fma(-L[i,p], x[p], s) for
// p < i (_trsm_leaf_generic!, level3.jl:309-321).  The host flattens the
// recursion into a list of leaf and update steps in the recursion's order; one
// CTA takes CW columns and runs the list with its columns in shared memory, so
// one launch gives the recursive solve's bits.
// ---------------------------------------------------------------------------
struct TrsmSteps {
    int count;
    int4 step[64];  // {kind (0 leaf, 1 update), a, b, c}: leaf rows [a, b); update rows [b, c) from [a, b)
};

static void trsm_steps_rec(int a, int b, TrsmSteps &st) {
    if (b - a <= 8) {
        st.step[st.count++] = make_int4(0, a, b, 0);
        return;
    }
    const int h = (b - a) / 2;
    trsm_steps_rec(a, a + h, st);
    st.step[st.count++] = make_int4(1, a, a + h, b);
    trsm_steps_rec(a + h, b, st);
}

constexpr int TR_TMAX = 128;

template <int CW>
__global__ void __launch_bounds__(256) k_trsm_refo(const double *__restrict__ L, i64 ldl, double *__restrict__ B,
                                                   i64 ldb, int t, i64 N, const __grid_constant__ TrsmSteps st) {
    // L is read through the L1 cache (threads of a warp that share a row read
    // the same element: one broadcast load), the CTA's columns stay in shared
    // memory: t x (CW + 1) doubles, several CTAs per SM.
    extern __shared__ __align__(16) double tr_smem[];
    double *X = tr_smem;
    constexpr int XP = CW + 1;
    const int tid = threadIdx.x;
    const i64 c0 = (i64)blockIdx.x * CW;
    const int cols = (int)((N - c0) < CW ? (N - c0) : CW);
    for (int e = tid; e < t * CW; e += 256) {
        const int i = e / CW, c = e - i * CW;
        X[i * XP + c] = (c < cols) ? B[(i64)i * ldb + c0 + c] : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < st.count; ++k) {
        const int4 o = st.step[k];
        if (o.x == 0) {
            // leaf of nl <= 8 rows: the column in registers, the triangle's
            // loads all issued up front (fully unrolled, predicated)
            if (tid < CW) {
                const int nl = o.z - o.y;
                double xv[8], lv[8][8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    xv[u] = (u < nl) ? X[(o.y + u) * XP + tid] : 0.0;
#pragma unroll
                    for (int pp = 0; pp < u; ++pp)
                        lv[u][pp] = (u < nl) ? __ldg(L + (i64)(o.y + u) * ldl + o.y + pp) : 0.0;
                }
#pragma unroll
                for (int u = 1; u < 8; ++u)
#pragma unroll
                    for (int pp = 0; pp < u; ++pp) xv[u] = fma(-lv[u][pp], xv[pp], xv[u]);
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (u < nl) X[(o.y + u) * XP + tid] = xv[u];
            }
        } else {
            // rows [o.z, o.w) -= L[rows, o.y:o.z] X[o.y:o.z]: a thread takes four
            // columns of up to two rows (register blocking; each element is
            // still one fma chain in pp order, then the subtraction)
            constexpr int NG = CW / 4, RGS = 256 / NG;
            const int cq = (tid % NG) * 4, rg = tid / NG;
            for (int r0 = o.z + rg; r0 < o.w; r0 += 2 * RGS) {
                const int r1 = r0 + RGS;
                const bool has1 = r1 < o.w;
                const double *L0 = L + (i64)r0 * ldl, *L1 = L + (i64)(has1 ? r1 : r0) * ldl;
                double a0[4] = {0.0, 0.0, 0.0, 0.0}, a1[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
                for (int pp = o.y; pp < o.z; ++pp) {
                    const double l0 = __ldg(L0 + pp), l1 = __ldg(L1 + pp);
                    const double *xr = X + pp * XP + cq;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        a0[u] = fma(l0, xr[u], a0[u]);
                        a1[u] = fma(l1, xr[u], a1[u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) X[r0 * XP + cq + u] -= a0[u];
                if (has1) {
#pragma unroll
                    for (int u = 0; u < 4; ++u) X[r1 * XP + cq + u] -= a1[u];
                }
            }
        }
        __syncthreads();
    }
    for (int e = tid; e < t * CW; e += 256) {
        const int i = e / CW, c = e - i * CW;
        if (c < cols) B[(i64)i * ldb + c0 + c] = X[i * XP + c];
    }
}

bool trsm_refo_applicable(int t) { return t >= 2 && t <= TR_TMAX; }

void launch_trsm_refo(const double *L, i64 ldl, double *B, i64 ldb, int t, i64 N, cudaStream_t s) {
    if (t <= 1 || N <= 0) return;
    if (t > TR_TMAX) throw CudaError{cudaErrorInvalidValue, "reference-order TRSM: triangle too large"};
    TrsmSteps st{};
    trsm_steps_rec(0, t, st);
    ProfScope ps(KC_TRSM_LEAF, s, (double)t * t * N, 2.0 * (double)t * N * 8);
    if (N <= 2048) {
        constexpr int CW = 8;
        const size_t smem = sizeof(double) * (size_t)t * (CW + 1);
        k_trsm_refo<CW><<<(unsigned)((N + CW - 1) / CW), 256, smem, s>>>(L, ldl, B, ldb, t, N, st);
    } else {
        constexpr int CW = 32;
        const size_t smem = sizeof(double) * (size_t)t * (CW + 1);
        k_trsm_refo<CW><<<(unsigned)((N + CW - 1) / CW), 256, smem, s>>>(L, ldl, B, ldb, t, N, st);
    }
    OXI_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Rank-k update in the order of a panel leaf's rank-1 steps (FP64): for every
// element of C (M x N, row-major), s = C; s = fma(-A[r,k], B[k,c], s) for
// k = 0..K-1.  Inside the reference's 32-column leaf (src/lapack/
// factorizations.jl:117-139) the columns right of step k receive exactly this
// sequence, so a leaf narrower than 32 columns followed by this update (and a
// substitution solve of its rows) reproduces the 32-column leaf's bits.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_rankk_seq(double *__restrict__ C, i64 ldc, const double *__restrict__ A,
                                                   i64 lda, const double *__restrict__ B, i64 ldb, int M, int N,
                                                   int K) {
    const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (i64)M * N) return;
    const int r = (int)(idx / N), c = (int)(idx - (i64)r * N);
    const double *a = A + (i64)r * lda;
    double sv = C[(i64)r * ldc + c];
    for (int k = 0; k < K; ++k) sv = fma(-a[k], B[(i64)k * ldb + c], sv);
    C[(i64)r * ldc + c] = sv;
}

void launch_rankk_seq(double *C, i64 ldc, const double *A, i64 lda, const double *B, i64 ldb, i64 M, i64 N,
                      i64 K, cudaStream_t s) {
    if (M <= 0 || N <= 0 || K <= 0) return;
    ProfScope ps(KC_GEMM_REF, s, 2.0 * M * N * K, 8.0 * (2.0 * M * N + M * K + K * N));
    const i64 tot = M * N;
    k_rankk_seq<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(C, ldc, A, lda, B, ldb, (int)M, (int)N, (int)K);
    OXI_LAUNCH_CHECK();
}

template void launch_trsm_fused<double>(const double *, i64, double *, i64, int, i64, cudaStream_t);
template void launch_trsm_fused<float>(const float *, i64, float *, i64, int, i64, cudaStream_t);

template void launch_trsm_leaf<double>(const double *, i64, double *, i64, int, i64, cudaStream_t, bool);
template void launch_trsm_leaf<float>(const float *, i64, float *, i64, int, i64, cudaStream_t, bool);

// ---------------------------------------------------------------------------
// Reference-order GEMM: C <- C - A*B, s_ij = sum_p fma(A_ip, B_pj, s) in p order
// from zero, then C_ij - s_ij -- the arithmetic of src/blas/gemm.jl:286-298 with
// alpha = -1, beta = 1.  64 x 64 tiles, 16-deep k slabs, 4 x 4 per thread.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_gemm_ref(T *__restrict__ C, i64 ldc, const T *__restrict__ A,
                                                  i64 lda, const T *__restrict__ B, i64 ldb, i64 M,
                                                  i64 N, i64 K) {
    __shared__ T As[16][64 + 1];
    __shared__ T Bs[16][64 + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const i64 m0 = (i64)blockIdx.y * 64, n0 = (i64)blockIdx.x * 64;
    T acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = T(0);
    for (i64 k0 = 0; k0 < K; k0 += 16) {
        for (int e = threadIdx.x; e < 64 * 16; e += 256) {
            const int r = e >> 4, kk = e & 15;   // A: row r, k kk (k contiguous)
            const i64 gi = m0 + r, gk = k0 + kk;
            As[kk][r] = (gi < M && gk < K) ? A[gi * lda + gk] : T(0);
            const int kr = e >> 6, cc = e & 63;  // B: k kr, col cc (n contiguous)
            const i64 gk2 = k0 + kr, gj = n0 + cc;
            Bs[kr][cc] = (gk2 < K && gj < N) ? B[gk2 * ldb + gj] : T(0);
        }
        __syncthreads();
        const int kmax = (int)((K - k0) < 16 ? (K - k0) : 16);
        for (int p = 0; p < kmax; ++p) {
            T a[4], b[4];
#pragma unroll
            for (int x = 0; x < 4; ++x) a[x] = As[p][ty + 16 * x];
#pragma unroll
            for (int y = 0; y < 4; ++y) b[y] = Bs[p][tx + 16 * y];
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) {
            const i64 gi = m0 + ty + 16 * x, gj = n0 + tx + 16 * y;
            if (gi < M && gj < N) C[gi * ldc + gj] = C[gi * ldc + gj] - acc[x][y];
        }
}

template <typename T>
void launch_gemm_ref(T *C, i64 ldc, const T *A, i64 lda, const T *B, i64 ldb, i64 M, i64 N, i64 K,
                     cudaStream_t s) {
    if (M <= 0 || N <= 0 || K <= 0) return;
    dim3 grid((unsigned)((N + 63) / 64), (unsigned)((M + 63) / 64));
    ProfScope ps(KC_GEMM_REF, s, 2.0 * M * N * K, (double)sizeof(T) * (2.0 * M * N + M * K + K * N));
    k_gemm_ref<T><<<grid, 256, 0, s>>>(C, ldc, A, lda, B, ldb, M, N, K);
    OXI_LAUNCH_CHECK();
}
// ---------------------------------------------------------------------------
// Register-blocked CUDA-core GEMM for the FP32 panel (C <- C - A*B, row-major):
// 128 x BN tile, 16-deep k slabs double-buffered through registers, 8 x (BN/16)
// outputs per thread (strided so shared-memory reads broadcast or are
// conflict-free).
// ---------------------------------------------------------------------------
template <typename T, int BN>
__global__ void __launch_bounds__(256) k_gemm_simt(T *__restrict__ C, i64 ldc, const T *__restrict__ A,
                                                   i64 lda, const T *__restrict__ B, i64 ldb, i64 M,
                                                   i64 N, i64 K) {
    constexpr int BM = 128, BK = 16, TN = BN / 16;
    __shared__ T As[2][BK][BM + 4];
    __shared__ T Bs[2][BK][BN + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const i64 m0 = (i64)blockIdx.y * BM, n0 = (i64)blockIdx.x * BN;
    T acc[8][TN];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = 0; b < TN; ++b) acc[a][b] = T(0);
    constexpr int AL = BM * BK / 256, BL = BK * BN / 256;
    T ra[AL], rb[BL];
    auto gload = [&](i64 k0) {
#pragma unroll
        for (int q = 0; q < AL; ++q) {
            const int e = threadIdx.x + q * 256;
            const int r = e / BK, kk = e % BK;
            const i64 gi = m0 + r, gk = k0 + kk;
            ra[q] = (gi < M && gk < K) ? A[gi * lda + gk] : T(0);
        }
#pragma unroll
        for (int q = 0; q < BL; ++q) {
            const int e = threadIdx.x + q * 256;
            const int kr = e / BN, cc = e % BN;
            const i64 gk = k0 + kr, gj = n0 + cc;
            rb[q] = (gk < K && gj < N) ? B[gk * ldb + gj] : T(0);
        }
    };
    auto sstore = [&](int buf) {
#pragma unroll
        for (int q = 0; q < AL; ++q) {
            const int e = threadIdx.x + q * 256;
            As[buf][e % BK][e / BK] = ra[q];
        }
#pragma unroll
        for (int q = 0; q < BL; ++q) {
            const int e = threadIdx.x + q * 256;
            Bs[buf][e / BN][e % BN] = rb[q];
        }
    };
    gload(0);
    sstore(0);
    __syncthreads();
    int buf = 0;
    for (i64 k0 = 0; k0 < K; k0 += BK) {
        const bool more = k0 + BK < K;
        if (more) gload(k0 + BK);
#pragma unroll
        for (int p = 0; p < BK; ++p) {
            T a[8], b[TN];
#pragma unroll
            for (int x = 0; x < 8; ++x) a[x] = As[buf][p][ty + 16 * x];
#pragma unroll
            for (int y = 0; y < TN; ++y) b[y] = Bs[buf][p][tx + 16 * y];
#pragma unroll
            for (int x = 0; x < 8; ++x)
#pragma unroll
                for (int y = 0; y < TN; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
        }
        if (more) {
            sstore(buf ^ 1);
            __syncthreads();
            buf ^= 1;
        }
    }
#pragma unroll
    for (int x = 0; x < 8; ++x) {
        const i64 gi = m0 + ty + 16 * x;
        if (gi >= M) continue;
#pragma unroll
        for (int y = 0; y < TN; ++y) {
            const i64 gj = n0 + tx + 16 * y;
            if (gj < N) C[gi * ldc + gj] -= acc[x][y];
        }
    }
}

template <typename T>
void launch_gemm_simt(T *C, i64 ldc, const T *A, i64 lda, const T *B, i64 ldb, i64 M, i64 N, i64 K,
                      cudaStream_t s) {
    if (M <= 0 || N <= 0 || K <= 0) return;
    ProfScope ps(KC_GEMM_REF, s, 2.0 * M * N * K, (double)sizeof(T) * (2.0 * M * N + M * K + K * N));
    if (N <= 64) {
        dim3 grid((unsigned)((N + 63) / 64), (unsigned)((M + 127) / 128));
        k_gemm_simt<T, 64><<<grid, 256, 0, s>>>(C, ldc, A, lda, B, ldb, M, N, K);
    } else {
        dim3 grid((unsigned)((N + 127) / 128), (unsigned)((M + 127) / 128));
        k_gemm_simt<T, 128><<<grid, 256, 0, s>>>(C, ldc, A, lda, B, ldb, M, N, K);
    }
    OXI_LAUNCH_CHECK();
}
template void launch_gemm_simt<float>(float *, i64, const float *, i64, const float *, i64, i64, i64, i64, cudaStream_t);

// ---------------------------------------------------------------------------
// Right-looking step inside an FP32 panel, after a KW-wide leaf:
//   U12 <- L11^-1 A12     (L11 the leaf's KW x KW unit lower block, A12 the
//                          panel's N columns right of the leaf in those rows)
//   A22 <- A22 - L21 U12  (L21 the leaf's M rows below L11)
// in ONE launch.  Every CTA solves the 64-column slice of U12 it needs (a
// KW-step substitution, one thread per column, L11 from shared memory), the
// CTAs of the first row tile write it to ubuf (the next leaf, or a copy,
// moves it into place once no CTA reads A12 any more), and each CTA then
// updates its 128 x 64 tile of A22 (K = KW).
// ---------------------------------------------------------------------------
template <int KW>
__global__ void __launch_bounds__(256, 2) k_panel_rl(float *__restrict__ P, i64 ld, int M, int N,
                                                  float *__restrict__ ubuf) {
    constexpr int BM = 128, BN = 64;
    __shared__ float Ls[KW][KW + 1];
    __shared__ __align__(16) float Us[KW][BN + 4];
    __shared__ __align__(16) float As[KW][BM + 4];  // the L21 tile, transposed
    const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
    const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM;
    for (int e = t; e < KW * KW; e += 256) Ls[e / KW][e % KW] = P[(i64)(e / KW) * ld + e % KW];
    for (int e = t; e < KW * BN; e += 256) {
        const int i = e / BN, j = e % BN;
        Us[i][j] = (n0 + j < N) ? P[(i64)i * ld + KW + n0 + j] : 0.f;
    }
    for (int e = t; e < BM * KW; e += 256) {
        const int r = e / KW, k = e % KW;
        As[k][r] = (m0 + r < M) ? P[(i64)(KW + m0 + r) * ld + k] : 0.f;
    }
    __syncthreads();
    if (t < BN) {
        float x[KW];
#pragma unroll
        for (int i = 0; i < KW; ++i) x[i] = Us[i][t];
#pragma unroll
        for (int p = 0; p < KW; ++p)
#pragma unroll
            for (int i = p + 1; i < KW; ++i) x[i] = fmaf(-Ls[i][p], x[p], x[i]);
#pragma unroll
        for (int i = 0; i < KW; ++i) Us[i][t] = x[i];
        if (blockIdx.y == 0 && n0 + t < N) {  // not into A12: other CTAs may still read it
#pragma unroll
            for (int i = 0; i < KW; ++i) ubuf[(i64)i * N + n0 + t] = x[i];
        }
    }
    __syncthreads();
    float c[8][4];
#pragma unroll
    for (int x = 0; x < 8; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) {
            const int r = m0 + ty + 16 * x, col = n0 + tx + 16 * y;
            c[x][y] = (r < M && col < N) ? P[(i64)(KW + r) * ld + KW + col] : 0.f;
        }
#pragma unroll 8
    for (int k = 0; k < KW; ++k) {
        float a[8], b[4];
#pragma unroll
        for (int x = 0; x < 8; ++x) a[x] = As[k][ty + 16 * x];
#pragma unroll
        for (int y = 0; y < 4; ++y) b[y] = Us[k][tx + 16 * y];
#pragma unroll
        for (int x = 0; x < 8; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) c[x][y] = fmaf(-a[x], b[y], c[x][y]);
    }
#pragma unroll
    for (int x = 0; x < 8; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) {
            const int r = m0 + ty + 16 * x, col = n0 + tx + 16 * y;
            if (r < M && col < N) P[(i64)(KW + r) * ld + KW + col] = c[x][y];
        }
}

void launch_panel_rl(float *P, i64 ld, int kw, i64 M, i64 N, float *ubuf, cudaStream_t s) {
    if (N <= 0) return;
    dim3 grid((unsigned)((N + 63) / 64), (unsigned)std::max<i64>(1, (M + 127) / 128));
    ProfScope ps(KC_GEMM_REF, s, 2.0 * (double)std::max<i64>(M, 0) * N * kw + (double)kw * kw * N,
                 4.0 * (2.0 * std::max<i64>(M, 0) * N + (double)(M + kw) * kw + 2.0 * kw * N));
    if (kw == 32) k_panel_rl<32><<<grid, 256, 0, s>>>(P, ld, (int)M, (int)N, ubuf);
    else if (kw == 16) k_panel_rl<16><<<grid, 256, 0, s>>>(P, ld, (int)M, (int)N, ubuf);
    else if (kw == 8) k_panel_rl<8><<<grid, 256, 0, s>>>(P, ld, (int)M, (int)N, ubuf);
    else throw CudaError{cudaErrorInvalidValue, "right-looking panel step: leaf width 8, 16 or 32"};
    OXI_LAUNCH_CHECK();
}

template void launch_gemm_ref<double>(double *, i64, const double *, i64, const double *, i64, i64, i64, i64, cudaStream_t);
template void launch_gemm_ref<float>(float *, i64, const float *, i64, const float *, i64, i64, i64, i64, cudaStream_t);

}  // namespace oxi
