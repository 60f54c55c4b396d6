// Complex (ComplexF64) partial-pivoted LU and its solves.
//
// Replaces _lu_factor! / _lu_panel! for Complex{Float64} (src/lapack/
// factorizations.jl:30-152: blocked right-looking with nb = 128, recursive
// panel with 16-column leaves for complex types (:113), the complex pivot rule
// of _lu_pivot (:92-107): the largest abs2, strict '>' so the first row wins,
// redone with abs when the largest square is not finite) and ldiv! with
// trans 'N' / 'T' / 'C' (src/api/linalg_api.jl:168-184).
//
// Layout: the caller's interleaved column-major A is split into two row-major
// FP64 planes (real, imaginary) in the handle's working matrix, so that a row
// interchange moves contiguous segments and the trailing update is four real
// products on the FP64 tensor cores (DMMA):
//   Cr -= Ar Br;  Cr -= (-Ai) Bi;  Ci -= Ar Bi;  Ci -= Ai Br,
// with -Ai a negated copy of the panel's imaginary plane.  The panel's leaves
// run in one CTA each (16 columns, every row of the panel), their interchanges
// are then applied to the other columns (laswp), and the U block row is solved
// by a unit-lower substitution kernel.
#include <cooperative_groups.h>
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>
#include "oxi_internal.h"

namespace oxi {

namespace {
constexpr int ZLEAF = 16;      // complex leaf (the reference's _lu_leaf for complex types)
constexpr int ZLEAF_NT = 1024;
inline i64 zrup(i64 x, i64 a) { return (x + a - 1) / a * a; }
}  // namespace

struct zd {
    double r, i;
};
__device__ __forceinline__ zd zmul(zd a, zd b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
// c - a b: the product, then the difference (muladd(-a, b, c) of the reference)
__device__ __forceinline__ zd zmsub(zd c, zd a, zd b) {
    return {c.r - (a.r * b.r - a.i * b.i), c.i - (a.r * b.i + a.i * b.r)};
}
// a / b, scaled by the larger of |b.r|, |b.i| (no spurious overflow)
__device__ __forceinline__ zd zdivd(zd a, zd b) {
    double s = fmax(fabs(b.r), fabs(b.i));
    if (s == 0.0) s = 1.0;  // a zero divisor: the quotients below become infinite or NaN
    const double br = b.r / s, bi = b.i / s, ar = a.r / s, ai = a.i / s;
    const double den = br * br + bi * bi;
    return {(ar * br + ai * bi) / den, (ai * br - ar * bi) / den};
}

// 1 / b, scaled by the larger of |b.r|, |b.i| (no spurious overflow)
__device__ __forceinline__ zd zrecip(zd b) {
    double s = fmax(fabs(b.r), fabs(b.i));
    if (s == 0.0) s = 1.0;
    const double br = b.r / s, bi = b.i / s;
    const double den = (br * br + bi * bi) * s;
    return {br / den, -bi / den};
}

// (key, position) argmax over the CTA: the largest key, the smallest position
// among equal keys; keys are non-negative doubles (NaN never enters).
__device__ __forceinline__ void cta_argmax(double &key, int &pos, double *s_key, int *s_pos) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int off = 16; off > 0; off >>= 1) {
        const double ok = __shfl_xor_sync(0xffffffffu, key, off);
        const int op = __shfl_xor_sync(0xffffffffu, pos, off);
        if (ok > key || (ok == key && op < pos)) { key = ok; pos = op; }
    }
    if (lane == 0) { s_key[warp] = key; s_pos[warp] = pos; }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        key = lane < nw ? s_key[lane] : -1.0;
        pos = lane < nw ? s_pos[lane] : INT_MAX;
        for (int off = 16; off > 0; off >>= 1) {
            const double ok = __shfl_xor_sync(0xffffffffu, key, off);
            const int op = __shfl_xor_sync(0xffffffffu, pos, off);
            if (ok > key || (ok == key && op < pos)) { key = ok; pos = op; }
        }
        if (lane == 0) { s_key[0] = key; s_pos[0] = pos; }
    }
    __syncthreads();
    key = s_key[0];
    pos = s_pos[0];
    __syncthreads();
}

// Leaf: the m x w (w <= 16) block at (Wr, Wi) (row-major planes, ld), one CTA.
// Column j: the pivot row (largest abs2 among rows >= j; with abs when that
// square is not finite; the row itself when nothing beats it), the interchange
// within the leaf's columns, the multipliers l = a / d and the rank-1 update of
// the leaf's later columns.  ipiv gets gofs + p + 1, info the first zero pivot.
__global__ void __launch_bounds__(ZLEAF_NT) k_zleaf(double *__restrict__ Wr, double *__restrict__ Wi, i64 ld, int m,
                                                    int w, i64 gofs, int64_t *__restrict__ ipiv,
                                                    int64_t *__restrict__ info) {
    __shared__ double s_key[32];
    __shared__ int s_pos[32];
    __shared__ zd s_prow[ZLEAF];
    const int tid = threadIdx.x;
    const int q = m < w ? m : w;
    for (int j = 0; j < q; ++j) {
        // candidates by abs2
        double key = -1.0;
        int pos = INT_MAX;
        bool nonfinite = false;
        for (int i = j + tid; i < m; i += ZLEAF_NT) {
            const double ar = Wr[(i64)i * ld + j], ai = Wi[(i64)i * ld + j];
            const double v = ar * ar + ai * ai;
            if (v == v && v > key) { key = v; pos = i; }
        }
        // the reference starts from row j: a NaN there keeps row j
        {
            const double ar = Wr[(i64)j * ld + j], ai = Wi[(i64)j * ld + j];
            const double v0 = ar * ar + ai * ai;
            if (v0 != v0) { key = (tid == 0) ? INFINITY : -1.0; pos = (tid == 0) ? j : INT_MAX; }
        }
        cta_argmax(key, pos, s_key, s_pos);
        nonfinite = !(key < INFINITY);
        if (nonfinite) {  // redo with abs (hypot) when the largest square overflowed
            double k2 = -1.0;
            int p2 = INT_MAX;
            for (int i = j + tid; i < m; i += ZLEAF_NT) {
                const double v = hypot(Wr[(i64)i * ld + j], Wi[(i64)i * ld + j]);
                if (v == v && v > k2) { k2 = v; p2 = i; }
            }
            const double v0 = hypot(Wr[(i64)j * ld + j], Wi[(i64)j * ld + j]);
            if (v0 != v0) { k2 = (tid == 0) ? INFINITY : -1.0; p2 = (tid == 0) ? j : INT_MAX; }
            cta_argmax(k2, p2, s_key, s_pos);
            pos = p2;
        }
        const int p = (pos == INT_MAX) ? j : pos;
        if (tid == 0) ipiv[gofs + j] = gofs + p + 1;
        if (p != j && tid < w) {  // the interchange within the leaf's columns
            const double tr = Wr[(i64)j * ld + tid], ti = Wi[(i64)j * ld + tid];
            Wr[(i64)j * ld + tid] = Wr[(i64)p * ld + tid];
            Wi[(i64)j * ld + tid] = Wi[(i64)p * ld + tid];
            Wr[(i64)p * ld + tid] = tr;
            Wi[(i64)p * ld + tid] = ti;
        }
        __syncthreads();
        if (tid < w) s_prow[tid] = {Wr[(i64)j * ld + tid], Wi[(i64)j * ld + tid]};
        __syncthreads();
        const zd d = s_prow[j];
        if (d.r == 0.0 && d.i == 0.0) {
            if (tid == 0 && *info == 0) *info = gofs + j + 1;
            continue;
        }
        // the multipliers a / d as a times the reciprocal of d, formed once per
        // column (the reference divides each element; the results agree to
        // rounding)
        const zd dinv = zrecip(d);
        for (int i = j + 1 + tid; i < m; i += ZLEAF_NT) {
            double *rr = Wr + (i64)i * ld, *ri = Wi + (i64)i * ld;
            const zd l = zmul({rr[j], ri[j]}, dinv);
            rr[j] = l.r;
            ri[j] = l.i;
            for (int c = j + 1; c < w; ++c) {
                const zd v = zmsub({rr[c], ri[c]}, l, s_prow[c]);
                rr[c] = v.r;
                ri[c] = v.i;
            }
        }
        __syncthreads();
    }
}

// The same leaf on a cluster of CS CTAs (1..16) that hold the panel's rows in
// shared memory (CTA r: rows [r RP, (r + 1) RP), both planes, 16 columns), so a
// column step reads no global memory: each CTA's candidate (the largest abs2
// and, for the overflow rule, the largest abs, of its rows below j, first index
// on ties), one cluster barrier, every CTA picks the same pivot from the CS
// candidates and |a_jj| (row j lives in CTA 0: j < 16 <= RP), reads the pivot
// row and row j through distributed shared memory, a second barrier, the two
// owners write the interchanged rows, then each CTA eliminates its own rows.
// Cluster barriers are hardware barriers every CTA meets the same number of
// times; there is no spin wait.
namespace cgz = cooperative_groups;
constexpr int ZCL_NT = 512;
constexpr int ZCL_MAXRP = 768;  // rows per CTA (192 KB of shared memory)
struct ZCand {
    double k2, kh;  // largest abs2 / abs among the CTA's rows below j (-1: none)
    int p2, ph;     // their rows (INT_MAX: none)
};
__device__ __forceinline__ void zcand_combine(double &k, int &p, double k2, int p2) {
    if (k2 > k || (k2 == k && p2 < p)) { k = k2; p = p2; }
}
__global__ void __launch_bounds__(ZCL_NT, 1) k_zleaf_cl(double *__restrict__ Wr, double *__restrict__ Wi, i64 ld, int m,
                                                         int w, int RP, i64 gofs, int64_t *__restrict__ ipiv,
                                                         int64_t *__restrict__ info) {
    cgz::cluster_group cl = cgz::this_cluster();
    const int CS = (int)cl.num_blocks(), cr = (int)cl.block_rank();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    extern __shared__ double2 zcl[];  // [RP][ZLEAF] complex
    __shared__ ZCand s_cand[2];
    __shared__ double s_rk[ZCL_NT / 32][2];
    __shared__ int s_rp[ZCL_NT / 32][2];
    __shared__ zd s_prow[ZLEAF], s_jrow[ZLEAF];
    __shared__ int s_piv[ZLEAF], s_info;
    const int r0 = cr * RP;
    const int nr = max(0, min(m - r0, RP));
    if (tid == 0) s_info = 0;
    for (int e = tid; e < nr * ZLEAF; e += ZCL_NT) {
        const int li = e / ZLEAF, c = e - li * ZLEAF;
        const i64 g = (i64)(r0 + li) * ld + c;
        zcl[e] = (c < w) ? make_double2(Wr[g], Wi[g]) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const int q = m < w ? m : w;
    for (int j = 0; j < q; ++j) {
        const int par = j & 1;
        // (1) this CTA's candidates among its rows below j
        double k2 = -1.0, kh = -1.0;
        int p2 = INT_MAX, ph = INT_MAX;
        for (int li = max(0, j + 1 - r0) + tid; li < nr; li += ZCL_NT) {
            const double2 a = zcl[li * ZLEAF + j];
            const double v2 = a.x * a.x + a.y * a.y, vh = hypot(a.x, a.y);
            if (v2 == v2 && v2 > k2) { k2 = v2; p2 = r0 + li; }  // rows ascend per thread: first maximum
            if (vh == vh && vh > kh) { kh = vh; ph = r0 + li; }
        }
        for (int off = 16; off > 0; off >>= 1) {
            zcand_combine(k2, p2, __shfl_xor_sync(0xffffffffu, k2, off), __shfl_xor_sync(0xffffffffu, p2, off));
            zcand_combine(kh, ph, __shfl_xor_sync(0xffffffffu, kh, off), __shfl_xor_sync(0xffffffffu, ph, off));
        }
        if (lane == 0) { s_rk[warp][0] = k2; s_rp[warp][0] = p2; s_rk[warp][1] = kh; s_rp[warp][1] = ph; }
        __syncthreads();
        if (tid == 0) {
            for (int wv = 1; wv < ZCL_NT / 32; ++wv) {
                zcand_combine(k2, p2, s_rk[wv][0], s_rp[wv][0]);
                zcand_combine(kh, ph, s_rk[wv][1], s_rp[wv][1]);
            }
            s_cand[par] = ZCand{k2, kh, p2, ph};
        }
        cl.sync();  // (2) every CTA's candidate is published
        // (3) the pivot, identical in every CTA: _lu_pivot's abs2 scan from row j
        // with strict '>', redone with abs when that square is not finite
        double b2 = -1.0, bh = -1.0;
        int q2 = INT_MAX, qh = INT_MAX;
        for (int rr = 0; rr < CS; ++rr) {
            const ZCand cd = *cl.map_shared_rank(&s_cand[par], rr);
            zcand_combine(b2, q2, cd.k2, cd.p2);
            zcand_combine(bh, qh, cd.kh, cd.ph);
        }
        const double2 ajj = *cl.map_shared_rank(&zcl[j * ZLEAF + j], 0);
        const double v2 = ajj.x * ajj.x + ajj.y * ajj.y;
        int p = j;
        double best = v2;
        if (q2 != INT_MAX && b2 > v2) { best = b2; p = q2; }
        if (!(best < INFINITY)) {  // NaN start or an overflowing square: the abs scan
            const double vh = hypot(ajj.x, ajj.y);
            p = (qh != INT_MAX && bh > vh) ? qh : j;
        }
        // (4) the pivot row and row j through distributed shared memory
        const int cp = p / RP;
        if (tid < ZLEAF) {
            const double2 pv = *cl.map_shared_rank(&zcl[(p - cp * RP) * ZLEAF + tid], cp);
            s_prow[tid] = {pv.x, pv.y};
            const double2 jv = *cl.map_shared_rank(&zcl[j * ZLEAF + tid], 0);
            s_jrow[tid] = {jv.x, jv.y};
        }
        if (cr == 0 && tid == 0) s_piv[j] = p;
        cl.sync();  // (5) every CTA has read both rows before they are rewritten
        if (p != j && tid < ZLEAF) {
            if (cr == 0) zcl[j * ZLEAF + tid] = make_double2(s_prow[tid].r, s_prow[tid].i);
            if (cr == cp) zcl[(p - r0) * ZLEAF + tid] = make_double2(s_jrow[tid].r, s_jrow[tid].i);
        }
        __syncthreads();
        // (6) elimination of this CTA's rows below j
        const zd d = s_prow[j];
        if (d.r == 0.0 && d.i == 0.0) {
            if (cr == 0 && tid == 0 && s_info == 0) s_info = j + 1;
            continue;
        }
        const zd dinv = zrecip(d);
        for (int li = max(0, j + 1 - r0) + tid; li < nr; li += ZCL_NT) {
            double2 *row = zcl + li * ZLEAF;
            const double2 a = row[j];
            const zd l = zmul({a.x, a.y}, dinv);
            row[j] = make_double2(l.r, l.i);
            for (int c = j + 1; c < w; ++c) {
                const double2 b = row[c];
                const zd v = zmsub({b.x, b.y}, l, s_prow[c]);
                row[c] = make_double2(v.r, v.i);
            }
        }
        __syncthreads();
    }
    cl.sync();  // no CTA leaves while another may still read its rows
    for (int e = tid; e < nr * ZLEAF; e += ZCL_NT) {
        const int li = e / ZLEAF, c = e - li * ZLEAF;
        if (c < w) {
            const i64 g = (i64)(r0 + li) * ld + c;
            Wr[g] = zcl[e].x;
            Wi[g] = zcl[e].y;
        }
    }
    if (cr == 0) {
        if (tid < q) ipiv[gofs + tid] = gofs + s_piv[tid] + 1;
        if (tid == 0 && s_info != 0 && *info == 0) *info = gofs + s_info;
    }
}

// laswp: the interchanges ipiv[k0 .. k0+cnt) (global 1-based rows, cnt <= 16)
// on columns [c_lo, c_hi) of both planes.  Their net effect is at most 2 cnt
// row moves (dst <- src); thread 0 of each CTA folds the sequence into that
// list, then every thread moves its column: all sources read, then all
// destinations written (one round trip instead of cnt dependent swaps).
constexpr int ZSWP_MAX = 2 * ZLEAF;
__global__ void k_zlaswp(double *__restrict__ Wr, double *__restrict__ Wi, i64 ld, const int64_t *__restrict__ ipiv,
                         i64 k0, int cnt, i64 c_lo, i64 c_hi, i64 skip_lo, i64 skip_hi) {
    __shared__ i64 s_dst[ZSWP_MAX], s_src[ZSWP_MAX];
    __shared__ int s_n;
    if (threadIdx.x == 0) {
        i64 key[ZSWP_MAX], val[ZSWP_MAX];  // position -> row now there (absent: itself)
        int nk = 0;
        auto find = [&](i64 x) {
            for (int q = 0; q < nk; ++q)
                if (key[q] == x) return q;
            key[nk] = x;
            val[nk] = x;
            return nk++;
        };
        for (int t = 0; t < cnt; ++t) {
            const i64 j = k0 + t, p = ipiv[j] - 1;
            if (p == j) continue;
            const int a = find(j), b = find(p);
            const i64 tmp = val[a];
            val[a] = val[b];
            val[b] = tmp;
        }
        int nm = 0;
        for (int q = 0; q < nk; ++q)
            if (val[q] != key[q]) {
                s_dst[nm] = key[q];
                s_src[nm] = val[q];
                ++nm;
            }
        s_n = nm;
    }
    __syncthreads();
    const int nm = s_n;
    const i64 c = c_lo + (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (nm == 0 || c >= c_hi || (c >= skip_lo && c < skip_hi)) return;
    double vr[ZSWP_MAX], vi[ZSWP_MAX];
#pragma unroll
    for (int q = 0; q < ZSWP_MAX; ++q)
        if (q < nm) {
            vr[q] = Wr[s_src[q] * ld + c];
            vi[q] = Wi[s_src[q] * ld + c];
        }
#pragma unroll
    for (int q = 0; q < ZSWP_MAX; ++q)
        if (q < nm) {
            Wr[s_dst[q] * ld + c] = vr[q];
            Wi[s_dst[q] * ld + c] = vi[q];
        }
}

// B (t x N at (Br, Bi), ld) <- L^-1 B, L the unit lower t x t block at (Lr, Li),
// t <= ZT_MAXT: a CTA per 32 columns, the t x 32 tile in shared memory; once
// row i is final every later row r is updated, x_r -= l_ri x_i (8 row groups of
// a warp each, its lanes across the columns: l_ri is one broadcast load).
constexpr int ZT_NT = 256, ZT_CW = 32, ZT_MAXT = 128;
__global__ void __launch_bounds__(ZT_NT) k_ztrsm_lunit(const double *__restrict__ Lr, const double *__restrict__ Li,
                                                       double *__restrict__ Br, double *__restrict__ Bi, i64 ld,
                                                       int t, i64 N) {
    extern __shared__ double2 zt[];  // [t][ZT_CW]
    const int tid = threadIdx.x, cl = tid & (ZT_CW - 1), rg = tid / ZT_CW;
    constexpr int RG = ZT_NT / ZT_CW;
    const i64 c0 = (i64)blockIdx.x * ZT_CW;
    const bool live = c0 + cl < N;
    for (int r = rg; r < t; r += RG)
        zt[r * ZT_CW + cl] = live ? make_double2(Br[(i64)r * ld + c0 + cl], Bi[(i64)r * ld + c0 + cl])
                                  : make_double2(0.0, 0.0);
    __syncthreads();
    for (int i = 0; i < t - 1; ++i) {
        const double2 xv = zt[i * ZT_CW + cl];
        const zd xi = {xv.x, xv.y};
        for (int r = i + 1 + rg; r < t; r += RG) {
            const zd l = {__ldg(Lr + (i64)r * ld + i), __ldg(Li + (i64)r * ld + i)};
            const double2 bv = zt[r * ZT_CW + cl];
            const zd v = zmsub({bv.x, bv.y}, l, xi);
            zt[r * ZT_CW + cl] = make_double2(v.r, v.i);
        }
        __syncthreads();
    }
    if (live)
        for (int r = rg + (rg == 0 ? RG : 0); r < t; r += RG) {  // row 0 is unchanged
            const double2 v = zt[r * ZT_CW + cl];
            Br[(i64)r * ld + c0 + cl] = v.x;
            Bi[(i64)r * ld + c0 + cl] = v.y;
        }
}

// dst = -src (rows x cols, row-major, lds / ldd)
__global__ void k_negate(const double *__restrict__ src, i64 lds, double *__restrict__ dst, i64 ldd, i64 rows,
                         i64 cols) {
    const i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= rows * cols) return;
    const i64 r = idx / cols, c = idx - r * cols;
    dst[r * ldd + c] = -src[r * lds + c];
}

// interleaved column-major (m x n, lda) <-> two row-major planes (ld)
__global__ void k_z_split(const double2 *__restrict__ A, i64 lda, double *__restrict__ Wr, double *__restrict__ Wi,
                          i64 ld, i64 m, i64 n) {
    __shared__ double2 tile[32][33];
    const i64 i0 = (i64)blockIdx.x * 32, j0 = (i64)blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {
        const i64 i = i0 + tx, j = j0 + r;
        if (i < m && j < n) tile[r][tx] = A[i + j * lda];
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const i64 i = i0 + r, j = j0 + tx;
        if (i < m && j < n) {
            const double2 v = tile[tx][r];
            Wr[i * ld + j] = v.x;
            Wi[i * ld + j] = v.y;
        }
    }
}
__global__ void k_z_merge(const double *__restrict__ Wr, const double *__restrict__ Wi, i64 ld, double2 *__restrict__ A,
                          i64 lda, i64 m, i64 n) {
    __shared__ double2 tile[32][33];
    const i64 i0 = (i64)blockIdx.x * 32, j0 = (i64)blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {
        const i64 i = i0 + r, j = j0 + tx;
        if (i < m && j < n) tile[r][tx] = make_double2(Wr[i * ld + j], Wi[i * ld + j]);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const i64 i = i0 + tx, j = j0 + r;
        if (i < m && j < n) A[i + j * lda] = tile[tx][r];
    }
}

struct ZRun {
    oxi_handle_s *h;
    double *Wr, *Wi;
    i64 ld, m, n;
    int64_t *ipiv, *info;
    double *neg;  // -Ai scratch (m x (nb + 2))
    i64 nb;       // panel width (lu_factor's blocksize, 128 by default)
};

// C -= A B on complex planes (row-major, common ld): four FP64 tensor-core
// products, the imaginary part of A negated once into scratch.
static void zgemm_minus(ZRun &R, i64 cr, i64 cc, i64 ar, i64 ac, i64 br, i64 bc, i64 M, i64 N, i64 K) {
    if (M <= 0 || N <= 0 || K <= 0) return;
    cudaStream_t s = R.h->stream;
    const i64 ld = R.ld;
    double *Cr = R.Wr + cr * ld + cc, *Ci = R.Wi + cr * ld + cc;
    const double *Ar = R.Wr + ar * ld + ac, *Ai = R.Wi + ar * ld + ac;
    const double *Bre = R.Wr + br * ld + bc, *Bim = R.Wi + br * ld + bc;
    const i64 ldn = zrup(K, 2);
    k_negate<<<(unsigned)((M * K + 255) / 256), 256, 0, s>>>(Ai, ld, R.neg, ldn, M, K);
    OXI_LAUNCH_CHECK();
    launch_gemm_dmma(Cr, ld, Ar, ld, Bre, ld, M, N, K, s);
    launch_gemm_dmma(Cr, ld, R.neg, ldn, Bim, ld, M, N, K, s);
    launch_gemm_dmma(Ci, ld, Ar, ld, Bim, ld, M, N, K, s);
    launch_gemm_dmma(Ci, ld, Ai, ld, Bre, ld, M, N, K, s);
}

static void ztrsm(ZRun &R, i64 r0, i64 c0, int t, i64 bc, i64 N) {
    if (t <= 1 || N <= 0) return;
    const i64 ld = R.ld;
    if (t > ZT_MAXT) {  // a wider block (blocksize > 128): the top rows, their update of the rest, the rest
        const int h = ZT_MAXT;
        ztrsm(R, r0, c0, h, bc, N);
        zgemm_minus(R, r0 + h, bc, r0 + h, c0, r0, bc, t - h, N, h);
        ztrsm(R, r0 + h, c0 + h, t - h, bc, N);
        return;
    }
    const int smem = (int)(sizeof(double2) * t * ZT_CW);
    set_max_dyn_smem((const void *)k_ztrsm_lunit, (int)(sizeof(double2) * ZT_MAXT * ZT_CW));
    k_ztrsm_lunit<<<(unsigned)((N + ZT_CW - 1) / ZT_CW), ZT_NT, smem, R.h->stream>>>(
        R.Wr + r0 * ld + c0, R.Wi + r0 * ld + c0, R.Wr + r0 * ld + bc, R.Wi + r0 * ld + bc, ld, t, N);
    OXI_LAUNCH_CHECK();
}

static void zlaswp(ZRun &R, i64 k0, int cnt, i64 c_lo, i64 c_hi, i64 skip_lo, i64 skip_hi) {
    if (c_hi <= c_lo || cnt <= 0) return;
    if (cnt > ZLEAF) throw CudaError{cudaErrorInvalidValue, "more interchanges than a complex leaf makes"};
    const i64 cols = c_hi - c_lo;
    k_zlaswp<<<(unsigned)((cols + 127) / 128), 128, 0, R.h->stream>>>(R.Wr, R.Wi, R.ld, R.ipiv, k0, cnt, c_lo, c_hi,
                                                                        skip_lo, skip_hi);
    OXI_LAUNCH_CHECK();
}

// _lu_panel! on columns [c0, c0+nc), rows [c0, m): the leaf's interchanges go
// to every other column of the matrix right after it (the reference applies
// them to the panel's columns in the recursion and to the rest per panel; each
// column receives the same sequence)
static void zpanel(ZRun &R, i64 c0, i64 nc) {
    const i64 mrows = R.m - c0;
    if (mrows <= 0 || nc <= 0) return;
    if (nc <= ZLEAF) {
        if (mrows <= (i64)ZCL_MAXRP * 16) {
            // rows over a cluster of up to 16 CTAs, in shared memory
            int cs = (int)std::min<i64>(16, std::max<i64>(1, (mrows + 511) / 512));
            int rp = (int)((mrows + cs - 1) / cs);
            while (rp > ZCL_MAXRP) rp = (int)((mrows + (++cs) - 1) / cs);
            const size_t smem = sizeof(double2) * (size_t)rp * ZLEAF;
            set_max_dyn_smem((const void *)k_zleaf_cl, (int)(sizeof(double2) * ZCL_MAXRP * ZLEAF));
            if (cs > 8) OXI_CUDA(cudaFuncSetAttribute(k_zleaf_cl, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(cs);
            cfg.blockDim = dim3(ZCL_NT);
            cfg.dynamicSmemBytes = smem;
            cfg.stream = R.h->stream;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = cs;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            OXI_CUDA(cudaLaunchKernelEx(&cfg, k_zleaf_cl, R.Wr + c0 * R.ld + c0, R.Wi + c0 * R.ld + c0, R.ld,
                                        (int)mrows, (int)nc, rp, c0, R.ipiv, R.info));
        } else {
            k_zleaf<<<1, ZLEAF_NT, 0, R.h->stream>>>(R.Wr + c0 * R.ld + c0, R.Wi + c0 * R.ld + c0, R.ld, (int)mrows,
                                                     (int)nc, c0, R.ipiv, R.info);
        }
        OXI_LAUNCH_CHECK();
        const int cnt = (int)std::min<i64>(nc, mrows);
        zlaswp(R, c0, cnt, 0, R.n, c0, c0 + nc);
        return;
    }
    const i64 h = nc / 2;
    zpanel(R, c0, h);
    ztrsm(R, c0, c0, (int)h, c0 + h, nc - h);
    if (mrows > h) {
        zgemm_minus(R, c0 + h, c0 + h, c0 + h, c0, c0, c0 + h, mrows - h, nc - h, h);
        zpanel(R, c0 + h, nc - h);
    }
}

static void zgetrf_planes(ZRun &R) {
    const i64 q = std::min(R.m, R.n);
    for (i64 f = 0; f < q; f += R.nb) {
        const i64 l = std::min(q, f + R.nb);
        zpanel(R, f, l - f);
        if (l >= R.n) continue;
        ztrsm(R, f, f, (int)(l - f), l, R.n - l);
        if (l >= R.m) continue;
        zgemm_minus(R, l, l, l, f, f, l, R.m - l, R.n - l, l - f);
    }
}

// ---- solves: one CTA per right-hand side, the substitutions row by row with
// a CTA-wide dot product per row (factor rows are contiguous in column-major
// only along columns, so each dot product reads one row of the triangle) ----
__device__ __forceinline__ zd cta_sum(zd v, zd *s_buf) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int off = 16; off > 0; off >>= 1) {
        v.r += __shfl_xor_sync(0xffffffffu, v.r, off);
        v.i += __shfl_xor_sync(0xffffffffu, v.i, off);
    }
    if (lane == 0) s_buf[warp] = v;
    __syncthreads();
    zd t = {0.0, 0.0};
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { t.r += s_buf[w].r; t.i += s_buf[w].i; }
    __syncthreads();
    return t;  // valid in thread 0
}

// x <- op(T)^-1 x for the n x n factor LU (interleaved column-major):
// lower (unit L) or upper (U), op = none / transpose / conjugate transpose.
__global__ void __launch_bounds__(256) k_ztrsv(const double2 *__restrict__ LU, i64 lda, double2 *__restrict__ X,
                                               i64 ldx, int n, int lower_solve, int unit, int transposed,
                                               int conjugate) {
    __shared__ zd s_buf[8];
    double2 *x = X + (i64)blockIdx.x * ldx;
    for (int step = 0; step < n; ++step) {
        const int i = lower_solve ? step : n - 1 - step;
        zd acc = {0.0, 0.0};
        const int p0 = lower_solve ? 0 : i + 1, p1 = lower_solve ? i : n;
        for (int p = p0 + threadIdx.x; p < p1; p += 256) {
            const double2 a2 = transposed ? LU[p + (i64)i * lda] : LU[i + (i64)p * lda];
            const zd a = {a2.x, conjugate ? -a2.y : a2.y};
            const double2 xp = x[p];
            const zd pr = zmul(a, {xp.x, xp.y});
            acc.r += pr.r;
            acc.i += pr.i;
        }
        acc = cta_sum(acc, s_buf);
        if (threadIdx.x == 0) {
            const double2 b = x[i];
            zd v = {b.x - acc.r, b.y - acc.i};
            if (!unit) {
                const double2 d2 = LU[i + (i64)i * lda];
                v = zdivd(v, {d2.x, conjugate ? -d2.y : d2.y});
            }
            x[i] = make_double2(v.r, v.i);
        }
        __syncthreads();
    }
}

// x <- T^-1 x for the untransposed factors, column by column with x in shared
// memory: the forward unit-lower solve (x_i -= l_ij x_j for i > j once x_j is
// final) or the backward upper one (x_j /= u_jj, then x_i -= u_ij x_j for
// i < j).  Each step reads one column of the factor, contiguous in memory.
// One CTA per right-hand side; n <= ZCOLS_MAXN.
constexpr int ZCOLS_NT = 512;
constexpr int ZCOLS_MAXN = 12288;
__global__ void __launch_bounds__(ZCOLS_NT) k_ztrsv_cols(const double2 *__restrict__ LU, i64 lda,
                                                         double2 *__restrict__ X, i64 ldx, int n, int lower) {
    // a step's column entries for this thread are loaded together into
    // registers before any is used: one global latency per step, not one per row
    constexpr int PER = ZCOLS_MAXN / ZCOLS_NT;
    extern __shared__ double2 zx[];
    double2 *x = X + (i64)blockIdx.x * ldx;
    const int tid = threadIdx.x;
    for (int i = tid; i < n; i += ZCOLS_NT) zx[i] = x[i];
    __syncthreads();
    double2 cv[PER];
    if (lower) {
        for (int j = 0; j < n - 1; ++j) {
            const double2 *col = LU + (i64)j * lda;
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const int i = j + 1 + tid + q * ZCOLS_NT;
                if (i < n) cv[q] = col[i];
            }
            const double2 xv = zx[j];
            const zd xj = {xv.x, xv.y};
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const int i = j + 1 + tid + q * ZCOLS_NT;
                if (i < n) {
                    const double2 b = zx[i];
                    const zd v = zmsub({b.x, b.y}, {cv[q].x, cv[q].y}, xj);
                    zx[i] = make_double2(v.r, v.i);
                }
            }
            __syncthreads();
        }
        for (int i = tid; i < n; i += ZCOLS_NT) x[i] = zx[i];
    } else {
        // zx[j] is not written in step j (every thread divides it for itself),
        // and not read after it: the solution goes straight to x[j]
        for (int j = n - 1; j >= 0; --j) {
            const double2 *col = LU + (i64)j * lda;
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const int i = tid + q * ZCOLS_NT;
                if (i < j) cv[q] = col[i];
            }
            const double2 xv = zx[j], d = col[j];
            const zd xj = zdivd({xv.x, xv.y}, {d.x, d.y});
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const int i = tid + q * ZCOLS_NT;
                if (i < j) {
                    const double2 b = zx[i];
                    const zd v = zmsub({b.x, b.y}, {cv[q].x, cv[q].y}, xj);
                    zx[i] = make_double2(v.r, v.i);
                }
            }
            if (tid == 0) x[j] = make_double2(xj.r, xj.i);
            __syncthreads();
        }
    }
}

// the interchanges on the columns of X: forward (before the 'N' solves) or in
// reverse (after the 'T' / 'C' solves), one thread per right-hand side
__global__ void k_zperm(double2 *__restrict__ X, i64 ldx, int n, int nrhs, const int64_t *__restrict__ ipiv,
                        int reverse) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nrhs) return;
    double2 *x = X + (i64)c * ldx;
    for (int s = 0; s < n; ++s) {
        const int j = reverse ? n - 1 - s : s;
        const int p = (int)ipiv[j] - 1;
        if (p != j) {
            const double2 t = x[j];
            x[j] = x[p];
            x[p] = t;
        }
    }
}

}  // namespace oxi

extern "C" int oxi_zgetrf(oxi_handle_t h, int64_t m, int64_t n, void *dA, int64_t lda, int64_t *d_ipiv,
                          int64_t *h_info) {
    using namespace oxi;
    if (!h || !h_info || m < 0 || n < 0 || lda < std::max<int64_t>(1, m)) return OXI_EINVAL;
    *h_info = 0;
    if (m == 0 || n == 0) return OXI_OK;
    if (!dA || !d_ipiv || m >= (1ll << 31) || n >= (1ll << 31)) return OXI_EINVAL;
    if ((uintptr_t)dA % 16) return OXI_EINVAL;  // ComplexF64 elements are 16-byte aligned
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        AbortScope ab(h);
        const i64 ld = zrup(n, 32), nb = std::max<i64>(1, h->opt.blocksize);
        double *W = (double *)h->work.get(sizeof(double) * (2 * (size_t)m * ld + (size_t)m * (nb + 2) + 64));
        ZRun R{h, W, W + (size_t)m * ld, ld, m, n, d_ipiv, nullptr, W + 2 * (size_t)m * ld, nb};
        char *sc = (char *)h->scratch.get(kScratchBytes);
        R.info = (int64_t *)sc;
        cudaStream_t s = h->stream;
        OXI_CUDA(cudaMemsetAsync(R.info, 0, sizeof(int64_t), s));
        dim3 g((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32));
        k_z_split<<<g, dim3(32, 8), 0, s>>>((const double2 *)dA, lda, R.Wr, R.Wi, ld, m, n);
        OXI_LAUNCH_CHECK();
        zgetrf_planes(R);
        k_z_merge<<<g, dim3(32, 8), 0, s>>>(R.Wr, R.Wi, ld, (double2 *)dA, lda, m, n);
        OXI_LAUNCH_CHECK();
        int64_t *hi = (int64_t *)h->host_ws.get(64);
        OXI_CUDA(cudaMemcpyAsync(hi, R.info, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        queue_abort_read(h, (int *)(hi + 2));
        OXI_CUDA(cudaStreamSynchronize(s));
        *h_info = hi[0];
        const int we = check_abort(h, (const int *)(hi + 2));
        if (we != OXI_OK) return we;
        return hi[0] > 0 ? OXI_ESINGULAR : OXI_OK;
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

extern "C" int oxi_zgetrs(oxi_handle_t h, char trans, int64_t n, int64_t nrhs, const void *dLU, int64_t lda,
                          const int64_t *d_ipiv, void *dB, int64_t ldb) {
    using namespace oxi;
    if (!h) return OXI_EINVAL;
    if (trans != 'N' && trans != 'T' && trans != 'C') return OXI_EINVAL;
    if (n < 0 || nrhs < 0 || lda < std::max<int64_t>(1, n) || ldb < std::max<int64_t>(1, n)) return OXI_EINVAL;
    if (n == 0 || nrhs == 0) return OXI_OK;
    if (!dLU || !d_ipiv || !dB || n >= (1ll << 31) || nrhs >= (1ll << 31)) return OXI_EINVAL;
    if ((uintptr_t)dLU % 16 || (uintptr_t)dB % 16) return OXI_EINVAL;
    try {
        ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        AbortScope ab(h);
        // the pivots are validated on the host (one copy of n entries)
        std::vector<int64_t> ip(n);
        OXI_CUDA(cudaMemcpyAsync(ip.data(), d_ipiv, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, h->stream));
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        for (i64 j = 0; j < n; ++j)
            if (ip[j] < 1 || ip[j] > n) return OXI_EINVAL;
        cudaStream_t s = h->stream;
        const double2 *LU = (const double2 *)dLU;
        double2 *X = (double2 *)dB;
        const unsigned gp = (unsigned)((nrhs + 127) / 128);
        if (trans == 'N') {
            k_zperm<<<gp, 128, 0, s>>>(X, ldb, (int)n, (int)nrhs, d_ipiv, 0);
            OXI_LAUNCH_CHECK();
            if (n <= ZCOLS_MAXN) {
                const int smem = (int)(sizeof(double2) * n);
                set_max_dyn_smem((const void *)k_ztrsv_cols, (int)(sizeof(double2) * ZCOLS_MAXN));
                k_ztrsv_cols<<<(unsigned)nrhs, ZCOLS_NT, smem, s>>>(LU, lda, X, ldb, (int)n, 1);
                OXI_LAUNCH_CHECK();
                k_ztrsv_cols<<<(unsigned)nrhs, ZCOLS_NT, smem, s>>>(LU, lda, X, ldb, (int)n, 0);
                OXI_LAUNCH_CHECK();
            } else {
                k_ztrsv<<<(unsigned)nrhs, 256, 0, s>>>(LU, lda, X, ldb, (int)n, 1, 1, 0, 0);
                OXI_LAUNCH_CHECK();
                k_ztrsv<<<(unsigned)nrhs, 256, 0, s>>>(LU, lda, X, ldb, (int)n, 0, 0, 0, 0);
                OXI_LAUNCH_CHECK();
            }
        } else {
            const int cj = trans == 'C';
            // U^T (U^H) is lower, non-unit; L^T (L^H) upper, unit
            k_ztrsv<<<(unsigned)nrhs, 256, 0, s>>>(LU, lda, X, ldb, (int)n, 1, 0, 1, cj);
            OXI_LAUNCH_CHECK();
            k_ztrsv<<<(unsigned)nrhs, 256, 0, s>>>(LU, lda, X, ldb, (int)n, 0, 1, 1, cj);
            OXI_LAUNCH_CHECK();
            k_zperm<<<gp, 128, 0, s>>>(X, ldb, (int)n, (int)nrhs, d_ipiv, 1);
            OXI_LAUNCH_CHECK();
        }
        int *he = (int *)h->host_ws.get(64);
        queue_abort_read(h, he);
        OXI_CUDA(cudaStreamSynchronize(s));
        return check_abort(h, he);
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}
