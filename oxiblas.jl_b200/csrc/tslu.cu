// Tournament-pivoting leaf (TSLU, the panel step of communication-avoiding LU)
// for the FP32 factorization inside the mixed-precision solve.
//
// The mixed solve needs a stable low-precision factor, not the reference's
// pivot sequence (refinement restores FP64 accuracy; the plain FP64 path keeps
// partial pivoting and its pivot parity).  Partial pivoting serialises every
// column of a tall leaf behind a cluster-wide arg-max; tournament pivoting
// picks the leaf's W pivot rows by a reduction tree instead:
//   level 0: each warp takes 64 rows and runs partial-pivoting elimination on
//            them (rows stay in registers), nominating W candidate rows;
//   level l: the last of two sibling warps to finish (an atomic counter per
//            node, no waiting) stacks both nominations (2W rows, their
//            ORIGINAL values re-read) and eliminates again, nominating W;
//   root:    its elimination leaves the winners' rows as L11 \ U11; it writes
//            the LAPACK interchange sequence, the (dst, src) moves of the net
//            permutation and info, and saves the rows the winners displace.
// k_tslu_apply then writes every row in its final position: the winners'
// factored rows on top, every other row as l = a U11^-1 (one warp per row, the
// inverse formed once by the root); one extra CTA moves the panel's other
// columns and the panel row map as the partial-pivoting leaf does.
//
// Measured on B200 this leaf is SLOWER than the cluster leaf (about 245 us
// against 81 us per 16384 x 32 leaf): a node's elimination runs on one warp,
// about 6.8K instructions at about 10 cycles each (no other warp to hide the
// latency, instruction-cache misses of the unrolled code), and the tree puts
// log2(m / 64) + 1 such nodes on the critical path.  It is therefore off by
// default (OXI_OPT_TOURNAMENT = 0) and kept as a tested option.
#include <algorithm>
#include <climits>
#include "oxi_internal.h"

namespace oxi {

namespace {
constexpr int TS_W = 32;           // leaf width
constexpr int TS_CH = 2 * TS_W;    // rows per warp at level 0 (= candidates per node)
constexpr int TS_APPLY_NT = 256;
constexpr int TS_MAXLEV = 16;

__device__ __forceinline__ uint32_t redux_max(uint32_t v) {
    uint32_t r;
    asm volatile("redux.sync.max.u32 %0, %1, 0xffffffff;" : "=r"(r) : "r"(v));
    return r;
}
__device__ __forceinline__ uint32_t redux_min(uint32_t v) {
    uint32_t r;
    asm volatile("redux.sync.min.u32 %0, %1, 0xffffffff;" : "=r"(r) : "r"(v));
    return r;
}
// 0 = no candidate; otherwise 1 + the bits of |v| (|v| >= 0 orders like its
// bits); NaN and 0 both map to 1, the lowest key a candidate can have.
__device__ __forceinline__ uint32_t ts_key(float v) {
    if (!(v == v)) return 1u;
    return __float_as_uint(fabsf(v)) + 1u;
}
}  // namespace

struct TsluTree {
    int nlev;
    int size[TS_MAXLEV];  // nodes per level
    int off[TS_MAXLEV];   // first node id of each level
};

// Elimination with partial pivoting on the cc <= 64 candidate rows s_c[] of
// the leaf (lane holds candidates lane and lane + 32).  Returns the number of
// pivots chosen (<= wact) with their rows in s_out[] in pivot order.  At the
// root, each winner's row as it stands when chosen -- its L11 \ U11 row -- is
// written to top[j][*].
__device__ int ts_eliminate(const float *__restrict__ P, i64 ld, int wact, const int *s_c, int cc, int *s_out,
                            float *s_prow, bool root, float *__restrict__ top) {
    const int lane = threadIdx.x;
    float a[2][TS_W];
    int pos[2];
    bool live[2];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int e = lane + 32 * s;
        pos[s] = (e < cc) ? s_c[e] : -1;
        live[s] = pos[s] >= 0;
        const float *row = live[s] ? P + (i64)pos[s] * ld : nullptr;
#pragma unroll
        for (int c = 0; c < TS_W; ++c) a[s][c] = (live[s] && c < wact) ? row[c] : 0.f;
    }
    int nsel = 0;
    bool done = false;  // uniform across the warp
#pragma unroll
    for (int j = 0; j < TS_W; ++j) {
        if (done || j >= wact) continue;
        const uint32_t k0 = live[0] ? ts_key(a[0][j]) : 0u;
        const uint32_t k1 = live[1] ? ts_key(a[1][j]) : 0u;
        const bool take1 = k1 > k0 || (k1 == k0 && k1 != 0u && pos[1] < pos[0]);
        const uint32_t bk = take1 ? k1 : k0;
        const int bp = take1 ? pos[1] : pos[0];
        const uint32_t kmax = redux_max(bk);
        if (kmax == 0u) {  // no candidate left
            done = true;
            continue;
        }
        const int win = (int)redux_min((bk == kmax && bk != 0u) ? (uint32_t)bp : (uint32_t)INT_MAX);
        const bool own = bk == kmax && bp == win;
        if (own) {  // this lane holds the winner: publish its row and retire it
#pragma unroll
            for (int c = 0; c < TS_W; ++c) {
                const float v = take1 ? a[1][c] : a[0][c];
                s_prow[c] = v;
                if (root) top[j * TS_W + c] = v;
            }
            if (take1) live[1] = false;
            else live[0] = false;
            s_out[j] = win;
        }
        __syncwarp();
        const float d = s_prow[j];
        if (d != 0.f) {
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                if (!live[s]) continue;
                const float l = a[s][j] / d;
                a[s][j] = l;
#pragma unroll
                for (int c = j + 1; c < TS_W; ++c) a[s][c] = fmaf(-l, s_prow[c], a[s][c]);
            }
        }
        nsel = j + 1;
        __syncwarp();
    }
    return nsel;
}

__global__ void __launch_bounds__(32)
k_tslu_tree(const float *__restrict__ P, i64 ld, int m, int wact, TsluTree tr, int *__restrict__ cand,
            int *__restrict__ ccnt, int *__restrict__ arrive, float *__restrict__ top, float *__restrict__ disp,
            float *__restrict__ uinv, i64 gofs, int64_t *__restrict__ ipiv, int64_t *__restrict__ info,
            int *__restrict__ moves, int *__restrict__ nmoves) {
    __shared__ int s_c[TS_CH];
    __shared__ int s_out[TS_W];
    __shared__ __align__(16) float s_prow[TS_W];
    __shared__ int s_pos[TS_CH], s_row[TS_CH];  // root: the rows involved in the interchanges
    const int lane = threadIdx.x;
    int lev = 0, node = blockIdx.x;
    int cc = min(TS_CH, m - node * TS_CH);
    for (int e = lane; e < TS_CH; e += 32) s_c[e] = (e < cc) ? node * TS_CH + e : -1;
    __syncwarp();
    for (;;) {
        const bool root = lev == tr.nlev - 1;
        const int nsel = ts_eliminate(P, ld, wact, s_c, cc, s_out, s_prow, root, top);
        __syncwarp();
        if (root) {
            const int q = nsel;
            __shared__ float sT[TS_W][TS_W + 1];
            for (int e = lane; e < TS_W * TS_W; e += 32) sT[e / TS_W][e % TS_W] = __ldcg(&top[e]);
            __syncwarp();
            // info: the first zero on U11's diagonal
            if (lane == 0) {
                int z = 0;
                for (int j = 0; j < q; ++j)
                    if (sT[j][j] == 0.f) { z = j + 1; break; }
                if (z && *info == 0) *info = gofs + z;
            }
            // U11^-1, column `lane` by back substitution (rows past the pivots: identity)
            {
                const int c = lane;
                float x[TS_W];
#pragma unroll
                for (int i = TS_W - 1; i >= 0; --i) {
                    float v;
                    if (i >= q) v = (i == c) ? 1.f : 0.f;
                    else if (i > c) v = 0.f;
                    else {
                        v = (i == c) ? 1.f : 0.f;
#pragma unroll
                        for (int k = i + 1; k < TS_W; ++k) v = fmaf(-sT[i][k], x[k], v);
                        v = v / sT[i][i];
                    }
                    x[i] = v;
                }
#pragma unroll
                for (int i = 0; i < TS_W; ++i) uinv[i * TS_W + c] = x[i];
            }
            // the rows the winners will displace, original values
            for (int e = lane; e < q * TS_W; e += 32) {
                const int x = e / TS_W, c = e - x * TS_W;
                disp[e] = (c < wact) ? P[(i64)x * ld + c] : 0.f;
            }
            // interchange sequence: entries (position, row) for positions 0..q-1 and
            // for every winner below them; entry e lives in lane e % 32
            int ne = q;
            if (lane == 0) {
                for (int x = 0; x < q; ++x) { s_pos[x] = x; s_row[x] = x; }
                for (int j = 0; j < q; ++j)
                    if (s_out[j] >= q) { s_pos[ne] = s_out[j]; s_row[ne] = s_out[j]; ++ne; }
            }
            ne = __shfl_sync(0xffffffffu, ne, 0);
            __syncwarp();
            for (int j = 0; j < q; ++j) {
                const int w = s_out[j];
                const unsigned m1 = __ballot_sync(0xffffffffu, (lane < ne && s_row[lane] == w) ||
                                                                   (lane + 32 < ne && s_row[lane + 32] == w));
                const int l1 = __ffs(m1) - 1;
                const int e1 = (s_row[l1] == w && l1 < ne) ? l1 : l1 + 32;
                const int cur = s_pos[e1];
                if (lane == 0) {
                    ipiv[gofs + j] = gofs + cur + 1;
                    // entry of position j is entry j (positions 0..q-1 keep their entries)
                    const int rj = s_row[j];
                    s_row[j] = w;
                    s_row[e1] = rj;
                }
                __syncwarp();
            }
            // moves of the net permutation (positions relative to the leaf)
            if (lane == 0) {
                int k = 0;
                for (int e = 0; e < ne; ++e)
                    if (s_pos[e] != s_row[e]) {
                        moves[2 * k] = s_pos[e];
                        moves[2 * k + 1] = s_row[e];
                        ++k;
                    }
                *nmoves = k;
                ccnt[0] = q;  // read by the apply kernel: the number of winners
            }
            return;
        }
        // publish this node's nominations, then the last of two siblings continues
        const int id = tr.off[lev] + node;
        for (int e = lane; e < TS_W; e += 32) cand[(i64)id * TS_W + e] = (e < nsel) ? s_out[e] : -1;
        if (lane == 0) ccnt[id + 1] = nsel;
        const int parent = node >> 1;
        const bool alone = (node ^ 1) >= tr.size[lev];
        if (!alone) {
            __threadfence();
            __syncwarp();  // every lane's stores are fenced before lane 0 announces them
            int old = 0;
            if (lane == 0) old = atomicAdd(&arrive[tr.off[lev + 1] + parent], 1);
            old = __shfl_sync(0xffffffffu, old, 0);
            if (old == 0) return;  // the sibling, still running, carries on
            __threadfence();
        }
        const int left = tr.off[lev] + (node & ~1);
        const int nl = __ldcg(&ccnt[left + 1]);
        const int nr = alone ? 0 : __ldcg(&ccnt[left + 2]);
        for (int e = lane; e < TS_CH; e += 32) {
            int v = -1;
            if (e < nl) v = __ldcg(&cand[(i64)left * TS_W + e]);
            else if (e - nl < nr) v = __ldcg(&cand[(i64)(left + 1) * TS_W + (e - nl)]);
            s_c[e] = v;
        }
        cc = nl + nr;
        __syncwarp();
        node = parent;
        ++lev;
    }
}

// Rows in final positions: the winners' L11 \ U11 rows on top, every other row
// l = a U11^-1 -- one warp per row, lane c computing l_c (a 128-byte row read
// and written whole).  The last CTA moves the panel's other columns and the row map.
__global__ void __launch_bounds__(TS_APPLY_NT)
k_tslu_apply(float *__restrict__ P, i64 ld, int m, int wact, const float *__restrict__ top,
             const float *__restrict__ disp, const float *__restrict__ uinv, const int *__restrict__ ccnt,
             int *__restrict__ arrive, int nodes, const int *__restrict__ moves, const int *__restrict__ nmoves,
             LeafPanel pn) {
    __shared__ float sUi[TS_W][TS_W + 1];
    __shared__ int s_dst[2 * TS_W], s_src[2 * TS_W];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int q = ccnt[0];
    const int cnt = min(*nmoves, 2 * TS_W);
    for (int e = t; e < TS_W * TS_W; e += TS_APPLY_NT) sUi[e / TS_W][e % TS_W] = uinv[e];
    for (int e = t; e < 2 * TS_W; e += TS_APPLY_NT) {
        s_dst[e] = (e < cnt) ? moves[2 * e] : -1;
        s_src[e] = (e < cnt) ? moves[2 * e + 1] : -1;
    }
    // reset the tree's arrival counters for the next leaf
    for (int e = blockIdx.x * TS_APPLY_NT + t; e < nodes; e += gridDim.x * TS_APPLY_NT) arrive[e] = 0;
    __syncthreads();
    if (blockIdx.x == gridDim.x - 1) {
        // the leaf's interchanges on the panel's other columns (all sources of a
        // column read before any destination of it is written) and on the row map
        if (cnt == 0) return;
        if (pn.nother > 0) {
            const int cpc = max(1, (TS_APPLY_NT * 8) / cnt);  // whole columns per pass
            for (int c0 = 0; c0 < pn.nother; c0 += cpc) {
                const int ncol = min(cpc, pn.nother - c0);
                float vals[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int e = t + k * TS_APPLY_NT;
                    if (e < cnt * ncol) {  // consecutive threads: consecutive columns of one row
                        const int oc = c0 + e % ncol, mv = e / ncol;
                        const int col = oc < pn.left_n ? pn.pc_lo + oc : pn.right_lo + (oc - pn.left_n);
                        vals[k] = P[(i64)s_src[mv] * ld + (col - pn.leaf_c0)];
                    }
                }
                __syncthreads();
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int e = t + k * TS_APPLY_NT;
                    if (e < cnt * ncol) {
                        const int oc = c0 + e % ncol, mv = e / ncol;
                        const int col = oc < pn.left_n ? pn.pc_lo + oc : pn.right_lo + (oc - pn.left_n);
                        P[(i64)s_dst[mv] * ld + (col - pn.leaf_c0)] = vals[k];
                    }
                }
                __syncthreads();
            }
        }
        if (pn.map) {
            int v = 0;
            if (t < cnt) v = pn.map[pn.map_off + s_src[t]];
            __syncthreads();
            if (t < cnt) pn.map[pn.map_off + s_dst[t]] = v;
        }
        return;
    }
    const int nwarps = (gridDim.x - 1) * (TS_APPLY_NT / 32);
    for (int x = blockIdx.x * (TS_APPLY_NT / 32) + warp; x < m; x += nwarps) {
        float *dst = P + (i64)x * ld;
        if (x < q) {
            if (lane < wact) dst[lane] = top[x * TS_W + lane];
            continue;
        }
        // a displaced row (moved here from above, saved by the root) or this row in place
        const unsigned hit = __ballot_sync(0xffffffffu, s_dst[lane] == x || s_dst[lane + 32] == x);
        const float *row = dst;
        if (hit) {
            const int h = __ffs(hit) - 1;
            const int e = (s_dst[h] == x) ? h : h + 32;
            row = disp + (i64)s_src[e] * TS_W;
        }
        const float a = (lane < wact) ? row[lane] : 0.f;
        float l = 0.f;
#pragma unroll
        for (int p = 0; p < TS_W; ++p) {
            const float ap = __shfl_sync(0xffffffffu, a, p);
            if (p < q) l = fmaf(ap, sUi[p][lane], l);  // U11^-1 is upper triangular
        }
        if (q < wact && lane >= q) l = a;  // columns past the pivots (a degenerate leaf) stay
        if (lane < wact) dst[lane] = l;
    }
}

// Workspace layout (ints/floats): cand [nodes][W], ccnt [1 + nodes], arrive [nodes],
// top [W][W], disp [W][W], uinv [W][W].
static size_t tslu_ws_bytes(int nodes) {
    return sizeof(int) * ((size_t)nodes * TS_W + (nodes + 1) + nodes) + sizeof(float) * 3 * TS_W * TS_W + 256;
}

bool tslu_applicable(i64 m) { return m > 2 * TS_CH && (m + TS_CH - 1) / TS_CH <= (1 << (TS_MAXLEV - 2)); }

void launch_tslu_leaf(oxi_handle_s *h, float *P, i64 ld, i64 m, int w, i64 gofs, int64_t *ipiv, int64_t *info,
                      int *moves, int *nmoves, cudaStream_t s, LeafPanel pn) {
    if (w > TS_W || !tslu_applicable(m)) throw CudaError{cudaErrorInvalidValue, "tournament leaf shape"};
    TsluTree tr{};
    int sz = (int)((m + TS_CH - 1) / TS_CH), nodes = 0;
    tr.nlev = 0;
    for (;;) {
        tr.size[tr.nlev] = sz;
        tr.off[tr.nlev] = nodes;
        nodes += sz;
        ++tr.nlev;
        if (sz == 1) break;
        sz = (sz + 1) / 2;
    }
    // one workspace sized for the tallest leaf this engine accepts, zeroed once
    const int max_nodes = 2 * (1 << (TS_MAXLEV - 2)) + TS_MAXLEV;
    const bool fresh = h->tslu_ws.bytes < tslu_ws_bytes(max_nodes);
    char *ws = (char *)h->tslu_ws.get(tslu_ws_bytes(max_nodes));
    if (fresh) OXI_CUDA(cudaMemsetAsync(ws, 0, h->tslu_ws.bytes, s));
    int *cand = (int *)ws;
    int *ccnt = cand + (size_t)max_nodes * TS_W;
    int *arrive = ccnt + max_nodes + 1;
    float *top = (float *)(arrive + max_nodes);
    float *disp = top + TS_W * TS_W;
    float *uinv = disp + TS_W * TS_W;
    const int nchunk = tr.size[0];
    ProfScope ps(KC_LEAF, s, 0.0, 2.0 * (double)m * w * sizeof(float));
    k_tslu_tree<<<nchunk, 32, 0, s>>>(P, ld, (int)m, w, tr, cand, ccnt, arrive, top, disp, uinv, gofs, ipiv, info,
                                      moves, nmoves);
    OXI_LAUNCH_CHECK();
    // row blocks: 8 rows (warps) per CTA, about 4 rows per warp; plus the move CTA
    const int blocks = (int)std::min<i64>((m + 31) / 32, 4 * 148) + 1;
    k_tslu_apply<<<blocks, TS_APPLY_NT, 0, s>>>(P, ld, (int)m, w, top, disp, uinv, ccnt, arrive, nodes, moves,
                                                nmoves, pn);
    OXI_LAUNCH_CHECK();
}

}  // namespace oxi
