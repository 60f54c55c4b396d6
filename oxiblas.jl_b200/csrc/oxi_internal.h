// Internal declarations shared by the translation units of liboxiblas_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include "../../include/oxiblas_b200.h"
#include "profile.h"

namespace oxi {

using i64 = int64_t;

// Error plumbing: every CUDA call on the host side goes through OXI_CUDA, which
// records the message on the handle and returns OXI_ECUDA from the entry point.
struct CudaError {
    cudaError_t code;
    const char *what;
};

#define OXI_CUDA(expr)                                                                 \
    do {                                                                               \
        cudaError_t oxi_e_ = (expr);                                                   \
        if (oxi_e_ != cudaSuccess) throw ::oxi::CudaError{oxi_e_, #expr};             \
    } while (0)

#define OXI_LAUNCH_CHECK()              \
    do {                                \
        ::oxi::count_launch();          \
        OXI_CUDA(cudaGetLastError());   \
    } while (0)

// Fixed layout of the handle's small control block (allocated once at this size,
// so pointers into it stay valid for the whole call).
constexpr size_t kScratchBytes = 65536;
constexpr size_t kScratchErrOff = 1024;     // the abort block (16 bytes), then other int error words
constexpr size_t kScratchStallOff = 1984;   // flag of the missing-producer test hook (never set)
constexpr size_t kScratchScalOff = 2048;    // double scalars of the mixed path
constexpr size_t kScratchTrsvOff = 8192;    // triangular-solve tickets and flags
constexpr int kTrsvCtlInts = (int)((kScratchBytes - kScratchTrsvOff) / sizeof(int));

// Device workspace owned by a handle; grows monotonically.
struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    void *get(size_t need) {
        if (need <= bytes) return ptr;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        need = (need + 255) & ~size_t(255);
        OXI_CUDA(cudaMalloc(&ptr, need));
        bytes = need;
        return ptr;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

struct PinnedBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    void *get(size_t need) {
        if (need <= bytes) return ptr;
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
        OXI_CUDA(cudaMallocHost(&ptr, need));
        bytes = need;
        return ptr;
    }
    void release() {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

struct Options {
    i64 blocksize = 128;   // lu_factor default (factorizations.jl:17)
    int gemm = 0;          // 0 tensor-core engine, 1 reference summation order
    i64 trsm_leaf = 32;    // recursive TRSM leaf
    int lookahead = 1;          // overlap panel k+1 with the trailing update of panel k
    i64 mixed_blocksize = 256;  // panel width of the mixed-precision factorization
    int stop_normwise = 0;      // IR stop test: 0 componentwise (reference), 1 normwise
    int graphs = 1;             // replay repeated factorizations as CUDA graphs
    int tournament = 0;         // mixed solve: tournament pivoting in the FP32 leaves (off: slower, see tslu.cu)
    int gmres_restart = 30;
    double gmres_tol = 1e-4;    // inner relative tolerance of GMRES-IR
};

// Precision of the trailing update inside an FP32 factorization.
enum TrailingKind { TRAIL_NATIVE = 0, TRAIL_BF16 = 1, TRAIL_FP16 = 2, TRAIL_BF16X3 = 4, TRAIL_FP16X3 = 5 };

}  // namespace oxi

struct oxi_handle_s {
    int device = 0;
    cudaStream_t stream = nullptr;
    oxi::Options opt;
    int64_t wait_limit_ns = 0;      // bounded-wait limit of this handle's calls (0: kWaitLimitNs)
    int64_t wait_limit_dev = -1;    // the value last written into the abort block
    int64_t stall_at = 0;           // OXI_OPT_TEST_MISSING_PRODUCER: > 0 arms the hook before that leaf
    std::string last_error;
    int sm_count = 148;
    // workspaces
    oxi::DeviceBuffer work;      // row-major working matrix
    oxi::DeviceBuffer scratch;   // small control data (moves, counters, info)
    oxi::DeviceBuffer solve_ws;  // solve workspace
    oxi::DeviceBuffer mixed_ws;  // mixed-precision workspace
    oxi::DeviceBuffer perm_ws;   // row permutation of the last solve
    oxi::PinnedBuffer host_ws;   // pinned host staging
    oxi::DeviceBuffer tc_ws;     // 16-bit GEMM operands
    oxi::DeviceBuffer tc_ws2;    // the same for a second, concurrent trailing update
    int tc_slot = 0;             // which of the two operand buffers (and scale slots) to use
    // the last A operand converted into tc_ws: the lookahead's second trailing
    // update has the same L21 and reuses it instead of converting it again
    struct TcA16 {
        const float *src = nullptr;
        int64_t lda = 0, M = 0, K = 0;
        int kind = -1;
        const void *a16 = nullptr;
    } tc_last_a;
    int gemm_ctas = 0;           // > 0: cap on the persistent tensor-core GEMM's CTAs;
                                 // -k: at most k GPC-filling clusters, one GPC spared
    cudaStream_t la_stream = nullptr;        // lookahead: the trailing update's stream
    cudaStream_t la_main = nullptr;          // lookahead: the panels' stream (highest priority)
    cudaEvent_t la_in = nullptr, la_out = nullptr;  // caller's stream -> la_main -> caller's stream
    cudaEvent_t la_fork = nullptr, la_join = nullptr;
    oxi::DeviceBuffer xtag_ws;   // tagged solution words of the triangular solves
    oxi::DeviceBuffer trsv_ws;   // per-block solve operators of getrs (inverse + two coupling blocks)
    oxi::DeviceBuffer rowmap_ws; // per-panel row map and composite move list
    oxi::DeviceBuffer tslu_ws;   // tournament-pivoting tree of the FP32 leaves
    int tslu = 0;                // 1 inside the mixed solve's FP32 factor: tournament leaves
    int trailing = 0;            // oxi::TrailingKind for getrf_rowmajor<float>
    oxi::Profiler prof;
    cudaStream_t aux_stream = nullptr;      // capturable stream used when the caller's is legacy
    cudaEvent_t aux_fork = nullptr, aux_join = nullptr;
    // CUDA graph of the last factorization (replayed when the same shape and
    // buffers come back)
    struct GraphCache {
        bool valid = false;
        int seen = 0;
        uint64_t nlaunch = 0;  // kernel launches one replay performs (launch counter)
        uint64_t key[12] = {};
        cudaGraphExec_t exec = nullptr;
        cudaGraph_t graph = nullptr;
        void reset() {
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
            exec = nullptr;
            graph = nullptr;
            valid = false;
            seen = 0;
        }
    } gcache;
    // batched small LU: tuning per mode (0 FP64, 1 FP32 factor + FP64 refinement),
    // queue/status block, per-CTA FP32 working matrices, graph of the last call
    struct BatchTune {
        bool tuned = false;
        int n_smem = 0;
        int nb[8] = {};
    } btune[2];
    oxi::DeviceBuffer batch_ctl, batch_wsp;
    struct BatchGraph {
        std::vector<uint64_t> key;
        int seen = 0;
        uint64_t nlaunch = 0;  // kernel launches one replay performs (launch counter)
        cudaGraphExec_t exec = nullptr;
        cudaGraph_t graph = nullptr;
        void reset() {
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
            exec = nullptr;
            graph = nullptr;
            seen = 0;
            key.clear();
        }
    } bgraph;
};

namespace oxi {

// The abort block of a handle: 16 bytes at kScratchErrOff of its scratch.
// int 0 is the sticky abort code of the running call (0: healthy; set by the
// first bounded wait that gives up, read by every later wait and kernel entry
// of the call), int 1 the mixed path's non-finite flag, ints 2-3 the wait limit
// in ns (0: kWaitLimitNs).  Each handle has its own block, so calls on
// different handles never see each other's timeouts.
//
// AbortScope (entry points): makes the handle's abort word the one the
// launchers of this host thread pass to their kernels (t_abort), clears the
// word on the handle's stream, and writes the wait limit when it changed.
// queue_abort_read enqueues the word's copy into *hdst (pinned) on the
// handle's stream; after the stream is idle, check_abort returns OXI_ETIMEOUT
// if it was set, else OXI_OK.
extern thread_local int *t_abort;
inline int *cur_abort() { return t_abort; }
int *abort_word(oxi_handle_s *h);
struct AbortScope {
    int *saved;
    int *word;
    explicit AbortScope(oxi_handle_s *h);
    ~AbortScope() { t_abort = saved; }
};
void queue_abort_read(oxi_handle_s *h, int *hdst);
int check_abort(oxi_handle_s *h, const int *hsrc);

// Test hook of the bounded waits (OXI_OPT_TEST_MISSING_PRODUCER): a one-thread
// kernel waits for a handle-owned flag that no kernel sets -- the wait of a
// consumer whose producer was never launched -- and so makes the call's
// abort word trip after the wait limit.
void launch_await_missing_producer(oxi_handle_s *h, cudaStream_t s);
// Called before every leaf launch of a factorization: launches the test hook
// before the armed leaf (h->stall_at counts leaves down to it).
void maybe_stall_before_leaf(oxi_handle_s *h, cudaStream_t s);

// Raise a kernel's dynamic shared-memory limit to `bytes`, once per device
// (the attribute belongs to the device's context).  A kernel keeps ONE limit,
// its largest use, so launches captured in a CUDA graph never see it lowered.
void set_max_dyn_smem(const void *func, int bytes);

// ---- kernels launched by the drivers (defined in lu_kernels.cu / gemm_*.cu) ----

// Column-major (m x n, lda) -> row-major (m x n, ldw) and back.
template <typename TS, typename TD>
void launch_cm_to_rm(const TS *A, i64 lda, TD *W, i64 ldw, i64 m, i64 n, cudaStream_t s);
template <typename TS, typename TD>
void launch_rm_to_cm(const TS *W, i64 ldw, TD *A, i64 lda, i64 m, i64 n, cudaStream_t s);

// Leaf LU of the row-major block P (m rows x w columns, ld), one thread-block
// cluster.  Writes ipiv[gofs + j], *info (first zero pivot, global 1-based), and
// the (dst, src) row-move list of the net permutation (positions relative to P).
// In-leaf application of the leaf's row interchanges to the rest of its panel
// (columns [pc_lo, pc_lo + left_n) and [right_lo, right_lo + nother - left_n),
// absolute) and to the panel row map (map[map_off + position]); nother = 0 and
// map = null switch it off.
// Other panel columns (panel width minus the leaf's) that the in-leaf row moves
// reach; wider panels apply each leaf's interchanges with separate row moves.
constexpr int LEAF_MAX_OTHER = 256;

// gemm_ctas = -k asks the persistent tensor-core GEMM for at most k clusters of
// GEMM_GPC_CLUSTER CTAs (one GPC each), always leaving at least one GPC free
constexpr int GEMM_GPC_CLUSTER = 16;

struct LeafPanel {
    int nother = 0, left_n = 0, pc_lo = 0, right_lo = 0, leaf_c0 = 0, map_off = 0;
    int *map = nullptr;
    // a pending block copy the leaf performs first: u_rows x u_cols elements,
    // row-major at u_src (leading dimension u_cols) to u_dst (the leaf's ld)
    const void *u_src = nullptr;
    void *u_dst = nullptr;
    int u_rows = 0, u_cols = 0;
    // set the move counter back to zero at the end (saves the next leaf's memset)
    int reset_nmoves = 0;
    // the call's abort word (set by launch_leaf)
    int *abort = nullptr;
};

// Tournament-pivoting leaf (FP32, mixed solve only): same contract as
// launch_leaf (pivots, info, moves, in-panel moves through pn).
bool tslu_applicable(i64 m);
// FP32 right-looking panel step after a kw-wide leaf at P (the leaf's diagonal
// corner): U12 <- L11^-1 A12 and A22 -= L21 U12 for the panel's N columns right
// of the leaf and the M rows below it.  U12 goes to ubuf (kw x N, row-major):
// the launch's CTAs all read A12, so it is copied into place afterwards.
void launch_panel_rl(float *P, i64 ld, int kw, i64 M, i64 N, float *ubuf, cudaStream_t s);
void launch_tslu_leaf(oxi_handle_s *h, float *P, i64 ld, i64 m, int w, i64 gofs, int64_t *ipiv, int64_t *info,
                      int *moves, int *nmoves, cudaStream_t s, LeafPanel pn);

template <typename T>
void launch_leaf(T *P, i64 ld, i64 m, int w, i64 gofs, int64_t *ipiv, int64_t *info,
                 int *moves, int *nmoves, int leafw, cudaStream_t s, LeafPanel pn = LeafPanel());
// Widest leaf width whose register capacity holds m rows.
template <typename T> int leaf_width_for(i64 m);

// Apply a row-move list (positions relative to row r0) to columns [c_lo, c_hi)
// of the row-major matrix W, skipping columns [skip_lo, skip_hi).
template <typename T>
void launch_rowmoves(T *W, i64 ld, i64 r0, const int *moves, const int *nmoves, i64 c_lo,
                     i64 c_hi, i64 skip_lo, i64 skip_hi, cudaStream_t s);

// Per-panel composition of the leaves' row permutations (see lu_kernels.cu).
void launch_rowmap_init(int *map, i64 len, int *zero0, int *zero1, cudaStream_t s);
void launch_rowmap_apply(int *map, i64 offset, const int *moves, const int *nmoves, cudaStream_t s);
void launch_rowmap_extract(const int *map, i64 len, int *list, int *cnt, cudaStream_t s);
template <typename T>
void launch_rowmoves_big(T *W, i64 ld, i64 r0, const int *list, const int *cnt, int maxcnt, i64 c_lo,
                         i64 c_hi, cudaStream_t s);

// B (t x N, row-major) <- L^-1 B, L unit lower t x t (t <= 32), row-major.
template <typename T>
void launch_trsm_leaf(const T *L, i64 ldl, T *B, i64 ldb, int t, i64 N, cudaStream_t s,
                      bool ref_order);
// Fused blocked TRSM, unit lower L with t <= 256 (one launch).
template <typename T>
void launch_trsm_fused(const T *L, i64 ldl, T *B, i64 ldb, int t, i64 N, cudaStream_t s);
// Reference-order TRSM for FP64 (t <= 128): the recursive solve's operations,
// element by element, in one launch (see lu_kernels.cu).
bool trsm_refo_applicable(int t);
void launch_trsm_refo(const double *L, i64 ldl, double *B, i64 ldb, int t, i64 N, cudaStream_t s);
// C (M x N) <- C - A (M x K) B (K x N), row-major, as K sequential fma steps per
// element starting from C (the order of a panel leaf's rank-1 updates).
void launch_rankk_seq(double *C, i64 ldc, const double *A, i64 lda, const double *B, i64 ldb, i64 M, i64 N,
                      i64 K, cudaStream_t s);
// FP32 register-blocked CUDA-core GEMM (any summation order).
template <typename T>
void launch_gemm_simt(T *C, i64 ldc, const T *A, i64 lda, const T *B, i64 ldb, i64 M, i64 N, i64 K,
                      cudaStream_t s);

// C (M x N) <- C - A (M x K) * B (K x N), all row-major.  Reference order:
// one FMA chain per output along k, then C - s.
template <typename T>
void launch_gemm_ref(T *C, i64 ldc, const T *A, i64 lda, const T *B, i64 ldb, i64 M, i64 N,
                     i64 K, cudaStream_t s);
// FP64 tensor-core (DMMA, TMA-fed) version.  upper_only: only the tiles that
// reach the upper triangle of C (M == N, a symmetric update) are computed.
void launch_gemm_dmma(double *C, i64 ldc, const double *A, i64 lda, const double *B, i64 ldb,
                      i64 M, i64 N, i64 K, cudaStream_t s, bool upper_only = false);

// tcgen05 GEMM: C (FP32 row-major) -= scale * A16 * B16^T, 16-bit K-major operands.
void launch_gemm_tc(int fmt, float *C, i64 ldc, const void *A16, i64 lda16, const void *B16,
                    i64 ldb16, i64 M, i64 N, i64 K, float scale, const float *d_scale,
                    cudaStream_t s, int max_ctas = 0);
void launch_cvt_rows16(int fmt, const float *src, i64 lds, void *dst, i64 ldd, i64 rows, i64 cols,
                       float scale, const float *d_scale, cudaStream_t s);
void launch_cvt_transpose16(int fmt, const float *src, i64 lds, void *dst, i64 ldd, i64 rows,
                            i64 cols, float scale, const float *d_scale, cudaStream_t s);
// C -= A*B for the trailing update of an FP32 factorization in h->trailing precision.
void gemm_trailing_f32(oxi_handle_s *h, float *C, i64 ldc, const float *A, i64 lda,
                       const float *B, i64 ldb, i64 M, i64 N, i64 K);

// Cholesky of the lower triangle of a column-major matrix, in place as the upper
// triangle of its row-major view (potrf.cu); work holds potrf_work_elems(n)
// elements.  FP32 runs its symmetric update in h->trailing precision.
size_t potrf_work_elems(i64 n);
// The lookahead's two streams (panels at the highest priority, the trailing
// update at the lowest) and its events, created once per handle.
void ensure_lookahead_streams(oxi_handle_s *h);
template <typename T>
void potrf_rowmajor(oxi_handle_s *h, T *U, i64 ld, i64 n, int64_t *d_info, T *work);
// Solves with a column-major lower Cholesky factor L: the block operators of L
// and of L^T (lu_block_inverse_elems(n) elements each), then L L^T X = B in
// place with them (solve.cu).
template <typename T>
void chol_block_ops(oxi_handle_s *h, const T *L, i64 ldl, i64 n, T *P1, T *P2);
template <typename T>
void chol_solve_ops(oxi_handle_s *h, const T *L, i64 ldl, i64 n, T *X, i64 ldx, i64 nrhs, int *d_err,
                    const T *P1, const T *P2);

// getrf_rowmajor through the handle's graph cache (same shape, buffers and
// options: replay; second occurrence: capture; otherwise direct launches).
template <typename T>
void getrf_rowmajor_cached(oxi_handle_s *h, T *W, i64 ld, i64 m, i64 n, int64_t *d_ipiv,
                           int64_t *d_info, int *d_moves, int *d_nmoves);

// Host driver: blocked right-looking getrf on a row-major working matrix.
template <typename T>
void getrf_rowmajor(oxi_handle_s *h, T *W, i64 ld, i64 m, i64 n, int64_t *d_ipiv,
                    int64_t *d_info, int *d_moves, int *d_nmoves);

// Driver helpers reused by the mixed-precision and batched paths.
template <typename T>
void gemm_minus(oxi_handle_s *h, T *C, i64 ldc, const T *A, i64 lda, const T *B, i64 ldb,
                i64 M, i64 N, i64 K);
template <typename T>
void trsm_lower_unit(oxi_handle_s *h, const T *L, i64 ldl, T *B, i64 ldb, i64 t, i64 N);

// Solve with a device-resident 0-based row permutation (A[perm, :] = L U) and
// column-major factors; B (n x nrhs, ldb) is overwritten.  *d_err becomes
// nonzero when a bounded device wait expired.
template <typename T>
void getrs_perm(oxi_handle_s *h, char trans, i64 n, i64 nrhs, const T *LU, i64 lda,
                const int64_t *d_perm, T *B, i64 ldb, int *d_err);
void perm_from_ipiv(const int64_t *ipiv, i64 q, i64 m, int64_t *perm);
// L then U solves with ROW-major factors (W, ld), X column-major n x nrhs, in place.
template <typename T>
void lu_solve_rowmajor(oxi_handle_s *h, const T *W, i64 ld, i64 n, T *X, i64 ldx, i64 nrhs,
                       int *d_err, const T *DinvL = nullptr, const T *DinvU = nullptr);
// Inverses of the 64 x 64 diagonal blocks of L (unit) and U of row-major factors.
template <typename T>
void lu_block_inverses_rowmajor(oxi_handle_s *h, const T *W, i64 ld, i64 n, T *DinvL, T *DinvU);
i64 lu_block_inverse_elems(i64 n);

}  // namespace oxi
