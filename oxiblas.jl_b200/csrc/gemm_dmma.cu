// FP64 trailing-update GEMM on the tensor cores: C <- C - A*B, row-major.
//
// sm_100a has no FP64 kind for tcgen05.mma; the FP64 tensor path is DMMA
// (mma.sync.aligned.m16n8k4 .f64), which this kernel feeds from TMA.
// CTA tile 128 x 64, k slab 16, 4-stage mbarrier pipeline:
//   warp 8      producer: one lane issues the TMA loads of each stage;
//   warps 0..7  consumers: 4 x 2 warp grid, 32 x 32 per warp (2 x 4 MMAs per k4).
// A stage holds A[128 x 16] with the 128-byte swizzle (conflict-free fragment
// loads) and B[16 x 64] as eight 16 x 8 boxes laid side by side (each k row of a
// box is 64 contiguous bytes, so a fragment load reads 256 contiguous bytes).
// The product s = A*B is accumulated from zero and subtracted at the end, the
// form of the reference's gemm!(C, A, B, -1, 1) (src/blas/gemm.jl:286-298).
#include "tma_util.cuh"

namespace oxi {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        OXI_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess)
            throw CudaError{cudaErrorNotSupported, "cuTensorMapEncodeTiled unavailable"};
        fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

void make_tmap_2d(CUtensorMap *tm, CUtensorMapDataType dt, int esize, const void *base, i64 cols,
                  i64 rows, i64 ld, int box_cols, int box_rows, CUtensorMapSwizzle swz) {
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * esize)};
    cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = tensor_map_encoder()(tm, dt, 2, const_cast<void *>(base), dims, strides, box, estr,
                                      CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw CudaError{cudaErrorInvalidValue, "cuTensorMapEncodeTiled"};
}

namespace {
constexpr int BM = 128, BN = 64, BK = 16, STAGES = 4;
constexpr int A_STAGE_BYTES = BM * BK * 8;  // 16 KB
constexpr int B_STAGE_BYTES = BK * BN * 8;  // 8 KB
constexpr int STAGE_BYTES = A_STAGE_BYTES + B_STAGE_BYTES;
constexpr int NCONSUMER_WARPS = 8;
constexpr int NTHREADS = (NCONSUMER_WARPS + 1) * 32;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
}  // namespace

__global__ void __launch_bounds__(NTHREADS, 2)
k_gemm_dmma(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
            double *__restrict__ C, i64 ldc, int M, int N, int K, int *__restrict__ ab, int upper_only) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~uintptr_t(1023));
    uint64_t *full = (uint64_t *)(smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    // upper_only (a symmetric rank-k update of the upper triangle): tiles that
    // lie wholly below the diagonal are not computed
    if (upper_only && m0 > n0 + BN - 1) return;
    const int KT = (K + BK - 1) / BK;

    __shared__ int s_skip;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NCONSUMER_WARPS);
        }
        s_skip = aborted(ab) ? 1 : 0;  // one reading for the whole CTA
        fence_barrier_init();
    }
    __syncthreads();
    if (s_skip) return;  // the call was aborted by an earlier wait

    if (warp == NCONSUMER_WARPS) {
        // ---------------- producer ----------------
        if (lane == 0) {
            prefetch_tmap(&tmA);
            prefetch_tmap(&tmB);
            for (int kt = 0; kt < KT; ++kt) {
                const int s = kt % STAGES;
                if (kt >= STAGES) {
                    if (!mbar_wait<false>(&empty[s], ((kt / STAGES) + 1) & 1, ab, 2)) break;
                }
                uint8_t *sa = smem + s * STAGE_BYTES;
                uint8_t *sb = sa + A_STAGE_BYTES;
                mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
                tma_load_2d(sa, &tmA, &full[s], kt * BK, m0);
#pragma unroll
                for (int g = 0; g < BN / 8; ++g)
                    tma_load_2d(sb + g * (BK * 8 * 8), &tmB, &full[s], n0 + 8 * g, kt * BK);
            }
        }
        return;
    }

    // ---------------- consumers ----------------
    const int wm = warp & 3, wn = warp >> 2;  // 4 x 2 warps
    const int gid = lane >> 2, tig = lane & 3;
    double acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0;

    for (int kt = 0; kt < KT; ++kt) {
        const int s = kt % STAGES;
        if (!mbar_wait<false>(&full[s], (kt / STAGES) & 1, ab, 2)) return;
        const uint8_t *sa = smem + s * STAGE_BYTES;
        const uint8_t *sb = sa + A_STAGE_BYTES;
#pragma unroll
        for (int k4 = 0; k4 < BK / 4; ++k4) {
            double af[2][2], bf[4];
            const int kc = k4 * 4 + tig;  // k column within the slab
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int r = wm * 32 + mt * 16 + gid + 8 * h;
                    // 128B swizzle: 16-byte chunk index XOR (row mod 8)
                    const int off = r * 128 + ((((kc * 8) >> 4) ^ (r & 7)) << 4) + ((kc * 8) & 15);
                    af[mt][h] = *(const double *)(sa + off);
                }
            }
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int g = (wn * 32 + nt * 8) >> 3;
                bf[nt] = *(const double *)(sb + g * (BK * 64) + kc * 64 + gid * 8);
            }
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt)
                    asm volatile(
                        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, "
                        "{%6}, {%0,%1,%2,%3};"
                        : "+d"(acc[mt][nt][0]), "+d"(acc[mt][nt][1]), "+d"(acc[mt][nt][2]),
                          "+d"(acc[mt][nt][3])
                        : "d"(af[mt][0]), "d"(af[mt][1]), "d"(bf[nt]));
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }

    // epilogue: C -= acc.  The eight C pairs of a row are loaded before any is
    // used so their round trips overlap (16-byte accesses when aligned).  A
    // symmetric update's tile that crosses the diagonal writes only the
    // elements on and above it (the other triangle stays as it was).
    const bool vec2 = ((ldc & 1) == 0) && ((((uintptr_t)C) & 15) == 0) && !(upper_only && m0 + BM - 1 > n0);
    const int cmin_row = upper_only ? 1 : 0;  // 1: column c is written only when c >= r
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = m0 + wm * 32 + mt * 16 + gid + 8 * h;
            if (r >= M) continue;
            double *crow = C + (i64)r * ldc;
            double2 cv[4];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int c = n0 + wn * 32 + nt * 8 + 2 * tig;
                if (c + 1 < N && vec2) cv[nt] = __ldcs((const double2 *)(crow + c));
                else {
                    cv[nt].x = (c < N && (!cmin_row || c >= r)) ? crow[c] : 0.0;
                    cv[nt].y = (c + 1 < N && (!cmin_row || c + 1 >= r)) ? crow[c + 1] : 0.0;
                }
            }
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int c = n0 + wn * 32 + nt * 8 + 2 * tig;
                double2 v;
                v.x = cv[nt].x - acc[mt][nt][2 * h];
                v.y = cv[nt].y - acc[mt][nt][2 * h + 1];
                if (c + 1 < N && vec2) __stcs((double2 *)(crow + c), v);
                else {
                    if (c < N && (!cmin_row || c >= r)) crow[c] = v.x;
                    if (c + 1 < N && (!cmin_row || c + 1 >= r)) crow[c + 1] = v.y;
                }
            }
        }
}

void launch_gemm_dmma(double *C, i64 ldc, const double *A, i64 lda, const double *B, i64 ldb, i64 M,
                      i64 N, i64 K, cudaStream_t s, bool upper_only) {
    if (M <= 0 || N <= 0 || K <= 0) return;
    const bool aligned = ((uintptr_t)A % 16 == 0) && ((uintptr_t)B % 16 == 0) && (lda % 2 == 0) &&
                         (ldb % 2 == 0) && M < (1 << 30) && N < (1 << 30) && K < (1 << 30);
    if (!aligned) {  // TMA needs 16-byte aligned bases and pitches (the whole block: same results)
        if (upper_only)  // the plain kernel would write both triangles; callers align first
            throw CudaError{cudaErrorInvalidValue, "symmetric update needs 16-byte aligned operands"};
        launch_gemm_ref<double>(C, ldc, A, lda, B, ldb, M, N, K, s);
        return;
    }
    CUtensorMap tmA, tmB;
    make_tmap_2d(&tmA, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, A, K, M, lda, BK, BM,
                 CU_TENSOR_MAP_SWIZZLE_128B);
    make_tmap_2d(&tmB, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, B, N, K, ldb, 8, BK,
                 CU_TENSOR_MAP_SWIZZLE_NONE);
    set_max_dyn_smem((const void *)k_gemm_dmma, SMEM_BYTES);
    dim3 grid((unsigned)((N + BN - 1) / BN), (unsigned)((M + BM - 1) / BM));
    ProfScope ps(KC_GEMM_DMMA, s, (upper_only ? 1.0 : 2.0) * M * N * K, 8.0 * (2.0 * M * N + M * K + K * N));
    k_gemm_dmma<<<grid, NTHREADS, SMEM_BYTES, s>>>(tmA, tmB, C, ldc, (int)M, (int)N, (int)K, cur_abort(),
                                                   upper_only ? 1 : 0);
    OXI_LAUNCH_CHECK();
}

}  // namespace oxi
