// Mixed-precision trailing update on the 5th-generation tensor cores:
//   C (FP32, row-major) <- C - scale * (A * B^T)
// A: M x K, B: N x K, both 16-bit (BF16 or FP16) and K-major (K contiguous),
// accumulated in FP32 in tensor memory (tcgen05.mma kind::f16).
//
// Tile 128 x 256, k slab 64 (one 128-byte swizzle atom per row), a 2-stage TMA
// ring for the operands, the whole FP32 C tile (128 KB) in shared memory, and
// two TMEM accumulators so that a tile's epilogue overlaps the next tile's MMAs
// (see k_gemm_tc).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include "tma_util.cuh"

namespace oxi {

namespace tc {
constexpr int BM = 128, BN = 256, BK = 64, STAGES = 2;
constexpr int A_BYTES = BM * BK * 2;  // 16 KB
constexpr int B_BYTES = BN * BK * 2;  // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int CBOX_COLS = 32;                    // one 128-byte swizzle atom per row
constexpr int NCBOX = BN / CBOX_COLS;            // 8 boxes across the tile
constexpr int CBOX_BYTES = BM * CBOX_COLS * 4;   // 16 KB
constexpr int C_BYTES = NCBOX * CBOX_BYTES;      // 128 KB: the whole FP32 C tile
constexpr int NTHREADS = 256;
constexpr int TMEM_COLS = 256;  // per accumulator buffer (two buffers)
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + C_BYTES + 1024 + 256;
}  // namespace tc

// UMMA shared-memory descriptor, K-major operand in the 128-byte swizzle
// layout TMA writes (rows of 128 bytes, 8-row groups 1024 bytes apart).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t smem_addr) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFF);  // start address
    d |= (uint64_t)1 << 16;                       // leading byte offset (unused for SW128 K-major)
    d |= (uint64_t)(1024 >> 4) << 32;             // stride byte offset: 8 rows x 128 B
    d |= (uint64_t)1 << 46;                       // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                       // SWIZZLE_128B
    return d;
}

// Instruction descriptor: D=F32, A/B format (0 F16, 1 BF16), K-major both, M, N.
__host__ __device__ constexpr uint32_t umma_idesc_f16(int ab_format, int M, int N) {
    return (1u << 4) | ((uint32_t)ab_format << 7) | ((uint32_t)ab_format << 10) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *tm, const void *src, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
            (uint64_t)tm),
        "r"(smem_u32(src)), "r"(x), "r"(y)
        : "memory");
}

// Bounded wait that also gives up when another role of the CTA has given up.
// A wait that runs past the call's limit records it in the call's abort word
// ab.  The word itself is read at entry only: with TMA loads and MMAs of its
// own in flight, the CTA must not leave because some other kernel failed.
__device__ __forceinline__ bool mbar_wait_ab(uint64_t *bar, uint32_t parity, volatile int *abort_flag,
                                             int *ab) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    const uint64_t lim = wait_limit_ns(ab);
    for (;;) {
        for (int it = 0; it < 256; ++it)
            if (mbar_try_wait(bar, parity)) return true;
        if (*abort_flag) return false;
        if (global_ns() - t0 > lim) break;
    }
    raise_abort(ab, 5);
    *abort_flag = 1;
    return false;
}

// Persistent, warp-specialised tcgen05 GEMM (one CTA per SM, tiles strided by
// the grid):
//   warp 0 lane 0   operand producer: A/B slabs by TMA into a 2-stage ring
//   warp 1 lane 0   MMA issuer into one of two 256-column TMEM accumulators
//   warp 2 lane 0   C producer: the tile's FP32 C (eight 32-column boxes, 128-byte
//                   swizzle) by TMA, once the previous tile has been stored
//   warps 4..7      epilogue warpgroup: TMEM -> registers, C - scale*D in shared
//                   memory, TMA store -- overlapping the next tile's MMAs
template <int AB_FORMAT>
__global__ void __launch_bounds__(256, 1)
k_gemm_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
          const __grid_constant__ CUtensorMap tmC, int M, int N, int K, float scale,
          const float *__restrict__ d_scale, int *__restrict__ ab) {
    using namespace tc;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~uintptr_t(1023));
    uint8_t *sC = smem + STAGES * STAGE_BYTES;
    uint64_t *full = (uint64_t *)(sC + C_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;  // [2]
    uint64_t *tempty = tfull + 2;      // [2]
    uint64_t *cfull = tempty + 2;      // [NCBOX]: C box loaded
    uint64_t *cempty = cfull + NCBOX;  // [NCBOX]: C box stored (read out of shared memory)
    uint32_t *tmem_slot = (uint32_t *)(cempty + NCBOX);
    volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int KT = (K + BK - 1) / BK;
    const int tilesN = (N + BN - 1) / BN, tilesM = (M + BM - 1) / BM;
    const int ntiles = tilesM * tilesN;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 4);
        }
        for (int c = 0; c < NCBOX; ++c) {
            mbar_init(&cfull[c], 1);
            mbar_init(&cempty[c], 1);
        }
        *abort_flag = aborted(ab) ? 1 : 0;  // an aborted call: every role skips its loop
        fence_barrier_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(2 * TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        tc_fence_before();
    }
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        prefetch_tmap(&tmA);
        prefetch_tmap(&tmB);
        int kb = 0;
        for (int tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x) {
            const int m0 = (tile / tilesN) * BM, n0 = (tile % tilesN) * BN;
            for (int kt = 0; kt < KT; ++kt, ++kb) {
                const int s = kb % STAGES;
                if (kb >= STAGES && !mbar_wait_ab(&empty[s], ((kb / STAGES) + 1) & 1, abort_flag, ab)) break;
                uint8_t *sa = smem + s * STAGE_BYTES;
                mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
                tma_load_2d(sa, &tmA, &full[s], kt * BK, m0);
                tma_load_2d(sa + A_BYTES, &tmB, &full[s], kt * BK, n0);
            }
        }
    } else if (warp == 1 && lane == 0) {
        constexpr uint32_t idesc = umma_idesc_f16(AB_FORMAT, BM, BN);
        int kb = 0, li = 0;
        for (int tile = blockIdx.x; tile < ntiles && !*abort_flag; tile += gridDim.x, ++li) {
            const int b = li & 1;
            if (li >= 2 && !mbar_wait_ab(&tempty[b], ((li >> 1) + 1) & 1, abort_flag, ab)) break;
            tc_fence_after();
            const uint32_t dacc = tmem + (uint32_t)(b * TMEM_COLS);
            for (int kt = 0; kt < KT; ++kt, ++kb) {
                const int s = kb % STAGES;
                if (!mbar_wait_ab(&full[s], (kb / STAGES) & 1, abort_flag, ab)) break;
                tc_fence_after();
                const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
                const uint64_t da = umma_desc_sw128(sa), db = umma_desc_sw128(sa + A_BYTES);
#pragma unroll
                for (int k = 0; k < BK / 16; ++k) {
                    const uint64_t adv = (uint64_t)((k * 32) >> 4);  // 16 elements = 32 bytes
                    const uint32_t acc = (kt > 0 || k > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dacc),
                        "l"(da + adv), "l"(db + adv), "r"(idesc), "r"(acc));
                }
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                        smem_u32(&empty[s]))
                    : "memory");
            }
            asm volatile(
                "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                    smem_u32(&tfull[b]))
                : "memory");
        }
    } else if (warp == 2 && lane == 0) {
        // C producer: box by box, each as soon as the previous tile's store
        // of that box has left shared memory
        prefetch_tmap(&tmC);
        int li = 0;
        bool go = true;
        for (int tile = blockIdx.x; go && tile < ntiles && !*abort_flag; tile += gridDim.x, ++li) {
            const int m0 = (tile / tilesN) * BM, n0 = (tile % tilesN) * BN;
            for (int bx = 0; bx < NCBOX; ++bx) {
                if (li >= 1 && !mbar_wait_ab(&cempty[bx], (li - 1) & 1, abort_flag, ab)) {
                    go = false;
                    break;
                }
                mbar_arrive_expect_tx(&cfull[bx], CBOX_BYTES);
                tma_load_2d(sC + bx * CBOX_BYTES, &tmC, &cfull[bx], n0 + bx * CBOX_COLS, m0);
            }
        }
    } else if (warp >= 4) {
        const int ew = warp - 4;          // TMEM lane quadrant of this warp
        const int r = ew * 32 + lane;     // tile row owned by this thread
        const float sc = d_scale ? scale * (*d_scale) : scale;
        // Box by box: wait for the box's C (and, for the first box, the
        // accumulator), C - scale * D into shared memory, TMA store of the box;
        // the store of box c is confirmed read before box c's slot is handed
        // back to the producer, one box later.  Every wait's outcome is made
        // uniform over the four warps before they meet at a named barrier.
        int li = 0;
        bool go = true;
        for (int tile = blockIdx.x; go && tile < ntiles; tile += gridDim.x, ++li) {
            const int m0 = (tile / tilesN) * BM, n0 = (tile % tilesN) * BN;
            const int b = li & 1;
            const uint32_t base = tmem + (uint32_t)(b * TMEM_COLS) + ((uint32_t)(ew * 32) << 16);
#pragma unroll 1
            for (int c = 0; c < NCBOX; ++c) {
                const bool ok = (c > 0 || mbar_wait_ab(&tfull[b], (li >> 1) & 1, abort_flag, ab)) &&
                                mbar_wait_ab(&cfull[c], li & 1, abort_flag, ab);
                uint32_t all_ok;
                asm volatile(
                    "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n"
                    " bar.red.and.pred q, 1, 128, p;\n selp.u32 %0, 1, 0, q;\n}\n"
                    : "=r"(all_ok)
                    : "r"((uint32_t)ok)
                    : "memory");
                if (!all_ok) {
                    go = false;
                    break;
                }
                if (c == 0) tc_fence_after();
                uint32_t v[32];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
                    "%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
                      "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
                      "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
                      "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
                      "=r"(v[31])
                    : "r"(base + (uint32_t)(c * 32)));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (c == NCBOX - 1) {  // the accumulator is drained: the MMA warp may reuse it
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&tempty[b]);
                }
                uint8_t *rowp = sC + c * CBOX_BYTES + r * 128;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    float4 *p4 = (float4 *)(rowp + ((q ^ (r & 7)) << 4));  // 128-byte swizzle
                    float4 x = *p4;
                    x.x -= sc * __uint_as_float(v[4 * q + 0]);
                    x.y -= sc * __uint_as_float(v[4 * q + 1]);
                    x.z -= sc * __uint_as_float(v[4 * q + 2]);
                    x.w -= sc * __uint_as_float(v[4 * q + 3]);
                    *p4 = x;
                }
                fence_proxy_async();  // shared-memory writes -> visible to the TMA (async proxy)
                asm volatile("bar.sync 1, 128;" ::: "memory");
                if (ew == 0 && lane == 0) {
                    tma_store_2d(&tmC, sC + c * CBOX_BYTES, n0 + c * CBOX_COLS, m0);
                    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                    if (c > 0) {
                        asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
                        mbar_arrive(&cempty[c - 1]);  // box c-1's slot may be refilled
                    }
                    if (c == NCBOX - 1) {
                        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                        mbar_arrive(&cempty[c]);
                    }
                }
            }
        }
        if (ew == 0 && lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(2 * TMEM_COLS));
    }
}

// ---- operand conversion (FP32 row-major -> 16-bit K-major) ----
template <typename H> __device__ __forceinline__ H to_half_t(float x);
template <> __device__ __forceinline__ __nv_bfloat16 to_half_t<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
template <> __device__ __forceinline__ __half to_half_t<__half>(float x) { return __float2half_rn(x); }

// dst[r][c] = src[r][c] * scale (same orientation): the A operand (L21).
template <typename H>
__global__ void k_cvt_rows(const float *__restrict__ src, i64 lds, H *__restrict__ dst, i64 ldd,
                           int rows, int cols, float scale, const float *__restrict__ d_scale) {
    const float s = d_scale ? scale * (*d_scale) : scale;
    const i64 r = blockIdx.y;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x)
        dst[r * ldd + c] = to_half_t<H>(src[r * lds + c] * s);
}

// dst[c][r] = src[r][c] * scale (transposed): the B operand (U12 -> N x K).
template <typename H>
__global__ void k_cvt_transpose(const float *__restrict__ src, i64 lds, H *__restrict__ dst,
                                i64 ldd, int rows, int cols, float scale,
                                const float *__restrict__ d_scale) {
    __shared__ float tile[32][33];
    const float s = d_scale ? scale * (*d_scale) : scale;
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int k = ty; k < 32; k += 8) {
        const int r = r0 + k, c = c0 + tx;
        tile[k][tx] = (r < rows && c < cols) ? src[(i64)r * lds + c] : 0.f;
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int c = c0 + k, r = r0 + tx;
        if (c < cols && r < rows) dst[(i64)c * ldd + r] = to_half_t<H>(tile[tx][k] * s);
    }
}

// Split operands: x = hi + lo with hi = H(x s), lo = H(x s - hi) (s: the operand's
// power-of-two scale, 1 for BF16).  A row becomes [hi | hi | lo] and a B row
// [hi | lo | hi] along K, so one GEMM over 3K accumulates A_hi B_hi + A_hi B_lo
// + A_lo B_hi; the dropped A_lo B_lo term is ~2^-16 (BF16) or ~2^-22 (FP16)
// relative.  FP32-accumulated products from 16-bit tensor-core operands.
template <typename H>
__device__ __forceinline__ float from_half_t(H x);
template <> __device__ __forceinline__ float from_half_t<__nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }
template <> __device__ __forceinline__ float from_half_t<__half>(__half x) { return __half2float(x); }

template <typename H>
__global__ void k_cvt_rows_split3(const float *__restrict__ src, i64 lds, H *__restrict__ dst, i64 ldd, int rows,
                                  int cols, float scale, const float *__restrict__ d_scale) {
    const float sc = d_scale ? scale * (*d_scale) : scale;
    const i64 r = blockIdx.y;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x) {
        const float x = src[r * lds + c] * sc;
        const H hi = to_half_t<H>(x);
        const H lo = to_half_t<H>(x - from_half_t<H>(hi));
        H *d = dst + r * ldd;
        d[c] = hi;
        d[cols + c] = hi;
        d[2 * cols + c] = lo;
    }
}
template <typename H>
__global__ void k_cvt_transpose_split3(const float *__restrict__ src, i64 lds, H *__restrict__ dst, i64 ldd,
                                       int rows, int cols, float scale, const float *__restrict__ d_scale) {
    __shared__ float tile[32][33];
    const float sc = d_scale ? scale * (*d_scale) : scale;
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int k = ty; k < 32; k += 8) {
        const int r = r0 + k, c = c0 + tx;
        tile[k][tx] = (r < rows && c < cols) ? src[(i64)r * lds + c] : 0.f;
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int c = c0 + k, r = r0 + tx;  // dst row c (an N index), K position r
        if (c < cols && r < rows) {
            const float x = tile[tx][k] * sc;
            const H hi = to_half_t<H>(x);
            const H lo = to_half_t<H>(x - from_half_t<H>(hi));
            H *d = dst + (i64)c * ldd;
            d[r] = hi;
            d[rows + r] = lo;
            d[2 * rows + r] = hi;
        }
    }
}

// ---- host ----
void launch_gemm_tc(int fmt /*0 fp16, 1 bf16*/, float *C, i64 ldc, const void *A16, i64 lda16,
                    const void *B16, i64 ldb16, i64 M, i64 N, i64 K, float scale,
                    const float *d_scale, cudaStream_t s, int max_ctas) {
    using namespace tc;
    if (M <= 0 || N <= 0 || K <= 0) return;
    CUtensorMap tmA, tmB, tmC;
    const CUtensorMapDataType dt = fmt == 1 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    make_tmap_2d(&tmA, dt, 2, A16, K, M, lda16, BK, BM, CU_TENSOR_MAP_SWIZZLE_128B);
    make_tmap_2d(&tmB, dt, 2, B16, K, N, ldb16, BK, BN, CU_TENSOR_MAP_SWIZZLE_128B);
    make_tmap_2d(&tmC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, C, N, M, ldc, CBOX_COLS, BM,
                 CU_TENSOR_MAP_SWIZZLE_128B);
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        OXI_CUDA(cudaGetDevice(&dev));
        OXI_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    const i64 tiles = ((N + BN - 1) / BN) * ((M + BM - 1) / BM);
    const void *kern = fmt == 1 ? (const void *)k_gemm_tc<1> : (const void *)k_gemm_tc<0>;
    set_max_dyn_smem(kern, SMEM_BYTES);
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(NTHREADS);
    cfg.dynamicSmemBytes = SMEM_BYTES;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    if (max_ctas < 0) {
        // Persistent CTAs in at most -max_ctas clusters of GEMM_GPC_CLUSTER: each
        // cluster fills the SMs of one GPC, and at least one cluster fewer than
        // fit leaves a whole GPC to a concurrent leaf LU (a cluster of up to 16
        // CTAs on one GPC).  The kernel itself uses no cluster feature.
        static int ncl[2] = {-1, -1};
        int &nc = ncl[fmt == 1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = GEMM_GPC_CLUSTER;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        if (nc < 0) {
            OXI_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            cfg.gridDim = dim3(GEMM_GPC_CLUSTER);
            int v = 0;
            if (cudaOccupancyMaxActiveClusters(&v, kern, &cfg) != cudaSuccess) {
                cudaGetLastError();
                v = 0;
            }
            nc = v;
        }
        if (nc >= 2) {
            const i64 want = (tiles + GEMM_GPC_CLUSTER - 1) / GEMM_GPC_CLUSTER * GEMM_GPC_CLUSTER;
            const int use = std::min(nc - 1, -max_ctas);
            cfg.gridDim = dim3((unsigned)std::min<i64>(want, (i64)use * GEMM_GPC_CLUSTER));
        } else {  // no whole GPC to spare: plain launch leaving some SMs
            cfg.attrs = nullptr;
            cfg.numAttrs = 0;
            cfg.gridDim = dim3((unsigned)std::min<i64>(tiles, std::max(1, sms - 24)));
        }
    } else {
        cfg.gridDim = dim3((unsigned)std::min<i64>(tiles, max_ctas > 0 ? std::min(max_ctas, sms) : sms));
    }
    ProfScope ps(KC_GEMM_TC, s, 2.0 * M * N * K, 8.0 * M * N + 2.0 * (M + N) * K);
    if (fmt == 1)
        OXI_CUDA(cudaLaunchKernelEx(&cfg, k_gemm_tc<1>, tmA, tmB, tmC, (int)M, (int)N, (int)K, scale, d_scale, cur_abort()));
    else
        OXI_CUDA(cudaLaunchKernelEx(&cfg, k_gemm_tc<0>, tmA, tmB, tmC, (int)M, (int)N, (int)K, scale, d_scale, cur_abort()));
    OXI_LAUNCH_CHECK();
}

void launch_cvt_rows16(int fmt, const float *src, i64 lds, void *dst, i64 ldd, i64 rows, i64 cols,
                       float scale, const float *d_scale, cudaStream_t s) {
    if (rows <= 0 || cols <= 0) return;
    dim3 grid((unsigned)std::min<i64>((cols + 255) / 256, 64), (unsigned)rows);
    ProfScope ps(KC_CONVERT, s, 0.0, 6.0 * rows * cols);
    if (fmt == 1)
        k_cvt_rows<__nv_bfloat16><<<grid, 256, 0, s>>>(src, lds, (__nv_bfloat16 *)dst, ldd, (int)rows, (int)cols, scale, d_scale);
    else
        k_cvt_rows<__half><<<grid, 256, 0, s>>>(src, lds, (__half *)dst, ldd, (int)rows, (int)cols, scale, d_scale);
    OXI_LAUNCH_CHECK();
}

void launch_cvt_transpose16(int fmt, const float *src, i64 lds, void *dst, i64 ldd, i64 rows,
                            i64 cols, float scale, const float *d_scale, cudaStream_t s) {
    if (rows <= 0 || cols <= 0) return;
    dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
    ProfScope ps(KC_CONVERT, s, 0.0, 6.0 * rows * cols);
    if (fmt == 1)
        k_cvt_transpose<__nv_bfloat16><<<grid, dim3(32, 8), 0, s>>>(src, lds, (__nv_bfloat16 *)dst, ldd, (int)rows, (int)cols, scale, d_scale);
    else
        k_cvt_transpose<__half><<<grid, dim3(32, 8), 0, s>>>(src, lds, (__half *)dst, ldd, (int)rows, (int)cols, scale, d_scale);
    OXI_LAUNCH_CHECK();
}

}  // namespace oxi

namespace oxi {

// FP16 operand scaling: L21 has |l| <= 1 under partial pivoting and is scaled by
// 2^14; U12 is scaled by the power of two that brings max|U12| into [2^14, 2^15),
// so neither operand overflows FP16 and small entries keep their precision.  The
// GEMM epilogue multiplies by the inverse of both scales (exact powers of two).
__global__ void k_absmax_f32(const float *__restrict__ src, i64 lds, int rows, int cols,
                             unsigned int *__restrict__ out) {
    float mx = 0.f;
    const int r = blockIdx.y;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < cols; c += gridDim.x * blockDim.x)
        mx = fmaxf(mx, fabsf(src[(i64)r * lds + c]));
    for (int off = 16; off > 0; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(mx));
}
__global__ void k_fp16_scales(const unsigned int *__restrict__ umax_bits, float *__restrict__ sc) {
    const float umax = __uint_as_float(*umax_bits);
    int e = 0;
    if (umax > 0.f && isfinite(umax)) frexpf(umax, &e);  // umax in [2^(e-1), 2^e)
    const int su = 15 - e;                                 // umax * 2^su in [2^14, 2^15)
    sc[0] = ldexpf(1.f, su);                               // U12 scale
    sc[1] = ldexpf(1.f, -(su + 14));                       // epilogue: 2^-14 * 2^-su
}

// The lookahead's second trailing update (operand slot 1) multiplies the same
// L21 as the first (slot 0), converted just before on the first stream, which
// the second stream waits for; slot 0 is not rewritten until the second update
// has finished.  Reuse that conversion.
static const void *reuse_a16(const oxi_handle_s *h, const float *A, i64 lda, i64 M, i64 K) {
    const auto &r = h->tc_last_a;
    if (h->tc_slot != 1 || r.src != A || r.lda != lda || r.M != M || r.K != K || r.kind != h->trailing) return nullptr;
    return r.a16;
}
static void note_a16(oxi_handle_s *h, const float *A, i64 lda, i64 M, i64 K, const void *a16) {
    if (h->tc_slot != 0) return;
    h->tc_last_a = {A, lda, M, K, h->trailing, a16};
}

void gemm_trailing_f32(oxi_handle_s *h, float *C, i64 ldc, const float *A, i64 lda, const float *B,
                       i64 ldb, i64 M, i64 N, i64 K) {
    if (M <= 0 || N <= 0 || K <= 0) return;
    if (((uintptr_t)C % 16) != 0 || (ldc * 4) % 16 != 0) {
        // the C tile travels by TMA: stage an unaligned C through an aligned copy
        const i64 ldp = (N + 3) / 4 * 4;
        float *Cp = (float *)h->solve_ws.get(sizeof(float) * (size_t)M * ldp);
        OXI_CUDA(cudaMemcpy2DAsync(Cp, ldp * 4, C, ldc * 4, N * 4, M, cudaMemcpyDeviceToDevice, h->stream));
        gemm_trailing_f32(h, Cp, ldp, A, lda, B, ldb, M, N, K);
        OXI_CUDA(cudaMemcpy2DAsync(C, ldc * 4, Cp, ldp * 4, N * 4, M, cudaMemcpyDeviceToDevice, h->stream));
        return;
    }
    if (h->trailing == TRAIL_BF16X3 || h->trailing == TRAIL_FP16X3) {
        const bool f16 = h->trailing == TRAIL_FP16X3;
        const i64 K3 = 3 * K, ldk3 = (K3 + 7) / 8 * 8;
        DeviceBuffer &tcw = h->tc_slot ? h->tc_ws2 : h->tc_ws;
        char *ws = (char *)tcw.get((size_t)(M + N) * ldk3 * 2 + 1024);
        void *A16 = ws;
        void *B16 = (void *)(((uintptr_t)(ws + (size_t)M * ldk3 * 2) + 255) & ~uintptr_t(255));
        cudaStream_t s = h->stream;
        float *scal = nullptr;
        if (f16) {  // the FP16 operand scales (see k_fp16_scales)
            scal = (float *)((char *)h->scratch.get(kScratchBytes) + kScratchScalOff + 1536 + 256 * h->tc_slot);
            unsigned int *umax = (unsigned int *)(scal + 4);
            OXI_CUDA(cudaMemsetAsync(umax, 0, sizeof(unsigned int), s));
            k_absmax_f32<<<dim3((unsigned)std::min<i64>((N + 255) / 256, 16), (unsigned)K), 256, 0, s>>>(
                B, ldb, (int)K, (int)N, umax);
            OXI_LAUNCH_CHECK();
            k_fp16_scales<<<1, 1, 0, s>>>(umax, scal);
            OXI_LAUNCH_CHECK();
        }
        if (const void *prev = reuse_a16(h, A, lda, M, K)) {
            A16 = const_cast<void *>(prev);
        } else {
            ProfScope ps(KC_CONVERT, s, 0.0, 10.0 * (double)M * K);
            dim3 g((unsigned)std::min<i64>((K + 255) / 256, 64), (unsigned)M);
            if (f16)
                k_cvt_rows_split3<__half><<<g, 256, 0, s>>>(A, lda, (__half *)A16, ldk3, (int)M, (int)K, 16384.f,
                                                            nullptr);
            else
                k_cvt_rows_split3<__nv_bfloat16><<<g, 256, 0, s>>>(A, lda, (__nv_bfloat16 *)A16, ldk3, (int)M,
                                                                   (int)K, 1.f, nullptr);
            OXI_LAUNCH_CHECK();
            note_a16(h, A, lda, M, K, A16);
        }
        {
            ProfScope ps(KC_CONVERT, s, 0.0, 10.0 * (double)N * K);
            dim3 g((unsigned)((N + 31) / 32), (unsigned)((K + 31) / 32));
            if (f16)
                k_cvt_transpose_split3<__half><<<g, dim3(32, 8), 0, s>>>(B, ldb, (__half *)B16, ldk3, (int)K,
                                                                         (int)N, 1.f, scal);
            else
                k_cvt_transpose_split3<__nv_bfloat16><<<g, dim3(32, 8), 0, s>>>(B, ldb, (__nv_bfloat16 *)B16, ldk3,
                                                                                (int)K, (int)N, 1.f, nullptr);
            OXI_LAUNCH_CHECK();
        }
        if (f16) launch_gemm_tc(0, C, ldc, A16, ldk3, B16, ldk3, M, N, K3, 1.f, scal + 1, s, h->gemm_ctas);
        else launch_gemm_tc(1, C, ldc, A16, ldk3, B16, ldk3, M, N, K3, 1.f, nullptr, s, h->gemm_ctas);
        return;
    }
    const int fmt = (h->trailing == TRAIL_BF16) ? 1 : 0;
    const i64 ldk = (K + 7) / 8 * 8;
    DeviceBuffer &tcw = h->tc_slot ? h->tc_ws2 : h->tc_ws;
    char *ws = (char *)tcw.get((size_t)(M + N) * ldk * 2 + 1024);
    void *A16 = ws;
    void *B16 = ws + (size_t)M * ldk * 2;
    B16 = (void *)(((uintptr_t)B16 + 255) & ~uintptr_t(255));
    float *scal = (float *)((char *)h->scratch.get(kScratchBytes) + kScratchScalOff + 1536 + 256 * h->tc_slot);
    cudaStream_t s = h->stream;
    const void *prev = reuse_a16(h, A, lda, M, K);
    if (prev) A16 = const_cast<void *>(prev);
    if (fmt == 1) {
        if (!prev) {
            launch_cvt_rows16(1, A, lda, A16, ldk, M, K, 1.f, nullptr, s);
            note_a16(h, A, lda, M, K, A16);
        }
        launch_cvt_transpose16(1, B, ldb, B16, ldk, K, N, 1.f, nullptr, s);
        launch_gemm_tc(1, C, ldc, A16, ldk, B16, ldk, M, N, K, 1.f, nullptr, s, h->gemm_ctas);
    } else {
        unsigned int *umax = (unsigned int *)(scal + 4);
        OXI_CUDA(cudaMemsetAsync(umax, 0, sizeof(unsigned int), s));
        k_absmax_f32<<<dim3((unsigned)std::min<i64>((N + 255) / 256, 16), (unsigned)K), 256, 0, s>>>(
            B, ldb, (int)K, (int)N, umax);
        OXI_LAUNCH_CHECK();
        k_fp16_scales<<<1, 1, 0, s>>>(umax, scal);
        OXI_LAUNCH_CHECK();
        if (!prev) {
            launch_cvt_rows16(0, A, lda, A16, ldk, M, K, 16384.f, nullptr, s);
            note_a16(h, A, lda, M, K, A16);
        }
        launch_cvt_transpose16(0, B, ldb, B16, ldk, K, N, 1.f, scal, s);
        launch_gemm_tc(0, C, ldc, A16, ldk, B16, ldk, M, N, K, 1.f, scal + 1, s, h->gemm_ctas);
    }
}

}  // namespace oxi
