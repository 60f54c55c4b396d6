// TMA / mbarrier helpers (inline PTX, sm_90+ forms available on sm_100a) and the
// host-side tensor-map encoder obtained from the driver at run time.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "oxi_internal.h"

namespace oxi {

// Waits on the GPU are bounded in time: a waiter that has seen no progress for
// the call's wait limit (kWaitLimitNs unless the handle sets another) records an
// error code in the call's abort word and gives up instead of hanging the device.
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s; legitimate waits are microseconds

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// The abort block of a call (handle-owned, see AbortBlock in oxi_internal.h):
// int 0 is the sticky abort code, ints 2-3 the wait limit in ns (0: default).
// Once any wait of the call gives up, every later wait and every kernel entry
// of the same call sees the code and returns at once, so one broken wait costs
// one wait limit, not one per launch.
__device__ __forceinline__ bool aborted(const int *ab) {
    return ab != nullptr && *(const volatile int *)ab != 0;
}
__device__ __forceinline__ uint64_t wait_limit_ns(const int *ab) {
    if (!ab) return kWaitLimitNs;
    const uint64_t v = *(const volatile unsigned long long *)(ab + 2);
    return v ? v : kWaitLimitNs;
}
__device__ __forceinline__ void raise_abort(int *ab, int code) {
    if (ab) atomicCAS(ab, 0, code);
}
// Bookkeeping of a polling loop: call once per poll; true when the loop must
// stop (this wait ran past the limit, recorded as `code`, or the call was
// aborted elsewhere).  The clock and the abort word are read every `every` polls.
template <uint32_t every = 256>
__device__ __forceinline__ bool spin_give_up(uint32_t &it, uint64_t t0, int *ab, int code) {
    if ((++it & (every - 1)) != 0) return false;
    if (aborted(ab)) return true;
    if (global_ns() - t0 > wait_limit_ns(ab)) {
        raise_abort(ab, code);
        return true;
    }
    return false;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait; returns false when it ran past the call's limit (recording
// `code` in the abort word ab) or, with POLL_ABORT, when the call has been
// aborted elsewhere.  Kernels with asynchronous copies or tensor-core work in
// flight (TMA loads, tcgen05.mma) wait with POLL_ABORT = false: leaving early
// because of another kernel's failure would let the CTA exit with its own
// transfers still landing; they read the abort word at entry only.
template <bool POLL_ABORT = true>
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *ab, int code) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        for (int it = 0; it < 256; ++it)
            if (mbar_try_wait(bar, parity)) return true;
        if (POLL_ABORT && aborted(ab)) return false;
        if (global_ns() - t0 > wait_limit_ns(ab)) break;
    }
    raise_abort(ab, code);
    return false;
}

// Address of the same shared-memory object in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_map_u32(const void *p, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}
// 16-byte store into (possibly another CTA's) shared memory that completes the
// given bytes on that CTA's mbarrier: the consumer waits on its own barrier,
// no cluster-wide barrier needed.
__device__ __forceinline__ void st_async_v4(uint32_t raddr, uint4 v, uint32_t rbar) {
    asm volatile(
        "st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(raddr),
        "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(rbar)
        : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tm, uint64_t *bar, int x,
                                            int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, "
        "%4}], [%2];" ::"r"(smem_u32(dst)),
        "l"((uint64_t)tm), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}
__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *tm) {
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)tm) : "memory");
}

// ---- host side ----
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// 2-D tensor map over a row-major matrix: `cols` contiguous elements per row,
// `rows` rows, `ld` elements between rows.  Box = box_cols x box_rows.
void make_tmap_2d(CUtensorMap *tm, CUtensorMapDataType dt, int esize, const void *base, i64 cols,
                  i64 rows, i64 ld, int box_cols, int box_rows, CUtensorMapSwizzle swz);

}  // namespace oxi
