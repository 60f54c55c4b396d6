// Handle life cycle, options, status strings, instrumentation and the
// standalone GEMM entry points.
#include <cstring>
#include <mutex>
#include <set>
#include <tuple>
#include <vector>
#include "oxi_internal.h"
#include "tma_util.cuh"

namespace oxi {
thread_local Profiler *t_prof = nullptr;

thread_local int *t_abort = nullptr;

int *abort_word(oxi_handle_s *h) {
    return (int *)((char *)h->scratch.get(kScratchBytes) + kScratchErrOff);
}

AbortScope::AbortScope(oxi_handle_s *h) : saved(t_abort), word(abort_word(h)) {
    if (h->wait_limit_dev != h->wait_limit_ns) {
        // first call of the handle, or the option changed: a blocking copy
        const uint64_t v = (uint64_t)h->wait_limit_ns;
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        OXI_CUDA(cudaMemcpy(word + 2, &v, sizeof(v), cudaMemcpyHostToDevice));
        h->wait_limit_dev = h->wait_limit_ns;
    }
    OXI_CUDA(cudaMemsetAsync(word, 0, 2 * sizeof(int), h->stream));
    t_abort = word;  // only once nothing above can throw
}

void queue_abort_read(oxi_handle_s *h, int *hdst) {
    OXI_CUDA(cudaMemcpyAsync(hdst, abort_word(h), sizeof(int), cudaMemcpyDeviceToHost, h->stream));
}

int check_abort(oxi_handle_s *h, const int *hsrc) {
    if (*hsrc == 0) return OXI_OK;
    static const char *what[] = {"", "leaf pivot exchange", "FP64 tensor-core GEMM pipeline",
                                 "triangular-solve chain", "low-precision conversion",
                                 "tensor-core GEMM pipeline", "missing producer (test hook)"};
    const int c = *hsrc;
    h->last_error = std::string("a bounded device wait timed out (") +
                    ((c > 0 && c < 7) ? what[c] : "unknown") + "); the call's results are void";
    return OXI_ETIMEOUT;
}

// One thread polls a flag nobody writes, with the call's bounded wait.
__global__ void k_await_missing_producer(const int *__restrict__ flag, int *__restrict__ ab) {
    if (aborted(ab)) return;
    const uint64_t t0 = global_ns();
    uint32_t it = 0;
    while (*(const volatile int *)flag == 0)
        if (spin_give_up<64>(it, t0, ab, 6)) return;
}

void launch_await_missing_producer(oxi_handle_s *h, cudaStream_t s) {
    int *flag = (int *)((char *)h->scratch.get(kScratchBytes) + kScratchStallOff);
    OXI_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));  // the flag starts clear; nothing sets it
    k_await_missing_producer<<<1, 1, 0, s>>>(flag, cur_abort());
    OXI_LAUNCH_CHECK();
}

void maybe_stall_before_leaf(oxi_handle_s *h, cudaStream_t s) {
    if (h->stall_at <= 0) return;
    if (--h->stall_at == 0) launch_await_missing_producer(h, s);
}

void set_max_dyn_smem(const void *func, int bytes) {
    static std::mutex mu;
    static std::set<std::tuple<const void *, int, int>> done;
    int dev = 0;
    OXI_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (done.count(std::make_tuple(func, dev, bytes))) return;
    OXI_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    done.insert(std::make_tuple(func, dev, bytes));
}
}

extern "C" {

int oxi_create(oxi_handle_t *out) {
    if (!out) return OXI_EINVAL;
    *out = nullptr;
    oxi_handle_s *h = new (std::nothrow) oxi_handle_s();
    if (!h) return OXI_ENOMEM;
    if (cudaGetDevice(&h->device) != cudaSuccess) {
        delete h;
        return OXI_ECUDA;
    }
    cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device);
    *out = h;
    return OXI_OK;
}

int oxi_destroy(oxi_handle_t h) {
    if (!h) return OXI_EINVAL;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    else cudaDeviceSynchronize();
    h->work.release();
    h->scratch.release();
    h->solve_ws.release();
    h->mixed_ws.release();
    h->perm_ws.release();
    h->tc_ws.release();
    h->tc_ws2.release();
    h->xtag_ws.release();
    h->rowmap_ws.release();
    h->tslu_ws.release();
    h->gcache.reset();
    h->bgraph.reset();
    h->batch_ctl.release();
    h->batch_wsp.release();
    if (h->aux_stream) cudaStreamDestroy(h->aux_stream);
    if (h->la_stream) cudaStreamDestroy(h->la_stream);
    if (h->la_main) cudaStreamDestroy(h->la_main);
    if (h->la_in) cudaEventDestroy(h->la_in);
    if (h->la_out) cudaEventDestroy(h->la_out);
    if (h->la_fork) cudaEventDestroy(h->la_fork);
    if (h->la_join) cudaEventDestroy(h->la_join);
    if (h->aux_fork) cudaEventDestroy(h->aux_fork);
    if (h->aux_join) cudaEventDestroy(h->aux_join);
    h->host_ws.release();
    delete h;
    return OXI_OK;
}

int oxi_set_stream(oxi_handle_t h, void *stream) {
    if (!h) return OXI_EINVAL;
    h->stream = (cudaStream_t)stream;
    return OXI_OK;
}

const char *oxi_status_string(int s) {
    switch (s) {
        case OXI_OK: return "ok";
        case OXI_EINVAL: return "invalid argument";
        case OXI_ESINGULAR: return "singular matrix (zero pivot)";
        case OXI_ENONFINITE: return "non-finite input";
        case OXI_EOVERFLOW: return "overflow in low-precision conversion";
        case OXI_ECUDA: return "CUDA error";
        case OXI_ETIMEOUT: return "device wait timed out";
        case OXI_ENOMEM: return "out of memory";
        case OXI_ENOTCONVERGED: return "refinement did not converge";
        case OXI_ENOTPOSDEF: return "matrix is not positive definite";
        case OXI_ESCRATCH:
            return "size exceeds the fixed scratch of oxi_dgetrs_noalloc "
                   "(n <= 65536 and n * nrhs <= 917504)";
        default: return "unknown status";
    }
}

const char *oxi_last_error(oxi_handle_t h) { return h ? h->last_error.c_str() : ""; }

int oxi_set_option(oxi_handle_t h, int option, int64_t value) {
    if (!h) return OXI_EINVAL;
    switch (option) {
        case OXI_OPT_BLOCKSIZE:
            if (value < 1) return OXI_EINVAL;  // "blocksize must be positive"
            h->opt.blocksize = value;
            return OXI_OK;
        case OXI_OPT_GEMM:
            if (value != 0 && value != 1) return OXI_EINVAL;
            h->opt.gemm = (int)value;
            return OXI_OK;
        case OXI_OPT_TRSM_LEAF:
            if (value < 1 || value > 32) return OXI_EINVAL;
            h->opt.trsm_leaf = value;
            return OXI_OK;
        case OXI_OPT_LOOKAHEAD:
            h->opt.lookahead = value ? 1 : 0;
            h->gcache.reset();
            return OXI_OK;
        case OXI_OPT_MIXED_BLOCKSIZE:
            if (value < 1) return OXI_EINVAL;
            h->opt.mixed_blocksize = value;
            return OXI_OK;
        case OXI_OPT_STOP_NORMWISE:
            h->opt.stop_normwise = value ? 1 : 0;
            return OXI_OK;
        case OXI_OPT_GMRES_RESTART:
            if (value < 2 || value > 62) return OXI_EINVAL;
            h->opt.gmres_restart = (int)value;
            return OXI_OK;
        case OXI_OPT_GRAPHS:
            h->opt.graphs = value ? 1 : 0;
            if (!value) {
                h->gcache.reset();
                h->bgraph.reset();
            }
            return OXI_OK;
        case OXI_OPT_TOURNAMENT:
            h->opt.tournament = value ? 1 : 0;
            return OXI_OK;
        case OXI_OPT_WAIT_LIMIT_US:
            if (value < 1000 || value > 60000000) return OXI_EINVAL;  // 1 ms .. 60 s
            h->wait_limit_ns = value * 1000;
            return OXI_OK;
        case OXI_OPT_TEST_MISSING_PRODUCER:
            if (value < 0) return OXI_EINVAL;
            h->stall_at = value;
            if (value) h->gcache.reset();
            return OXI_OK;
        default: return OXI_EINVAL;
    }
}

int oxi_get_option(oxi_handle_t h, int option, int64_t *value) {
    if (!h || !value) return OXI_EINVAL;
    switch (option) {
        case OXI_OPT_BLOCKSIZE: *value = h->opt.blocksize; return OXI_OK;
        case OXI_OPT_GEMM: *value = h->opt.gemm; return OXI_OK;
        case OXI_OPT_TRSM_LEAF: *value = h->opt.trsm_leaf; return OXI_OK;
        case OXI_OPT_LOOKAHEAD: *value = h->opt.lookahead; return OXI_OK;
        case OXI_OPT_MIXED_BLOCKSIZE: *value = h->opt.mixed_blocksize; return OXI_OK;
        case OXI_OPT_STOP_NORMWISE: *value = h->opt.stop_normwise; return OXI_OK;
        case OXI_OPT_GMRES_RESTART: *value = h->opt.gmres_restart; return OXI_OK;
        case OXI_OPT_GRAPHS: *value = h->opt.graphs; return OXI_OK;
        case OXI_OPT_TOURNAMENT: *value = h->opt.tournament; return OXI_OK;
        case OXI_OPT_WAIT_LIMIT_US:
            *value = (h->wait_limit_ns ? h->wait_limit_ns : (int64_t)oxi::kWaitLimitNs) / 1000;
            return OXI_OK;
        case OXI_OPT_TEST_MISSING_PRODUCER: *value = h->stall_at; return OXI_OK;
        default: return OXI_EINVAL;
    }
}

// Column-major C -= A*B is the row-major C^T -= B^T A^T: the row-major kernels
// run on the same memory with the operands swapped.
int oxi_dgemm_update(oxi_handle_t h, int64_t m, int64_t n, int64_t k, double *dC, int64_t ldc,
                     const double *dA, int64_t lda, const double *dB, int64_t ldb) {
    if (!h || m < 0 || n < 0 || k < 0) return OXI_EINVAL;
    if (m == 0 || n == 0 || k == 0) return OXI_OK;
    if (!dC || !dA || !dB || ldc < m || lda < m || ldb < k) return OXI_EINVAL;
    try {
        oxi::ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        oxi::AbortScope ab(h);
        oxi::gemm_minus<double>(h, dC, ldc, dB, ldb, dA, lda, n, m, k);
        int *he = (int *)h->host_ws.get(64);
        oxi::queue_abort_read(h, he);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        return oxi::check_abort(h, he);
    } catch (const oxi::CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

int oxi_sgemm_update_lowp(oxi_handle_t h, int prec, int64_t m, int64_t n, int64_t k, float *dC,
                          int64_t ldc, const float *dA, int64_t lda, const float *dB, int64_t ldb) {
    if (!h || m < 0 || n < 0 || k < 0) return OXI_EINVAL;
    if (prec != OXI_PREC_FP32 && prec != OXI_PREC_BF16 && prec != OXI_PREC_FP16 && prec != OXI_PREC_BF16X3 &&
        prec != OXI_PREC_FP16X3)
        return OXI_EINVAL;
    if (m == 0 || n == 0 || k == 0) return OXI_OK;
    if (!dC || !dA || !dB || ldc < m || lda < m || ldb < k) return OXI_EINVAL;
    const int saved = h->trailing;
    try {
        oxi::ProfGuard pg(&h->prof);
        OXI_CUDA(cudaSetDevice(h->device));
        oxi::AbortScope ab(h);
        h->trailing = prec;  // OXI_PREC_{FP32,BF16,FP16,BF16X3,FP16X3} == TRAIL_{NATIVE,...,FP16X3}
        if (prec == OXI_PREC_FP32)
            oxi::gemm_minus<float>(h, dC, ldc, dB, ldb, dA, lda, n, m, k);
        else
            oxi::gemm_trailing_f32(h, dC, ldc, dB, ldb, dA, lda, n, m, k);
        h->trailing = saved;
        int *he = (int *)h->host_ws.get(64);
        oxi::queue_abort_read(h, he);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        return oxi::check_abort(h, he);
    } catch (const oxi::CudaError &e) {
        h->trailing = saved;
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

int oxi_profile_enable(oxi_handle_t h, int on) {
    if (!h) return OXI_EINVAL;
    h->gcache.reset();  // profiled launches are recorded individually
    h->bgraph.reset();
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    h->prof.recycle();
    h->prof.enabled = on != 0;
    return OXI_OK;
}

int oxi_profile_read(oxi_handle_t h, int kind, int64_t *launches, double *total_ms, double *flops,
                     double *bytes) {
    if (!h || kind < 0 || kind >= oxi::KC_COUNT) return OXI_EINVAL;
    cudaSetDevice(h->device);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return OXI_ECUDA;
    int64_t cnt = 0;
    double ms = 0, fl = 0, by = 0;
    for (auto &r : h->prof.recs) {
        if (r.kind != kind) continue;
        float t = 0;
        if (cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess) continue;
        ++cnt;
        ms += t;
        fl += r.flops;
        by += r.bytes;
    }
    if (launches) *launches = cnt;
    if (total_ms) *total_ms = ms;
    if (flops) *flops = fl;
    if (bytes) *bytes = by;
    return OXI_OK;
}

int oxi_profile_timeline(oxi_handle_t h, int64_t max, double *out, int64_t *count) {
    if (!h || !count || (max > 0 && !out)) return OXI_EINVAL;
    cudaSetDevice(h->device);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return OXI_ECUDA;
    std::vector<cudaStream_t> seen;
    int64_t k = 0;
    const auto &recs = h->prof.recs;
    for (size_t i = 0; i < recs.size(); ++i) {
        if (k >= max) { ++k; continue; }
        float t0 = 0, t1 = 0;
        if (cudaEventElapsedTime(&t0, recs[0].a, recs[i].a) != cudaSuccess ||
            cudaEventElapsedTime(&t1, recs[0].a, recs[i].b) != cudaSuccess)
            return OXI_ECUDA;
        size_t sid = 0;
        while (sid < seen.size() && seen[sid] != recs[i].s) ++sid;
        if (sid == seen.size()) seen.push_back(recs[i].s);
        out[4 * k] = recs[i].kind;
        out[4 * k + 1] = (double)sid;
        out[4 * k + 2] = t0;
        out[4 * k + 3] = t1;
        ++k;
    }
    *count = k;
    return OXI_OK;
}

int oxi_launch_count(oxi_handle_t h, int64_t *count) {
    if (!h || !count) return OXI_EINVAL;
    *count = (int64_t)h->prof.launches;
    return OXI_OK;
}

int oxi_launch_count_reset(oxi_handle_t h) {
    if (!h) return OXI_EINVAL;
    h->prof.launches = 0;
    return OXI_OK;
}

}  // extern "C"

// B (n x m, column-major, ldb) = A^T for the m x n column-major A (lda), with
// 4-, 8- or 16-byte elements: the column-major copy of a row-major host array
// (a row-major m x n array is the column-major n x m matrix A^T) that the other
// entry points take.  A tiled transpose at HBM speed, stream-ordered.
extern "C" int oxi_transpose(oxi_handle_t h, int elem_bytes, int64_t m, int64_t n, const void *dA, int64_t lda,
                             void *dB, int64_t ldb) {
    using namespace oxi;
    if (!h || m < 0 || n < 0 || lda < std::max<int64_t>(1, m) || ldb < std::max<int64_t>(1, n)) return OXI_EINVAL;
    if (elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16) return OXI_EINVAL;
    if (m == 0 || n == 0) return OXI_OK;
    if (!dA || !dB) return OXI_EINVAL;
    try {
        OXI_CUDA(cudaSetDevice(h->device));
        if (elem_bytes == 4)
            launch_cm_to_rm<float, float>((const float *)dA, lda, (float *)dB, ldb, m, n, h->stream);
        else if (elem_bytes == 8)
            launch_cm_to_rm<double, double>((const double *)dA, lda, (double *)dB, ldb, m, n, h->stream);
        else
            launch_cm_to_rm<double2, double2>((const double2 *)dA, lda, (double2 *)dB, ldb, m, n, h->stream);
        return OXI_OK;
    } catch (const CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}
