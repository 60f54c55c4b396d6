// Handle life cycle, options, status strings and the standalone GEMM entry point.
#include <cstring>
#include "oxi_internal.h"

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
        oxi::gemm_minus<double>(h, dC, ldc, dB, ldb, dA, lda, n, m, k);
        OXI_CUDA(cudaStreamSynchronize(h->stream));
        return OXI_OK;
    } catch (const oxi::CudaError &e) {
        h->last_error = std::string(e.what) + ": " + cudaGetErrorString(e.code);
        return OXI_ECUDA;
    }
}

}  // extern "C"
