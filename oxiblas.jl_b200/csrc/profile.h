// Launch counting and per-kernel-class timing (CUDA events on the launching
// stream), switched on per handle.  Entry points install the handle's profiler
// for the duration of the call (ProfGuard); launchers open a ProfScope.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

namespace oxi {

enum KernelClass {
    KC_LEAF = 0, KC_ROWMOVES, KC_TRSM_LEAF, KC_GEMM_REF, KC_GEMM_DMMA, KC_GEMM_TC, KC_CONVERT,
    KC_TRSV, KC_RESIDUAL, KC_OTHER, KC_COUNT
};

struct Profiler {
    bool enabled = false;
    uint64_t launches = 0;
    struct Rec {
        int kind;
        cudaEvent_t a, b;
        double flops, bytes;
        cudaStream_t s;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t take() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    void recycle() {
        for (auto &r : recs) { pool.push_back(r.a); pool.push_back(r.b); }
        recs.clear();
    }
    ~Profiler() {
        recycle();
        for (auto e : pool) cudaEventDestroy(e);
    }
};

extern thread_local Profiler *t_prof;

inline void count_launch() {
    if (t_prof) ++t_prof->launches;
}

struct ProfScope {
    Profiler *p;
    cudaStream_t s;
    size_t idx = 0;
    ProfScope(int kind, cudaStream_t st, double flops, double bytes) : p(t_prof), s(st) {
        if (!p || !p->enabled) { p = nullptr; return; }
        Profiler::Rec r{kind, p->take(), p->take(), flops, bytes, st};
        cudaEventRecord(r.a, s);
        idx = p->recs.size();
        p->recs.push_back(r);
    }
    ~ProfScope() {
        if (p) cudaEventRecord(p->recs[idx].b, s);
    }
};

struct ProfGuard {
    Profiler *saved;
    explicit ProfGuard(Profiler *p) : saved(t_prof) { t_prof = p; }
    ~ProfGuard() { t_prof = saved; }
};

}  // namespace oxi
