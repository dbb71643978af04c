// Per-kernel-class device timing with CUDA events on the context stream.
// Off by default; when on, every launch wrapper call is bracketed by an event
// pair and amr_profile_collect() turns the pairs into milliseconds.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "amr_internal.h"

namespace amr {

enum KernelClass {
    KC_GHOST = 0, KC_FLUX, KC_REFLUX, KC_ADD_DIFS, KC_INJECT, KC_MAX_DT, KC_REFINE, KC_PROLONG,
    KC_RELAX, KC_VDOWN, KC_PHI_BOUND, KC_DPHI_BOUND, KC_FORCES, KC_ERROR, KC_SOURCE, KC_PHYS_BOUND,
    KC_CORRECT, KC_PHI_TIME, KC_OTHER, KC_FUSED, KC_COUNT
};

struct Profiler {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    struct Pending {
        int cls;
        cudaEvent_t a, b;
        long long units;
    };
    std::vector<Pending> pending;
    double ms[KC_COUNT] = {};
    long long launches[KC_COUNT] = {};
    long long units[KC_COUNT] = {};  // bricks (or items) processed
    long long kernels = 0;           // kernels launched, counted whether or not timing is on
    cudaEvent_t take() {
        if (pool.empty()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            return e;
        }
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    void begin(int cls, cudaStream_t s, cudaEvent_t* a) {
        (void)cls;
        *a = nullptr;
        if (!on) return;
        *a = take();
        cudaEventRecord(*a, s);
    }
    void end(int cls, cudaStream_t s, cudaEvent_t a, long long n) {
        if (!on || !a) return;
        cudaEvent_t b = take();
        cudaEventRecord(b, s);
        pending.push_back({cls, a, b, n});
    }
    void collect() {
        for (auto& p : pending) {
            float t = 0.0f;
            if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) {
                ms[p.cls] += t;
                launches[p.cls]++;
                units[p.cls] += p.units;
            }
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    void reset() {
        collect();
        for (int i = 0; i < KC_COUNT; i++) {
            ms[i] = 0.0;
            launches[i] = 0;
            units[i] = 0;
        }
    }
    ~Profiler() {
        for (auto& p : pending) {
            cudaEventDestroy(p.a);
            cudaEventDestroy(p.b);
        }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

// RAII bracket for one launch wrapper call
struct ProfScope {
    Profiler& p;
    int cls;
    cudaStream_t s;
    cudaEvent_t a;
    long long n;
    long long tally0;  // launch tally when the bracket opened
    ProfScope(Profiler& p_, int cls_, cudaStream_t s_, long long n_ = 0)
        : p(p_), cls(cls_), s(s_), n(n_), tally0(g_launch_tally) {
        p.begin(cls, s, &a);
    }
    ~ProfScope() {
        p.kernels += g_launch_tally - tally0;
        p.end(cls, s, a, n);
    }
};

}  // namespace amr
