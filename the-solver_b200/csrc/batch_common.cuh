// Pieces shared by the two batched PDHG drivers (block-diagonal and shared-matrix):
// the 1e30 sentinel tests of sk_solve, an order-independent max of non-negative
// doubles for the per-LP gates, and the column / row masses that define the
// diagonal steps of sk_solve's first-order loop (c/src/sk_solve.c:868-880).
#pragma once

#include "engine.cuh"

#include <chrono>

namespace b200 {
namespace batch {

__device__ __forceinline__ bool sk_inf(double v) { return v >= 1.0e30; }
__device__ __forceinline__ bool sk_neg_inf(double v) { return v <= -1.0e30; }

// max of non-negative doubles through their bit patterns (order-independent)
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* slot, double v) {
    if (!(v > 0.0)) {
        if (isnan(v)) atomicMax(slot, 0x7ff8000000000000ull);
        return;
    }
    atomicMax(slot, static_cast<unsigned long long>(__double_as_longlong(v)));
}

__device__ __forceinline__ double slot_value(unsigned long long b) {
    return __longlong_as_double(static_cast<long long>(b));
}

// Sequential |a| sums per CSR row in stored order (the reference's order).
static __global__ void k_abs_sums(int rows, const int* __restrict__ ptr, const double* __restrict__ val,
                                  double* __restrict__ out) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += blockDim.x * gridDim.x) {
        double s = 0.0;
        for (int p = ptr[r]; p < ptr[r + 1]; ++p) s += fabs(val[p]);
        out[r] = s;
    }
}

// CUDA events around the iteration loop of a batched solve (timing level >= 1):
// the device time from the first window to the last check, idle gaps included.
struct LoopEvents {
    cudaEvent_t a = nullptr, b = nullptr;
    bool on = false;
    LoopEvents(bool enabled, cudaStream_t s) : on(enabled) {
        if (on && (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess ||
                   cudaEventRecord(a, s) != cudaSuccess))
            on = false;
    }
    double stop(cudaStream_t s) {
        float ms = 0.f;
        if (on && cudaEventRecord(b, s) == cudaSuccess && cudaEventSynchronize(b) == cudaSuccess)
            cudaEventElapsedTime(&ms, a, b);
        on = false;
        return ms;
    }
    ~LoopEvents() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

inline double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace batch
}  // namespace b200
