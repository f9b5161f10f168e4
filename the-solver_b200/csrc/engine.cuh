// Internal declarations of the B200 PDHG engine (not installed).
//
// Device layout of a matrix ("plan"), shared by every solve that uses it:
//   A    : the caller's CSR (int32 offsets / int32 columns / f64 values) plus a
//          row-tile schedule tile_row[0..ntiles] (see build_tiles)
//   A^T  : a second CSR holding the transpose (rows of A^T = columns of A, the
//          row indices of A ascending inside each), with its own tile schedule
// Both products are gathers, so every sum has a fixed order and results are
// bit-reproducible run to run.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <memory>
#include <mutex>
#include <vector>

#include "sankhya_b200.h"
#include "sankhya_cuda.h"

namespace b200 {

// ------------------------------------------------------------------ errors

int fail_msg(const char* message);                 // sets last error, returns -1
int fail_cuda(const char* operation, cudaError_t); // sets last error, returns -1
void clear_error();

#define B200_TRY(expr, label)                                  \
    do {                                                       \
        cudaError_t b200_err_ = (expr);                        \
        if (b200_err_ != cudaSuccess) return fail_cuda(label, b200_err_); \
    } while (0)

// ----------------------------------------------------------- tile schedule

constexpr int kThreads = 256;          // threads per tile block
constexpr int kWarps = kThreads / 32;
constexpr int kTileNnz = 2048;         // nonzeros staged in shared memory per tile
constexpr int kShortRow = 32;          // rows up to this length: one thread, sequential sum
constexpr int kMaxTileRows = 4096;     // cap on rows per tile (keeps empty-row runs balanced)

// Greedy row tiles: consecutive rows whose nonzeros fit kTileNnz; a row longer
// than kTileNnz is a tile of its own and is reduced by the whole block.
std::vector<int> build_tiles(int rows, const int* row_offsets);

struct TileCsr {
    int rows = 0, cols = 0, nnz = 0, ntiles = 0;
    const int* ptr = nullptr;
    const int* idx = nullptr;
    const double* val = nullptr;
    const int* tile_row = nullptr;
};

// Owns everything a solve needs for one matrix beyond the caller's CSR.
struct Plan {
    int device = 0;
    TileCsr a;          // view of the caller's CSR + owned tiles
    TileCsr at;         // owned transpose + tiles
    int* d_tile_a = nullptr;
    int* d_at_ptr = nullptr;
    int* d_at_idx = nullptr;
    double* d_at_val = nullptr;
    int* d_tile_at = nullptr;
    double row_mass_max = 0.0;   // filled lazily by users that need it
    std::mutex workspace_mutex;  // serialises solves that share this plan's workspace
    std::vector<void*> workspace; // cached per-plan device buffers (freed with the plan)
    size_t workspace_bytes = 0;
    ~Plan();
};

// Builds A^T and both tile schedules from host CSR arrays (host-side counting
// sort, O(nnz)). d_ptr/d_idx/d_val are the device copies of the same CSR.
int make_plan(const SankhyaCudaCSR* m, const int* h_ptr, const int* h_idx, const double* h_val,
              std::shared_ptr<Plan>* out);

// Registered plan of a handle made by sankhya_cuda_csr_create, else a plan
// built now from the handle's device arrays (copied back to the host once).
int get_plan(const SankhyaCudaCSR* m, std::shared_ptr<Plan>* out);
void register_plan(const void* key, std::shared_ptr<Plan> plan);
void unregister_plan(const void* key);

// ------------------------------------------------------------- streams/timing

cudaStream_t engine_stream();   // one non-blocking stream per host thread and device
int grid_for(const void* kernel, int ntiles);

struct TimingState {
    int level = 0;
    SankhyaB200Timing last{};
};
TimingState& timing();

// ------------------------------------------------------- device arithmetic
// Explicit round-to-nearest intrinsics: no multiply-add contraction, so the
// elementwise updates round exactly like the reference's host C code.

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// cuda/src/sankhya_cuda_lp.cu:13-17: only IEEE infinities are absent bounds.
__device__ __forceinline__ double box_ieee(double v, double lo, double hi) {
    if (!isinf(lo) && v < lo) v = lo;
    if (!isinf(hi) && v > hi) v = hi;
    return v;
}
// c/src/sk_solve.c:18-24: the 1e30 sentinel (SK_INFINITY) marks absent bounds.
__device__ __forceinline__ double box_sk(double v, double lo, double hi) {
    if (!(lo <= -1.0e30) && v < lo) v = lo;
    if (!(hi >= 1.0e30) && v > hi) v = hi;
    return v;
}
__device__ __forceinline__ bool has_lower_gate(double v) { return isfinite(v) && v > -5.0e29; }
__device__ __forceinline__ bool has_upper_gate(double v) { return isfinite(v) && v < 5.0e29; }

// ------------------------------------------------------------- reductions

struct NoAcc {
    static constexpr int kSlots = 0;
    __device__ __forceinline__ void init() {}
};

// NS reduction slots; bit k of SumMask set = slot k is a sum, else a max.
template <int NS, unsigned SumMask>
struct Slots {
    static constexpr int kSlots = NS;
    double v[NS];
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int k = 0; k < NS; ++k) v[k] = 0.0;
    }
    __device__ __forceinline__ void max(int k, double x) { v[k] = fmax(v[k], x); }
    __device__ __forceinline__ void add(int k, double x) { v[k] += x; }
};

template <unsigned SumMask>
__device__ __forceinline__ double slot_op(int k, double a, double b) {
    return ((SumMask >> k) & 1u) ? a + b : fmax(a, b);
}

// Fixed-shape block reduction; thread 0's result lands in partial[blockIdx.x*NS+k].
template <int NS, unsigned SumMask>
__device__ void block_store(Slots<NS, SumMask>& acc, double* __restrict__ partial, double* smem) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        double v = acc.v[k];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            v = slot_op<SumMask>(k, v, __shfl_xor_sync(0xffffffffu, v, off));
        if (lane == 0) smem[warp * NS + k] = v;
    }
    __syncthreads();
    if (threadIdx.x < NS) {
        const int k = threadIdx.x;
        double r = smem[k];
        for (int w = 1; w < kWarps; ++w) r = slot_op<SumMask>(k, r, smem[w * NS + k]);
        partial[blockIdx.x * NS + k] = r;
    }
    __syncthreads();
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// --------------------------------------------------- fused tiled SpMV kernel
//
// One block walks tiles blockIdx.x, blockIdx.x + gridDim.x, ... For each tile
// it stages val[p] * v[idx[p]] for the tile's nonzeros in shared memory
// (coalesced val/idx streams, gathers of v from L2), then reduces rows:
//   rows of <= kShortRow entries: one thread, sequential sum from 0.0 in
//     stored order (the exact rounding of a serial CPU loop),
//   longer rows in a tile: one warp, lane-strided partials + xor tree,
//   a row longer than kTileNnz: the whole block, strided partials + fixed tree.
// Epi::row(r, sum, acc) consumes every row exactly once; Epi::finish reduces
// the per-thread accumulators of reducing epilogues.

template <class Epi>
__global__ void __launch_bounds__(kThreads) k_tiled(TileCsr A, const double* __restrict__ v, Epi epi) {
    __shared__ double prod[kTileNnz];
    __shared__ double red[kWarps * 8];
    typename Epi::Acc acc;
    acc.init();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
        const int r0 = A.tile_row[t], r1 = A.tile_row[t + 1];
        const int p0 = __ldg(A.ptr + r0), p1 = __ldg(A.ptr + r1);
        if (p1 - p0 > kTileNnz) {
            double s = 0.0;
            for (int p = p0 + tid; p < p1; p += kThreads)
                s += __ldcs(A.val + p) * __ldg(v + __ldcs(A.idx + p));
            s = warp_sum(s);
            if (lane == 0) red[warp] = s;
            __syncthreads();
            if (tid == 0) {
                double total = red[0];
                for (int w = 1; w < kWarps; ++w) total += red[w];
                epi.row(r0, total, acc);
            }
            __syncthreads();
            continue;
        }
#pragma unroll 4
        for (int p = p0 + tid; p < p1; p += kThreads)
            prod[p - p0] = dmul(__ldcs(A.val + p), __ldg(v + __ldcs(A.idx + p)));
        __syncthreads();
        for (int r = r0 + tid; r < r1; r += kThreads) {
            const int q0 = __ldg(A.ptr + r) - p0, q1 = __ldg(A.ptr + r + 1) - p0;
            if (q1 - q0 <= kShortRow) {
                double s = 0.0;
                for (int q = q0; q < q1; ++q) s = dadd(s, prod[q]);
                epi.row(r, s, acc);
            }
        }
        for (int r = r0 + warp; r < r1; r += kWarps) {
            const int q0 = __ldg(A.ptr + r) - p0, q1 = __ldg(A.ptr + r + 1) - p0;
            if (q1 - q0 > kShortRow) {
                double s = 0.0;
                for (int q = q0 + lane; q < q1; q += 32) s += prod[q];
                s = warp_sum(s);
                if (lane == 0) epi.row(r, s, acc);
            }
        }
        __syncthreads();
    }
    epi.finish(acc, red);
}

// Plain product y = A v.
struct StoreEpi {
    double* y;
    using Acc = NoAcc;
    __device__ __forceinline__ void row(int r, double s, NoAcc&) const { y[r] = s; }
    __device__ __forceinline__ void finish(NoAcc&, double*) const {}
};

template <class Epi>
inline int launch_tiled(const TileCsr& A, const double* v, const Epi& epi, cudaStream_t stream,
                        int grid) {
    if (A.ntiles == 0) return 0;
    k_tiled<Epi><<<grid, kThreads, 0, stream>>>(A, v, epi);
    return 0;
}

template <class Epi>
inline int tiled_grid(const TileCsr& A) {
    return grid_for(reinterpret_cast<const void*>(&k_tiled<Epi>), A.ntiles);
}

// Final fixed-order combine of per-block partials: out[k] = op_g partial[g*NS+k].
template <int NS, unsigned SumMask>
__global__ void k_combine(const double* __restrict__ partial, int nblocks, double* __restrict__ out) {
    __shared__ double smem[kThreads];
    for (int k = 0; k < NS; ++k) {
        double r = 0.0;
        for (int g = threadIdx.x; g < nblocks; g += kThreads) r = slot_op<SumMask>(k, r, partial[g * NS + k]);
        smem[threadIdx.x] = r;
        __syncthreads();
        for (int s = kThreads / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) smem[threadIdx.x] = slot_op<SumMask>(k, smem[threadIdx.x], smem[threadIdx.x + s]);
            __syncthreads();
        }
        if (threadIdx.x == 0) out[k] = smem[0];
        __syncthreads();
    }
}

// ------------------------------------------------------------- small kernels

__global__ void k_fill(double* __restrict__ out, double value, int n);
__global__ void k_copy(double* __restrict__ dst, const double* __restrict__ src, int n);

inline int elem_grid(int n) {
    int g = (n + kThreads - 1) / kThreads;
    return g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g);
}

// ---------------------------------------------------------- device buffers

// Simple owning device array (cudaMalloc / cudaFree).
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { if (p) cudaFree(p); }
    int alloc(size_t b, const char* what) {
        if (p) { cudaFree(p); p = nullptr; }
        bytes = b;
        if (b == 0) return 0;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) { p = nullptr; return fail_cuda(what, e); }
        return 0;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace b200
