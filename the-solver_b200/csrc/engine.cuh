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
#include <cuda_bf16.h>

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

constexpr int kThreads = 256;          // threads per block (8 warps)
constexpr int kWarps = kThreads / 32;
constexpr int kChunkNnz = 256;         // nonzeros per warp chunk (8 per lane)
constexpr int kChunkRows = 32;         // rows per warp chunk (one owning lane each)
constexpr int kPerLane = kChunkNnz / 32;
constexpr int kShortRow = 32;          // rows up to this length: owning lane, sequential sum

// Warp chunks: consecutive rows with at most kChunkNnz nonzeros and at most
// kChunkRows rows; a row longer than kChunkNnz is a chunk of its own. Returns
// the chunk boundaries as (row, first nonzero) pairs, ntiles + 1 of them.
std::vector<int> build_tiles(int rows, const int* row_offsets);
// Stable transpose of a device CSR (rows x cols, nnz): tptr[cols + 1], tidx and
// tval receive A^T with each of its rows in ascending source-row order. Device
// work on `stream`; returns 0 or -1 (an index outside [0, cols) is an error).
int device_transpose(int rows, int cols, int nnz, const int* ptr, const int* idx, const double* val, int* tptr,
                     int* tidx, double* tval, cudaStream_t stream);

// A CSR with its warp-chunk schedule; T is the value type (double, or float
// for the FP32 inner iterations of the refined PDLP).
template <class T>
struct TileCsrT {
    int rows = 0, cols = 0, nnz = 0, ntiles = 0;
    const int* ptr = nullptr;
    const int* idx = nullptr;
    const T* val = nullptr;
    const int2* tile = nullptr;   // chunk boundaries: (first row, first nonzero)

    template <class U>
    TileCsrT<U> with_values(const U* v) const {
        TileCsrT<U> o;
        o.rows = rows; o.cols = cols; o.nnz = nnz; o.ntiles = ntiles;
        o.ptr = ptr; o.idx = idx; o.val = v; o.tile = tile;
        return o;
    }
};
using TileCsr = TileCsrT<double>;

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
    int* d_a_idx = nullptr;         // owned copies of A when the caller's arrays are not
    double* d_a_val = nullptr;      // 16-byte aligned (the bulk L2 prefetch of a chunk needs it)
    const void* src_idx = nullptr;  // the handle's device_column_indices / device_values at
    const void* src_val = nullptr;  // planning time: a handle pointing elsewhere is another matrix
    double row_mass_max = 0.0;   // filled lazily by users that need it
    std::mutex workspace_mutex;   // held by the solve that uses `solve_cache`
    std::shared_ptr<void> solve_cache; // workspace + captured graphs of the last fixed-step solve
    ~Plan();
};

// Builds A^T and both tile schedules from host CSR arrays (host-side counting
// sort, O(nnz)). d_ptr/d_idx/d_val are the device copies of the same CSR.
int make_plan(const SankhyaCudaCSR* m, const int* h_ptr, const int* h_idx, const double* h_val,
              std::shared_ptr<Plan>* out);

// Registered plan of a handle made by sankhya_cuda_csr_create, else a plan
// built now from the handle's device arrays (copied back to the host once).
// Fails (-1) when the plan lives on another device than the current one: its
// arrays are that device's memory.
int get_plan(const SankhyaCudaCSR* m, std::shared_ptr<Plan>* out);
// Registered plan only (never builds one, never allocates): -1 with a message
// when the handle has none, points at other arrays than the planned ones, or the
// plan lives on another device than the current one.
int find_plan(const SankhyaCudaCSR* m, std::shared_ptr<Plan>* out);
void register_plan(const void* key, std::shared_ptr<Plan> plan);
void unregister_plan(const void* key);

// ------------------------------------------------------------- streams/timing

cudaStream_t engine_stream();   // one non-blocking stream per host thread and device
int grid_for(const void* kernel, int ntiles, int dynamic_smem = 0);

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
__device__ __forceinline__ float dadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float dmul(float a, float b) { return __fmul_rn(a, b); }

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

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// --------------------------------------------------- fused tiled SpMV kernel
//
// Warp-granular: every warp of a persistent grid walks warp chunks
// gw, gw + total_warps, ... independently (no block-wide barrier on the path).
// For a chunk of rows [r0, r1) and nonzeros [p0, p1):
//   0. lane 0 asks the TMA unit to pull the warp's NEXT chunk of values and
//      column indices into L2 (cp.async.bulk.prefetch.L2, no shared memory, no
//      completion to wait for), so that chunk's loads below hit L2, not HBM;
//   1. lane l owns row r0 + l and prefetches that row's epilogue data
//      (Epi::load: y, bounds, steps, ...) into registers;
//   2. lane l loads values and column indices p0 + l + 32 k (k < 8, coalesced,
//      evict-first) and issues its 8 gathers v[idx] back to back (the vectors
//      stay L2-resident);
//   3. products go to the warp's 2 KB shared-memory slice; rows of at most
//      kShortRow entries are summed by their owning lane sequentially in stored
//      order from 0.0 (the exact rounding of a serial CPU loop), longer rows by
//      the whole warp (lane-strided partials, xor tree);
//   4. Epi::store / Epi::row finishes the PDHG step for the row.
// A row longer than kChunkNnz is a chunk of its own, streamed by the warp.
// Reducing epilogues keep per-thread accumulators; Epi::finish combines them
// per block in a fixed order.

struct Empty {};

template <class E, class = void>
struct HasLoad {
    static constexpr bool value = false;
};
template <class E>
struct HasLoad<E, decltype(void(&E::load))> {
    static constexpr bool value = true;
};

template <class Epi, bool = HasLoad<Epi>::value>
struct RowPre {
    using type = Empty;
    static __device__ __forceinline__ type load(const Epi&, int) { return {}; }
    template <class T>
    static __device__ __forceinline__ void apply(const Epi& e, int r, T s, const type&, typename Epi::Acc& acc) {
        e.row(r, s, acc);
    }
};
template <class Epi>
struct RowPre<Epi, true> {
    using type = typename Epi::Row;
    static __device__ __forceinline__ type load(const Epi& e, int r) { return e.load(r); }
    template <class T>
    static __device__ __forceinline__ void apply(const Epi& e, int r, T s, const type& pre, typename Epi::Acc& acc) {
        e.store(r, s, pre, acc);
    }
};

// Bulk L2 prefetch of [first, last) elements of a 16-byte-aligned array; the
// range is shrunk to its 16-byte-aligned interior so it never leaves the array.
template <class T>
__device__ __forceinline__ void prefetch_l2(const T* base, int first, int last) {
    constexpr int per = 16 / static_cast<int>(sizeof(T));
    const int a = (first + per - 1) / per * per, b = last / per * per;
    if (b > a)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(base + a),
                     "r"(static_cast<unsigned>((b - a) * static_cast<int>(sizeof(T))))
                     : "memory");
}

// A stored matrix value as the arithmetic type T (the identity unless the values
// are kept narrower than the vectors, e.g. bf16 values with fp32 vectors).
template <class T, class V>
__device__ __forceinline__ T load_value(const V* p) {
    return static_cast<T>(__ldcs(p));
}
template <>
__device__ __forceinline__ float load_value<float, __nv_bfloat16>(const __nv_bfloat16* p) {
    return __bfloat162float(__ldcs(p));
}

template <class Epi, class T, class V = T>
__global__ void __launch_bounds__(kThreads) k_tiled(TileCsrT<V> A, const T* __restrict__ v, Epi epi) {
    using P = RowPre<Epi>;
    __shared__ T prod[kWarps][kChunkNnz];
    __shared__ double red[kWarps * 8];
    typename Epi::Acc acc;
    acc.init();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = gridDim.x * kWarps;
    T* sp = prod[warp];
    const unsigned full = 0xffffffffu;
    int t = blockIdx.x * kWarps + warp;
    int2 b0 = t < A.ntiles ? __ldg(A.tile + t) : make_int2(0, 0);
    int2 b1 = t < A.ntiles ? __ldg(A.tile + t + 1) : make_int2(0, 0);
    for (; t < A.ntiles; t += nw) {
        const int r0 = b0.x, r1 = b1.x, p0 = b0.y, p1 = b1.y;
        const int tn = t + nw;
        int2 n0 = b1, n1 = b1;
        if (tn < A.ntiles) {
            n0 = __ldg(A.tile + tn);
            n1 = __ldg(A.tile + tn + 1);
            if (lane == 0 && n1.y - n0.y <= kChunkNnz) {
                prefetch_l2(A.val, n0.y, n1.y);
                prefetch_l2(A.idx, n0.y, n1.y);
            }
        }
        const int my = r0 + lane;
        const bool owns = my < r1;
        typename P::type pre{};
        int q0 = 0, q1 = 0;
        if (owns) {
            pre = P::load(epi, my);
            q0 = __ldg(A.ptr + my) - p0;
            q1 = __ldg(A.ptr + my + 1) - p0;
        }
        if (p1 - p0 > kChunkNnz) {
            T s0 = T(0), s1 = T(0);
            int p = p0 + lane;
            for (; p + 32 < p1; p += 64) {
                s0 += load_value<T>(A.val + p) * __ldg(v + __ldcs(A.idx + p));
                s1 += load_value<T>(A.val + p + 32) * __ldg(v + __ldcs(A.idx + p + 32));
            }
            if (p < p1) s0 += load_value<T>(A.val + p) * __ldg(v + __ldcs(A.idx + p));
            const T s = warp_sum(s0 + s1);
            if (lane == 0) P::apply(epi, r0, s, pre, acc);
            b0 = n0;
            b1 = n1;
            continue;
        }
        int col[kPerLane];
        T a[kPerLane];
#pragma unroll
        for (int k = 0; k < kPerLane; ++k) {
            const int p = p0 + 32 * k + lane;
            col[k] = 0;
            a[k] = T(0);
            if (p < p1) {
                col[k] = __ldcs(A.idx + p);
                a[k] = load_value<T>(A.val + p);
            }
        }
#pragma unroll
        for (int k = 0; k < kPerLane; ++k)
            if (p0 + 32 * k + lane < p1) a[k] = dmul(a[k], __ldg(v + col[k]));
#pragma unroll
        for (int k = 0; k < kPerLane; ++k)
            if (p0 + 32 * k + lane < p1) sp[32 * k + lane] = a[k];
        __syncwarp();
        const int len = q1 - q0;
        if (owns && len <= kShortRow) {
            T s = T(0);
            for (int q = q0; q < q1; ++q) s = dadd(s, sp[q]);
            P::apply(epi, my, s, pre, acc);
        }
        unsigned long_rows = __ballot_sync(full, owns && len > kShortRow);
        while (long_rows) {
            const int l = __ffs(long_rows) - 1;
            long_rows &= long_rows - 1;
            const int lq0 = __shfl_sync(full, q0, l), lq1 = __shfl_sync(full, q1, l);
            T s = T(0);
            for (int q = lq0 + lane; q < lq1; q += 32) s += sp[q];
            s = warp_sum(s);
            if (lane == l) P::apply(epi, my, s, pre, acc);
        }
        __syncwarp();
        b0 = n0;
        b1 = n1;
    }
    epi.finish(acc, red);
}

// Plain product y = A v.
template <class T = double>
struct StoreEpiT {
    T* y;
    using Acc = NoAcc;
    __device__ __forceinline__ void row(int r, T s, NoAcc&) const { y[r] = s; }
    __device__ __forceinline__ void finish(NoAcc&, double*) const {}
};
using StoreEpi = StoreEpiT<double>;

template <class Epi, class T = double, class V = T>
inline int tiled_grid(const TileCsrT<V>& A) {
    const void* k = reinterpret_cast<const void*>(&k_tiled<Epi, T, V>);
    return grid_for(k, (A.ntiles + kWarps - 1) / kWarps, 0);
}

template <class Epi, class T, class V>
inline int launch_tiled(const TileCsrT<V>& A, const T* v, const Epi& epi, cudaStream_t stream, int grid) {
    if (A.ntiles == 0) return 0;
    k_tiled<Epi, T, V><<<grid, kThreads, 0, stream>>>(A, v, epi);
    return 0;
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
