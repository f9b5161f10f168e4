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

struct TileCsr {
    int rows = 0, cols = 0, nnz = 0, ntiles = 0;
    const int* ptr = nullptr;
    const int* idx = nullptr;
    const double* val = nullptr;
    const int2* tile = nullptr;   // chunk boundaries: (first row, first nonzero)
    unsigned int* err = nullptr;  // counts bounded device waits that gave up (may be null)
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
    unsigned int* d_err = nullptr;  // wait-timeout counter shared by this plan's launches
    int* d_a_idx = nullptr;         // owned copies of A when the caller's arrays are
    double* d_a_val = nullptr;      // not 16-byte aligned (TMA bulk copies need it)
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
int get_plan(const SankhyaCudaCSR* m, std::shared_ptr<Plan>* out);
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
// Warp-granular: every warp of a persistent grid walks warp chunks
// gw, gw + total_warps, ... independently (no block-wide barrier on the path).
// Each warp owns a double-buffered shared-memory slice. Lane 0 brings a chunk's
// values and column indices in with two 1-D TMA bulk copies (cp.async.bulk,
// completion counted on the slice's mbarrier), issued one chunk ahead, so the
// HBM latency of the matrix stream overlaps the work on the current chunk:
//   1. lane l owns row r0 + l and prefetches that row's epilogue data
//      (Epi::load: y, bounds, steps, ...);
//   2. lane l takes column indices p0 + l + 32 k (k < 8) from shared memory and
//      issues its gathers v[idx] back to back (the vectors stay L2-resident),
//      then overwrites each value slot with val[p] * v[idx[p]];
//   3. rows of at most kShortRow entries are summed by their owning lane
//      sequentially in stored order from 0.0 (the exact rounding of a serial
//      CPU loop), longer rows by the whole warp (lane-strided partials, xor tree);
//   4. Epi::store / Epi::row finishes the PDHG step for the row.
// A row longer than kChunkNnz is a chunk of its own, streamed from global memory
// by the warp. The copies cover the 16-byte-aligned interior of the chunk
// ([p0 rounded down, p1 rounded down) to 2 doubles / 4 ints); the at most 1 value
// and 3 indices past the last aligned boundary are read with plain loads, so no
// copy leaves the arrays. Waits are bounded: a wait that gives up counts in A.err
// and the warp stops after draining its copies. Reducing epilogues keep per-thread
// accumulators; Epi::finish combines them per block in a fixed order.

constexpr int kStageVal = kChunkNnz + 2;  // doubles per buffer
constexpr int kStageIdx = kChunkNnz + 4;  // ints per buffer
struct WarpStage {
    double val[2][kStageVal];
    int idx[2][kStageIdx];
    unsigned long long bar[2];
};
constexpr int kTiledSmem = kWarps * static_cast<int>(sizeof(WarpStage));
constexpr long long kWaitLimit = 1ll << 22;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    for (long long i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

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
    static __device__ __forceinline__ void apply(const Epi& e, int r, double s, const type&,
                                                 typename Epi::Acc& acc) {
        e.row(r, s, acc);
    }
};
template <class Epi>
struct RowPre<Epi, true> {
    using type = typename Epi::Row;
    static __device__ __forceinline__ type load(const Epi& e, int r) { return e.load(r); }
    static __device__ __forceinline__ void apply(const Epi& e, int r, double s, const type& pre,
                                                 typename Epi::Acc& acc) {
        e.store(r, s, pre, acc);
    }
};

struct Chunk {
    int r0, r1, p0, p1, a0v, a1v, a0i, a1i;
    __device__ __forceinline__ bool streamed() const { return p1 - p0 > kChunkNnz; }
};

__device__ __forceinline__ Chunk chunk_at(const TileCsr& A, int t) {
    const int2 b0 = __ldg(A.tile + t), b1 = __ldg(A.tile + t + 1);
    Chunk c;
    c.r0 = b0.x;
    c.r1 = b1.x;
    c.p0 = b0.y;
    c.p1 = b1.y;
    c.a0v = c.p0 & ~1;
    c.a1v = max(c.a0v, c.p1 & ~1);
    c.a0i = c.p0 & ~3;
    c.a1i = max(c.a0i, c.p1 & ~3);
    return c;
}

// Lane 0: both bulk copies of a staged chunk into buffer b of the warp's slice.
__device__ __forceinline__ void issue_chunk(const TileCsr& A, const Chunk& c, WarpStage& ws, int b) {
    const unsigned vb = static_cast<unsigned>(c.a1v - c.a0v) * 8u;
    const unsigned ib = static_cast<unsigned>(c.a1i - c.a0i) * 4u;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_arrive_expect(&ws.bar[b], vb + ib);
    if (vb) bulk_load(ws.val[b], A.val + c.a0v, vb, &ws.bar[b]);
    if (ib) bulk_load(ws.idx[b], A.idx + c.a0i, ib, &ws.bar[b]);
}

template <class Epi>
__global__ void __launch_bounds__(kThreads, 4) k_tiled(TileCsr A, const double* __restrict__ v, Epi epi) {
    using P = RowPre<Epi>;
    extern __shared__ __align__(16) unsigned char dyn[];
    __shared__ double red[kWarps * 8];
    typename Epi::Acc acc;
    acc.init();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    WarpStage& ws = reinterpret_cast<WarpStage*>(dyn)[warp];
    const int nw = gridDim.x * kWarps;
    const unsigned full = 0xffffffffu;
    if (lane == 0) {
        mbar_init(&ws.bar[0], 1);
        mbar_init(&ws.bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    unsigned phase = 0;   // bit b: parity to wait for on buffer b
    unsigned pending = 0; // bit b: a copy into buffer b is in flight
    bool aborted = false;
    int t = blockIdx.x * kWarps + warp;
    Chunk cur{};
    if (t < A.ntiles) {
        cur = chunk_at(A, t);
        if (!cur.streamed()) {
            if (lane == 0) issue_chunk(A, cur, ws, 0);
            pending |= 1u;
        }
    }
    for (int k = 0; t < A.ntiles; ++k, t += nw) {
        const int b = k & 1;
        const int tn = t + nw;
        Chunk nxt{};
        if (tn < A.ntiles) {
            nxt = chunk_at(A, tn);
            if (!nxt.streamed()) {
                if (lane == 0) issue_chunk(A, nxt, ws, b ^ 1);
                pending |= 2u >> b;  // bit (b ^ 1)
            }
        }
        const int my = cur.r0 + lane;
        const bool owns = my < cur.r1;
        typename P::type pre{};
        int q0 = 0, q1 = 0;
        if (owns) {
            pre = P::load(epi, my);
            q0 = __ldg(A.ptr + my) - cur.a0v;
            q1 = __ldg(A.ptr + my + 1) - cur.a0v;
        }
        if (cur.streamed()) {
            double s0 = 0.0, s1 = 0.0;
            int p = cur.p0 + lane;
            for (; p + 32 < cur.p1; p += 64) {
                s0 += __ldcs(A.val + p) * __ldg(v + __ldcs(A.idx + p));
                s1 += __ldcs(A.val + p + 32) * __ldg(v + __ldcs(A.idx + p + 32));
            }
            if (p < cur.p1) s0 += __ldcs(A.val + p) * __ldg(v + __ldcs(A.idx + p));
            const double s = warp_sum(s0 + s1);
            if (lane == 0) P::apply(epi, cur.r0, s, pre, acc);
            cur = nxt;
            continue;
        }
        const bool ok = mbar_wait(&ws.bar[b], (phase >> b) & 1u);
        phase ^= 1u << b;
        pending &= ~(1u << b);
        if (!__all_sync(full, ok)) {
            if (lane == 0 && A.err) atomicAdd(A.err, 1u);
            aborted = true;
            break;
        }
        double* sval = ws.val[b];
        const int* sidx = ws.idx[b];
        int col[kPerLane];
        double g[kPerLane];
#pragma unroll
        for (int e = 0; e < kPerLane; ++e) {
            const int p = cur.p0 + 32 * e + lane;
            col[e] = 0;
            if (p < cur.p1) col[e] = p < cur.a1i ? sidx[p - cur.a0i] : __ldg(A.idx + p);
        }
#pragma unroll
        for (int e = 0; e < kPerLane; ++e)
            g[e] = cur.p0 + 32 * e + lane < cur.p1 ? __ldg(v + col[e]) : 0.0;
#pragma unroll
        for (int e = 0; e < kPerLane; ++e) {
            const int p = cur.p0 + 32 * e + lane;
            if (p < cur.p1) {
                const double a = p < cur.a1v ? sval[p - cur.a0v] : __ldg(A.val + p);
                sval[p - cur.a0v] = dmul(a, g[e]);
            }
        }
        __syncwarp();
        const int len = q1 - q0;
        if (owns && len <= kShortRow) {
            double s = 0.0;
            for (int q = q0; q < q1; ++q) s = dadd(s, sval[q]);
            P::apply(epi, my, s, pre, acc);
        }
        unsigned long_rows = __ballot_sync(full, owns && len > kShortRow);
        while (long_rows) {
            const int l = __ffs(long_rows) - 1;
            long_rows &= long_rows - 1;
            const int lq0 = __shfl_sync(full, q0, l), lq1 = __shfl_sync(full, q1, l);
            double s = 0.0;
            for (int q = lq0 + lane; q < lq1; q += 32) s += sval[q];
            s = warp_sum(s);
            if (lane == l) P::apply(epi, my, s, pre, acc);
        }
        __syncwarp();
        cur = nxt;
    }
    if (aborted && lane == 0) {
        // drain copies still in flight before the slice is released
        for (int b = 0; b < 2; ++b)
            if (pending & (1u << b)) mbar_wait(&ws.bar[b], (phase >> b) & 1u);
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
inline int tiled_grid(const TileCsr& A) {
    const void* k = reinterpret_cast<const void*>(&k_tiled<Epi>);
    return grid_for(k, (A.ntiles + kWarps - 1) / kWarps, kTiledSmem);
}

template <class Epi>
inline int launch_tiled(const TileCsr& A, const double* v, const Epi& epi, cudaStream_t stream,
                        int grid) {
    if (A.ntiles == 0) return 0;
    k_tiled<Epi><<<grid, kThreads, kTiledSmem, stream>>>(A, v, epi);
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
