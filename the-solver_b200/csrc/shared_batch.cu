// Batched PDHG over LPs that share one constraint matrix and differ in their
// cost and bounds: the node relaxations of a branch-and-bound search, which the
// reference solves one at a time on the same model with only the column bounds
// swapped in (milp_solve_lp, c/src/sk_milp.c:432-459). Every LP runs the first-
// order loop of sk_solve (c/src/sk_solve.c:849-954) with its own gates, exactly
// as sankhya_b200_batch_pdhg does for a block-diagonal batch.
//
// Layout. The per-LP vectors live batch-minor on the device: element j of LP k
// at j * bp + k, bp = batch rounded up to 32. A row of the shared matrix is read
// once per iteration for all LPs; its "gathers" become contiguous 256-byte
// loads of 32 LPs' values (one slab), and a warp carries a few slabs through
// the row, one LP per lane and slab. Each LP's row sum runs over
// the row's entries in stored order with unfused products and adds, the order
// and rounding of sk_solve's serial CSC loops (and of the single-LP kernels'
// short-row path), so every LP's iterates equal a separate solve's bit for bit.
// Costs and row bounds may be given once for all LPs (kept as one vector).
#include "batch_common.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace b200 {

namespace {

using batch::atomic_max_nonneg;
using batch::k_abs_sums;
using batch::now_s;
using batch::sk_inf;
using batch::sk_neg_inf;
using batch::slot_value;

// Warp shapes: S 32-LP slabs carried by one warp, gathers of A row entries issued
// together. Every shape sums each LP in stored order, so all give the same bits;
// the fastest for a (matrix, batch width) is picked by timing (schedule 0) or
// fixed by the caller (schedule 1..3).
struct Shape {
    int slabs, ahead;
};
constexpr Shape kShapes[3] = {{1, 8}, {2, 4}, {4, 4}};

// Each epilogue prefetches its per-(row, LP) data into L1 before the gathers
// (prefetch: no registers held), reads it after them (load) and finishes the step
// with the row sum (store).

// sk_solve.c:901-906 per (row, LP), with LP freezing
struct MultiDualEpi {
    const double* __restrict__ y;
    const double* __restrict__ rl;
    const double* __restrict__ ru;
    const double* __restrict__ sig;
    const int* __restrict__ done;
    double* __restrict__ y_new;
    int bp, rows_per_lp;
    struct Row {
        double y, lo, hi;
        int frozen;
    };
    __device__ __forceinline__ Row load(int i, int k) const {
        const size_t e = static_cast<size_t>(i) * bp + k, b = rows_per_lp ? e : static_cast<size_t>(i);
        return Row{y[e], rl[b], ru[b], done[k]};
    }
    __device__ __forceinline__ void prefetch(int i, int k) const {
        const size_t e = static_cast<size_t>(i) * bp + k, b = rows_per_lp ? e : static_cast<size_t>(i);
        asm volatile("prefetch.global.L1 [%0];" ::"l"(y + e));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(rl + b));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(ru + b));
    }
    __device__ __forceinline__ void store(int i, int k, double act, const Row& r) const {
        const size_t e = static_cast<size_t>(i) * bp + k;
        if (r.frozen) {
            y_new[e] = r.y;
            return;
        }
        const double s = sig[i];
        const double trial = dadd(r.y, dmul(s, act));
        y_new[e] = dsub(trial, dmul(s, box_sk(ddiv(trial, s), r.lo, r.hi)));
    }
};

// sk_solve.c:918-923 (LP, no Q) per (column, LP), with LP freezing
struct MultiPrimalEpi {
    const double* __restrict__ x;
    const double* __restrict__ c;
    const double* __restrict__ tau;
    const double* __restrict__ cl;
    const double* __restrict__ cu;
    const int* __restrict__ done;
    double* __restrict__ x_new;
    double* __restrict__ x_bar;
    int bp, c_per_lp;
    struct Row {
        double x, c, lo, hi;
        int frozen;
    };
    __device__ __forceinline__ Row load(int j, int k) const {
        const size_t e = static_cast<size_t>(j) * bp + k;
        return Row{x[e], c[c_per_lp ? e : static_cast<size_t>(j)], cl[e], cu[e], done[k]};
    }
    __device__ __forceinline__ void prefetch(int j, int k) const {
        const size_t e = static_cast<size_t>(j) * bp + k;
        asm volatile("prefetch.global.L1 [%0];" ::"l"(x + e));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(cl + e));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(cu + e));
    }
    __device__ __forceinline__ void store(int j, int k, double g, const Row& r) const {
        const size_t e = static_cast<size_t>(j) * bp + k;
        if (r.frozen) {
            x_new[e] = r.x;
            return;
        }
        double xn = dsub(r.x, dmul(tau[j], dadd(dadd(r.c, 0.0), g)));
        xn = box_sk(xn, r.lo, r.hi);
        x_new[e] = xn;
        x_bar[e] = dsub(dmul(2.0, xn), r.x);
    }
};

struct MultiStoreEpi {
    double* __restrict__ out;
    int bp;
    struct Row {};
    __device__ __forceinline__ Row load(int, int) const { return {}; }
    __device__ __forceinline__ void prefetch(int, int) const {}
    __device__ __forceinline__ void store(int i, int k, double s, const Row&) const {
        out[static_cast<size_t>(i) * bp + k] = s;
    }
};

// One warp per (row, group of 32 S LPs): out(r, k) = sum_p a_p v[col_p, k] in
// stored order for every LP k of the group. The gathers of AH entries are issued
// before their products are added, in order, to each LP's sum.
template <class Epi, int S, int AH>
__global__ void __launch_bounds__(kThreads) k_multi(int rows, int groups, int bp, const int* __restrict__ ptr,
                                                    const int* __restrict__ idx, const double* __restrict__ val,
                                                    const double* __restrict__ v, Epi epi) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long units = static_cast<long long>(rows) * groups;
    const long long nw = static_cast<long long>(gridDim.x) * kWarps;
    for (long long u = static_cast<long long>(blockIdx.x) * kWarps + (threadIdx.x >> 5); u < units; u += nw) {
        const int r = static_cast<int>(u / groups), g = static_cast<int>(u % groups);
        const int k0 = g * 32 * S;
        const int ns = min(S, (bp - k0) >> 5);
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (s < ns) epi.prefetch(r, k0 + 32 * s + lane);
        double acc[S];
#pragma unroll
        for (int s = 0; s < S; ++s) acc[s] = 0.0;
        const int p0 = __ldg(ptr + r), p1 = __ldg(ptr + r + 1);
        for (int pb = p0; pb < p1; pb += 32) {
            const int cnt = min(32, p1 - pb);
            int ci = 0;
            double ai = 0.0;
            if (lane < cnt) {
                ci = __ldg(idx + pb + lane);
                ai = __ldg(val + pb + lane);
            }
            for (int e0 = 0; e0 < cnt; e0 += AH) {
                double g8[AH][S];
#pragma unroll
                for (int q = 0; q < AH; ++q) {
                    const int col = __shfl_sync(full, ci, min(e0 + q, 31));
                    const double* src = v + static_cast<size_t>(col) * bp + k0 + lane;
#pragma unroll
                    for (int s = 0; s < S; ++s)
                        g8[q][s] = (e0 + q < cnt && s < ns) ? __ldg(src + 32 * s) : 0.0;
                }
#pragma unroll
                for (int q = 0; q < AH; ++q) {
                    const double a = __shfl_sync(full, ai, min(e0 + q, 31));
                    if (e0 + q < cnt) {
#pragma unroll
                        for (int s = 0; s < S; ++s) acc[s] = dadd(acc[s], dmul(a, g8[q][s]));
                    }
                }
            }
        }
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (s < ns) epi.store(r, k0 + 32 * s + lane, acc[s], epi.load(r, k0 + 32 * s + lane));
    }
}

// LP-major [batch][len] (the caller's layout) <-> batch-minor [len][bp], 32 x 32 tiles.
__global__ void k_to_batch_minor(int len, int batch, int bp, const double* __restrict__ in, double* __restrict__ out) {
    __shared__ double tile[32][33];
    const int j0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
        const int k = k0 + dy, j = j0 + threadIdx.x;
        tile[dy][threadIdx.x] = (k < batch && j < len) ? in[static_cast<size_t>(k) * len + j] : 0.0;
    }
    __syncthreads();
    for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
        const int j = j0 + dy, k = k0 + threadIdx.x;
        if (j < len && k < bp) out[static_cast<size_t>(j) * bp + k] = tile[threadIdx.x][dy];
    }
}

__global__ void k_from_batch_minor(int len, int batch, int bp, const double* __restrict__ in, double* __restrict__ out) {
    __shared__ double tile[32][33];
    const int j0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
        const int j = j0 + dy, k = k0 + threadIdx.x;
        tile[dy][threadIdx.x] = (j < len && k < bp) ? in[static_cast<size_t>(j) * bp + k] : 0.0;
    }
    __syncthreads();
    for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
        const int k = k0 + dy, j = j0 + threadIdx.x;
        if (k < batch && j < len) out[static_cast<size_t>(k) * len + j] = tile[threadIdx.x][dy];
    }
}

// Initial point of every LP (sk_solve.c:882-884): x = box(0), x_bar = x.
__global__ void k_multi_init(size_t total, const double* __restrict__ cl, const double* __restrict__ cu,
                             double* __restrict__ x, double* __restrict__ x_bar) {
    for (size_t e = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; e < total;
         e += static_cast<size_t>(blockDim.x) * gridDim.x) {
        const double v = box_sk(0.0, cl[e], cu[e]);
        x[e] = v;
        x_bar[e] = v;
    }
}

// Per-LP maxima over rows (sk_solve.c:82-95 violation; max |y - y_prev|).
// Block (32, 8): lane x = LP within the slab blockIdx.y, y strides the rows.
__global__ void k_multi_rows_check(int m, int bp, int rows_per_lp, const double* __restrict__ act,
                                   const double* __restrict__ y, const double* __restrict__ y_prev,
                                   const double* __restrict__ rl, const double* __restrict__ ru,
                                   const int* __restrict__ done, unsigned long long* __restrict__ viol,
                                   unsigned long long* __restrict__ dstep) {
    __shared__ double sv[8][32], sd[8][32];
    const int k = blockIdx.y * 32 + threadIdx.x;
    double v = 0.0, d = 0.0;
    if (!done[k]) {
        for (int i = blockIdx.x * blockDim.y + threadIdx.y; i < m; i += gridDim.x * blockDim.y) {
            const size_t e = static_cast<size_t>(i) * bp + k, b = rows_per_lp ? e : static_cast<size_t>(i);
            const double a = act[e];
            double t = 0.0;
            if (!sk_neg_inf(rl[b]) && rl[b] - a > t) t = rl[b] - a;
            if (!sk_inf(ru[b]) && a - ru[b] > t) t = a - ru[b];
            v = (t > v || isnan(t)) ? t : v;
            const double s = fabs(y[e] - y_prev[e]);
            d = (s > d || isnan(s)) ? s : d;
        }
    }
    sv[threadIdx.y][threadIdx.x] = v;
    sd[threadIdx.y][threadIdx.x] = d;
    __syncthreads();
    if (threadIdx.y == 0 && !done[k]) {
        for (int w = 1; w < 8; ++w) {
            v = (sv[w][threadIdx.x] > v || isnan(sv[w][threadIdx.x])) ? sv[w][threadIdx.x] : v;
            d = (sd[w][threadIdx.x] > d || isnan(sd[w][threadIdx.x])) ? sd[w][threadIdx.x] : d;
        }
        atomic_max_nonneg(&viol[k], v);
        atomic_max_nonneg(&dstep[k], d);
    }
}

// Per-LP maxima over columns: |x|_inf and max |x_bar - x|.
__global__ void k_multi_cols_check(int n, int bp, const double* __restrict__ x, const double* __restrict__ x_bar,
                                   const int* __restrict__ done, unsigned long long* __restrict__ scale,
                                   unsigned long long* __restrict__ step) {
    __shared__ double ss[8][32], st[8][32];
    const int k = blockIdx.y * 32 + threadIdx.x;
    double a = 0.0, b = 0.0;
    if (!done[k]) {
        for (int j = blockIdx.x * blockDim.y + threadIdx.y; j < n; j += gridDim.x * blockDim.y) {
            const size_t e = static_cast<size_t>(j) * bp + k;
            const double s = fabs(x[e]), t = fabs(x_bar[e] - x[e]);
            a = (s > a || isnan(s)) ? s : a;
            b = (t > b || isnan(t)) ? t : b;
        }
    }
    ss[threadIdx.y][threadIdx.x] = a;
    st[threadIdx.y][threadIdx.x] = b;
    __syncthreads();
    if (threadIdx.y == 0 && !done[k]) {
        for (int w = 1; w < 8; ++w) {
            a = (ss[w][threadIdx.x] > a || isnan(ss[w][threadIdx.x])) ? ss[w][threadIdx.x] : a;
            b = (st[w][threadIdx.x] > b || isnan(st[w][threadIdx.x])) ? st[w][threadIdx.x] : b;
        }
        atomic_max_nonneg(&scale[k], a);
        atomic_max_nonneg(&step[k], b);
    }
}

// Largest column and row mass of the shared matrix (one block).
__global__ void k_mass_max(int n, const double* __restrict__ cmass, int m, const double* __restrict__ rmass,
                           double* __restrict__ out) {
    __shared__ double sc[kThreads], sr[kThreads];
    double a = 0.0, b = 0.0;
    for (int j = threadIdx.x; j < n; j += blockDim.x) a = fmax(a, cmass[j]);
    for (int i = threadIdx.x; i < m; i += blockDim.x) b = fmax(b, rmass[i]);
    sc[threadIdx.x] = a;
    sr[threadIdx.x] = b;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sc[threadIdx.x] = fmax(sc[threadIdx.x], sc[threadIdx.x + w]);
            sr[threadIdx.x] = fmax(sr[threadIdx.x], sr[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sc[0];
        out[1] = sr[0];
    }
}

__global__ void k_mass_steps(int len, const double* __restrict__ mass, double* __restrict__ steps) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < len; j += blockDim.x * gridDim.x)
        steps[j] = 0.9 / (1.0 + mass[j]);
}

// One thread per LP: the gates of sk_solve.c:926-953 (anorm of the shared
// matrix, sk_solve.c:877-880); clears the maxima.
__global__ void k_multi_gate(int batch, int iteration, int last, double ptol, double dtol,
                             unsigned long long* __restrict__ viol, unsigned long long* __restrict__ dstep,
                             unsigned long long* __restrict__ scale, unsigned long long* __restrict__ step,
                             const double* __restrict__ massmax, int* __restrict__ done, int* __restrict__ iters,
                             double* __restrict__ report, unsigned int* __restrict__ remaining) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < batch; k += blockDim.x * gridDim.x) {
        if (done[k]) continue;
        const double v = slot_value(viol[k]), ds = slot_value(dstep[k]);
        const double sc = fmax(1.0, slot_value(scale[k])), st = slot_value(step[k]);
        const double anorm = sqrt(massmax[0] * massmax[1]);
        report[4 * k + 0] = v;
        report[4 * k + 1] = st;
        report[4 * k + 2] = ds;
        report[4 * k + 3] = anorm;
        viol[k] = dstep[k] = scale[k] = step[k] = 0ull;
        iters[k] = iteration;
        if (v <= ptol && st <= ptol * sc && ds <= dtol * (1.0 + anorm)) {
            done[k] = 1;
        } else if (!last) {
            atomicAdd(remaining, 1u);
        }
    }
}

__global__ void k_mark_padding(int batch, int bp, int* __restrict__ done) {
    const int k = batch + blockIdx.x * blockDim.x + threadIdx.x;
    if (k < bp) done[k] = 1;
}

template <class Epi, int S, int AH>
void launch_shape(int rows, int bp, const TileCsr& M, const double* v, const Epi& epi, cudaStream_t st) {
    if (rows == 0) return;
    const int groups = (bp + 32 * S - 1) / (32 * S);
    const long long blocks = (static_cast<long long>(rows) * groups + kWarps - 1) / kWarps;
    const int grid = grid_for(reinterpret_cast<const void*>(&k_multi<Epi, S, AH>),
                              static_cast<int>(std::min<long long>(blocks, 1 << 30)), 0);
    k_multi<Epi, S, AH><<<grid, kThreads, 0, st>>>(rows, groups, bp, M.ptr, M.idx, M.val, v, epi);
}

template <class Epi>
void launch_multi(int shape, int rows, int bp, const TileCsr& M, const double* v, const Epi& epi, cudaStream_t st) {
    switch (shape) {
        case 0: launch_shape<Epi, kShapes[0].slabs, kShapes[0].ahead>(rows, bp, M, v, epi, st); break;
        case 1: launch_shape<Epi, kShapes[1].slabs, kShapes[1].ahead>(rows, bp, M, v, epi, st); break;
        default: launch_shape<Epi, kShapes[2].slabs, kShapes[2].ahead>(rows, bp, M, v, epi, st); break;
    }
}

// Fastest shape for one iteration (dual + primal step) of this matrix at this
// batch width, timed with CUDA events on the solve's own data (outputs to scratch),
// cached per (device, matrix, width).
int autotuned_shape(const TileCsr& A, const TileCsr& AT, int bp, const MultiDualEpi& dual, const double* x_bar,
                    const MultiPrimalEpi& primal, const double* y, cudaStream_t st) {
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, int, int, int>, int> cache;
    int device = 0;
    cudaGetDevice(&device);
    const auto key = std::make_tuple(device, static_cast<const void*>(A.ptr), A.rows, A.nnz, bp);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return 1;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return 1;
    }
    int best = 1;
    float best_ms = 0.f;
    for (int shape = 0; shape < 3; ++shape) {
        auto pair = [&]() {
            launch_multi(shape, A.rows, bp, A, x_bar, dual, st);
            launch_multi(shape, AT.rows, bp, AT, y, primal, st);
        };
        pair();
        cudaEventRecord(e0, st);
        for (int r = 0; r < 5; ++r) pair();
        cudaEventRecord(e1, st);
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) continue;
        if (shape == 0 || ms < best_ms) {
            best = shape;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = best;
    return best;
}

}  // namespace

}  // namespace b200

using namespace b200;

extern "C" int sankhya_b200_shared_batch_pdhg(const SankhyaCudaCSR* matrix, int batch, const double* c, int c_per_lp,
                                              const double* rlow, const double* rupp, int row_bounds_per_lp,
                                              const double* clow, const double* cupp, int col_bounds_per_lp,
                                              const SankhyaB200BatchSettings* settings, double* x_out, double* y_out,
                                              SankhyaB200BatchResult* results) {
    clear_error();
    (void)cudaGetLastError();
    SankhyaB200BatchSettings s;
    sankhya_b200_batch_default_settings(&s);
    if (settings) {
        if (settings->struct_version != 1) return fail_msg("unsupported settings struct_version");
        s = *settings;
    }
    if (!matrix || batch <= 0 || !c || !rlow || !rupp || !clow || !cupp || !x_out || !results)
        return fail_msg("invalid shared batch arguments");
    if (s.max_iterations <= 0 || s.check_every <= 0 || !(s.primal_tol > 0.0) || !(s.dual_tol > 0.0) ||
        s.time_limit < 0.0 || s.schedule < 0 || s.schedule > 3)
        return fail_msg("invalid batch settings");
    const int m = matrix->rows, n = matrix->cols;
    if (m < 0 || n <= 0) return fail_msg("invalid matrix dimensions");
    const size_t bp = (static_cast<size_t>(batch) + 31) / 32 * 32;
    const size_t nc = c_per_lp ? static_cast<size_t>(batch) * n : static_cast<size_t>(n);
    const size_t nr = row_bounds_per_lp ? static_cast<size_t>(batch) * m : static_cast<size_t>(m);
    const size_t ncol = col_bounds_per_lp ? static_cast<size_t>(batch) * n : static_cast<size_t>(n);
    for (size_t j = 0; j < nc; ++j)
        if (!std::isfinite(c[j])) return fail_msg("invalid cost or column bound");
    for (size_t j = 0; j < ncol; ++j)
        if (std::isnan(clow[j]) || std::isnan(cupp[j]) || clow[j] > cupp[j])
            return fail_msg("invalid cost or column bound");
    for (size_t i = 0; i < nr; ++i)
        if (std::isnan(rlow[i]) || std::isnan(rupp[i]) || rlow[i] > rupp[i]) return fail_msg("invalid row bound");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) return fail_msg("no CUDA device available");
    std::shared_ptr<Plan> plan;
    if (get_plan(matrix, &plan)) return -1;
    const double t0 = now_s();
    cudaStream_t stream = engine_stream();

    auto al = [](size_t bytes) { return (bytes + 255) / 256 * 256; };
    const size_t NB = al(sizeof(double) * n * bp), MB = al(sizeof(double) * static_cast<size_t>(m) * bp);
    const size_t nb = al(sizeof(double) * n), mb = al(sizeof(double) * static_cast<size_t>(m));
    const size_t kb = al(sizeof(double) * bp);
    const size_t stage = std::max(NB, MB);
    // batch-minor: x[2], x_bar, cl, cu, (c); y[2], act, (rl, ru); shared: tau, cmass,
    // sig, rmass, (c), (rl, ru); per-LP slots; staging for the layout changes
    const size_t total = 6 * NB + (c_per_lp ? NB : nb) + 3 * MB + (row_bounds_per_lp ? 2 * MB : 2 * mb) + 2 * nb +
                         2 * mb + 12 * kb + stage + 4096;
    DevBuf blob;
    if (blob.alloc(total, "cudaMalloc shared batch workspace")) return -1;
    char* p = blob.as<char>();
    auto take = [&](size_t b) { char* r = p; p += b; return reinterpret_cast<double*>(r); };
    double *xb0 = take(NB), *xb1 = take(NB), *xbar = take(NB), *dcl = take(NB), *dcu = take(NB), *tune = take(NB);
    double* dc = take(c_per_lp ? NB : nb);
    double *yb0 = take(MB), *yb1 = take(MB), *act = take(MB);
    double* drl = take(row_bounds_per_lp ? MB : mb);
    double* dru = take(row_bounds_per_lp ? MB : mb);
    double *tau = take(nb), *cmass = take(nb), *sig = take(mb), *rmass = take(mb);
    auto* viol = reinterpret_cast<unsigned long long*>(take(kb));
    auto* dstep = reinterpret_cast<unsigned long long*>(take(kb));
    auto* scale = reinterpret_cast<unsigned long long*>(take(kb));
    auto* step = reinterpret_cast<unsigned long long*>(take(kb));
    int* done = reinterpret_cast<int*>(take(kb));
    int* iters = reinterpret_cast<int*>(take(kb));
    double* report = take(4 * kb);
    double* massmax = take(2 * kb);
    double* staging = take(stage);
    unsigned int* counters = reinterpret_cast<unsigned int*>(take(256));

    const int bpi = static_cast<int>(bp);
    const dim3 tblock(32, 8);
    // LP-major host array -> batch-minor device array (per-LP), or one shared vector
    auto upload = [&](const double* host, int len, bool per_lp, double* dst) -> int {
        if (len == 0) return 0;
        if (!per_lp) {
            B200_TRY(cudaMemcpyAsync(dst, host, sizeof(double) * len, cudaMemcpyHostToDevice, stream), "upload");
            return 0;
        }
        B200_TRY(cudaMemcpyAsync(staging, host, sizeof(double) * static_cast<size_t>(batch) * len,
                                 cudaMemcpyHostToDevice, stream),
                 "upload");
        k_to_batch_minor<<<dim3((len + 31) / 32, bpi / 32), tblock, 0, stream>>>(len, batch, bpi, staging, dst);
        return 0;
    };
    // a shared vector replicated into every LP's slot (column bounds are per LP inside)
    auto upload_replicated = [&](const double* host, int len, double* dst) -> int {
        if (len == 0) return 0;
        std::vector<double> rep(static_cast<size_t>(batch) * len);
        for (int k = 0; k < batch; ++k) std::memcpy(rep.data() + static_cast<size_t>(k) * len, host, sizeof(double) * len);
        B200_TRY(cudaMemcpyAsync(staging, rep.data(), sizeof(double) * rep.size(), cudaMemcpyHostToDevice, stream),
                 "upload");
        k_to_batch_minor<<<dim3((len + 31) / 32, bpi / 32), tblock, 0, stream>>>(len, batch, bpi, staging, dst);
        B200_TRY(cudaStreamSynchronize(stream), "upload");
        return 0;
    };
    if (upload(c, n, c_per_lp != 0, dc)) return -1;
    if (col_bounds_per_lp) {
        if (upload(clow, n, true, dcl) || upload(cupp, n, true, dcu)) return -1;
    } else {
        if (upload_replicated(clow, n, dcl) || upload_replicated(cupp, n, dcu)) return -1;
    }
    if (upload(rlow, m, row_bounds_per_lp != 0, drl) || upload(rupp, m, row_bounds_per_lp != 0, dru)) return -1;
    if (m) B200_TRY(cudaMemsetAsync(yb0, 0, MB, stream), "zero y");
    B200_TRY(cudaMemsetAsync(viol, 0, 6 * kb, stream), "zero slots");
    B200_TRY(cudaMemsetAsync(counters, 0, 256, stream), "zero counters");
    if (bp > static_cast<size_t>(batch))
        k_mark_padding<<<1, 32, 0, stream>>>(batch, bpi, done);
    const TileCsr& A = plan->a;
    const TileCsr& AT = plan->at;
    if (m) k_abs_sums<<<elem_grid(m), kThreads, 0, stream>>>(m, A.ptr, A.val, rmass);
    k_abs_sums<<<elem_grid(n), kThreads, 0, stream>>>(n, AT.ptr, AT.val, cmass);
    k_mass_max<<<1, kThreads, 0, stream>>>(n, cmass, m, rmass, massmax);
    k_mass_steps<<<elem_grid(n), kThreads, 0, stream>>>(n, cmass, tau);
    if (m) k_mass_steps<<<elem_grid(m), kThreads, 0, stream>>>(m, rmass, sig);
    k_multi_init<<<elem_grid(static_cast<int>(std::min<size_t>(n * bp, 1u << 30))), kThreads, 0, stream>>>(
        n * bp, dcl, dcu, xb0, xbar);
    B200_TRY(cudaGetLastError(), "shared batch setup");
    unsigned int* host_counters = nullptr;
    B200_TRY(cudaMallocHost(reinterpret_cast<void**>(&host_counters), 64), "cudaMallocHost");
    struct Free {
        unsigned int* p;
        ~Free() { cudaFreeHost(p); }
    } free_host{host_counters};

    int shape = s.schedule - 1;
    if (s.schedule == 0) {
        // time on scratch outputs: y_new into the activity buffer, x_new / x_bar into
        // the staging buffer and the tuning buffer; iterates untouched
        shape = autotuned_shape(A, AT, bpi,
                                MultiDualEpi{yb0, drl, dru, sig, done, act, bpi, row_bounds_per_lp ? 1 : 0}, xbar,
                                MultiPrimalEpi{xb0, dc, tau, dcl, dcu, done, staging, tune, bpi, c_per_lp ? 1 : 0},
                                yb0, stream);
        B200_TRY(cudaGetLastError(), "shared batch schedule");
    }
    const dim3 check_rows(static_cast<unsigned>(std::max(1, std::min((m + 7) / 8, 4 * 148 * 8 * 32 / bpi))), bpi / 32);
    const dim3 check_cols(static_cast<unsigned>(std::max(1, std::min((n + 7) / 8, 4 * 148 * 8 * 32 / bpi))), bpi / 32);
    double* xb[2] = {xb0, xb1};
    double* yb[2] = {yb0, yb1};
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
    struct Graphs {
        std::map<std::pair<int, int>, cudaGraphExec_t>* g;
        ~Graphs() {
            for (auto& kv : *g)
                if (kv.second) cudaGraphExecDestroy(kv.second);
        }
    } graphs_guard{&graphs};
    int cur = 0, it = 0, launches = 0;
    auto iterate = [&]() {
        const int nx = cur ^ 1;
        launch_multi(shape, m, bpi, A, xbar, MultiDualEpi{yb[cur], drl, dru, sig, done, yb[nx], bpi,
                                                           row_bounds_per_lp ? 1 : 0},
                     stream);
        launch_multi(shape, n, bpi, AT, yb[nx],
                     MultiPrimalEpi{xb[cur], dc, tau, dcl, dcu, done, xb[nx], xbar, bpi, c_per_lp ? 1 : 0}, stream);
        cur = nx;
    };
    bool timed_out = false;
    int checks = 0;
    batch::LoopEvents loop_events(timing().level >= 1, stream);
    while (it < s.max_iterations) {
        const int next = std::min((it / s.check_every + 1) * s.check_every, s.max_iterations);
        int k = next - it;
        while (k > 0) {
            const int chunk = std::min(k, 64);
            auto key = std::make_pair(chunk, cur);
            auto g = graphs.find(key);
            if (g == graphs.end()) {
                const int saved = cur;
                cudaGraph_t graph;
                B200_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
                for (int i = 0; i < chunk; ++i) iterate();
                B200_TRY(cudaStreamEndCapture(stream, &graph), "end capture");
                cudaGraphExec_t exec;
                cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
                cudaGraphDestroy(graph);
                if (e != cudaSuccess) return fail_cuda("graph instantiate", e);
                g = graphs.emplace(key, exec).first;
                cur = saved;
            }
            B200_TRY(cudaGraphLaunch(g->second, stream), "graph launch");
            launches += (m ? 2 : 1) * chunk;
            cur ^= (chunk & 1);
            k -= chunk;
        }
        it = next;
        const bool last = it >= s.max_iterations;
        ++checks;
        B200_TRY(cudaMemsetAsync(counters, 0, 4, stream), "zero counter");
        if (m) {
            launch_multi(shape, m, bpi, A, xb[cur], MultiStoreEpi{act, bpi}, stream);
            k_multi_rows_check<<<check_rows, tblock, 0, stream>>>(m, bpi, row_bounds_per_lp ? 1 : 0, act, yb[cur],
                                                                  yb[cur ^ 1], drl, dru, done, viol, dstep);
        }
        k_multi_cols_check<<<check_cols, tblock, 0, stream>>>(n, bpi, xb[cur], xbar, done, scale, step);
        k_multi_gate<<<elem_grid(batch), kThreads, 0, stream>>>(batch, it, last ? 1 : 0, s.primal_tol, s.dual_tol,
                                                                viol, dstep, scale, step, massmax, done, iters,
                                                                report, counters);
        launches += m ? 4 : 2;
        B200_TRY(cudaMemcpyAsync(host_counters, counters, 4, cudaMemcpyDeviceToHost, stream), "read");
        B200_TRY(cudaStreamSynchronize(stream), "shared batch check");
        if (host_counters[0] == 0) break;
        if (s.time_limit > 0.0 && now_s() - t0 >= s.time_limit) {
            timed_out = true;
            break;
        }
    }
    const double loop_ms = loop_events.stop(stream);
    std::vector<int> h_done(static_cast<size_t>(batch)), h_iters(static_cast<size_t>(batch));
    std::vector<double> h_report(static_cast<size_t>(batch) * 4);
    k_from_batch_minor<<<dim3((n + 31) / 32, bpi / 32), tblock, 0, stream>>>(n, batch, bpi, xb[cur], staging);
    B200_TRY(cudaMemcpyAsync(x_out, staging, sizeof(double) * static_cast<size_t>(batch) * n, cudaMemcpyDeviceToHost,
                             stream),
             "download x");
    if (y_out && m) {
        B200_TRY(cudaStreamSynchronize(stream), "download x");
        k_from_batch_minor<<<dim3((m + 31) / 32, bpi / 32), tblock, 0, stream>>>(m, batch, bpi, yb[cur], staging);
        B200_TRY(cudaMemcpyAsync(y_out, staging, sizeof(double) * static_cast<size_t>(batch) * m,
                                 cudaMemcpyDeviceToHost, stream),
                 "download y");
    }
    B200_TRY(cudaMemcpyAsync(h_done.data(), done, sizeof(int) * batch, cudaMemcpyDeviceToHost, stream), "download");
    B200_TRY(cudaMemcpyAsync(h_iters.data(), iters, sizeof(int) * batch, cudaMemcpyDeviceToHost, stream), "download");
    B200_TRY(cudaMemcpyAsync(h_report.data(), report, sizeof(double) * 4 * batch, cudaMemcpyDeviceToHost, stream),
             "download");
    B200_TRY(cudaStreamSynchronize(stream), "shared batch download");
    for (int k = 0; k < batch; ++k) {
        SankhyaB200BatchResult& r = results[k];
        r.status = h_done[k] ? 0 : (timed_out ? 2 : 1);
        r.iterations = h_done[k] ? h_iters[k] : it;
        const double* ck = c + (c_per_lp ? static_cast<size_t>(k) * n : 0);
        const double* xk = x_out + static_cast<size_t>(k) * n;
        double obj = 0.0;
        for (int j = 0; j < n; ++j) obj += ck[j] * xk[j];
        r.objective = obj;
        r.row_violation = h_report[4 * k + 0];
        r.step = h_report[4 * k + 1];
        r.dual_step = h_report[4 * k + 2];
        r.anorm = h_report[4 * k + 3];
    }
    TimingState& ts = timing();
    ts.last = SankhyaB200Timing{};
    ts.last.iterations = it;
    ts.last.kernel_launches = launches;
    ts.last.checkpoints = checks;
    ts.last.loop_ms = loop_ms;
    return 0;
}
