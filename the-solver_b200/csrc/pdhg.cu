// Fixed-step PDHG behind the reference C ABI (the five *_pdhg entry points)
// and the sk_solve loop replacement.
//
// One iteration is two fused launches over the tiled CSR store:
//   A-side   y_new_i = prox(y_i + s_i (A x_bar)_i)           (dual step)
//   A'-side  x_new_j = proj((x_j - t_j (c_j + (A'y_new)_j + ..)) / (1 + t_j q_j)),
//            x_bar_j = extrapolation                          (primal step)
// plus, for an explicit Hessian, one Q x product between them. A window of
// iterations between checkpoints is captured once as a CUDA graph and
// replayed. A checkpoint is two more fused products (A x and A'y, each with
// its residual terms reduced in the epilogue) and a 100-byte copy to the host.
//
// Two arithmetic contracts are kept, selected per entry point:
//   SemCuda  the CUDA prototype, cuda/src/sankhya_cuda_lp.cu:26-52, 101-385
//            (IEEE-infinity bounds, x_bar = x + theta (x - x_old), 5-gate check)
//   SemSk    the CPU loop of c/src/sk_solve.c:849-954 (1e30 sentinel bounds,
//            x_bar = 2 x_new - x_old, mass-based steps, 20-iteration checks)
#include "engine.cuh"
#include "fixed_epi.cuh"

#include <algorithm>
#include <chrono>
#include <climits>
#include <limits>
#include <map>
#include <tuple>

namespace b200 {

// ===================================================================== epilogues

// c/src/sk_solve.c:901-906 (dual step, and max |y_new - y| for the gate)
struct DualSkEpi {
    const double* __restrict__ y;
    const double* __restrict__ rl;
    const double* __restrict__ ru;
    const double* __restrict__ sig;
    double* __restrict__ y_new;
    double* __restrict__ partial;
    using Acc = Slots<1, 0u>;
    struct Row {
        double y, lo, hi, s;
    };
    __device__ __forceinline__ Row load(int i) const { return Row{y[i], rl[i], ru[i], sig[i]}; }
    __device__ __forceinline__ void store(int i, double act, const Row& r, Acc& acc) const {
        const double trial = dadd(r.y, dmul(r.s, act));
        const double yn = dsub(trial, dmul(r.s, box_sk(ddiv(trial, r.s), r.lo, r.hi)));
        y_new[i] = yn;
        acc.max(0, fabs(dsub(yn, r.y)));
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

// c/src/sk_solve.c:908-923 (primal step with optional diagonal prox / explicit Q x)
struct PrimalSkEpi {
    const double* __restrict__ x;
    const double* __restrict__ c;
    const double* __restrict__ tauv;
    const double* __restrict__ qx;    // explicit Q x or null
    const double* __restrict__ qdiag; // diagonal Q or null
    const double* __restrict__ cl;
    const double* __restrict__ cu;
    double* __restrict__ x_new;
    double* __restrict__ x_bar;
    using Acc = NoAcc;
    struct Row {
        double x, c, t, lo, hi, qd, qx;
    };
    __device__ __forceinline__ Row load(int j) const {
        return Row{x[j], c[j], tauv[j], cl[j], cu[j], qdiag ? qdiag[j] : 0.0, qx ? qx[j] : 0.0};
    }
    __device__ __forceinline__ void store(int j, double g, const Row& r, Acc&) const {
        double xn;
        if (qdiag) {
            xn = ddiv(dsub(r.x, dmul(r.t, dadd(r.c, g))), dadd(1.0, dmul(r.t, r.qd)));
        } else {
            xn = dsub(r.x, dmul(r.t, dadd(dadd(r.c, r.qx), g)));
        }
        xn = box_sk(xn, r.lo, r.hi);
        x_new[j] = xn;
        x_bar[j] = dsub(dmul(2.0, xn), r.x);
    }
    __device__ __forceinline__ void finish(Acc&, double*) const {}
};

__device__ __forceinline__ bool sk_inf(double v) { return v >= 1.0e30; }
__device__ __forceinline__ bool sk_neg_inf(double v) { return v <= -1.0e30; }

// sk checkpoint, rows of A: stores the activity; slots 0 primal violation
// (c/src/sk_solve.c:82-95), 1 row dual infeasibility, 2 row complementarity
// (the row half of sk_verify, c/src/sk_core.c:471-498).
struct CheckRowsSkEpi {
    const double* __restrict__ y;
    const double* __restrict__ rl;
    const double* __restrict__ ru;
    double* __restrict__ act_out;
    double* __restrict__ partial;
    using Acc = Slots<3, 0u>;
    __device__ __forceinline__ void row(int i, double act, Acc& acc) const {
        const double lo = rl[i], hi = ru[i], yv = y[i];
        act_out[i] = act;
        if (!sk_neg_inf(lo)) acc.max(0, lo - act);
        if (!sk_inf(hi)) acc.max(0, act - hi);
        const bool atlo = !sk_neg_inf(lo) && fabs(act - lo) <= 1e-9;
        const bool athi = !sk_inf(hi) && fabs(act - hi) <= 1e-9;
        if (atlo && athi) {
        } else if (atlo) {
            acc.max(1, yv);
        } else if (athi) {
            acc.max(1, -yv);
        } else {
            acc.max(1, fabs(yv));
        }
        if (yv < 0.0) {
            if (sk_neg_inf(lo)) acc.max(1, -yv);
            else acc.max(2, -yv * fabs(act - lo));
        } else if (yv > 0.0) {
            if (sk_inf(hi)) acc.max(1, yv);
            else acc.max(2, yv * fabs(hi - act));
        }
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

// sk checkpoint, columns (QP): slots 0 column primal violation, 1 dual
// infeasibility, 2 complementarity, 3 objective c'x + x'Qx/2 (sum), 4 step
// max|x_bar - x|, 5 scale max|x| (c/src/sk_core.c:415-470, sk_solve.c:933-936).
struct CheckColsSkEpi {
    const double* __restrict__ x;
    const double* __restrict__ x_bar;
    const double* __restrict__ c;
    const double* __restrict__ qx;
    const double* __restrict__ cl;
    const double* __restrict__ cu;
    double* __restrict__ partial;
    using Acc = Slots<6, 1u << 3>;
    __device__ __forceinline__ void row(int j, double aty, Acc& acc) const {
        const double xj = x[j], lo = cl[j], hi = cu[j];
        const double qxj = qx ? qx[j] : 0.0;
        const double r = c[j] + qxj + aty;
        if (!isfinite(xj)) acc.max(0, INFINITY);
        if (!sk_neg_inf(lo)) acc.max(0, lo - xj);
        if (!sk_inf(hi)) acc.max(0, xj - hi);
        const bool atlo = !sk_neg_inf(lo) && fabs(xj - lo) <= 1e-9;
        const bool athi = !sk_inf(hi) && fabs(xj - hi) <= 1e-9;
        if (atlo && athi) {
        } else if (atlo) {
            acc.max(1, -r);
        } else if (athi) {
            acc.max(1, r);
        } else {
            acc.max(1, fabs(r));
        }
        if (r > 0.0 && sk_neg_inf(lo)) acc.max(1, r);
        else if (r < 0.0 && sk_inf(hi)) acc.max(1, -r);
        if (r > 0.0 && !sk_neg_inf(lo)) acc.max(2, r * fabs(xj - lo));
        else if (r < 0.0 && !sk_inf(hi)) acc.max(2, -r * fabs(hi - xj));
        acc.add(3, c[j] * xj + 0.5 * xj * qxj);
        acc.max(4, fabs(x_bar[j] - xj));
        acc.max(5, fabs(xj));
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

// sk checkpoint for LP: step and scale only (no product needed).
__global__ void k_sk_step_scale(const double* __restrict__ x, const double* __restrict__ x_bar, int n,
                                double* __restrict__ partial) {
    __shared__ double smem[kWarps * 2];
    Slots<2, 0u> acc;
    acc.init();
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) {
        acc.max(0, fabs(x_bar[j] - x[j]));
        acc.max(1, fabs(x[j]));
    }
    block_store(acc, partial, smem);
}

// Q x for a diagonal Q (sk_solve.c:909: qx_j = qdiag_j x_j).
__global__ void k_diag_mul(const double* __restrict__ qd, const double* __restrict__ xv, double* __restrict__ out,
                           int n) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) out[j] = qd[j] * xv[j];
}

__global__ void k_init_box_sk(int n, const double* __restrict__ lo, const double* __restrict__ hi,
                              double* __restrict__ x, double* __restrict__ x_bar) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) {
        const double v = box_sk(0.0, lo[j], hi[j]);
        x[j] = v;
        x_bar[j] = v;
    }
}

// =================================================================== solver

enum class Sem { Cuda, Sk };

// Device state of one solve; one allocation carved into aligned vectors.
struct Workspace {
    DevBuf blob;
    double *c = nullptr, *rl = nullptr, *ru = nullptr, *cl = nullptr, *cu = nullptr;
    double *qdiag = nullptr, *tauv = nullptr, *sigv = nullptr;
    double *x[2] = {nullptr, nullptr}, *y[2] = {nullptr, nullptr};
    double *x_bar = nullptr, *qx = nullptr, *x_prev = nullptr, *act = nullptr;
    double *part_a = nullptr, *part_b = nullptr, *part_c = nullptr, *out = nullptr;
    unsigned int* flags = nullptr;
    int n = 0, m = 0;

    int allocate(int n_, int m_, int max_grid) {
        n = n_;
        m = m_;
        const size_t nb = (static_cast<size_t>(n) * 8 + 255) / 256 * 256;
        const size_t mb = (static_cast<size_t>(m) * 8 + 255) / 256 * 256;
        const size_t pb = (static_cast<size_t>(max_grid) * 8 * 8 + 255) / 256 * 256;
        const size_t total = 11 * nb + 6 * mb + 3 * pb + 512;
        if (blob.alloc(total, "cudaMalloc PDHG workspace")) return -1;
        char* p = blob.as<char>();
        auto take = [&](size_t b) { double* r = reinterpret_cast<double*>(p); p += b; return r; };
        c = take(nb); cl = take(nb); cu = take(nb); qdiag = take(nb); tauv = take(nb);
        x[0] = take(nb); x[1] = take(nb); x_bar = take(nb); qx = take(nb); x_prev = take(nb);
        take(nb);
        rl = take(mb); ru = take(mb); sigv = take(mb); y[0] = take(mb); y[1] = take(mb); act = take(mb);
        part_a = take(pb); part_b = take(pb); part_c = take(pb); out = take(256);
        flags = reinterpret_cast<unsigned int*>(take(256));
        return 0;
    }
};

// A host-visible pinned slot for checkpoint results, one per thread.
static double* pinned_out() {
    struct Holder {
        double* p = nullptr;
        ~Holder() { if (p) cudaFreeHost(p); }
    };
    thread_local Holder h;
    if (!h.p && cudaMallocHost(reinterpret_cast<void**>(&h.p), 64 * sizeof(double)) != cudaSuccess) h.p = nullptr;
    return h.p;
}

// Captured iteration graphs, keyed by everything a captured launch bakes in.
struct GraphKey {
    cudaStream_t stream;
    const void* q;
    int has_qdiag, has_steps, chunk, parity, sem;
    double tau, sigma, theta;
    bool operator<(const GraphKey& o) const {
        return std::tie(stream, q, has_qdiag, has_steps, chunk, parity, sem, tau, sigma, theta) <
               std::tie(o.stream, o.q, o.has_qdiag, o.has_steps, o.chunk, o.parity, o.sem, o.tau, o.sigma, o.theta);
    }
};

struct GraphMap {
    std::map<GraphKey, cudaGraphExec_t> map;
    GraphMap() = default;
    GraphMap(const GraphMap&) = delete;
    GraphMap& operator=(const GraphMap&) = delete;
    ~GraphMap() {
        for (auto& kv : map)
            if (kv.second) cudaGraphExecDestroy(kv.second);
    }
};

// Per-plan cache of the fixed-step solver's device state: a later call with
// the same shape reuses the workspace and the graphs captured over it.
struct FixedCache {
    Workspace w;
    GraphMap graphs;
};

struct Solver {
    Sem sem;
    cudaStream_t stream;
    const TileCsr* A;
    const TileCsr* AT;
    const TileCsr* Q;  // explicit Hessian (rows of Q) or null
    Workspace* w;
    bool has_qdiag = false, has_steps = false;
    double tau = 0, sigma = 0, theta = 1;
    int cur = 0;
    int grid_dual = 1, grid_primal = 1, grid_q = 1;
    int launches = 0;
    GraphMap local_graphs;
    GraphMap* graphs = &local_graphs;

    void setup_grids() {
        if (sem == Sem::Cuda) {
            grid_dual = tiled_grid<DualCudaEpi>(*A);
            grid_primal = tiled_grid<PrimalCudaEpi>(*AT);
        } else {
            grid_dual = tiled_grid<DualSkEpi>(*A);
            grid_primal = tiled_grid<PrimalSkEpi>(*AT);
        }
        if (Q) grid_q = tiled_grid<StoreEpi>(*Q);
    }

    // One PDHG iteration from buffer cur into buffer cur^1.
    void iterate(cudaEvent_t* ev) {
        const int nx = cur ^ 1;
        if (ev) cudaEventRecord(ev[0], stream);
        if (sem == Sem::Cuda) {
            launch_tiled(*A, w->x_bar,
                         DualCudaEpi{w->y[cur], w->rl, w->ru, has_steps ? w->sigv : nullptr, sigma, w->y[nx]},
                         stream, grid_dual);
        } else {
            launch_tiled(*A, w->x_bar, DualSkEpi{w->y[cur], w->rl, w->ru, w->sigv, w->y[nx], w->part_c}, stream,
                         grid_dual);
        }
        if (ev) cudaEventRecord(ev[1], stream);
        if (Q) {
            launch_tiled(*Q, w->x[cur], StoreEpi{w->qx}, stream, grid_q);
            ++launches;
        }
        if (ev) cudaEventRecord(ev[2], stream);
        if (sem == Sem::Cuda) {
            launch_tiled(*AT, w->y[nx],
                         PrimalCudaEpi{w->x[cur], w->c, has_steps ? w->tauv : nullptr, Q ? w->qx : nullptr,
                                       has_qdiag ? w->qdiag : nullptr, w->cl, w->cu, tau, theta, w->x[nx], w->x_bar},
                         stream, grid_primal);
        } else {
            launch_tiled(*AT, w->y[nx],
                         PrimalSkEpi{w->x[cur], w->c, w->tauv, Q ? w->qx : nullptr, has_qdiag ? w->qdiag : nullptr,
                                     w->cl, w->cu, w->x[nx], w->x_bar},
                         stream, grid_primal);
        }
        if (ev) cudaEventRecord(ev[3], stream);
        launches += 2;
        cur = nx;
    }

    // Runs k iterations: direct launches with per-kernel events at timing
    // level 2, else replayed CUDA graphs of up to 64 iterations.
    int run(int k) {
        TimingState& ts = timing();
        if (ts.level >= 2) {
            cudaEvent_t ev[4];
            for (auto& e : ev) cudaEventCreate(&e);
            for (int i = 0; i < k; ++i) {
                iterate(ev);
                cudaEventSynchronize(ev[3]);
                float a = 0, b = 0;
                cudaEventElapsedTime(&a, ev[0], ev[1]);
                cudaEventElapsedTime(&b, ev[2], ev[3]);
                ts.last.dual_kernel_ms += a;
                ts.last.primal_kernel_ms += b;
                ts.last.per_kernel_samples += 1;
            }
            for (auto& e : ev) cudaEventDestroy(e);
            return 0;
        }
        while (k > 0) {
            const int chunk = k > 64 ? 64 : k;
            const GraphKey key{stream, Q, has_qdiag ? 1 : 0, has_steps ? 1 : 0, chunk, cur, static_cast<int>(sem),
                               tau, sigma, theta};
            auto it = graphs->map.find(key);
            if (it == graphs->map.end()) {
                const int saved_cur = cur, saved_launches = launches;
                cudaGraph_t g;
                B200_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
                for (int i = 0; i < chunk; ++i) iterate(nullptr);
                B200_TRY(cudaStreamEndCapture(stream, &g), "end capture");
                cudaGraphExec_t exec;
                cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return fail_cuda("graph instantiate", e);
                it = graphs->map.emplace(key, exec).first;
                cur = saved_cur;
                launches = saved_launches;
            }
            B200_TRY(cudaGraphLaunch(it->second, stream), "graph launch");
            launches += chunk * (Q ? 3 : 2);
            cur ^= (chunk & 1);
            k -= chunk;
        }
        return 0;
    }
};

static double now_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}


struct EventTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    bool on;
    cudaStream_t s;
    EventTimer(bool enabled, cudaStream_t stream) : on(enabled), s(stream) {
        if (on) { cudaEventCreate(&a); cudaEventCreate(&b); cudaEventRecord(a, s); }
    }
    double stop() {
        if (!on) return 0.0;
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        on = false;
        return ms;
    }
    ~EventTimer() { if (on) { cudaEventDestroy(a); cudaEventDestroy(b); } }
};

// cuda/src/sankhya_cuda_lp.cu:101-385, on the device.
static int solve_fixed(const SankhyaCudaCSR* matrix, const SankhyaCudaCSR* hessian, const double* qdiag,
                       const double* c, const double* rl, const double* ru, const double* cl, const double* cu,
                       SankhyaCudaLPSettings s, const double* pstep, const double* dstep, double* solution,
                       double* dual_solution, SankhyaCudaLPResult* result) {
    clear_error();
    (void)cudaGetLastError();  // a caller's earlier non-sticky error is not ours
    if (result == nullptr) return fail_msg("null result");
    result->status = -1;
    result->iterations = 0;
    result->objective = std::numeric_limits<double>::quiet_NaN();
    result->maximum_row_violation = std::numeric_limits<double>::infinity();
    result->maximum_step = std::numeric_limits<double>::infinity();
    result->maximum_kkt_residual = std::numeric_limits<double>::infinity();
    result->maximum_dual_residual = std::numeric_limits<double>::infinity();
    result->maximum_complementarity = std::numeric_limits<double>::infinity();
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) return fail_msg("no CUDA device available");
    if (matrix == nullptr || c == nullptr || rl == nullptr || ru == nullptr || cl == nullptr || cu == nullptr ||
        solution == nullptr)
        return fail_msg("null model or solution pointer");
    if (s.max_iterations <= 0 || s.check_every <= 0 || s.theta < 0.0 || s.theta > 1.0 || s.tolerance <= 0.0 ||
        s.time_limit < 0.0)
        return fail_msg("invalid PDHG settings");
    if ((pstep == nullptr) != (dstep == nullptr)) return fail_msg("exactly one step vector given");
    if (pstep == nullptr && (s.tau <= 0.0 || s.sigma <= 0.0)) return fail_msg("non-positive scalar step");
    const int rows = matrix->rows, cols = matrix->cols;
    if (rows < 0 || cols < 0) return fail_msg("negative dimension");
    if (hessian != nullptr && (qdiag != nullptr || hessian->rows != cols || hessian->cols != cols))
        return fail_msg("invalid Hessian");
    // The per-element checks of sankhya_cuda_lp.cu:136-153 run on the device
    // right after the upload (k_validate_fixed), before any iteration.

    std::shared_ptr<Plan> plan, qplan;
    if (get_plan(matrix, &plan)) return -1;
    if (hessian != nullptr && get_plan(hessian, &qplan)) return -1;
    TimingState& ts = timing();
    ts.last = SankhyaB200Timing{};
    const bool timed = ts.level >= 1;
    cudaStream_t stream = engine_stream();
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, plan->device);

    // The plan's cached workspace and graphs, unless another thread holds them.
    std::unique_lock<std::mutex> lock(plan->workspace_mutex, std::try_to_lock);
    std::shared_ptr<FixedCache> cache;
    if (lock.owns_lock()) {
        cache = std::static_pointer_cast<FixedCache>(plan->solve_cache);
        if (!cache || cache->w.n != cols || cache->w.m != rows) {
            plan->solve_cache.reset();
            cache = std::make_shared<FixedCache>();
            if (cache->w.allocate(cols, rows, sms * 8)) return -1;
            plan->solve_cache = cache;
        }
    } else {
        cache = std::make_shared<FixedCache>();
        if (cache->w.allocate(cols, rows, sms * 8)) return -1;
    }
    Workspace* w = &cache->w;

    const size_t nb = sizeof(double) * static_cast<size_t>(cols), mb = sizeof(double) * static_cast<size_t>(rows);
    EventTimer t_h2d(timed, stream);
    if (cols > 0) {
        B200_TRY(cudaMemcpyAsync(w->c, c, nb, cudaMemcpyHostToDevice, stream), "upload c");
        B200_TRY(cudaMemcpyAsync(w->cl, cl, nb, cudaMemcpyHostToDevice, stream), "upload col_lower");
        B200_TRY(cudaMemcpyAsync(w->cu, cu, nb, cudaMemcpyHostToDevice, stream), "upload col_upper");
        if (qdiag) B200_TRY(cudaMemcpyAsync(w->qdiag, qdiag, nb, cudaMemcpyHostToDevice, stream), "upload diagonal");
        if (pstep) B200_TRY(cudaMemcpyAsync(w->tauv, pstep, nb, cudaMemcpyHostToDevice, stream), "upload primal steps");
    }
    if (rows > 0) {
        B200_TRY(cudaMemcpyAsync(w->rl, rl, mb, cudaMemcpyHostToDevice, stream), "upload row_lower");
        B200_TRY(cudaMemcpyAsync(w->ru, ru, mb, cudaMemcpyHostToDevice, stream), "upload row_upper");
        if (dstep) B200_TRY(cudaMemcpyAsync(w->sigv, dstep, mb, cudaMemcpyHostToDevice, stream), "upload dual steps");
        B200_TRY(cudaMemsetAsync(w->y[0], 0, mb, stream), "zero y");
    }
    if (cols > 0) k_init_box_ieee<<<elem_grid(cols), kThreads, 0, stream>>>(cols, w->cl, w->cu, w->x[0], w->x_bar);
    B200_TRY(cudaMemsetAsync(w->flags, 0, sizeof(unsigned int), stream), "clear flags");
    k_validate_fixed<<<elem_grid(std::max(rows, cols)), kThreads, 0, stream>>>(
        cols, rows, w->c, w->cl, w->cu, w->rl, w->ru, pstep ? w->tauv : nullptr, dstep ? w->sigv : nullptr,
        qdiag ? w->qdiag : nullptr, w->flags);
    B200_TRY(cudaGetLastError(), "init launch");
    {
        unsigned int* hflags = reinterpret_cast<unsigned int*>(pinned_out() + 48);
        B200_TRY(cudaMemcpyAsync(hflags, w->flags, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream), "flags");
        B200_TRY(cudaStreamSynchronize(stream), "validation");
        const unsigned int f = *hflags;
        if (f & 1u) return fail_msg("invalid cost or column bound");
        if (f & 2u) return fail_msg("invalid row bound");
        if (f & 4u) return fail_msg("invalid primal step");
        if (f & 8u) return fail_msg("invalid dual step");
        if (f & 16u) return fail_msg("invalid quadratic diagonal");
    }
    ts.last.h2d_ms = t_h2d.stop();

    Solver sv;
    sv.sem = Sem::Cuda;
    sv.stream = stream;
    sv.A = &plan->a;
    sv.AT = &plan->at;
    sv.Q = qplan ? &qplan->a : nullptr;
    sv.w = w;
    // graphs over an explicit Hessian bake in that matrix's pointers: keep them per call
    sv.graphs = hessian == nullptr ? &cache->graphs : &sv.local_graphs;
    sv.has_qdiag = qdiag != nullptr;
    sv.has_steps = pstep != nullptr;
    sv.tau = s.tau;
    sv.sigma = s.sigma;
    sv.theta = s.theta;
    sv.setup_grids();
    const int grid_rows = tiled_grid<CheckRowsCudaEpi>(plan->a);
    const int grid_cols = tiled_grid<CheckColsCudaEpi>(plan->at);
    const int nb_rows = plan->a.ntiles ? grid_rows : 0, nb_cols = plan->at.ntiles ? grid_cols : 0;
    double* host = pinned_out();
    if (!host) return fail_msg("cudaMallocHost checkpoint slot");

    bool have_prev = false;
    int final_iteration = s.max_iterations, it = 0;
    const double started = now_seconds();
    while (it < s.max_iterations) {
        if (s.time_limit > 0.0 && (it + 1) % s.check_every == 1 && now_seconds() - started >= s.time_limit) {
            final_iteration = it;
            result->status = 2;
            break;
        }
        const long long next_ll = (static_cast<long long>(it) / s.check_every + 1) * s.check_every;
        const int next = static_cast<int>(std::min<long long>(next_ll, s.max_iterations));
        {
            EventTimer t_loop(timed, stream);
            if (sv.run(next - it)) return -1;
            ts.last.loop_ms += t_loop.stop();
        }
        ts.last.iterations += next - it;
        it = next;
        // ---- checkpoint: A x and A'y with their residual terms reduced in the epilogues
        EventTimer t_chk(timed, stream);
        const int cx = sv.cur;
        launch_tiled(plan->a, w->x[cx], CheckRowsCudaEpi{w->y[cx], w->rl, w->ru, w->part_a}, stream, grid_rows);
        if (sv.Q) launch_tiled(*sv.Q, w->x[cx], StoreEpi{w->qx}, stream, sv.grid_q);
        launch_tiled(plan->at, w->y[cx],
                     CheckColsCudaEpi{w->x[cx], w->x_prev, w->c, qdiag ? w->qdiag : nullptr, sv.Q ? w->qx : nullptr,
                                      w->cl, w->cu, w->part_b},
                     stream, grid_cols);
        k_combine<5, 0u><<<1, kThreads, 0, stream>>>(w->part_a, nb_rows, w->out);
        k_combine<7, 1u << 1><<<1, kThreads, 0, stream>>>(w->part_b, nb_cols, w->out + 8);
        sv.launches += 4 + (sv.Q ? 1 : 0);
        B200_TRY(cudaMemcpyAsync(host, w->out, 16 * sizeof(double), cudaMemcpyDeviceToHost, stream), "read checkpoint");
        B200_TRY(cudaStreamSynchronize(stream), "checkpoint");
        ts.last.checkpoint_ms += t_chk.stop();
        ts.last.checkpoints += 1;
        const double nonfinite = std::max(host[0], host[8]);
        const double objective = host[9];
        if (nonfinite > 0.0 || !std::isfinite(objective)) {
            result->status = -2;
            ts.last.kernel_launches = sv.launches;
            return -2;
        }
        const double violation = std::max(0.0, host[1]);
        const double kkt = std::max(host[2], host[12]);
        const double dual_residual = std::max(host[3], host[13]);
        const double complementarity = std::max(host[4], host[14]);
        const double step = have_prev ? host[10] : std::numeric_limits<double>::infinity();
        const double scale = std::max(1.0, host[11]);
        have_prev = true;
        result->objective = objective;
        result->maximum_row_violation = violation;
        result->maximum_step = step;
        result->maximum_kkt_residual = kkt;
        result->maximum_dual_residual = dual_residual;
        result->maximum_complementarity = complementarity / (1.0 + std::fabs(objective));
        if (violation <= s.tolerance && step <= s.tolerance * scale && kkt <= s.tolerance &&
            dual_residual <= s.tolerance && result->maximum_complementarity <= s.tolerance) {
            final_iteration = it;
            result->status = 0;
            break;
        }
    }
    if (result->status < 0) result->status = 1;
    result->iterations = final_iteration;
    EventTimer t_d2h(timed, stream);
    if (cols > 0) B200_TRY(cudaMemcpyAsync(solution, w->x[sv.cur], nb, cudaMemcpyDeviceToHost, stream), "download x");
    if (dual_solution != nullptr && rows > 0)
        B200_TRY(cudaMemcpyAsync(dual_solution, w->y[sv.cur], mb, cudaMemcpyDeviceToHost, stream), "download y");
    B200_TRY(cudaStreamSynchronize(stream), "download");
    ts.last.d2h_ms = t_d2h.stop();
    ts.last.kernel_launches = sv.launches;
    if (ts.last.per_kernel_samples > 0) {
        ts.last.dual_kernel_ms /= ts.last.per_kernel_samples;
        ts.last.primal_kernel_ms /= ts.last.per_kernel_samples;
    }
    return 0;
}

// ================================================================ sk bridge

// Device copies of a matrix given in CSC (the reference's sk_csc) and of its
// CSR. The CSC is uploaded as stored and is the CSR of the transpose; the CSR is
// built on the device by a stable transpose (each row's columns ascending, the
// order of sk_solve's scatter csc_mv).
struct OwnedPair {
    DevBuf ptr, idx, val, tiles, tptr, tidx, tval, ttiles;
    TileCsr a, at;
    int upload_csc(int rows, int cols, const int* p, const int* i, const double* x) {
        const int nnz = p[cols];
        const size_t nz = static_cast<size_t>(nnz > 0 ? nnz : 1);
        std::vector<int> tb = build_tiles(cols, p);
        if (ptr.alloc((static_cast<size_t>(rows) + 1) * 4, "cudaMalloc A") || idx.alloc(nz * 4, "cudaMalloc A") ||
            val.alloc(nz * 8, "cudaMalloc A") || tptr.alloc((static_cast<size_t>(cols) + 1) * 4, "cudaMalloc A^T") ||
            tidx.alloc(nz * 4, "cudaMalloc A^T") || tval.alloc(nz * 8, "cudaMalloc A^T") ||
            ttiles.alloc(tb.size() * 4, "cudaMalloc tiles"))
            return -1;
        B200_TRY(cudaMemcpy(tptr.p, p, tptr.bytes, cudaMemcpyHostToDevice), "upload A^T");
        if (nnz) {
            B200_TRY(cudaMemcpy(tidx.p, i, static_cast<size_t>(nnz) * 4, cudaMemcpyHostToDevice), "upload A^T");
            B200_TRY(cudaMemcpy(tval.p, x, static_cast<size_t>(nnz) * 8, cudaMemcpyHostToDevice), "upload A^T");
        }
        B200_TRY(cudaMemcpy(ttiles.p, tb.data(), ttiles.bytes, cudaMemcpyHostToDevice), "upload tiles");
        if (device_transpose(cols, rows, nnz, tptr.as<int>(), tidx.as<int>(), tval.as<double>(), ptr.as<int>(),
                             idx.as<int>(), val.as<double>(), nullptr))
            return -1;
        std::vector<int> rp(static_cast<size_t>(rows) + 1);
        B200_TRY(cudaMemcpy(rp.data(), ptr.p, rp.size() * 4, cudaMemcpyDeviceToHost), "read A offsets");
        std::vector<int> ta = build_tiles(rows, rp.data());
        if (tiles.alloc(ta.size() * 4, "cudaMalloc tiles")) return -1;
        B200_TRY(cudaMemcpy(tiles.p, ta.data(), tiles.bytes, cudaMemcpyHostToDevice), "upload tiles");
        a = TileCsr{rows, cols, nnz, static_cast<int>(ta.size()) / 2 - 1, ptr.as<int>(), idx.as<int>(),
                    val.as<double>(), tiles.as<int2>()};
        at = TileCsr{cols, rows, nnz, static_cast<int>(tb.size()) / 2 - 1, tptr.as<int>(), tidx.as<int>(),
                     tval.as<double>(), ttiles.as<int2>()};
        return 0;
    }
};

static int sk_loop(const sk_model* m, const sk_options* o, double* x, double* y, double* activity,
                   SankhyaB200LoopResult* res) {
    const int n = m->ncol, r = m->nrow;
    const int max_it = (o && o->iteration_limit > 0 && o->iteration_limit < 2147483647LL)
                           ? static_cast<int>(o->iteration_limit) : 100000;
    const int check_every = 20;
    const double ptol = o->primal_tol, dtol = o->dual_tol, time_limit = o->time_limit;
    const sk_csc* q = m->Q;

    // Host setup, exactly the reference's order of additions
    // (c/src/sk_solve.c:60-80 matrix_norm_bound, :863-870 diagonal test, :880-896 steps).
    std::vector<double> row_mass(static_cast<size_t>(r), 0.0), col_mass(static_cast<size_t>(n), 0.0);
    std::vector<double> anorm_rows(static_cast<size_t>(r), 0.0);
    double col_max = 0.0, row_max = 0.0;
    for (int j = 0; j < n; ++j) {
        double col_sum = 0.0;
        for (int p = m->A.p[j]; p < m->A.p[j + 1]; ++p) {
            const double v = std::fabs(m->A.x[p]);
            col_sum += v;
            anorm_rows[m->A.i[p]] += v;
        }
        if (col_sum > col_max) col_max = col_sum;
    }
    for (int i = 0; i < r; ++i) if (anorm_rows[i] > row_max) row_max = anorm_rows[i];
    const double anorm = (r && n) ? std::sqrt(col_max * row_max) : 0.0;
    for (int j = 0; j < n; ++j) {
        for (int p = m->A.p[j]; p < m->A.p[j + 1]; ++p) {
            row_mass[m->A.i[p]] += std::fabs(m->A.x[p]);
            col_mass[j] += std::fabs(m->A.x[p]);
        }
        if (q) for (int p = q->p[j]; p < q->p[j + 1]; ++p) col_mass[j] += std::fabs(q->x[p]);
    }
    std::vector<double> tauv(static_cast<size_t>(n)), sigv(static_cast<size_t>(r));
    for (int j = 0; j < n; ++j) tauv[j] = 0.9 / (1.0 + col_mass[j]);
    for (int i = 0; i < r; ++i) sigv[i] = 0.9 / (1.0 + row_mass[i]);
    bool diagonal = false;
    std::vector<double> qd;
    if (q) {
        diagonal = true;
        qd.assign(static_cast<size_t>(n), 0.0);
        for (int j = 0; j < n && diagonal; ++j)
            for (int p = q->p[j]; p < q->p[j + 1]; ++p) {
                if (q->i[p] != j) { diagonal = false; break; }
                qd[j] += q->x[p];
            }
    }

    cudaStream_t stream = engine_stream();
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    OwnedPair ap;
    if (ap.upload_csc(r, n, m->A.p, m->A.i, m->A.x)) return -1;
    OwnedPair qp;
    const bool explicit_q = q && !diagonal;
    if (explicit_q && qp.upload_csc(n, n, q->p, q->i, q->x)) return -1;
    Workspace w;
    if (w.allocate(n, r, sms * 8)) return -1;
    const size_t nb = sizeof(double) * static_cast<size_t>(n), mb = sizeof(double) * static_cast<size_t>(r);
    if (n) {
        B200_TRY(cudaMemcpyAsync(w.c, m->c, nb, cudaMemcpyHostToDevice, stream), "upload c");
        B200_TRY(cudaMemcpyAsync(w.cl, m->clow, nb, cudaMemcpyHostToDevice, stream), "upload clow");
        B200_TRY(cudaMemcpyAsync(w.cu, m->cupp, nb, cudaMemcpyHostToDevice, stream), "upload cupp");
        B200_TRY(cudaMemcpyAsync(w.tauv, tauv.data(), nb, cudaMemcpyHostToDevice, stream), "upload tau");
        if (q && diagonal) B200_TRY(cudaMemcpyAsync(w.qdiag, qd.data(), nb, cudaMemcpyHostToDevice, stream), "upload qdiag");
        k_init_box_sk<<<elem_grid(n), kThreads, 0, stream>>>(n, w.cl, w.cu, w.x[0], w.x_bar);
    }
    if (r) {
        B200_TRY(cudaMemcpyAsync(w.rl, m->rlow, mb, cudaMemcpyHostToDevice, stream), "upload rlow");
        B200_TRY(cudaMemcpyAsync(w.ru, m->rupp, mb, cudaMemcpyHostToDevice, stream), "upload rupp");
        B200_TRY(cudaMemcpyAsync(w.sigv, sigv.data(), mb, cudaMemcpyHostToDevice, stream), "upload sigma");
        B200_TRY(cudaMemsetAsync(w.y[0], 0, mb, stream), "zero y");
    }
    B200_TRY(cudaGetLastError(), "init launch");

    Solver sv;
    sv.sem = Sem::Sk;
    sv.stream = stream;
    sv.A = &ap.a;
    sv.AT = &ap.at;
    sv.Q = explicit_q ? &qp.a : nullptr;
    sv.w = &w;
    sv.has_qdiag = q && diagonal;
    sv.has_steps = true;
    sv.setup_grids();
    const int nb_dual = ap.a.ntiles ? sv.grid_dual : 0;
    const int grid_rows = tiled_grid<CheckRowsSkEpi>(ap.a);
    const int grid_cols = tiled_grid<CheckColsSkEpi>(ap.at);
    const int nb_rows = ap.a.ntiles ? grid_rows : 0, nb_cols = ap.at.ntiles ? grid_cols : 0;
    const int grid_step = elem_grid(n);
    double* host = pinned_out();
    if (!host) return fail_msg("cudaMallocHost checkpoint slot");
    TimingState& ts = timing();
    ts.last = SankhyaB200Timing{};

    int it = 0, converged = 0;
    double dual_step = std::numeric_limits<double>::infinity();
    bool activity_is_ax = false;
    const double start = now_seconds();
    while (it < max_it) {
        const int next = std::min((it / check_every + 1) * check_every, max_it);
        if (sv.run(next - it)) return -1;
        ts.last.iterations += next - it;
        it = next;
        const int cx = sv.cur;
        // dual step of the last iteration (written by every dual launch)
        k_combine<1, 0u><<<1, kThreads, 0, stream>>>(w.part_c, nb_dual, w.out + 24);
        if (time_limit > 0.0 && now_seconds() - start >= time_limit) {
            activity_is_ax = false;
            break;
        }
        launch_tiled(ap.a, w.x[cx], CheckRowsSkEpi{w.y[cx], w.rl, w.ru, w.act, w.part_a}, stream, grid_rows);
        k_combine<3, 0u><<<1, kThreads, 0, stream>>>(w.part_a, nb_rows, w.out);
        if (explicit_q) launch_tiled(qp.a, w.x[cx], StoreEpi{w.qx}, stream, sv.grid_q);
        if (q && diagonal && n) k_diag_mul<<<elem_grid(n), kThreads, 0, stream>>>(w.qdiag, w.x[cx], w.qx, n);
        if (q) {
            launch_tiled(ap.at, w.y[cx], CheckColsSkEpi{w.x[cx], w.x_bar, w.c, w.qx, w.cl, w.cu, w.part_b}, stream,
                         grid_cols);
            k_combine<6, 1u << 3><<<1, kThreads, 0, stream>>>(w.part_b, nb_cols, w.out + 8);
        } else {
            if (n) k_sk_step_scale<<<grid_step, kThreads, 0, stream>>>(w.x[cx], w.x_bar, n, w.part_b);
            k_combine<2, 0u><<<1, kThreads, 0, stream>>>(w.part_b, n ? grid_step : 0, w.out + 16);
        }
        B200_TRY(cudaMemcpyAsync(host, w.out, 32 * sizeof(double), cudaMemcpyDeviceToHost, stream), "read checkpoint");
        B200_TRY(cudaStreamSynchronize(stream), "checkpoint");
        ts.last.checkpoints += 1;
        activity_is_ax = true;
        dual_step = host[24];
        const double violation = host[0];
        double step, scale;
        bool ready = true;
        if (q) {
            step = host[12];
            scale = std::max(1.0, host[13]);
            const double pobj = m->objshift + host[11];
            const double pinf = std::max(std::max(0.0, host[0]), std::max(0.0, host[8]));
            const double dinf = std::max(std::max(0.0, host[1]), std::max(0.0, host[9]));
            const double comp = std::max(host[2], host[10]) / (1.0 + std::fabs(pobj));
            const double score = pinf + dinf + comp;
            ready = std::isfinite(score) && score <= 100.0 * (ptol + 2.0 * dtol);
        } else {
            step = host[16];
            scale = std::max(1.0, host[17]);
        }
        if (violation <= ptol && step <= ptol * scale && dual_step <= dtol * (1.0 + anorm) && ready) {
            converged = 1;
            break;
        }
    }
    if (!activity_is_ax) {
        // the reference leaves A x_bar of the last iteration in `activity`
        B200_TRY(cudaMemcpyAsync(host, w.out + 24, sizeof(double), cudaMemcpyDeviceToHost, stream), "read dual step");
        if (r) launch_tiled(ap.a, w.x_bar, StoreEpi{w.act}, stream, tiled_grid<StoreEpi>(ap.a));
        B200_TRY(cudaStreamSynchronize(stream), "activity");
        dual_step = host[0];
    }
    if (n) B200_TRY(cudaMemcpyAsync(x, w.x[sv.cur], nb, cudaMemcpyDeviceToHost, stream), "download x");
    if (r) {
        B200_TRY(cudaMemcpyAsync(y, w.y[sv.cur], mb, cudaMemcpyDeviceToHost, stream), "download y");
        B200_TRY(cudaMemcpyAsync(activity, w.act, mb, cudaMemcpyDeviceToHost, stream), "download activity");
    }
    B200_TRY(cudaStreamSynchronize(stream), "download");
    res->iterations = it;
    res->converged = converged;
    res->numeric_failure = 0;
    res->dual_step = dual_step;
    res->anorm = anorm;
    res->seconds = now_seconds() - start;
    ts.last.kernel_launches = sv.launches;
    return 0;
}

}  // namespace b200

using namespace b200;

extern "C" int sankhya_cuda_lp_pdhg(const SankhyaCudaCSR* matrix, const double* c, const double* row_lower,
                                    const double* row_upper, const double* col_lower, const double* col_upper,
                                    SankhyaCudaLPSettings settings, double* solution, SankhyaCudaLPResult* result) {
    return solve_fixed(matrix, nullptr, nullptr, c, row_lower, row_upper, col_lower, col_upper, settings, nullptr,
                       nullptr, solution, nullptr, result);
}

extern "C" int sankhya_cuda_diagonal_qp_pdhg(const SankhyaCudaCSR* matrix, const double* quadratic_diagonal,
                                             const double* c, const double* row_lower, const double* row_upper,
                                             const double* col_lower, const double* col_upper,
                                             SankhyaCudaLPSettings settings, double* solution,
                                             SankhyaCudaLPResult* result) {
    if (quadratic_diagonal == nullptr) return fail_msg("null quadratic diagonal");
    return solve_fixed(matrix, nullptr, quadratic_diagonal, c, row_lower, row_upper, col_lower, col_upper, settings,
                       nullptr, nullptr, solution, nullptr, result);
}

extern "C" int sankhya_cuda_sparse_qp_pdhg(const SankhyaCudaCSR* matrix, const SankhyaCudaCSR* hessian,
                                           const double* c, const double* row_lower, const double* row_upper,
                                           const double* col_lower, const double* col_upper,
                                           SankhyaCudaLPSettings settings, double* solution,
                                           SankhyaCudaLPResult* result) {
    if (hessian == nullptr) return fail_msg("null Hessian");
    return solve_fixed(matrix, hessian, nullptr, c, row_lower, row_upper, col_lower, col_upper, settings, nullptr,
                       nullptr, solution, nullptr, result);
}

extern "C" int sankhya_cuda_qp_pdhg_preconditioned(const SankhyaCudaCSR* matrix, const SankhyaCudaCSR* hessian,
                                                   const double* quadratic_diagonal, const double* c,
                                                   const double* row_lower, const double* row_upper,
                                                   const double* col_lower, const double* col_upper,
                                                   const double* primal_steps, const double* dual_steps,
                                                   SankhyaCudaLPSettings settings, double* solution,
                                                   SankhyaCudaLPResult* result) {
    if (primal_steps == nullptr || dual_steps == nullptr) return fail_msg("null step vector");
    return solve_fixed(matrix, hessian, quadratic_diagonal, c, row_lower, row_upper, col_lower, col_upper, settings,
                       primal_steps, dual_steps, solution, nullptr, result);
}

extern "C" int sankhya_cuda_qp_pdhg_preconditioned_with_dual(
    const SankhyaCudaCSR* matrix, const SankhyaCudaCSR* hessian, const double* quadratic_diagonal, const double* c,
    const double* row_lower, const double* row_upper, const double* col_lower, const double* col_upper,
    const double* primal_steps, const double* dual_steps, SankhyaCudaLPSettings settings, double* solution,
    double* dual_solution, SankhyaCudaLPResult* result) {
    if (primal_steps == nullptr || dual_steps == nullptr || dual_solution == nullptr)
        return fail_msg("null step vector or dual output");
    return solve_fixed(matrix, hessian, quadratic_diagonal, c, row_lower, row_upper, col_lower, col_upper, settings,
                       primal_steps, dual_steps, solution, dual_solution, result);
}

// What sk_model_validate requires of a model (c/src/sk_core.c:126-155), except
// vartype, which the loop never reads: a well-formed CSC for A (and Q) and finite
// costs with ordered, non-NaN bounds. sk_solve checks this before its loop; this
// entry checks it again because its host setup and device schedules index through
// the CSC arrays.
static bool sk_csc_ok(const sk_csc* a, int rows, int cols) {
    if (!a || a->nrow != rows || a->ncol != cols || a->nzmax < 0 || !a->p || a->p[0] != 0) return false;
    const int nnz = a->p[cols];
    if (nnz < 0 || nnz > a->nzmax || (nnz > 0 && (!a->i || !a->x))) return false;
    for (int j = 0; j < cols; ++j)
        if (a->p[j] > a->p[j + 1] || a->p[j + 1] > nnz) return false;
    for (int p = 0; p < nnz; ++p)
        if (a->i[p] < 0 || a->i[p] >= rows || !std::isfinite(a->x[p])) return false;
    return true;
}

static bool sk_model_ok(const sk_model* m) {
    if (!sk_csc_ok(&m->A, m->nrow, m->ncol) || (m->Q && !sk_csc_ok(m->Q, m->ncol, m->ncol))) return false;
    for (int j = 0; j < m->ncol; ++j)
        if (!std::isfinite(m->c[j]) || std::isnan(m->clow[j]) || std::isnan(m->cupp[j]) || m->clow[j] > m->cupp[j])
            return false;
    for (int i = 0; i < m->nrow; ++i)
        if (std::isnan(m->rlow[i]) || std::isnan(m->rupp[i]) || m->rlow[i] > m->rupp[i]) return false;
    return true;
}

extern "C" int sankhya_b200_pdhg_loop(const sk_model* model, const sk_options* options, double* x, double* y,
                                      double* activity, SankhyaB200LoopResult* result) {
    clear_error();
    if (!model || !options || !result || model->nrow < 0 || model->ncol < 0) {
        fail_msg("invalid sk loop arguments");
        return 1;
    }
    const int n = model->ncol, r = model->nrow;
    if ((n && (!x || !model->c || !model->clow || !model->cupp)) || (r && (!y || !activity || !model->rlow || !model->rupp)) ||
        !model->A.p || (model->Q && (!model->Q->p || model->Q->nrow != n || model->Q->ncol != n)) ||
        options->primal_tol <= 0.0 || options->dual_tol <= 0.0) {
        fail_msg("invalid sk loop arguments");
        return 1;
    }
    if (!sk_model_ok(model)) {
        fail_msg("invalid sk model (malformed CSC, non-finite cost, or NaN / crossed bound)");
        return 1;
    }
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
        fail_msg("no CUDA device available");
        return 7;
    }
    *result = SankhyaB200LoopResult{};
    (void)cudaGetLastError();  // a caller's earlier non-sticky error is not ours
    const int rc = sk_loop(model, options, x, y, activity, result);
    return rc == 0 ? 0 : 7;
}
