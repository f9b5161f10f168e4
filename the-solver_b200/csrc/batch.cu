// Batched PDHG: many independent LPs of uneven size advanced together in the
// same fused launches, each with the first-order loop of sk_solve
// (c/src/sk_solve.c:849-954): diagonal steps tau_j = 0.9/(1 + |A_:j|_1),
// sigma_i = 0.9/(1 + |A_i:|_1), x_bar = 2 x_new - x_old, and every
// check_every iterations its own gates: row violation <= primal_tol,
// max |x_bar - x| <= primal_tol * max(1, |x|_inf), max |y_new - y| <=
// dual_tol * (1 + anorm_k) with anorm_k = sqrt(max column mass * max row mass)
// of that LP.
//
// The batch is one block-diagonal CSR: LP k owns rows [row_seg[k], row_seg[k+1])
// and columns [col_seg[k], col_seg[k+1]). One PDHG iteration of the whole batch
// is the usual two fused launches (the A-side dual step, the A'-side primal
// step); a window of iterations is one CUDA graph. The gates are evaluated on
// the device with per-LP maxima (atomic max on the bit patterns of non-negative
// doubles, so the result does not depend on the order); an LP that passes is
// frozen (its iterates are carried through unchanged) and the host reads only
// the number of LPs still running. Per LP the arithmetic is exactly the
// single-LP loop's, so every LP's iterates equal a separate solve's bit for bit.
#include "batch_common.cuh"

#include <algorithm>
#include <cstring>
#include <limits>
#include <map>

namespace b200 {

namespace {

using batch::atomic_max_nonneg;
using batch::k_abs_sums;
using batch::sk_inf;
using batch::sk_neg_inf;
using batch::slot_value;

// sk_solve.c:901-906 with LP freezing
struct BatchDualEpi {
    const double* __restrict__ y;
    const double* __restrict__ rl;
    const double* __restrict__ ru;
    const double* __restrict__ sig;
    const int* __restrict__ seg;
    const int* __restrict__ done;
    double* __restrict__ y_new;
    using Acc = NoAcc;
    struct Row {
        double y, lo, hi, s;
        int frozen;
    };
    __device__ __forceinline__ Row load(int i) const { return Row{y[i], rl[i], ru[i], sig[i], done[seg[i]]}; }
    __device__ __forceinline__ void store(int i, double act, const Row& r, Acc&) const {
        if (r.frozen) {
            y_new[i] = r.y;
            return;
        }
        const double trial = dadd(r.y, dmul(r.s, act));
        y_new[i] = dsub(trial, dmul(r.s, box_sk(ddiv(trial, r.s), r.lo, r.hi)));
    }
    __device__ __forceinline__ void finish(Acc&, double*) const {}
};

// sk_solve.c:918-923 (LP, no Q) with LP freezing
struct BatchPrimalEpi {
    const double* __restrict__ x;
    const double* __restrict__ c;
    const double* __restrict__ tauv;
    const double* __restrict__ cl;
    const double* __restrict__ cu;
    const int* __restrict__ seg;
    const int* __restrict__ done;
    double* __restrict__ x_new;
    double* __restrict__ x_bar;
    using Acc = NoAcc;
    struct Row {
        double x, c, t, lo, hi;
        int frozen;
    };
    __device__ __forceinline__ Row load(int j) const { return Row{x[j], c[j], tauv[j], cl[j], cu[j], done[seg[j]]}; }
    __device__ __forceinline__ void store(int j, double g, const Row& r, Acc&) const {
        if (r.frozen) {
            x_new[j] = r.x;
            return;
        }
        double xn = dsub(r.x, dmul(r.t, dadd(dadd(r.c, 0.0), g)));
        xn = box_sk(xn, r.lo, r.hi);
        x_new[j] = xn;
        x_bar[j] = dsub(dmul(2.0, xn), r.x);
    }
    __device__ __forceinline__ void finish(Acc&, double*) const {}
};

// Check over rows: A x (stored as the activity), per-LP row violation
// (sk_solve.c:82-95) and max |y - y_prev| of the last iteration.
struct BatchRowsEpi {
    const double* __restrict__ y;
    const double* __restrict__ y_prev;
    const double* __restrict__ rl;
    const double* __restrict__ ru;
    const int* __restrict__ seg;
    const int* __restrict__ done;
    double* __restrict__ act_out;
    unsigned long long* __restrict__ viol;
    unsigned long long* __restrict__ dstep;
    using Acc = NoAcc;
    __device__ __forceinline__ void row(int i, double act, Acc&) const {
        const int k = seg[i];
        if (done[k]) return;
        act_out[i] = act;
        double v = 0.0;
        if (!sk_neg_inf(rl[i]) && rl[i] - act > v) v = rl[i] - act;
        if (!sk_inf(ru[i]) && act - ru[i] > v) v = act - ru[i];
        atomic_max_nonneg(&viol[k], v);
        atomic_max_nonneg(&dstep[k], fabs(y[i] - y_prev[i]));
    }
    __device__ __forceinline__ void finish(Acc&, double*) const {}
};

__global__ void k_batch_cols(int n, const double* __restrict__ x, const double* __restrict__ x_bar,
                             const int* __restrict__ seg, const int* __restrict__ done,
                             unsigned long long* __restrict__ scale, unsigned long long* __restrict__ step) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) {
        const int k = seg[j];
        if (done[k]) continue;
        atomic_max_nonneg(&scale[k], fabs(x[j]));
        atomic_max_nonneg(&step[k], fabs(x_bar[j] - x[j]));
    }
}

// One thread per LP: the gates of sk_solve.c:926-953; clears the maxima.
__global__ void k_batch_gate(int batch, int iteration, int last, double ptol, double dtol,
                             unsigned long long* __restrict__ viol, unsigned long long* __restrict__ dstep,
                             unsigned long long* __restrict__ scale, unsigned long long* __restrict__ step,
                             const unsigned long long* __restrict__ cmax, const unsigned long long* __restrict__ rmax,
                             int* __restrict__ done, int* __restrict__ iters, double* __restrict__ report,
                             unsigned int* __restrict__ remaining) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < batch; k += blockDim.x * gridDim.x) {
        if (done[k]) continue;
        const double v = slot_value(viol[k]), ds = slot_value(dstep[k]);
        const double sc = fmax(1.0, slot_value(scale[k])), st = slot_value(step[k]);
        const double anorm = sqrt(slot_value(cmax[k]) * slot_value(rmax[k]));
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

__global__ void k_steps_and_max(int len, const double* __restrict__ mass, const int* __restrict__ seg,
                                double* __restrict__ steps, unsigned long long* __restrict__ segmax) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < len; j += blockDim.x * gridDim.x) {
        steps[j] = 0.9 / (1.0 + mass[j]);
        atomic_max_nonneg(&segmax[seg[j]], mass[j]);
    }
}

// Block-diagonal structure: every nonzero of row i lies in the columns of i's LP.
__global__ void k_check_blocks(int rows, const int* __restrict__ ptr, const int* __restrict__ idx,
                               const int* __restrict__ rseg, const int* __restrict__ cseg,
                               unsigned int* __restrict__ bad) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += blockDim.x * gridDim.x) {
        const int k = rseg[r];
        for (int p = ptr[r]; p < ptr[r + 1]; ++p)
            if (cseg[idx[p]] != k) { atomicOr(bad, 1u); break; }
    }
}

__global__ void k_init_box(int n, const double* __restrict__ lo, const double* __restrict__ hi,
                           double* __restrict__ x, double* __restrict__ x_bar) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) {
        const double v = box_sk(0.0, lo[j], hi[j]);
        x[j] = v;
        x_bar[j] = v;
    }
}

using batch::now_s;

}  // namespace

}  // namespace b200

using namespace b200;

extern "C" void sankhya_b200_batch_default_settings(SankhyaB200BatchSettings* s) {
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->struct_version = 1;
    s->max_iterations = 100000;
    s->check_every = 20;
    s->primal_tol = 1e-7;
    s->dual_tol = 1e-7;
    s->time_limit = 0.0;
}

extern "C" int sankhya_b200_batch_pdhg(const SankhyaCudaCSR* matrix, int batch, const int* row_segments,
                                       const int* col_segments, const double* c, const double* rlow,
                                       const double* rupp, const double* clow, const double* cupp,
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
    if (!matrix || batch <= 0 || !row_segments || !col_segments || !c || !rlow || !rupp || !clow || !cupp || !x_out ||
        !results)
        return fail_msg("invalid batch arguments");
    if (s.max_iterations <= 0 || s.check_every <= 0 || !(s.primal_tol > 0.0) || !(s.dual_tol > 0.0) ||
        s.time_limit < 0.0)
        return fail_msg("invalid batch settings");
    const int m = matrix->rows, n = matrix->cols;
    if (row_segments[0] != 0 || col_segments[0] != 0 || row_segments[batch] != m || col_segments[batch] != n)
        return fail_msg("segments do not cover the matrix");
    for (int k = 0; k < batch; ++k)
        if (row_segments[k] > row_segments[k + 1] || col_segments[k] > col_segments[k + 1])
            return fail_msg("segments are not ordered");
    for (int j = 0; j < n; ++j)
        if (!std::isfinite(c[j]) || std::isnan(clow[j]) || std::isnan(cupp[j]) || clow[j] > cupp[j])
            return fail_msg("invalid cost or column bound");
    for (int i = 0; i < m; ++i)
        if (std::isnan(rlow[i]) || std::isnan(rupp[i]) || rlow[i] > rupp[i]) return fail_msg("invalid row bound");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) return fail_msg("no CUDA device available");
    std::shared_ptr<Plan> plan;
    if (get_plan(matrix, &plan)) return -1;
    const double t0 = now_s();
    cudaStream_t stream = engine_stream();

    // segment maps
    std::vector<int> rseg(static_cast<size_t>(m)), cseg(static_cast<size_t>(n));
    for (int k = 0; k < batch; ++k) {
        for (int i = row_segments[k]; i < row_segments[k + 1]; ++i) rseg[i] = k;
        for (int j = col_segments[k]; j < col_segments[k + 1]; ++j) cseg[j] = k;
    }
    const size_t nb = (static_cast<size_t>(n) * 8 + 255) / 256 * 256, mb = (static_cast<size_t>(m) * 8 + 255) / 256 * 256;
    const size_t kb = (static_cast<size_t>(batch) * 8 + 255) / 256 * 256;
    DevBuf blob;
    // 8 n-vectors + the column segment map, 7 m-vectors + the row segment map,
    // 12 per-LP slots, counters
    if (blob.alloc(9 * nb + 8 * mb + 12 * kb + 4096, "cudaMalloc batch workspace")) return -1;
    char* p = blob.as<char>();
    auto take = [&](size_t b) { char* r = p; p += b; return r; };
    double *dc = reinterpret_cast<double*>(take(nb)), *dcl = reinterpret_cast<double*>(take(nb)),
           *dcu = reinterpret_cast<double*>(take(nb)), *tau = reinterpret_cast<double*>(take(nb)),
           *xb0 = reinterpret_cast<double*>(take(nb)), *xb1 = reinterpret_cast<double*>(take(nb)),
           *xbar = reinterpret_cast<double*>(take(nb)), *cmass = reinterpret_cast<double*>(take(nb));
    double *drl = reinterpret_cast<double*>(take(mb)), *dru = reinterpret_cast<double*>(take(mb)),
           *sig = reinterpret_cast<double*>(take(mb)), *yb0 = reinterpret_cast<double*>(take(mb)),
           *yb1 = reinterpret_cast<double*>(take(mb)), *act = reinterpret_cast<double*>(take(mb)),
           *rmass = reinterpret_cast<double*>(take(mb));
    int* d_rseg = reinterpret_cast<int*>(take(mb));
    int* d_cseg = reinterpret_cast<int*>(take(nb));
    unsigned long long* viol = reinterpret_cast<unsigned long long*>(take(kb));
    unsigned long long* dstep = reinterpret_cast<unsigned long long*>(take(kb));
    unsigned long long* scale = reinterpret_cast<unsigned long long*>(take(kb));
    unsigned long long* step = reinterpret_cast<unsigned long long*>(take(kb));
    unsigned long long* cmax = reinterpret_cast<unsigned long long*>(take(kb));
    unsigned long long* rmax = reinterpret_cast<unsigned long long*>(take(kb));
    int* done = reinterpret_cast<int*>(take(kb));
    int* iters = reinterpret_cast<int*>(take(kb));
    double* report = reinterpret_cast<double*>(take(4 * kb));
    unsigned int* counters = reinterpret_cast<unsigned int*>(take(256));
    const size_t n8 = sizeof(double) * static_cast<size_t>(n), m8 = sizeof(double) * static_cast<size_t>(m);
    if (n) {
        B200_TRY(cudaMemcpyAsync(dc, c, n8, cudaMemcpyHostToDevice, stream), "upload c");
        B200_TRY(cudaMemcpyAsync(dcl, clow, n8, cudaMemcpyHostToDevice, stream), "upload clow");
        B200_TRY(cudaMemcpyAsync(dcu, cupp, n8, cudaMemcpyHostToDevice, stream), "upload cupp");
        B200_TRY(cudaMemcpyAsync(d_cseg, cseg.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream), "upload seg");
    }
    if (m) {
        B200_TRY(cudaMemcpyAsync(drl, rlow, m8, cudaMemcpyHostToDevice, stream), "upload rlow");
        B200_TRY(cudaMemcpyAsync(dru, rupp, m8, cudaMemcpyHostToDevice, stream), "upload rupp");
        B200_TRY(cudaMemcpyAsync(d_rseg, rseg.data(), sizeof(int) * m, cudaMemcpyHostToDevice, stream), "upload seg");
        B200_TRY(cudaMemsetAsync(yb0, 0, m8, stream), "zero y");
    }
    B200_TRY(cudaMemsetAsync(viol, 0, 6 * kb, stream), "zero maxima");
    B200_TRY(cudaMemsetAsync(done, 0, 2 * kb, stream), "zero flags");
    B200_TRY(cudaMemsetAsync(counters, 0, 256, stream), "zero counters");
    const TileCsr& A = plan->a;
    const TileCsr& AT = plan->at;
    const int ge = elem_grid(std::max(m, n));
    if (m) k_check_blocks<<<elem_grid(m), kThreads, 0, stream>>>(m, A.ptr, A.idx, d_rseg, d_cseg, counters + 1);
    if (m) k_abs_sums<<<elem_grid(m), kThreads, 0, stream>>>(m, A.ptr, A.val, rmass);
    if (n) k_abs_sums<<<elem_grid(n), kThreads, 0, stream>>>(n, AT.ptr, AT.val, cmass);
    if (n) k_steps_and_max<<<elem_grid(n), kThreads, 0, stream>>>(n, cmass, d_cseg, tau, cmax);
    if (m) k_steps_and_max<<<elem_grid(m), kThreads, 0, stream>>>(m, rmass, d_rseg, sig, rmax);
    if (n) k_init_box<<<elem_grid(n), kThreads, 0, stream>>>(n, dcl, dcu, xb0, xbar);
    B200_TRY(cudaGetLastError(), "batch setup");
    unsigned int* host_counters = nullptr;
    B200_TRY(cudaMallocHost(reinterpret_cast<void**>(&host_counters), 64), "cudaMallocHost");
    struct Free {
        unsigned int* p;
        ~Free() { cudaFreeHost(p); }
    } free_host{host_counters};
    B200_TRY(cudaMemcpyAsync(host_counters, counters, 8, cudaMemcpyDeviceToHost, stream), "read");
    B200_TRY(cudaStreamSynchronize(stream), "batch setup");
    if (host_counters[1]) return fail_msg("matrix is not block-diagonal over the given segments");

    double* xb[2] = {xb0, xb1};
    double* yb[2] = {yb0, yb1};
    const int grid_d = tiled_grid<BatchDualEpi>(A), grid_p = tiled_grid<BatchPrimalEpi>(AT);
    const int grid_r = tiled_grid<BatchRowsEpi>(A);
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
        launch_tiled(A, xbar, BatchDualEpi{yb[cur], drl, dru, sig, d_rseg, done, yb[nx]}, stream, grid_d);
        launch_tiled(AT, yb[nx], BatchPrimalEpi{xb[cur], dc, tau, dcl, dcu, d_cseg, done, xb[nx], xbar}, stream,
                     grid_p);
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
            launches += 2 * chunk;
            cur ^= (chunk & 1);
            k -= chunk;
        }
        it = next;
        const bool last = it >= s.max_iterations;
        ++checks;
        B200_TRY(cudaMemsetAsync(counters, 0, 4, stream), "zero counter");
        launch_tiled(A, xb[cur], BatchRowsEpi{yb[cur], yb[cur ^ 1], drl, dru, d_rseg, done, act, viol, dstep}, stream,
                     grid_r);
        if (n) k_batch_cols<<<elem_grid(n), kThreads, 0, stream>>>(n, xb[cur], xbar, d_cseg, done, scale, step);
        k_batch_gate<<<elem_grid(batch), kThreads, 0, stream>>>(batch, it, last ? 1 : 0, s.primal_tol, s.dual_tol, viol,
                                                                dstep, scale, step, cmax, rmax, done, iters, report,
                                                                counters);
        launches += 3;
        B200_TRY(cudaMemcpyAsync(host_counters, counters, 4, cudaMemcpyDeviceToHost, stream), "read");
        B200_TRY(cudaStreamSynchronize(stream), "batch check");
        if (host_counters[0] == 0) break;
        if (s.time_limit > 0.0 && now_s() - t0 >= s.time_limit) {
            timed_out = true;
            break;
        }
    }
    const double loop_ms = loop_events.stop(stream);
    std::vector<int> h_done(static_cast<size_t>(batch)), h_iters(static_cast<size_t>(batch));
    std::vector<double> h_report(static_cast<size_t>(batch) * 4);
    B200_TRY(cudaMemcpyAsync(x_out, xb[cur], n8, cudaMemcpyDeviceToHost, stream), "download x");
    if (y_out && m) B200_TRY(cudaMemcpyAsync(y_out, yb[cur], m8, cudaMemcpyDeviceToHost, stream), "download y");
    B200_TRY(cudaMemcpyAsync(h_done.data(), done, sizeof(int) * batch, cudaMemcpyDeviceToHost, stream), "download");
    B200_TRY(cudaMemcpyAsync(h_iters.data(), iters, sizeof(int) * batch, cudaMemcpyDeviceToHost, stream), "download");
    B200_TRY(cudaMemcpyAsync(h_report.data(), report, sizeof(double) * 4 * batch, cudaMemcpyDeviceToHost, stream),
             "download");
    B200_TRY(cudaStreamSynchronize(stream), "batch download");
    for (int k = 0; k < batch; ++k) {
        SankhyaB200BatchResult& r = results[k];
        r.status = h_done[k] ? 0 : (timed_out ? 2 : 1);
        r.iterations = h_done[k] ? h_iters[k] : it;
        double obj = 0.0;
        for (int j = col_segments[k]; j < col_segments[k + 1]; ++j) obj += c[j] * x_out[j];
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
