// Allocation-free variant of the fixed-step PDHG of sankhya_cuda_lp_pdhg.
//
// For callers that cannot allocate device memory while they solve: an embedding
// runtime that hands out all device memory from its own pool (a cudaMalloc behind
// its back fails or breaks its accounting), a process with a fixed device-memory
// budget that must not grow after start-up, or a service that cannot take the
// device-wide synchronisation cudaMalloc/cudaFree can impose on other streams. The fixed-step solve's scratch (iterate
// ping-pong buffers, x_bar, the checkpoint's x_prev, reduction partials, result
// slots) lives in this file-scope array instead of a cudaMalloc'd workspace.
// Every GPU that loads this library reserves it until the process exits.
#include "engine.cuh"
#include "fixed_epi.cuh"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <limits>
#include <mutex>

namespace b200 {
namespace {

double wall_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

constexpr size_t kNoAllocScratchDoubles = size_t(2) << 20;  // 16 MiB per device
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of g_noalloc_scratch per device, looked up once per device
// (cudaGetSymbolAddress with that device current). The first call on a device
// does this set-up; that first call should come before any stream capture.
double* noalloc_scratch_address(int device) {
    static std::mutex mu;
    static double* addr[64] = {};
    if (device < 0 || device >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return nullptr;
        addr[device] = static_cast<double*>(p);
    }
    return addr[device];
}

template <class Epi>
int noalloc_grid(const TileCsr& A, int sms) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void*>(&k_tiled<Epi, double>),
                                                  kThreads, 0);
    const int resident = std::max(1, per_sm) * std::max(1, sms);
    return std::max(1, std::min((A.ntiles + kWarps - 1) / kWarps, resident));
}

}  // namespace
}  // namespace b200

extern "C" int sankhya_b200_lp_pdhg_device_noalloc(const SankhyaCudaCSR* matrix, const double* d_c,
                                                   const double* d_row_lower, const double* d_row_upper,
                                                   const double* d_col_lower, const double* d_col_upper,
                                                   SankhyaCudaLPSettings s, double* d_solution,
                                                   SankhyaCudaLPResult* result) {
    using namespace b200;
    clear_error();
    (void)cudaGetLastError();
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
    if (matrix == nullptr || d_c == nullptr || d_row_lower == nullptr || d_row_upper == nullptr ||
        d_col_lower == nullptr || d_col_upper == nullptr || d_solution == nullptr)
        return fail_msg("null model or solution pointer");
    if (s.max_iterations <= 0 || s.check_every <= 0 || s.theta < 0.0 || s.theta > 1.0 || s.tolerance <= 0.0 ||
        s.time_limit < 0.0 || s.tau <= 0.0 || s.sigma <= 0.0)
        return fail_msg("invalid PDHG settings");
    std::shared_ptr<Plan> plan;
    if (find_plan(matrix, &plan)) return -1;  // also rejects a matrix made on another device
    const int rows = matrix->rows, cols = matrix->cols;
    const int device = plan->device;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    // scratch layout (doubles): x[2], x_bar, x_prev (cols each), y[2] (rows each),
    // two reduction-partial areas, 32 result slots and one flag word
    const size_t nb = (static_cast<size_t>(cols) + 31) / 32 * 32, mb = (static_cast<size_t>(rows) + 31) / 32 * 32;
    const size_t pb = static_cast<size_t>(sms) * 8 * 8;
    const size_t need = 4 * nb + 2 * mb + 2 * pb + 64;
    if (need > kNoAllocScratchDoubles) {
        char msg[200];
        std::snprintf(msg, sizeof(msg),
                      "problem too large for the allocation-free scratch: needs %zu doubles "
                      "(4*cols + 2*rows + partials), the limit is %zu",
                      need, kNoAllocScratchDoubles);
        return fail_msg(msg);
    }
    double* base = noalloc_scratch_address(device);
    if (!base) return fail_msg("cudaGetSymbolAddress of the allocation-free scratch failed");
    double* x[2] = {base, base + nb};
    double* x_bar = base + 2 * nb;
    double* x_prev = base + 3 * nb;
    double* y[2] = {base + 4 * nb, base + 4 * nb + mb};
    double* part_a = base + 4 * nb + 2 * mb;
    double* part_b = part_a + pb;
    double* out = part_b + pb;
    unsigned int* flags = reinterpret_cast<unsigned int*>(out + 32);
    cudaStream_t stream = 0;  // the legacy default stream, like the reference's device primitives

    // the previous call's contents stay in the array: clear what must start at zero
    B200_TRY(cudaMemsetAsync(flags, 0, sizeof(unsigned int), stream), "clear flags");
    if (rows) B200_TRY(cudaMemsetAsync(y[0], 0, sizeof(double) * rows, stream), "zero y");
    k_validate_fixed<<<elem_grid(std::max(rows, cols)), kThreads, 0, stream>>>(
        cols, rows, d_c, d_col_lower, d_col_upper, d_row_lower, d_row_upper, nullptr, nullptr, nullptr, flags);
    if (cols) k_init_box_ieee<<<elem_grid(cols), kThreads, 0, stream>>>(cols, d_col_lower, d_col_upper, x[0], x_bar);
    B200_TRY(cudaGetLastError(), "init launch");
    unsigned int hflags = 0;
    B200_TRY(cudaMemcpy(&hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost), "validation");
    if (hflags & 1u) return fail_msg("invalid cost or column bound");
    if (hflags & 2u) return fail_msg("invalid row bound");

    const TileCsr& A = plan->a;
    const TileCsr& AT = plan->at;
    const int gd = noalloc_grid<DualCudaEpi>(A, sms), gp = noalloc_grid<PrimalCudaEpi>(AT, sms);
    const int gr = noalloc_grid<CheckRowsCudaEpi>(A, sms), gc = noalloc_grid<CheckColsCudaEpi>(AT, sms);
    const int nb_rows = A.ntiles ? gr : 0, nb_cols = AT.ntiles ? gc : 0;
    int cur = 0, it = 0, final_iteration = s.max_iterations;
    bool have_prev = false;
    double host[16];
    const double started = wall_seconds();
    while (it < s.max_iterations) {
        if (s.time_limit > 0.0 && (it + 1) % s.check_every == 1 && wall_seconds() - started >= s.time_limit) {
            final_iteration = it;
            result->status = 2;
            break;
        }
        const long long next_ll = (static_cast<long long>(it) / s.check_every + 1) * s.check_every;
        const int next = static_cast<int>(std::min<long long>(next_ll, s.max_iterations));
        for (; it < next; ++it) {
            const int nx = cur ^ 1;
            launch_tiled(A, x_bar, DualCudaEpi{y[cur], d_row_lower, d_row_upper, nullptr, s.sigma, y[nx]}, stream, gd);
            launch_tiled(AT, y[nx],
                         PrimalCudaEpi{x[cur], d_c, nullptr, nullptr, nullptr, d_col_lower, d_col_upper, s.tau, s.theta,
                                       x[nx], x_bar},
                         stream, gp);
            cur = nx;
        }
        launch_tiled(A, x[cur], CheckRowsCudaEpi{y[cur], d_row_lower, d_row_upper, part_a}, stream, gr);
        launch_tiled(AT, y[cur],
                     CheckColsCudaEpi{x[cur], x_prev, d_c, nullptr, nullptr, d_col_lower, d_col_upper, part_b}, stream,
                     gc);
        k_combine<5, 0u><<<1, kThreads, 0, stream>>>(part_a, nb_rows, out);
        k_combine<7, 1u << 1><<<1, kThreads, 0, stream>>>(part_b, nb_cols, out + 8);
        B200_TRY(cudaGetLastError(), "checkpoint launch");
        B200_TRY(cudaMemcpy(host, out, 16 * sizeof(double), cudaMemcpyDeviceToHost), "read checkpoint");
        const double objective = host[9];
        if (std::max(host[0], host[8]) > 0.0 || !std::isfinite(objective)) {
            result->status = -2;
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
    if (cols) B200_TRY(cudaMemcpyAsync(d_solution, x[cur], sizeof(double) * cols, cudaMemcpyDeviceToDevice, stream),
                       "copy solution");
    B200_TRY(cudaStreamSynchronize(stream), "solve");
    return 0;
}
