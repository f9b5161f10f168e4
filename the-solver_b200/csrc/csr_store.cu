// Device CSR store: validation + upload (sankhya_cuda_csr_create/destroy), the
// private transpose and row-tile schedule kept beside each matrix, the
// thread-local error text, the engine stream and launch sizing.
//
// Reference behaviour followed: cuda/src/sankhya_cuda.cu:10-21 (error text),
// :116-152 (validation order and messages, destroy-before-create, zeroed
// handle on failure), :154-163 (destroy).
#include "engine.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <unordered_map>

namespace b200 {

namespace {
thread_local char g_last_error[512] = "";
}

int fail_msg(const char* message) {
    std::snprintf(g_last_error, sizeof(g_last_error), "%s", message);
    return -1;
}

int fail_cuda(const char* operation, cudaError_t error) {
    std::snprintf(g_last_error, sizeof(g_last_error), "%s: %s", operation, cudaGetErrorString(error));
    return -1;
}

void clear_error() { g_last_error[0] = '\0'; }

// ------------------------------------------------------------------ tiles

std::vector<int> build_tiles(int rows, const int* ptr) {
    std::vector<int> tiles;  // (row, nonzero) pairs
    tiles.reserve(static_cast<size_t>(rows) / 8 + 4);
    int r = 0;
    while (r < rows) {
        tiles.push_back(r);
        tiles.push_back(ptr[r]);
        const int len = ptr[r + 1] - ptr[r];
        if (len > kChunkNnz) {
            ++r;
            continue;
        }
        const int start = r;
        int nnz = 0;
        while (r < rows && r - start < kChunkRows) {
            const int l = ptr[r + 1] - ptr[r];
            if (nnz + l > kChunkNnz) break;
            nnz += l;
            ++r;
        }
    }
    tiles.push_back(rows);
    tiles.push_back(ptr[rows]);
    return tiles;
}

// ------------------------------------------------------------------ plans

Plan::~Plan() {
    int current = -1;
    cudaGetDevice(&current);
    if (current != device) cudaSetDevice(device);
    cudaFree(d_tile_a);
    cudaFree(d_at_ptr);
    cudaFree(d_at_idx);
    cudaFree(d_at_val);
    cudaFree(d_tile_at);
    cudaFree(d_a_idx);
    cudaFree(d_a_val);
    solve_cache.reset();
    if (current >= 0 && current != device) cudaSetDevice(current);
}

static int upload(void** dst, const void* src, size_t bytes, const char* what) {
    if (bytes == 0) { *dst = nullptr; return 0; }
    cudaError_t e = cudaMalloc(dst, bytes);
    if (e != cudaSuccess) { *dst = nullptr; return fail_cuda(what, e); }
    e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail_cuda(what, e);
    return 0;
}

int make_plan(const SankhyaCudaCSR* m, const int* h_ptr, const int* h_idx, const double* h_val,
              std::shared_ptr<Plan>* out) {
    auto plan = std::make_shared<Plan>();
    cudaGetDevice(&plan->device);
    plan->src_idx = m->device_column_indices;
    plan->src_val = m->device_values;
    const int rows = m->rows, cols = m->cols, nnz = m->nnz;

    std::vector<int> tiles_a = build_tiles(rows, h_ptr);
    // A^T built on the device by a stable transpose: each column of A (row of
    // A^T) lists its row indices ascending, the order of a counting sort over the
    // rows of A.
    const size_t nnz_alloc = static_cast<size_t>(nnz > 0 ? nnz : 1);
    B200_TRY(cudaMalloc(reinterpret_cast<void**>(&plan->d_at_ptr), (static_cast<size_t>(cols) + 1) * sizeof(int)),
             "cudaMalloc A^T offsets");
    B200_TRY(cudaMalloc(reinterpret_cast<void**>(&plan->d_at_idx), nnz_alloc * sizeof(int)), "cudaMalloc A^T indices");
    B200_TRY(cudaMalloc(reinterpret_cast<void**>(&plan->d_at_val), nnz_alloc * sizeof(double)), "cudaMalloc A^T values");
    if (device_transpose(rows, cols, nnz, static_cast<const int*>(m->device_row_offsets),
                         static_cast<const int*>(m->device_column_indices), static_cast<const double*>(m->device_values),
                         plan->d_at_ptr, plan->d_at_idx, plan->d_at_val, nullptr))
        return -1;
    std::vector<int> at_ptr(static_cast<size_t>(cols) + 1, 0);
    B200_TRY(cudaMemcpy(at_ptr.data(), plan->d_at_ptr, at_ptr.size() * sizeof(int), cudaMemcpyDeviceToHost),
             "read A^T offsets");
    std::vector<int> tiles_at = build_tiles(cols, at_ptr.data());

    if (upload(reinterpret_cast<void**>(&plan->d_tile_a), tiles_a.data(), tiles_a.size() * sizeof(int), "cudaMalloc tiles(A)") ||
        upload(reinterpret_cast<void**>(&plan->d_tile_at), tiles_at.data(), tiles_at.size() * sizeof(int), "cudaMalloc tiles(A^T)"))
        return -1;
    const int* a_idx = static_cast<const int*>(m->device_column_indices);
    const double* a_val = static_cast<const double*>(m->device_values);
    if ((reinterpret_cast<uintptr_t>(a_idx) | reinterpret_cast<uintptr_t>(a_val)) & 15u) {
        if (upload(reinterpret_cast<void**>(&plan->d_a_idx), h_idx, static_cast<size_t>(nnz) * sizeof(int), "cudaMalloc A indices") ||
            upload(reinterpret_cast<void**>(&plan->d_a_val), h_val, static_cast<size_t>(nnz) * sizeof(double), "cudaMalloc A values"))
            return -1;
        a_idx = plan->d_a_idx;
        a_val = plan->d_a_val;
    }

    plan->a.rows = rows;
    plan->a.cols = cols;
    plan->a.nnz = nnz;
    plan->a.ptr = static_cast<const int*>(m->device_row_offsets);
    plan->a.idx = a_idx;
    plan->a.val = a_val;
    plan->a.ntiles = static_cast<int>(tiles_a.size()) / 2 - 1;
    plan->a.tile = reinterpret_cast<const int2*>(plan->d_tile_a);
    plan->at.rows = cols;
    plan->at.cols = rows;
    plan->at.nnz = nnz;
    plan->at.ptr = plan->d_at_ptr;
    plan->at.idx = plan->d_at_idx;
    plan->at.val = plan->d_at_val;
    plan->at.ntiles = static_cast<int>(tiles_at.size()) / 2 - 1;
    plan->at.tile = reinterpret_cast<const int2*>(plan->d_tile_at);
    *out = std::move(plan);
    return 0;
}

namespace {
std::mutex g_registry_mutex;
std::unordered_map<const void*, std::shared_ptr<Plan>>& registry() {
    static auto* map = new std::unordered_map<const void*, std::shared_ptr<Plan>>();
    return *map;
}
}  // namespace

void register_plan(const void* key, std::shared_ptr<Plan> plan) {
    std::lock_guard<std::mutex> lock(g_registry_mutex);
    registry()[key] = std::move(plan);
}

void unregister_plan(const void* key) {
    std::shared_ptr<Plan> doomed;
    {
        std::lock_guard<std::mutex> lock(g_registry_mutex);
        auto it = registry().find(key);
        if (it == registry().end()) return;
        doomed = std::move(it->second);
        registry().erase(it);
    }
}

// The registered plan of m when it describes the same arrays (offsets, indices,
// values and sizes), else null.
static std::shared_ptr<Plan> registered(const SankhyaCudaCSR* m) {
    std::lock_guard<std::mutex> lock(g_registry_mutex);
    auto it = registry().find(m->device_row_offsets);
    if (it == registry().end()) return nullptr;
    const Plan& p = *it->second;
    if (p.a.rows != m->rows || p.a.cols != m->cols || p.a.nnz != m->nnz || p.src_idx != m->device_column_indices ||
        p.src_val != m->device_values)
        return nullptr;
    return it->second;
}

// A plan's arrays are memory of the device that was current when it was made.
static int check_device(const Plan& plan) {
    int current = -1;
    B200_TRY(cudaGetDevice(&current), "cudaGetDevice");
    if (current == plan.device) return 0;
    char msg[160];
    std::snprintf(msg, sizeof(msg), "the matrix was created on device %d but device %d is current", plan.device,
                  current);
    return fail_msg(msg);
}

int find_plan(const SankhyaCudaCSR* m, std::shared_ptr<Plan>* out) {
    if (m == nullptr) return fail_msg("null device CSR pointer");
    std::shared_ptr<Plan> p = registered(m);
    if (!p) return fail_msg("this entry point needs a matrix made by sankhya_cuda_csr_create and not changed since");
    if (check_device(*p)) return -1;
    *out = std::move(p);
    return 0;
}

int get_plan(const SankhyaCudaCSR* m, std::shared_ptr<Plan>* out) {
    if (m == nullptr) return fail_msg("null device CSR pointer");
    if (std::shared_ptr<Plan> p = registered(m)) {
        if (check_device(*p)) return -1;
        *out = std::move(p);
        return 0;
    }
    // A handle filled by the caller: bring its CSR back once and plan it.
    if (m->rows < 0 || m->cols < 0 || m->nnz < 0) return fail_msg("invalid device CSR dimensions");
    if (m->device_row_offsets == nullptr || (m->nnz > 0 && (m->device_column_indices == nullptr || m->device_values == nullptr)))
        return fail_msg("null device CSR pointer");
    std::vector<int> ptr(static_cast<size_t>(m->rows) + 1);
    std::vector<int> idx(static_cast<size_t>(m->nnz));
    std::vector<double> val(static_cast<size_t>(m->nnz));
    B200_TRY(cudaMemcpy(ptr.data(), m->device_row_offsets, ptr.size() * sizeof(int), cudaMemcpyDeviceToHost), "read CSR offsets");
    if (m->nnz > 0) {
        B200_TRY(cudaMemcpy(idx.data(), m->device_column_indices, idx.size() * sizeof(int), cudaMemcpyDeviceToHost), "read CSR indices");
        B200_TRY(cudaMemcpy(val.data(), m->device_values, val.size() * sizeof(double), cudaMemcpyDeviceToHost), "read CSR values");
    }
    if (ptr[0] != 0 || ptr[static_cast<size_t>(m->rows)] != m->nnz) return fail_msg("invalid CSR row-offset endpoints");
    for (int r = 0; r < m->rows; ++r)
        if (ptr[r] < 0 || ptr[r] > ptr[r + 1] || ptr[r + 1] > m->nnz) return fail_msg("invalid CSR row-offset ordering");
    for (int p = 0; p < m->nnz; ++p)
        if (idx[p] < 0 || idx[p] >= m->cols) return fail_msg("invalid CSR column index or coefficient");
    return make_plan(m, ptr.data(), idx.data(), val.data(), out);
}

// ------------------------------------------------------------ stream, grid

cudaStream_t engine_stream() {
    struct PerThread {
        cudaStream_t streams[64] = {};
        ~PerThread() {
            for (cudaStream_t s : streams)
                if (s) cudaStreamDestroy(s);
        }
    };
    thread_local PerThread state;
    int device = 0;
    cudaGetDevice(&device);
    if (device < 0 || device >= 64) return nullptr;
    if (!state.streams[device]) cudaStreamCreateWithFlags(&state.streams[device], cudaStreamNonBlocking);
    return state.streams[device];
}

int grid_for(const void* kernel, int ntiles, int dynamic_smem) {
    struct Entry { const void* k; int device; int blocks; };
    static std::mutex mu;
    static std::vector<Entry> cache;
    int device = 0;
    cudaGetDevice(&device);
    int resident = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        for (const Entry& e : cache)
            if (e.k == kernel && e.device == device) resident = e.blocks;
        if (resident == 0) {
            int per_sm = 0, sms = 0;
            if (dynamic_smem > 48 * 1024)
                cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dynamic_smem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, dynamic_smem);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
            resident = std::max(1, per_sm) * std::max(1, sms);
            cache.push_back({kernel, device, resident});
        }
    }
    return std::max(1, std::min(ntiles, resident));
}

TimingState& timing() {
    thread_local TimingState state;
    return state;
}

// ------------------------------------------------------------ small kernels

__global__ void k_fill(double* __restrict__ out, double value, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += blockDim.x * gridDim.x) out[i] = value;
}

__global__ void k_copy(double* __restrict__ dst, const double* __restrict__ src, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += blockDim.x * gridDim.x) dst[i] = src[i];
}

}  // namespace b200

using namespace b200;

extern "C" const char* sankhya_cuda_last_error(void) { return g_last_error; }

extern "C" void sankhya_b200_set_timing(int level) { timing().level = level; }

extern "C" void sankhya_b200_last_timing(SankhyaB200Timing* out) {
    if (out) *out = timing().last;
}

extern "C" void sankhya_cuda_csr_destroy(SankhyaCudaCSR* matrix) {
    if (matrix == nullptr) return;
    if (matrix->device_row_offsets) unregister_plan(matrix->device_row_offsets);
    cudaFree(matrix->device_row_offsets);
    cudaFree(matrix->device_column_indices);
    cudaFree(matrix->device_values);
    matrix->rows = matrix->cols = matrix->nnz = 0;
    matrix->device_row_offsets = nullptr;
    matrix->device_column_indices = nullptr;
    matrix->device_values = nullptr;
}

extern "C" int sankhya_cuda_csr_create(SankhyaCudaCSR* matrix, int rows, int cols, int nnz,
                                       const int* row_offsets, const int* column_indices,
                                       const double* values) {
    clear_error();
    if (matrix == nullptr || row_offsets == nullptr || rows < 0 || cols < 0 || nnz < 0 ||
        (nnz > 0 && (column_indices == nullptr || values == nullptr)))
        return fail_msg("invalid persistent CSR input");
    if (row_offsets[0] != 0 || row_offsets[rows] != nnz) return fail_msg("invalid CSR row-offset endpoints");
    for (int r = 0; r < rows; ++r)
        if (row_offsets[r] < 0 || row_offsets[r] > row_offsets[r + 1] || row_offsets[r + 1] > nnz)
            return fail_msg("invalid CSR row-offset ordering");
    for (int p = 0; p < nnz; ++p)
        if (column_indices[p] < 0 || column_indices[p] >= cols || !std::isfinite(values[p]))
            return fail_msg("invalid CSR column index or coefficient");
    int devices = 0;
    cudaError_t e = cudaGetDeviceCount(&devices);
    if (e != cudaSuccess) return fail_cuda("cudaGetDeviceCount", e);
    if (devices == 0) return fail_msg("no CUDA device available");
    sankhya_cuda_csr_destroy(matrix);
    matrix->rows = rows;
    matrix->cols = cols;
    matrix->nnz = nnz;
    std::shared_ptr<Plan> plan;
    if (upload(&matrix->device_row_offsets, row_offsets, sizeof(int) * (static_cast<size_t>(rows) + 1), "cudaMalloc row_offsets") ||
        (nnz > 0 && upload(&matrix->device_column_indices, column_indices, sizeof(int) * static_cast<size_t>(nnz), "cudaMalloc column_indices")) ||
        (nnz > 0 && upload(&matrix->device_values, values, sizeof(double) * static_cast<size_t>(nnz), "cudaMalloc values")) ||
        make_plan(matrix, row_offsets, column_indices, values, &plan)) {
        char saved[512];
        std::snprintf(saved, sizeof(saved), "%s", g_last_error);
        sankhya_cuda_csr_destroy(matrix);
        fail_msg(saved);
        return -1;
    }
    register_plan(matrix->device_row_offsets, std::move(plan));
    return 0;
}

extern "C" int sankhya_b200_csr_transpose(const SankhyaCudaCSR* matrix, int* at_ptr, int* at_idx, double* at_val) {
    clear_error();
    (void)cudaGetLastError();
    if (!matrix || !at_ptr || (matrix->nnz > 0 && (!at_idx || !at_val))) return fail_msg("invalid transpose arguments");
    std::shared_ptr<Plan> plan;
    if (get_plan(matrix, &plan)) return -1;
    const TileCsr& at = plan->at;
    B200_TRY(cudaMemcpy(at_ptr, at.ptr, (static_cast<size_t>(at.rows) + 1) * sizeof(int), cudaMemcpyDeviceToHost),
             "read A^T offsets");
    if (at.nnz > 0) {
        B200_TRY(cudaMemcpy(at_idx, at.idx, static_cast<size_t>(at.nnz) * sizeof(int), cudaMemcpyDeviceToHost),
                 "read A^T indices");
        B200_TRY(cudaMemcpy(at_val, at.val, static_cast<size_t>(at.nnz) * sizeof(double), cudaMemcpyDeviceToHost),
                 "read A^T values");
    }
    return 0;
}
