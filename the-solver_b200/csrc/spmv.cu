// Public sparse primitives: device-pointer SpMV / transpose SpMV / AXPY on the
// default stream, and the host-array SpMV / AXPY conveniences.
//
// Reference behaviour followed: cuda/src/sankhya_cuda.cu:78-106 (argument
// checks, early returns for empty shapes), :165-197 (device entry points),
// :199-284 (host entry points: copy in, compute, copy out).
#include "engine.cuh"

namespace b200 {

__global__ void k_axpy(int n, double alpha, const double* __restrict__ x, double* __restrict__ y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += blockDim.x * gridDim.x)
        y[i] = fma(alpha, x[i], y[i]);
}

static int ensure_device() {
    int devices = 0;
    cudaError_t e = cudaGetDeviceCount(&devices);
    if (e != cudaSuccess) return fail_cuda("cudaGetDeviceCount", e);
    return devices == 0 ? fail_msg("no CUDA device available") : 0;
}

}  // namespace b200

using namespace b200;

extern "C" int sankhya_cuda_spmv_device_f64(const SankhyaCudaCSR* matrix, const double* device_x,
                                            double* device_y) {
    clear_error();
    if (ensure_device()) return -1;
    if (matrix == nullptr) return fail_msg("null device CSR pointer");
    if (matrix->rows == 0) return 0;
    if (device_y == nullptr || (matrix->cols > 0 && device_x == nullptr))
        return fail_msg("null device CSR or vector pointer");
    std::shared_ptr<Plan> plan;
    if (get_plan(matrix, &plan)) return -1;
    const TileCsr& A = plan->a;
    launch_tiled(A, device_x, StoreEpi{device_y}, 0, tiled_grid<StoreEpi>(A));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail_cuda("CSR SpMV launch", e);
}

extern "C" int sankhya_cuda_spmv_transpose_device_f64(const SankhyaCudaCSR* matrix,
                                                      const double* device_y, double* device_x) {
    clear_error();
    if (ensure_device()) return -1;
    if (matrix == nullptr) return fail_msg("null device CSR pointer");
    if (matrix->rows == 0 || matrix->cols == 0) return 0;
    if (device_y == nullptr || device_x == nullptr)
        return fail_msg("null device CSR or transpose vector pointer");
    std::shared_ptr<Plan> plan;
    if (get_plan(matrix, &plan)) return -1;
    const TileCsr& AT = plan->at;
    launch_tiled(AT, device_y, StoreEpi{device_x}, 0, tiled_grid<StoreEpi>(AT));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail_cuda("transpose SpMV launch", e);
}

extern "C" int sankhya_cuda_axpy_device_f64(int n, double alpha, const double* device_x, double* device_y) {
    clear_error();
    if (ensure_device()) return -1;
    if (n < 0) return fail_msg("negative vector dimension");
    if (n == 0) return 0;
    if (device_x == nullptr || device_y == nullptr) return fail_msg("null device vector pointer");
    k_axpy<<<elem_grid(n), kThreads>>>(n, alpha, device_x, device_y);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : fail_cuda("AXPY launch", e);
}

extern "C" int sankhya_cuda_spmv_f64(int rows, int cols, int nnz, const int* row_offsets,
                                     const int* column_indices, const double* values,
                                     const double* x, double* y) {
    clear_error();
    if (rows < 0 || cols < 0 || nnz < 0) return fail_msg("negative CSR dimension");
    if (row_offsets == nullptr || y == nullptr ||
        (nnz > 0 && (column_indices == nullptr || values == nullptr)) || (cols > 0 && x == nullptr))
        return fail_msg("null CSR or vector pointer");
    if (rows == 0) return 0;
    // The reference launches on these arrays unchecked. An offset outside [0, nnz],
    // decreasing offsets or a column outside [0, cols) would send the kernel outside
    // its buffers, so those (and only those) are rejected here, before any device work;
    // every input the reference reads in bounds behaves as there.
    if (row_offsets[0] < 0 || row_offsets[rows] > nnz) return fail_msg("invalid CSR row-offset endpoints");
    for (int r = 0; r < rows; ++r)
        if (row_offsets[r] > row_offsets[r + 1]) return fail_msg("invalid CSR row-offset ordering");
    for (int p = row_offsets[0]; p < row_offsets[rows]; ++p)
        if (column_indices[p] < 0 || column_indices[p] >= cols) return fail_msg("invalid CSR column index");
    if (ensure_device()) return -1;
    std::vector<int> tiles = build_tiles(rows, row_offsets);
    DevBuf d_ptr, d_idx, d_val, d_x, d_y, d_tiles;
    if (d_ptr.alloc(sizeof(int) * (static_cast<size_t>(rows) + 1), "cudaMalloc row_offsets") ||
        d_idx.alloc(sizeof(int) * static_cast<size_t>(nnz), "cudaMalloc column_indices") ||
        d_val.alloc(sizeof(double) * static_cast<size_t>(nnz), "cudaMalloc values") ||
        d_x.alloc(sizeof(double) * static_cast<size_t>(cols), "cudaMalloc x") ||
        d_y.alloc(sizeof(double) * static_cast<size_t>(rows), "cudaMalloc y") ||
        d_tiles.alloc(sizeof(int) * tiles.size(), "cudaMalloc tiles"))
        return -1;
    B200_TRY(cudaMemcpy(d_ptr.p, row_offsets, d_ptr.bytes, cudaMemcpyHostToDevice), "cudaMemcpy row_offsets");
    if (nnz > 0) {
        B200_TRY(cudaMemcpy(d_idx.p, column_indices, d_idx.bytes, cudaMemcpyHostToDevice), "cudaMemcpy column_indices");
        B200_TRY(cudaMemcpy(d_val.p, values, d_val.bytes, cudaMemcpyHostToDevice), "cudaMemcpy values");
    }
    if (cols > 0) B200_TRY(cudaMemcpy(d_x.p, x, d_x.bytes, cudaMemcpyHostToDevice), "cudaMemcpy x");
    B200_TRY(cudaMemcpy(d_tiles.p, tiles.data(), d_tiles.bytes, cudaMemcpyHostToDevice), "cudaMemcpy tiles");
    TileCsr A;
    A.rows = rows;
    A.cols = cols;
    A.nnz = nnz;
    A.ptr = d_ptr.as<int>();
    A.idx = d_idx.as<int>();
    A.val = d_val.as<double>();
    A.ntiles = static_cast<int>(tiles.size()) / 2 - 1;
    A.tile = d_tiles.as<int2>();
    launch_tiled(A, d_x.as<double>(), StoreEpi{d_y.as<double>()}, 0, tiled_grid<StoreEpi>(A));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda("CSR SpMV launch", e);
    B200_TRY(cudaMemcpy(y, d_y.p, d_y.bytes, cudaMemcpyDeviceToHost), "cudaMemcpy y");
    return 0;
}

extern "C" int sankhya_cuda_axpy_f64(int n, double alpha, const double* x, double* y) {
    clear_error();
    if (n < 0) return fail_msg("negative vector dimension");
    if (n == 0) return 0;
    if (x == nullptr || y == nullptr) return fail_msg("null vector pointer");
    if (ensure_device()) return -1;
    DevBuf dx, dy;
    if (dx.alloc(sizeof(double) * static_cast<size_t>(n), "cudaMalloc x") ||
        dy.alloc(sizeof(double) * static_cast<size_t>(n), "cudaMalloc y"))
        return -1;
    B200_TRY(cudaMemcpy(dx.p, x, dx.bytes, cudaMemcpyHostToDevice), "cudaMemcpy AXPY input");
    B200_TRY(cudaMemcpy(dy.p, y, dy.bytes, cudaMemcpyHostToDevice), "cudaMemcpy AXPY input");
    k_axpy<<<elem_grid(n), kThreads>>>(n, alpha, dx.as<double>(), dy.as<double>());
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda("AXPY launch", e);
    B200_TRY(cudaMemcpy(y, dy.p, dy.bytes, cudaMemcpyDeviceToHost), "cudaMemcpy AXPY output");
    return 0;
}
