/* Drop-in C ABI of the B200 PDHG engine.
 *
 * Symbol-for-symbol replacement for the reference's cuda/include/sankhya_cuda.h:
 * the same function names, argument meaning, return codes and struct layouts, so
 * an application linked against the reference library (apps/sankhya_pdhg.cu,
 * apps/sankhya_qp_cuda.cu, the cuda/tests programs) links against libsankhya_cuda.so
 * built here without source changes. Each declaration cites the reference
 * declaration it replaces (path relative to the reference project).
 *
 * Engine-specific extensions live in sankhya_b200.h; nothing here changes
 * signature or layout.
 */
#ifndef SANKHYA_CUDA_H_B200
#define SANKHYA_CUDA_H_B200

#if defined(_WIN32) && defined(SANKHYA_CUDA_BUILD)
#define SANKHYA_CUDA_API __declspec(dllexport)
#else
#define SANKHYA_CUDA_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces cuda/include/sankhya_cuda.h:14-21. Three int dimensions and three
   device pointers to a canonical CSR (int32 offsets, int32 column indices,
   float64 values). Matrices made by sankhya_cuda_csr_create additionally own
   a private device-side transpose and row-tile schedule, found by the
   device_row_offsets pointer; the three public pointers stay a valid CSR. */
typedef struct SankhyaCudaCSR {
    int rows;
    int cols;
    int nnz;
    void* device_row_offsets;
    void* device_column_indices;
    void* device_values;
} SankhyaCudaCSR;

/* Replaces cuda/include/sankhya_cuda.h:25-32 (cuda/src/sankhya_cuda.cu:116-152).
   Validates offsets (0 .. nnz, non-decreasing), column range and finite values
   on the host before any allocation; returns 0 or -1 with
   sankhya_cuda_last_error() set. Any previous contents of *matrix are released
   first; on failure *matrix is left zeroed. */
SANKHYA_CUDA_API int sankhya_cuda_csr_create(
    SankhyaCudaCSR* matrix, int rows, int cols, int nnz,
    const int* row_offsets, const int* column_indices, const double* values);

/* Replaces cuda/include/sankhya_cuda.h:33 (sankhya_cuda.cu:154-163). */
SANKHYA_CUDA_API void sankhya_cuda_csr_destroy(SankhyaCudaCSR* matrix);

/* Replace cuda/include/sankhya_cuda.h:38-42 (sankhya_cuda.cu:165-197). Device
   pointers; the work is queued on CUDA's default stream and the call returns
   after launch. The transpose product is a deterministic gather over the
   stored transpose (the reference scatters with atomics). */
SANKHYA_CUDA_API int sankhya_cuda_spmv_device_f64(
    const SankhyaCudaCSR* matrix, const double* device_x, double* device_y);
SANKHYA_CUDA_API int sankhya_cuda_spmv_transpose_device_f64(
    const SankhyaCudaCSR* matrix, const double* device_y, double* device_x);
SANKHYA_CUDA_API int sankhya_cuda_axpy_device_f64(
    int n, double alpha, const double* device_x, double* device_y);

/* Replaces cuda/include/sankhya_cuda.h:44-52. Note that C aggregate
   initialisation with six values leaves time_limit at 0 (no limit). */
typedef struct SankhyaCudaLPSettings {
    int max_iterations;
    int check_every;
    double tau;
    double sigma;
    double theta;
    double tolerance;
    double time_limit; /* seconds, <= 0 disables the wall-clock limit */
} SankhyaCudaLPSettings;

/* Replaces cuda/include/sankhya_cuda.h:54-68. status: 0 converged,
   1 iteration limit, 2 time limit, negative error. Residual fields are those
   of the latest checkpoint (NaN / +inf until one has run). */
typedef struct SankhyaCudaLPResult {
    int status;
    int iterations;
    double objective;
    double maximum_row_violation;
    double maximum_step;
    double maximum_kkt_residual;
    double maximum_dual_residual;
    double maximum_complementarity;
} SankhyaCudaLPResult;

/* Replaces cuda/include/sankhya_cuda.h:72-81 (sankhya_cuda_lp.cu:387-393).
   min c'x s.t. row_lower <= A x <= row_upper, col_lower <= x <= col_upper.
   Model arrays and solution are host memory. Returns 0 (also at iteration or
   time limit), -1 on invalid input or CUDA error, -2 with result->status = -2
   when an iterate, A'y, Qx or the objective becomes non-finite. */
SANKHYA_CUDA_API int sankhya_cuda_lp_pdhg(
    const SankhyaCudaCSR* matrix, const double* c,
    const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper,
    SankhyaCudaLPSettings settings, double* solution, SankhyaCudaLPResult* result);

/* Replaces cuda/include/sankhya_cuda.h:85-99 (sankhya_cuda_lp.cu:426-437). */
SANKHYA_CUDA_API int sankhya_cuda_qp_pdhg_preconditioned_with_dual(
    const SankhyaCudaCSR* matrix, const SankhyaCudaCSR* hessian,
    const double* quadratic_diagonal, const double* c,
    const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper,
    const double* primal_steps, const double* dual_steps,
    SankhyaCudaLPSettings settings, double* solution, double* dual_solution,
    SankhyaCudaLPResult* result);

/* Replaces cuda/include/sankhya_cuda.h:106-116 (sankhya_cuda_lp.cu:395-403).
   min 0.5 sum q_i x_i^2 + c'x with an implicit diagonal proximal step. */
SANKHYA_CUDA_API int sankhya_cuda_diagonal_qp_pdhg(
    const SankhyaCudaCSR* matrix, const double* quadratic_diagonal, const double* c,
    const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper,
    SankhyaCudaLPSettings settings, double* solution, SankhyaCudaLPResult* result);

/* Replaces cuda/include/sankhya_cuda.h:121-131 (sankhya_cuda_lp.cu:405-413).
   Full symmetric Hessian Q (cols x cols), explicit Q x gradient at x. */
SANKHYA_CUDA_API int sankhya_cuda_sparse_qp_pdhg(
    const SankhyaCudaCSR* matrix, const SankhyaCudaCSR* hessian, const double* c,
    const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper,
    SankhyaCudaLPSettings settings, double* solution, SankhyaCudaLPResult* result);

/* Replaces cuda/include/sankhya_cuda.h:137-150 (sankhya_cuda_lp.cu:415-424).
   Caller-supplied finite positive per-column / per-row steps; tau and sigma
   are ignored and may be zero. */
SANKHYA_CUDA_API int sankhya_cuda_qp_pdhg_preconditioned(
    const SankhyaCudaCSR* matrix, const SankhyaCudaCSR* hessian,
    const double* quadratic_diagonal, const double* c,
    const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper,
    const double* primal_steps, const double* dual_steps,
    SankhyaCudaLPSettings settings, double* solution, SankhyaCudaLPResult* result);

/* Replaces cuda/include/sankhya_cuda.h:153-161 (sankhya_cuda.cu:199-252).
   Host arrays in and out; returns 0, -1 or a cudaError_t value. */
SANKHYA_CUDA_API int sankhya_cuda_spmv_f64(
    int rows, int cols, int nnz, const int* row_offsets, const int* column_indices,
    const double* values, const double* x, double* y);

/* Replaces cuda/include/sankhya_cuda.h:164 (sankhya_cuda.cu:254-284). */
SANKHYA_CUDA_API int sankhya_cuda_axpy_f64(int n, double alpha, const double* x, double* y);

/* Replaces cuda/include/sankhya_cuda.h:167. Thread-local text for the last
   non-zero return on this thread. */
SANKHYA_CUDA_API const char* sankhya_cuda_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
