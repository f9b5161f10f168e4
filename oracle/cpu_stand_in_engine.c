/* TEST INFRASTRUCTURE ONLY. A CPU stand-in for the four engine entry points that the
 * run_first_order integration block calls (sankhya_cuda_csr_create / _destroy,
 * sankhya_b200_pdlp_default_settings, sankhya_b200_pdlp_solve), answering with the
 * oracle's restatement of the restarted PDLP (orc_pdlp, no scaling). It lets the
 * reference's own LP driver, with the integration blocks spliced in, run its
 * first-order paths on a machine without a GPU: built as libsankhya_cuda_cpu_stand_in.so
 * (a name of its own, so that a process holding both never mistakes one for the other;
 * oracle/_ref/cpu_stand_in/) and linked in the engine's place.
 * The product never links it. */
#include <stdlib.h>
#include <string.h>

#include "../include/sankhya_b200.h"
#include "pdhg_oracle.h"

int sankhya_cuda_csr_create(SankhyaCudaCSR* m, int rows, int cols, int nnz, const int* row_offsets,
                            const int* column_indices, const double* values)
{
    if (!m || rows < 0 || cols < 0 || nnz < 0) return -1;
    int* p = (int*)malloc(sizeof(int) * (size_t)(rows + 1));
    int* i = (int*)malloc(sizeof(int) * (size_t)(nnz + 1));
    double* v = (double*)malloc(sizeof(double) * (size_t)(nnz + 1));
    if (!p || !i || !v) { free(p); free(i); free(v); return -1; }
    memcpy(p, row_offsets, sizeof(int) * (size_t)(rows + 1));
    memcpy(i, column_indices, sizeof(int) * (size_t)nnz);
    memcpy(v, values, sizeof(double) * (size_t)nnz);
    m->rows = rows;
    m->cols = cols;
    m->nnz = nnz;
    m->device_row_offsets = p;        /* host memory here: nothing else reads these fields */
    m->device_column_indices = i;
    m->device_values = v;
    return 0;
}

void sankhya_cuda_csr_destroy(SankhyaCudaCSR* m)
{
    if (!m) return;
    free(m->device_row_offsets);
    free(m->device_column_indices);
    free(m->device_values);
    memset(m, 0, sizeof(*m));
}

void sankhya_b200_pdlp_default_settings(SankhyaB200PdlpSettings* s)
{
    if (!s) return;
    memset(s, 0, sizeof(*s));
    s->struct_version = 4;
    s->max_iterations = 500000;
    s->restart_period = 64;
    s->power_iterations = 30;
    s->adaptive_step = 1;
    s->eps_optimal = 1e-8;
    s->eta_min_factor = 1e-6;
    s->eta_max_factor = 1e4;
    s->ruiz_tolerance = 1e-2;
}

int sankhya_b200_pdlp_solve(const SankhyaCudaCSR* matrix, const double* c, const double* row_lower,
                            const double* row_upper, const double* col_lower, const double* col_upper,
                            const SankhyaB200PdlpSettings* settings, const double* x0, const double* y0,
                            double* x_out, double* y_out, SankhyaB200PdlpResult* result)
{
    (void)x0;
    (void)y0;
    if (!matrix || !settings || !x_out || !result) return -1;
    memset(result, 0, sizeof(*result));
    orc_csr a;
    a.rows = matrix->rows;
    a.cols = matrix->cols;
    a.ptr = (const int*)matrix->device_row_offsets;
    a.idx = (const int*)matrix->device_column_indices;
    a.val = (const double*)matrix->device_values;
    orc_pdlp_params p;
    p.eps_optimal = settings->eps_optimal;
    p.max_iterations = settings->max_iterations;
    p.restart_period = settings->restart_period;
    p.power_iterations = settings->power_iterations;
    p.adaptive_step = settings->adaptive_step;
    p.eta_min_factor = settings->eta_min_factor;
    p.eta_max_factor = settings->eta_max_factor;
    double* y = y_out ? y_out : (double*)calloc((size_t)matrix->rows + 1, sizeof(double));
    if (!y) return -1;
    orc_pdlp_stats st;
    const int rc = orc_pdlp(&a, c, col_lower, col_upper, row_lower, row_upper, &p, x_out, y, &st);
    if (!y_out) free(y);
    result->status = st.converged ? 0 : 1;
    result->iterations = st.iterations;
    result->restarts = st.restarts;
    result->rejected_steps = st.rejected_steps;
    result->primal_objective = st.primal_objective;
    result->dual_objective = st.dual_objective;
    result->relative_primal_residual = st.relative_primal_residual;
    result->relative_dual_residual = st.relative_dual_residual;
    result->relative_gap = st.relative_gap;
    result->matrix_norm = st.matrix_norm;
    result->final_step_size = st.final_step_size;
    return rc == 0 ? 0 : -1;
}
