/* CPU restatement of the reference's PDHG / PDLP hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA
 * engine is compared against in tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py. The product never links or calls it.
 *
 * Every function restates one reference routine (paths are relative to the
 * reference project):
 *   orc_fixed_pdhg      cuda/src/sankhya_cuda_lp.cu:101-385   (solve_qp)
 *   orc_sk_loop         c/src/sk_solve.c:801-954              (solve_continuous loop)
 *   orc_sk_verify       c/src/sk_core.c:394-510               (sk_verify)
 *   orc_pdlp            src/cuda/GpuPdlp.cpp:179-534 and
 *                       src/cuda/PdlpKernels.cu:71-518        (restarted PDLP)
 *   orc_ruiz            src/lp/Scaling.cpp:11-92
 *   orc_pock_chambolle  src/lp/Scaling.cpp:111-145
 *   orc_pow2_scale      c/src/sk_scale.c:20-72
 *
 * Arithmetic is plain IEEE double with contraction disabled
 * (-ffp-contract=off); sparse products sum val*x terms sequentially in
 * stored order, starting from 0.0.
 */
#ifndef PDHG_ORACLE_H
#define PDHG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_csr {
    int rows;
    int cols;
    const int *ptr;
    const int *idx;
    const double *val;
} orc_csr;

/* Same field order as SankhyaCudaLPSettings / SankhyaCudaLPResult. */
typedef struct orc_settings {
    int max_iterations;
    int check_every;
    double tau;
    double sigma;
    double theta;
    double tolerance;
    double time_limit;
} orc_settings;

typedef struct orc_result {
    int status;
    int iterations;
    double objective;
    double maximum_row_violation;
    double maximum_step;
    double maximum_kkt_residual;
    double maximum_dual_residual;
    double maximum_complementarity;
} orc_result;

void orc_csr_spmv(const orc_csr *a, const double *x, double *y);
/* Builds the CSR of A^T (rows of A^T = columns of A, entries in ascending row
   order). tptr has cols+1 entries, tidx/tval nnz entries. */
void orc_csr_transpose(const orc_csr *a, int *tptr, int *tidx, double *tval);

int orc_fixed_pdhg(const orc_csr *a, const orc_csr *hessian, const double *quadratic_diagonal,
                   const double *c, const double *row_lower, const double *row_upper,
                   const double *col_lower, const double *col_upper, orc_settings settings,
                   const double *primal_steps, const double *dual_steps, double *solution,
                   double *dual_solution, orc_result *result);

/* sk_solve's continuous PDHG loop. a is the CSR of the model's A (columns in
   ascending order inside each row, which is what a CSC->CSR conversion
   yields); q the CSR of the full symmetric Q or NULL. SK_INFINITY (1e30)
   sentinels mark absent bounds. x, y, activity are outputs. */
typedef struct orc_sk_out {
    int iterations;
    int converged;
    double dual_step;
    double anorm;
} orc_sk_out;
int orc_sk_loop(const orc_csr *a, const orc_csr *q, const double *c, const double *rlow,
                const double *rupp, const double *clow, const double *cupp, int max_iterations,
                double primal_tol, double dual_tol, double time_limit, double *x, double *y,
                double *activity, orc_sk_out *out);

typedef struct orc_verify {
    double objective;
    double primal_infeasibility;
    double dual_infeasibility;
    double complementarity;
} orc_verify;
void orc_sk_verify(const orc_csr *a, const orc_csr *q, const double *c, double objshift,
                   const double *rlow, const double *rupp, const double *clow,
                   const double *cupp, const double *x, const double *y, orc_verify *out);

typedef struct orc_pdlp_params {
    double eps_optimal;
    int max_iterations;
    int restart_period;
    int power_iterations;
    int adaptive_step;
    double eta_min_factor;
    double eta_max_factor;
} orc_pdlp_params;

typedef struct orc_pdlp_stats {
    int converged;
    int iterations;
    int restarts;
    int rejected_steps;
    double primal_objective;
    double dual_objective;
    double relative_primal_residual;
    double relative_dual_residual;
    double relative_gap;
    double matrix_norm;
    double final_step_size;
} orc_pdlp_stats;

/* Bounds whose magnitude is >= 1e30 are treated as absent. */
int orc_pdlp(const orc_csr *a, const double *c, const double *lower, const double *upper,
             const double *row_lower, const double *row_upper, const orc_pdlp_params *params,
             double *x_out, double *y_out, orc_pdlp_stats *stats);

double orc_power_norm(const orc_csr *a, int iterations);

/* Scaling factors. row_scale has a->rows entries, col_scale a->cols. */
int orc_ruiz(const orc_csr *a, int max_iters, double tol, double *row_scale, double *col_scale);
void orc_pock_chambolle(const orc_csr *a, double alpha, double *row_scale, double *col_scale);
void orc_pow2_scale(const orc_csr *a, int passes, double *row_scale, double *col_scale);

#ifdef __cplusplus
}
#endif
#endif
