/* CPU restatement of the reference's PDHG / PDLP hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine, never part of
 * the product. See pdhg_oracle.h for the routine-by-routine map to the
 * reference sources. Compiled with -ffp-contract=off so a*b+c is always
 * two roundings, as in the reference's host code built by gcc for x86-64.
 */
#include "pdhg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static double wall_seconds(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static double dmax(double a, double b) { return a > b ? a : b; }

/* ------------------------------------------------------------ sparse core */

void orc_csr_spmv(const orc_csr *a, const double *x, double *y)
{
    int r, p;
    for (r = 0; r < a->rows; ++r) {
        double s = 0.0;
        for (p = a->ptr[r]; p < a->ptr[r + 1]; ++p) s += a->val[p] * x[a->idx[p]];
        y[r] = s;
    }
}

void orc_csr_transpose(const orc_csr *a, int *tptr, int *tidx, double *tval)
{
    int r, p, j;
    int *next;
    for (j = 0; j <= a->cols; ++j) tptr[j] = 0;
    for (p = 0; p < a->ptr[a->rows]; ++p) tptr[a->idx[p] + 1]++;
    for (j = 0; j < a->cols; ++j) tptr[j + 1] += tptr[j];
    next = (int *)malloc(sizeof(int) * (size_t)(a->cols > 0 ? a->cols : 1));
    for (j = 0; j < a->cols; ++j) next[j] = tptr[j];
    for (r = 0; r < a->rows; ++r)
        for (p = a->ptr[r]; p < a->ptr[r + 1]; ++p) {
            const int slot = next[a->idx[p]]++;
            tidx[slot] = r;
            tval[slot] = a->val[p];
        }
    free(next);
}

typedef struct owned_csr {
    orc_csr view;
    int *ptr;
    int *idx;
    double *val;
} owned_csr;

static int make_transpose(const orc_csr *a, owned_csr *t)
{
    const int nnz = a->ptr[a->rows];
    t->ptr = (int *)malloc(sizeof(int) * (size_t)(a->cols + 1));
    t->idx = (int *)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));
    t->val = (double *)malloc(sizeof(double) * (size_t)(nnz > 0 ? nnz : 1));
    if (!t->ptr || !t->idx || !t->val) {
        free(t->ptr); free(t->idx); free(t->val);
        return -1;
    }
    orc_csr_transpose(a, t->ptr, t->idx, t->val);
    t->view.rows = a->cols;
    t->view.cols = a->rows;
    t->view.ptr = t->ptr;
    t->view.idx = t->idx;
    t->view.val = t->val;
    return 0;
}

static void free_owned(owned_csr *t) { free(t->ptr); free(t->idx); free(t->val); }

/* ============================================================
 * cuda/src/sankhya_cuda_lp.cu:101-385  (solve_qp)
 * ============================================================ */

/* sankhya_cuda_lp.cu:13-17: only IEEE infinities are "no bound". */
static double box_ieee(double v, double lo, double hi)
{
    if (!isinf(lo) && v < lo) v = lo;
    if (!isinf(hi) && v > hi) v = hi;
    return v;
}

static int valid_lower(double v) { return !isnan(v) && !(isinf(v) && v > 0.0); }
static int valid_upper(double v) { return !isnan(v) && !(isinf(v) && v < 0.0); }
/* sankhya_cuda_lp.cu:91-97: the residual gates also honour the 1e30 sentinel. */
static int has_lower(double v) { return isfinite(v) && v > -5.0e29; }
static int has_upper(double v) { return isfinite(v) && v < 5.0e29; }

static void fixed_result_init(orc_result *r)
{
    r->status = -1;
    r->iterations = 0;
    r->objective = NAN;
    r->maximum_row_violation = INFINITY;
    r->maximum_step = INFINITY;
    r->maximum_kkt_residual = INFINITY;
    r->maximum_dual_residual = INFINITY;
    r->maximum_complementarity = INFINITY;
}

int orc_fixed_pdhg(const orc_csr *a, const orc_csr *hessian, const double *quadratic_diagonal,
                   const double *c, const double *row_lower, const double *row_upper,
                   const double *col_lower, const double *col_upper, orc_settings settings,
                   const double *primal_steps, const double *dual_steps, double *solution,
                   double *dual_solution, orc_result *result)
{
    int rows, cols, i, j, iteration, final_iteration, have_previous_x = 0, rc = 0;
    double *x, *x_new, *x_bar, *y, *y_new, *activity, *gradient, *qgrad, *prev_x, *aty;
    owned_csr at;
    double started;

    if (result == NULL) return -1;
    fixed_result_init(result);
    if (a == NULL || c == NULL || row_lower == NULL || row_upper == NULL || col_lower == NULL ||
        col_upper == NULL || solution == NULL)
        return -1;
    if (settings.max_iterations <= 0 || settings.check_every <= 0 || settings.theta < 0.0 ||
        settings.theta > 1.0 || settings.tolerance <= 0.0 || settings.time_limit < 0.0)
        return -1;
    if ((primal_steps == NULL) != (dual_steps == NULL)) return -1;
    if (primal_steps == NULL && (settings.tau <= 0.0 || settings.sigma <= 0.0)) return -1;
    rows = a->rows;
    cols = a->cols;
    if (rows < 0 || cols < 0) return -1;
    for (j = 0; j < cols; ++j)
        if (!isfinite(c[j]) || !valid_lower(col_lower[j]) || !valid_upper(col_upper[j]) ||
            col_lower[j] > col_upper[j])
            return -1;
    for (i = 0; i < rows; ++i)
        if (!valid_lower(row_lower[i]) || !valid_upper(row_upper[i]) || row_lower[i] > row_upper[i])
            return -1;
    if (primal_steps != NULL) {
        for (j = 0; j < cols; ++j)
            if (!isfinite(primal_steps[j]) || primal_steps[j] <= 0.0) return -1;
        for (i = 0; i < rows; ++i)
            if (!isfinite(dual_steps[i]) || dual_steps[i] <= 0.0) return -1;
    }
    if (hessian != NULL &&
        (quadratic_diagonal != NULL || hessian->rows != cols || hessian->cols != cols))
        return -1;
    if (quadratic_diagonal != NULL)
        for (j = 0; j < cols; ++j)
            if (!isfinite(quadratic_diagonal[j]) || quadratic_diagonal[j] < 0.0) return -1;

    if (make_transpose(a, &at) != 0) return -1;
    x = (double *)calloc((size_t)cols + 1, sizeof(double));
    x_new = (double *)calloc((size_t)cols + 1, sizeof(double));
    x_bar = (double *)calloc((size_t)cols + 1, sizeof(double));
    gradient = (double *)calloc((size_t)cols + 1, sizeof(double));
    qgrad = (double *)calloc((size_t)cols + 1, sizeof(double));
    prev_x = (double *)calloc((size_t)cols + 1, sizeof(double));
    aty = (double *)calloc((size_t)cols + 1, sizeof(double));
    y = (double *)calloc((size_t)rows + 1, sizeof(double));
    y_new = (double *)calloc((size_t)rows + 1, sizeof(double));
    activity = (double *)calloc((size_t)rows + 1, sizeof(double));

    for (j = 0; j < cols; ++j) x[j] = x_bar[j] = box_ieee(0.0, col_lower[j], col_upper[j]);
    final_iteration = settings.max_iterations;
    started = wall_seconds();
    for (iteration = 1; iteration <= settings.max_iterations; ++iteration) {
        double *swap;
        if (settings.time_limit > 0.0 && iteration % settings.check_every == 1 &&
            wall_seconds() - started >= settings.time_limit) {
            final_iteration = iteration - 1;
            result->status = 2;
            break;
        }
        /* sankhya_cuda_lp.cu:230-234 dual step on A*x_bar */
        orc_csr_spmv(a, x_bar, activity);
        for (i = 0; i < rows; ++i) {
            const double sigma = dual_steps ? dual_steps[i] : settings.sigma;
            const double trial = y[i] + sigma * activity[i];
            y_new[i] = trial - sigma * box_ieee(trial / sigma, row_lower[i], row_upper[i]);
        }
        /* :235 A^T y_new (the reference scatters with atomics; a gather in
           ascending row order is one of its admissible summation orders) */
        if (rows > 0 && cols > 0) orc_csr_spmv(&at.view, y_new, gradient);
        /* :236-238 explicit Hessian gradient uses x, not x_bar */
        if (hessian != NULL) orc_csr_spmv(hessian, x, qgrad);
        /* :239-245 primal step + extrapolation */
        for (j = 0; j < cols; ++j) {
            const double tau = primal_steps ? primal_steps[j] : settings.tau;
            const double curvature = quadratic_diagonal ? quadratic_diagonal[j] : 0.0;
            const double qg = hessian ? qgrad[j] : 0.0;
            const double trial = (x[j] - tau * (c[j] + gradient[j] + qg)) / (1.0 + tau * curvature);
            const double next = box_ieee(trial, col_lower[j], col_upper[j]);
            x_new[j] = next;
            x_bar[j] = next + settings.theta * (next - x[j]);
        }
        swap = x; x = x_new; x_new = swap;
        swap = y; y = y_new; y_new = swap;

        if (iteration % settings.check_every == 0 || iteration == settings.max_iterations) {
            double objective = 0.0, step, scale = 1.0, violation = 0.0, kkt = 0.0;
            double dual_residual = 0.0, complementarity = 0.0, objective_scale;
            orc_csr_spmv(a, x, activity);
            if (rows > 0 && cols > 0) orc_csr_spmv(&at.view, y, aty);
            for (j = 0; j < cols; ++j)
                if (!isfinite(x[j]) || !isfinite(aty[j])) { result->status = -2; rc = -2; goto done; }
            for (i = 0; i < rows; ++i)
                if (!isfinite(activity[i]) || !isfinite(y[i])) { result->status = -2; rc = -2; goto done; }
            if (hessian != NULL) {
                orc_csr_spmv(hessian, x, qgrad);
                for (j = 0; j < cols; ++j)
                    if (!isfinite(qgrad[j])) { result->status = -2; rc = -2; goto done; }
            }
            for (j = 0; j < cols; ++j) {
                objective += c[j] * x[j];
                if (quadratic_diagonal) objective += 0.5 * quadratic_diagonal[j] * x[j] * x[j];
                else if (hessian) objective += 0.5 * x[j] * qgrad[j];
            }
            if (!isfinite(objective)) { result->status = -2; rc = -2; goto done; }
            step = have_previous_x ? 0.0 : INFINITY;
            for (j = 0; j < cols; ++j) {
                if (have_previous_x) step = dmax(step, fabs(x[j] - prev_x[j]));
                scale = dmax(scale, fabs(x[j]));
                prev_x[j] = x[j];
            }
            have_previous_x = 1;
            for (i = 0; i < rows; ++i) {
                if (isfinite(row_lower[i])) violation = dmax(violation, row_lower[i] - activity[i]);
                if (isfinite(row_upper[i])) violation = dmax(violation, activity[i] - row_upper[i]);
            }
            violation = dmax(0.0, violation);
            for (i = 0; i < rows; ++i) {
                const double projected = box_ieee(activity[i] + y[i], row_lower[i], row_upper[i]);
                kkt = dmax(kkt, fabs(activity[i] - projected));
            }
            for (j = 0; j < cols; ++j) {
                const double qg = quadratic_diagonal ? quadratic_diagonal[j] * x[j]
                                                     : (hessian ? qgrad[j] : 0.0);
                const double g = c[j] + aty[j] + qg;
                const double projected = box_ieee(x[j] - g, col_lower[j], col_upper[j]);
                kkt = dmax(kkt, fabs(x[j] - projected));
            }
            for (j = 0; j < cols; ++j) {
                const double qg = quadratic_diagonal ? quadratic_diagonal[j] * x[j]
                                                     : (hessian ? qgrad[j] : 0.0);
                const double residual = c[j] + aty[j] + qg;
                const int at_lower = has_lower(col_lower[j]) && fabs(x[j] - col_lower[j]) <= 1e-9;
                const int at_upper = has_upper(col_upper[j]) && fabs(x[j] - col_upper[j]) <= 1e-9;
                if (at_lower && at_upper) {
                } else if (at_lower) {
                    dual_residual = dmax(dual_residual, -residual);
                } else if (at_upper) {
                    dual_residual = dmax(dual_residual, residual);
                } else {
                    dual_residual = dmax(dual_residual, fabs(residual));
                }
                if (residual > 0.0 && has_lower(col_lower[j]))
                    complementarity = dmax(complementarity, residual * fabs(x[j] - col_lower[j]));
                else if (residual < 0.0 && has_upper(col_upper[j]))
                    complementarity = dmax(complementarity, -residual * fabs(col_upper[j] - x[j]));
            }
            for (i = 0; i < rows; ++i) {
                const double mult = y[i];
                const double act = activity[i];
                const int at_lower = has_lower(row_lower[i]) && fabs(act - row_lower[i]) <= 1e-9;
                const int at_upper = has_upper(row_upper[i]) && fabs(act - row_upper[i]) <= 1e-9;
                if (at_lower && at_upper) {
                } else if (at_lower) {
                    dual_residual = dmax(dual_residual, mult);
                } else if (at_upper) {
                    dual_residual = dmax(dual_residual, -mult);
                } else {
                    dual_residual = dmax(dual_residual, fabs(mult));
                }
                if (mult < 0.0 && has_lower(row_lower[i]))
                    complementarity = dmax(complementarity, -mult * fabs(act - row_lower[i]));
                else if (mult > 0.0 && has_upper(row_upper[i]))
                    complementarity = dmax(complementarity, mult * fabs(row_upper[i] - act));
            }
            objective_scale = 1.0 + fabs(objective);
            result->objective = objective;
            result->maximum_row_violation = violation;
            result->maximum_step = step;
            result->maximum_kkt_residual = kkt;
            result->maximum_dual_residual = dual_residual;
            result->maximum_complementarity = complementarity / objective_scale;
            if (violation <= settings.tolerance && step <= settings.tolerance * scale &&
                kkt <= settings.tolerance && dual_residual <= settings.tolerance &&
                result->maximum_complementarity <= settings.tolerance) {
                final_iteration = iteration;
                result->status = 0;
                break;
            }
        }
    }
    if (result->status < 0) result->status = 1;
    result->iterations = final_iteration;
    for (j = 0; j < cols; ++j) solution[j] = x[j];
    if (dual_solution != NULL)
        for (i = 0; i < rows; ++i) dual_solution[i] = y[i];
done:
    free(x); free(x_new); free(x_bar); free(gradient); free(qgrad); free(prev_x); free(aty);
    free(y); free(y_new); free(activity);
    free_owned(&at);
    return rc;
}

/* ============================================================
 * c/src/sk_solve.c:801-954  (solve_continuous PDHG loop)
 * ============================================================ */

#define ORC_SK_INF 1.0e30
static int sk_is_inf(double v) { return v >= ORC_SK_INF; }
static int sk_is_neg_inf(double v) { return v <= -ORC_SK_INF; }

/* sk_solve.c:18-24 */
static double sk_clamp(double x, double lo, double hi)
{
    if (!sk_is_neg_inf(lo) && x < lo) x = lo;
    if (!sk_is_inf(hi) && x > hi) x = hi;
    return x;
}

/* sk_solve.c:82-95 */
static double sk_row_violation(int rows, const double *rlow, const double *rupp, const double *act)
{
    int i;
    double v = 0.0;
    for (i = 0; i < rows; ++i) {
        if (!sk_is_neg_inf(rlow[i]) && rlow[i] - act[i] > v) v = rlow[i] - act[i];
        if (!sk_is_inf(rupp[i]) && act[i] - rupp[i] > v) v = act[i] - rupp[i];
    }
    return v;
}

int orc_sk_loop(const orc_csr *a, const orc_csr *q, const double *c, const double *rlow,
                const double *rupp, const double *clow, const double *cupp, int max_iterations,
                double primal_tol, double dual_tol, double time_limit, double *x, double *y,
                double *activity, orc_sk_out *out)
{
    const int n = a->cols, r = a->rows, check_every = 20;
    int iteration, j, p, converged = 0, diagonal = 0;
    double *x_new, *x_bar, *y_new, *gradient, *qx = NULL, *qdiag = NULL, *tau_vec, *sigma_vec;
    double *row_mass, *col_mass, anorm, col_max = 0.0, row_max = 0.0, start;
    double dual_step = INFINITY;
    owned_csr at;

    if (make_transpose(a, &at) != 0) return -1;
    x_new = (double *)calloc((size_t)n + 1, sizeof(double));
    x_bar = (double *)calloc((size_t)n + 1, sizeof(double));
    gradient = (double *)calloc((size_t)n + 1, sizeof(double));
    tau_vec = (double *)calloc((size_t)n + 1, sizeof(double));
    col_mass = (double *)calloc((size_t)n + 1, sizeof(double));
    y_new = (double *)calloc((size_t)r + 1, sizeof(double));
    sigma_vec = (double *)calloc((size_t)r + 1, sizeof(double));
    row_mass = (double *)calloc((size_t)r + 1, sizeof(double));
    for (j = 0; j < r; ++j) y[j] = 0.0;
    if (q) {
        qx = (double *)calloc((size_t)n + 1, sizeof(double));
        qdiag = (double *)calloc((size_t)n + 1, sizeof(double));
        /* sk_solve.c:863-870: Q is diagonal when every stored entry sits on
           the diagonal; duplicates are summed. q is symmetric, so its CSR
           rows are its CSC columns. */
        diagonal = 1;
        for (j = 0; j < n && diagonal; ++j)
            for (p = q->ptr[j]; p < q->ptr[j + 1]; ++p) {
                if (q->idx[p] != j) { diagonal = 0; break; }
                qdiag[j] += q->val[p];
            }
        if (!diagonal) { free(qdiag); qdiag = NULL; }
    }
    for (j = 0; j < n; ++j) x[j] = x_bar[j] = sk_clamp(0.0, clow[j], cupp[j]);

    /* sk_solve.c:60-80 matrix_norm_bound and :880-896 step vectors. Column
       sums run over a column's entries in ascending row order (CSC order);
       row sums accumulate in ascending column order. */
    for (j = 0; j < n; ++j) {
        double s = 0.0;
        for (p = at.ptr[j]; p < at.ptr[j + 1]; ++p) s += fabs(at.val[p]);
        col_mass[j] = s;
        if (s > col_max) col_max = s;
    }
    for (j = 0; j < r; ++j) {
        double s = 0.0;
        for (p = a->ptr[j]; p < a->ptr[j + 1]; ++p) s += fabs(a->val[p]);
        row_mass[j] = s;
        if (s > row_max) row_max = s;
    }
    anorm = (r && n) ? sqrt(col_max * row_max) : 0.0;
    if (q)
        for (j = 0; j < n; ++j)
            for (p = q->ptr[j]; p < q->ptr[j + 1]; ++p) col_mass[j] += fabs(q->val[p]);
    for (j = 0; j < n; ++j) tau_vec[j] = 0.9 / (1.0 + col_mass[j]);
    for (j = 0; j < r; ++j) sigma_vec[j] = 0.9 / (1.0 + row_mass[j]);

    start = wall_seconds();
    for (iteration = 1; iteration <= max_iterations; ++iteration) {
        orc_csr_spmv(a, x_bar, activity);
        for (j = 0; j < r; ++j) {
            const double trial = y[j] + sigma_vec[j] * activity[j];
            y_new[j] = trial - sigma_vec[j] * sk_clamp(trial / sigma_vec[j], rlow[j], rupp[j]);
        }
        dual_step = 0.0;
        for (j = 0; j < r; ++j)
            if (fabs(y_new[j] - y[j]) > dual_step) dual_step = fabs(y_new[j] - y[j]);
        orc_csr_spmv(&at.view, y_new, gradient);
        if (q) {
            if (qdiag) for (j = 0; j < n; ++j) qx[j] = qdiag[j] * x[j];
            else orc_csr_spmv(q, x, qx);
        }
        for (j = 0; j < n; ++j) {
            if (qdiag)
                x_new[j] = (x[j] - tau_vec[j] * (c[j] + gradient[j])) / (1.0 + tau_vec[j] * qdiag[j]);
            else
                x_new[j] = x[j] - tau_vec[j] * (c[j] + (q ? qx[j] : 0.0) + gradient[j]);
            x_new[j] = sk_clamp(x_new[j], clow[j], cupp[j]);
            x_bar[j] = 2.0 * x_new[j] - x[j];
        }
        memcpy(x, x_new, (size_t)n * sizeof(double));
        memcpy(y, y_new, (size_t)r * sizeof(double));
        if (time_limit > 0.0 && wall_seconds() - start >= time_limit) break;
        if (iteration % check_every == 0 || iteration == max_iterations) {
            double step = 0.0, scale = 1.0;
            int ready = 1;
            orc_csr_spmv(a, x, activity);
            for (j = 0; j < n; ++j) if (fabs(x[j]) > scale) scale = fabs(x[j]);
            for (j = 0; j < n; ++j) if (fabs(x_bar[j] - x[j]) > step) step = fabs(x_bar[j] - x[j]);
            if (q) {
                orc_verify v;
                double score;
                orc_sk_verify(a, q, c, 0.0, rlow, rupp, clow, cupp, x, y, &v);
                score = v.primal_infeasibility + v.dual_infeasibility + v.complementarity;
                ready = isfinite(score) && score <= 100.0 * (primal_tol + 2.0 * dual_tol);
            }
            if (sk_row_violation(r, rlow, rupp, activity) <= primal_tol && step <= primal_tol * scale &&
                dual_step <= dual_tol * (1.0 + anorm) && ready) {
                converged = 1;
                break;
            }
        }
    }
    out->iterations = iteration > max_iterations ? max_iterations : iteration;
    out->converged = converged;
    out->dual_step = dual_step;
    out->anorm = anorm;
    free(x_new); free(x_bar); free(gradient); free(tau_vec); free(col_mass); free(y_new);
    free(sigma_vec); free(row_mass); free(qx); free(qdiag);
    free_owned(&at);
    return 0;
}

/* ============================================================
 * c/src/sk_core.c:394-510  (sk_verify)
 * ============================================================ */
void orc_sk_verify(const orc_csr *a, const orc_csr *q, const double *c, double objshift,
                   const double *rlow, const double *rupp, const double *clow,
                   const double *cupp, const double *x, const double *y, orc_verify *out)
{
    const int n = a->cols, m = a->rows;
    const double bt = 1e-9;
    int i, j, p;
    double pinf = 0.0, dinf = 0.0, comp = 0.0, pobj, dobj;
    double *act = (double *)calloc((size_t)m + 1, sizeof(double));
    double *rc = (double *)calloc((size_t)n + 1, sizeof(double));
    double *qx = (double *)calloc((size_t)n + 1, sizeof(double));
    owned_csr at;
    make_transpose(a, &at);

    /* act = A x accumulated column by column, i.e. ascending column order per row */
    orc_csr_spmv(a, x, act);
    pobj = objshift;
    for (j = 0; j < n; ++j) pobj += c[j] * x[j];
    if (q) {
        orc_csr_spmv(q, x, qx);
        for (j = 0; j < n; ++j) pobj += 0.5 * x[j] * qx[j];
    }
    for (i = 0; i < m; ++i) {
        if (!sk_is_neg_inf(rlow[i]) && rlow[i] - act[i] > pinf) pinf = rlow[i] - act[i];
        if (!sk_is_inf(rupp[i]) && act[i] - rupp[i] > pinf) pinf = act[i] - rupp[i];
    }
    for (j = 0; j < n; ++j) {
        if (!isfinite(x[j])) { pinf = INFINITY; break; }
        if (!sk_is_neg_inf(clow[j]) && clow[j] - x[j] > pinf) pinf = clow[j] - x[j];
        if (!sk_is_inf(cupp[j]) && x[j] - cupp[j] > pinf) pinf = x[j] - cupp[j];
    }
    dobj = objshift;
    if (y) {
        for (j = 0; j < n; ++j) {
            double r = c[j] + (q ? qx[j] : 0.0);
            for (p = at.ptr[j]; p < at.ptr[j + 1]; ++p) r += at.val[p] * y[at.idx[p]];
            rc[j] = r;
        }
        for (j = 0; j < n; ++j) {
            const int atlo = !sk_is_neg_inf(clow[j]) && fabs(x[j] - clow[j]) <= bt;
            const int athi = !sk_is_inf(cupp[j]) && fabs(x[j] - cupp[j]) <= bt;
            const double r = rc[j];
            if (atlo && athi) {
            } else if (atlo) {
                if (-r > dinf) dinf = -r;
            } else if (athi) {
                if (r > dinf) dinf = r;
            } else {
                if (fabs(r) > dinf) dinf = fabs(r);
            }
            if (r > 0.0) {
                if (sk_is_neg_inf(clow[j])) { if (r > dinf) dinf = r; }
                else dobj += r * clow[j];
            } else if (r < 0.0) {
                if (sk_is_inf(cupp[j])) { if (-r > dinf) dinf = -r; }
                else dobj += r * cupp[j];
            }
            if (r > 0.0 && !sk_is_neg_inf(clow[j])) {
                const double prod = r * fabs(x[j] - clow[j]);
                if (prod > comp) comp = prod;
            } else if (r < 0.0 && !sk_is_inf(cupp[j])) {
                const double prod = -r * fabs(cupp[j] - x[j]);
                if (prod > comp) comp = prod;
            }
        }
        for (i = 0; i < m; ++i) {
            const int atlo = !sk_is_neg_inf(rlow[i]) && fabs(act[i] - rlow[i]) <= bt;
            const int athi = !sk_is_inf(rupp[i]) && fabs(act[i] - rupp[i]) <= bt;
            const double yv = y[i];
            if (atlo && athi) {
            } else if (atlo) {
                if (yv > dinf) dinf = yv;
            } else if (athi) {
                if (-yv > dinf) dinf = -yv;
            } else {
                if (fabs(yv) > dinf) dinf = fabs(yv);
            }
            if (yv < 0.0) {
                if (sk_is_neg_inf(rlow[i])) { if (-yv > dinf) dinf = -yv; }
                else dobj -= yv * rlow[i];
                if (!sk_is_neg_inf(rlow[i])) {
                    const double prod = -yv * fabs(act[i] - rlow[i]);
                    if (prod > comp) comp = prod;
                }
            } else if (yv > 0.0) {
                if (sk_is_inf(rupp[i])) { if (yv > dinf) dinf = yv; }
                else dobj -= yv * rupp[i];
                if (!sk_is_inf(rupp[i])) {
                    const double prod = yv * fabs(rupp[i] - act[i]);
                    if (prod > comp) comp = prod;
                }
            }
        }
        out->complementarity = q ? comp / (1.0 + fabs(pobj)) : fabs(pobj - dobj) / (1.0 + fabs(pobj));
    } else {
        dinf = INFINITY;
        out->complementarity = INFINITY;
    }
    out->objective = pobj;
    out->primal_infeasibility = pinf > 0.0 ? pinf : 0.0;
    out->dual_infeasibility = dinf > 0.0 ? dinf : 0.0;
    free(act); free(rc); free(qx);
    free_owned(&at);
}

/* ============================================================
 * src/cuda/GpuPdlp.cpp + src/cuda/PdlpKernels.cu  (restarted PDLP)
 * ============================================================ */

#define PDLP_STEP_SAFETY 0.9
#define PDLP_MIN_WEIGHT 1e-6
#define PDLP_MAX_WEIGHT 1e6
#define PDLP_SMOOTHING 0.5
#define PDLP_SUFFICIENT 0.2
#define PDLP_NECESSARY 0.8
#define PDLP_ARTIFICIAL 0.36

static int bound_finite(double v) { return isfinite(v) && fabs(v) < 1e30; }

static double clamp_fm(double v, double lo, double hi)
{
    /* fmin/fmax clamp with absent bounds widened to +-inf (PdlpKernels.cu:42-47) */
    if (!bound_finite(lo)) lo = -INFINITY;
    if (!bound_finite(hi)) hi = INFINITY;
    return fmin(fmax(v, lo), hi);
}

/* GpuPdlp.cpp:179-211: power iteration on A^T A from v = 1/||1||. */
double orc_power_norm(const orc_csr *a, int iterations)
{
    const int n = a->cols, m = a->rows;
    int k, j;
    double nrm_sq = 0.0, lambda, norm;
    double *v = (double *)calloc((size_t)n + 1, sizeof(double));
    double *w = (double *)calloc((size_t)m + 1, sizeof(double));
    double *v2 = (double *)calloc((size_t)n + 1, sizeof(double));
    owned_csr at;
    make_transpose(a, &at);
    for (j = 0; j < n; ++j) v[j] = 1.0;
    for (j = 0; j < n; ++j) nrm_sq += v[j] * v[j];
    if (sqrt(nrm_sq) > 0.0) {
        const double inv = 1.0 / sqrt(nrm_sq);
        for (j = 0; j < n; ++j) v[j] *= inv;
    }
    for (k = 0; k < iterations; ++k) {
        orc_csr_spmv(a, v, w);
        orc_csr_spmv(&at.view, w, v2);
        nrm_sq = 0.0;
        for (j = 0; j < n; ++j) nrm_sq += v2[j] * v2[j];
        for (j = 0; j < n; ++j) v[j] = v2[j];
        if (sqrt(nrm_sq) > 0.0) {
            const double inv = 1.0 / sqrt(nrm_sq);
            for (j = 0; j < n; ++j) v[j] *= inv;
        }
    }
    lambda = sqrt(nrm_sq > 0.0 ? nrm_sq : 0.0);
    norm = sqrt(lambda);
    free(v); free(w); free(v2);
    free_owned(&at);
    return (norm > 0.0 && isfinite(norm)) ? norm : 1.0;
}

typedef struct pdlp_kkt {
    double primal, dual, gap, primal_obj, dual_obj, primal_move, dual_move;
} pdlp_kkt;

static double kkt_worst(const pdlp_kkt *k)
{
    const double a = k->primal > k->dual ? k->primal : k->dual;
    return a > k->gap ? a : k->gap;
}

/* PdlpKernels.cu:101-209 residual sums + GpuPdlp.cpp:226-250 relative measures */
static void pdlp_residuals(const orc_csr *a, const orc_csr *at, const double *x, const double *y,
                           double *ax, double *aty, const double *c, const double *lower,
                           const double *upper, const double *rl, const double *ru,
                           const double *x_restart, const double *y_restart, double cost_norm,
                           double bound_norm, pdlp_kkt *k)
{
    const int n = a->cols, m = a->rows;
    int i, j;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    orc_csr_spmv(a, x, ax);
    orc_csr_spmv(at, y, aty);
    for (j = 0; j < n; ++j) {
        const double xj = x[j], lo = lower[j], hi = upper[j];
        const double r = c[j] + aty[j];
        const int lf = bound_finite(lo), hf = bound_finite(hi);
        double viol = 0.0, term = 0.0, dx;
        acc[2] += c[j] * xj;
        acc[4] += xj * xj;
        dx = xj - x_restart[j];
        acc[6] += dx * dx;
        if (lf && hf) term = fmin(r * lo, r * hi);
        else if (lf) { viol = fmax(0.0, -r); term = fmax(0.0, r) * lo; }
        else if (hf) { viol = fmax(0.0, r); term = fmin(0.0, r) * hi; }
        else viol = fabs(r);
        acc[1] += viol * viol;
        acc[3] += term;
    }
    for (i = 0; i < m; ++i) {
        const double axi = ax[i], yi = y[i];
        const double pr = axi - clamp_fm(axi, rl[i], ru[i]);
        double support = 0.0, dy;
        acc[0] += pr * pr;
        acc[5] += yi * yi;
        dy = yi - y_restart[i];
        acc[7] += dy * dy;
        if (yi > 0.0) support = bound_finite(ru[i]) ? yi * ru[i] : 0.0;
        else if (yi < 0.0) support = bound_finite(rl[i]) ? yi * rl[i] : 0.0;
        acc[3] -= support;
    }
    k->primal = sqrt(fmax(0.0, acc[0])) / (1.0 + bound_norm);
    k->dual = sqrt(fmax(0.0, acc[1])) / (1.0 + cost_norm);
    k->primal_obj = acc[2];
    k->dual_obj = acc[3];
    k->gap = fabs(acc[2] - acc[3]) / (1.0 + fabs(acc[2]) + fabs(acc[3]));
    k->primal_move = sqrt(fmax(0.0, acc[6]));
    k->dual_move = sqrt(fmax(0.0, acc[7]));
    if (!isfinite(k->primal) || !isfinite(k->dual) || !isfinite(k->gap))
        k->primal = k->dual = k->gap = INFINITY;
}

int orc_pdlp(const orc_csr *a, const double *c, const double *lower, const double *upper,
             const double *row_lower, const double *row_upper, const orc_pdlp_params *params,
             double *x_out, double *y_out, orc_pdlp_stats *stats)
{
    const int n = a->cols, m = a->rows;
    int i, j, iteration = 0, windows_since_restart = 0, iterations_since_restart = 0;
    double cost_norm = 0.0, bl = 0.0, bu = 0.0, bound_norm, matrix_norm, eta_global, eta_min,
           eta_max, omega = 1.0, mu_at_restart = INFINITY, mu_previous = INFINITY;
    double eta, updates = 0.0, accept_count = 0.0, accepted_at_restart = 0.0;
    pdlp_kkt best = {1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0};
    owned_csr at;
    double *x, *x_bar, *x_sum, *x_restart, *x_avg, *aty, *x_cand;
    double *y, *y_sum, *y_restart, *y_avg, *ax_bar, *ax, *y_cand, *ax_cand, *ax_prev;

    memset(stats, 0, sizeof(*stats));
    if (make_transpose(a, &at) != 0) return -1;
#define NV(n_) (double *)calloc((size_t)(n_) + 1, sizeof(double))
    x = NV(n); x_bar = NV(n); x_sum = NV(n); x_restart = NV(n); x_avg = NV(n); aty = NV(n);
    x_cand = NV(n);
    y = NV(m); y_sum = NV(m); y_restart = NV(m); y_avg = NV(m); ax_bar = NV(m); ax = NV(m);
    y_cand = NV(m); ax_cand = NV(m); ax_prev = NV(m);
#undef NV
    for (j = 0; j < n; ++j) if (bound_finite(c[j])) cost_norm += c[j] * c[j];
    cost_norm = sqrt(cost_norm);
    for (i = 0; i < m; ++i) {
        if (bound_finite(row_lower[i])) bl += row_lower[i] * row_lower[i];
        if (bound_finite(row_upper[i])) bu += row_upper[i] * row_upper[i];
    }
    bound_norm = sqrt(sqrt(bl) * sqrt(bl) + sqrt(bu) * sqrt(bu));

    matrix_norm = orc_power_norm(a, params->power_iterations);
    stats->matrix_norm = matrix_norm;
    eta_global = PDLP_STEP_SAFETY / matrix_norm;
    eta_min = params->eta_min_factor / matrix_norm;
    eta_max = params->eta_max_factor / matrix_norm;
    if (cost_norm > 0.0 && bound_norm > 0.0)
        omega = fmin(PDLP_MAX_WEIGHT, fmax(PDLP_MIN_WEIGHT, cost_norm / bound_norm));
    eta = eta_global;

    while (iteration < params->max_iterations) {
        int period = params->restart_period;
        int k;
        double terms;
        pdlp_kkt current, average;
        int average_better;
        if (params->max_iterations - iteration < period) period = params->max_iterations - iteration;
        if (period <= 0) break;
        if (params->adaptive_step) {
            for (k = 0; k < period; ++k) {
                const double sigma = eta * omega, tau = eta / omega;
                double dx_sq = 0.0, dy_sq = 0.0, inter = 0.0, movement, eta_bar, kk, eta_next;
                int accept;
                /* PdlpKernels.cu:377-389 */
                for (i = 0; i < m; ++i) {
                    const double axb = 2.0 * ax[i] - ax_prev[i];
                    const double v = y[i] + sigma * axb;
                    y_cand[i] = v - sigma * clamp_fm(v / sigma, row_lower[i], row_upper[i]);
                }
                orc_csr_spmv(&at.view, y_cand, aty);
                /* :391-400 */
                for (j = 0; j < n; ++j)
                    x_cand[j] = clamp_fm(x[j] - tau * (c[j] + aty[j]), lower[j], upper[j]);
                orc_csr_spmv(a, x_cand, ax_cand);
                /* :405-494 */
                for (j = 0; j < n; ++j) { const double d = x_cand[j] - x[j]; dx_sq += d * d; }
                for (i = 0; i < m; ++i) {
                    const double dy = y_cand[i] - y[i];
                    dy_sq += dy * dy;
                    inter += dy * (ax_cand[i] - ax[i]);
                }
                inter = fabs(inter);
                movement = 0.5 * (omega * dx_sq + dy_sq / omega);
                eta_bar = (inter > 0.0 && movement > 0.0) ? movement / inter : eta_max;
                accept = eta <= eta_bar;
                kk = updates + 1.0;
                eta_next = fmin((1.0 - pow(kk + 1.0, -0.3)) * eta_bar, (1.0 + pow(kk + 1.0, -0.6)) * eta);
                if (!(eta_next > 0.0) || !isfinite(eta_next)) eta_next = eta;
                eta_next = fmin(fmax(eta_next, eta_min), eta_max);
                eta = eta_next;
                updates = kk;
                if (accept) {
                    /* :499-518 */
                    accept_count += 1.0;
                    for (j = 0; j < n; ++j) { x[j] = x_cand[j]; x_sum[j] += x_cand[j]; }
                    for (i = 0; i < m; ++i) {
                        y[i] = y_cand[i];
                        y_sum[i] += y_cand[i];
                        ax_prev[i] = ax[i];
                        ax[i] = ax_cand[i];
                    }
                }
            }
        } else {
            const double tau = eta_global / omega, sigma = eta_global * omega;
            for (k = 0; k < period; ++k) {
                orc_csr_spmv(a, x_bar, ax_bar);
                for (i = 0; i < m; ++i) {   /* PdlpKernels.cu:71-83 */
                    const double v = y[i] + sigma * ax_bar[i];
                    y[i] = v - sigma * clamp_fm(v / sigma, row_lower[i], row_upper[i]);
                    y_sum[i] += 1.0 * y[i];
                }
                orc_csr_spmv(&at.view, y, aty);
                for (j = 0; j < n; ++j) {   /* :85-97 */
                    const double xj = x[j];
                    const double xn = clamp_fm(xj - tau * (c[j] + aty[j]), lower[j], upper[j]);
                    x_bar[j] = 2.0 * xn - xj;
                    x[j] = xn;
                    x_sum[j] += 1.0 * xn;
                }
            }
        }
        iteration += period;
        iterations_since_restart += period;
        ++windows_since_restart;

        pdlp_residuals(a, &at.view, x, y, ax_cand, aty, c, lower, upper, row_lower, row_upper,
                       x_restart, y_restart, cost_norm, bound_norm, &current);
        if (!params->adaptive_step) {
            /* the fixed path evaluates into the live A x buffer (GpuPdlp.cpp:394) */
        }
        if (params->adaptive_step) {
            terms = accept_count - accepted_at_restart;
            if (terms < 1.0) terms = 1.0;
        } else {
            terms = (double)(windows_since_restart * params->restart_period);
        }
        for (j = 0; j < n; ++j) x_avg[j] = (1.0 / terms) * x_sum[j];
        for (i = 0; i < m; ++i) y_avg[i] = (1.0 / terms) * y_sum[i];
        pdlp_residuals(a, &at.view, x_avg, y_avg, ax_bar, aty, c, lower, upper, row_lower,
                       row_upper, x_restart, y_restart, cost_norm, bound_norm, &average);
        average_better = kkt_worst(&average) < kkt_worst(&current);
        best = average_better ? average : current;
        if (best.primal <= params->eps_optimal && best.dual <= params->eps_optimal &&
            best.gap <= params->eps_optimal) {
            if (average_better) {
                memcpy(x, x_avg, sizeof(double) * (size_t)n);
                memcpy(y, y_avg, sizeof(double) * (size_t)m);
            }
            stats->converged = 1;
            break;
        }
        {
            const double mu = kkt_worst(&best);
            const int sufficient = mu <= PDLP_SUFFICIENT * mu_at_restart;
            const int necessary = mu <= PDLP_NECESSARY * mu_at_restart && mu > mu_previous;
            const int artificial =
                (double)iterations_since_restart >= PDLP_ARTIFICIAL * (double)iteration;
            mu_previous = mu;
            if (!(sufficient || necessary || artificial)) continue;
            if (average_better) {
                memcpy(x, x_avg, sizeof(double) * (size_t)n);
                memcpy(y, y_avg, sizeof(double) * (size_t)m);
                memcpy(x_bar, x_avg, sizeof(double) * (size_t)n);
                if (params->adaptive_step) memcpy(ax, ax_bar, sizeof(double) * (size_t)m);
            } else {
                memcpy(x_bar, x, sizeof(double) * (size_t)n);
            }
            if (params->adaptive_step) {
                memcpy(ax_prev, ax, sizeof(double) * (size_t)m);
                accepted_at_restart = accept_count;
            }
            memset(x_sum, 0, sizeof(double) * (size_t)n);
            memset(y_sum, 0, sizeof(double) * (size_t)m);
            windows_since_restart = 0;
            iterations_since_restart = 0;
            mu_at_restart = mu;
            mu_previous = INFINITY;
            stats->restarts++;
            if (best.primal_move > 1e-14 && best.dual_move > 1e-14) {
                const double target = best.dual_move / best.primal_move;
                const double updated =
                    exp(PDLP_SMOOTHING * log(target) + (1.0 - PDLP_SMOOTHING) * log(omega));
                if (isfinite(updated))
                    omega = fmin(PDLP_MAX_WEIGHT, fmax(PDLP_MIN_WEIGHT, updated));
            }
            memcpy(x_restart, x, sizeof(double) * (size_t)n);
            memcpy(y_restart, y, sizeof(double) * (size_t)m);
        }
    }
    for (j = 0; j < n; ++j) x_out[j] = x[j];
    for (i = 0; i < m; ++i) y_out[i] = y[i];
    stats->iterations = iteration;
    stats->primal_objective = best.primal_obj;
    stats->dual_objective = best.dual_obj;
    stats->relative_primal_residual = best.primal;
    stats->relative_dual_residual = best.dual;
    stats->relative_gap = best.gap;
    stats->final_step_size = params->adaptive_step ? eta : eta_global;
    stats->rejected_steps = params->adaptive_step ? (int)(updates - accept_count) : 0;
    free(x); free(x_bar); free(x_sum); free(x_restart); free(x_avg); free(aty); free(x_cand);
    free(y); free(y_sum); free(y_restart); free(y_avg); free(ax_bar); free(ax); free(y_cand);
    free(ax_cand); free(ax_prev);
    free_owned(&at);
    return 0;
}

/* ============================================================
 * Scaling
 * ============================================================ */

/* src/lp/Scaling.cpp:11-92: simultaneous Ruiz infinity-norm equilibration;
   identity when it has not converged within max_iters. */
int orc_ruiz(const orc_csr *a, int max_iters, double tol, double *row_scale, double *col_scale)
{
    const int m = a->rows, n = a->cols, nnz = a->ptr[a->rows];
    int it, i, j, p, converged = 0;
    double *rn, *cn;
    owned_csr at;
    for (i = 0; i < m; ++i) row_scale[i] = 1.0;
    for (j = 0; j < n; ++j) col_scale[j] = 1.0;
    if (nnz == 0 || m == 0 || n == 0) return 1;
    make_transpose(a, &at);
    rn = (double *)calloc((size_t)m, sizeof(double));
    cn = (double *)calloc((size_t)n, sizeof(double));
    for (it = 0; it < max_iters; ++it) {
        double max_dev = 0.0;
        for (i = 0; i < m; ++i) {
            double best = 0.0;
            for (p = a->ptr[i]; p < a->ptr[i + 1]; ++p) {
                const double v = fabs(a->val[p]) * col_scale[a->idx[p]];
                if (v > best) best = v;
            }
            rn[i] = row_scale[i] * best;
        }
        for (j = 0; j < n; ++j) {
            double best = 0.0;
            for (p = at.ptr[j]; p < at.ptr[j + 1]; ++p) {
                const double v = fabs(at.val[p]) * row_scale[at.idx[p]];
                if (v > best) best = v;
            }
            cn[j] = col_scale[j] * best;
        }
        for (i = 0; i < m; ++i) if (rn[i] > 0.0 && fabs(rn[i] - 1.0) > max_dev) max_dev = fabs(rn[i] - 1.0);
        for (j = 0; j < n; ++j) if (cn[j] > 0.0 && fabs(cn[j] - 1.0) > max_dev) max_dev = fabs(cn[j] - 1.0);
        if (max_dev < tol) { converged = 1; break; }
        for (i = 0; i < m; ++i) if (rn[i] > 0.0) row_scale[i] /= sqrt(rn[i]);
        for (j = 0; j < n; ++j) if (cn[j] > 0.0) col_scale[j] /= sqrt(cn[j]);
    }
    if (!converged) {
        for (i = 0; i < m; ++i) row_scale[i] = 1.0;
        for (j = 0; j < n; ++j) col_scale[j] = 1.0;
    }
    free(rn); free(cn);
    free_owned(&at);
    return converged;
}

/* src/lp/Scaling.cpp:111-145 */
void orc_pock_chambolle(const orc_csr *a, double alpha, double *row_scale, double *col_scale)
{
    const int m = a->rows, n = a->cols;
    int i, j, p;
    double *racc = (double *)calloc((size_t)m + 1, sizeof(double));
    double *cacc = (double *)calloc((size_t)n + 1, sizeof(double));
    for (i = 0; i < m; ++i)
        for (p = a->ptr[i]; p < a->ptr[i + 1]; ++p) {
            const double v = fabs(a->val[p]);
            if (v == 0.0) continue;
            racc[i] += pow(v, 2.0 - alpha);
            cacc[a->idx[p]] += pow(v, alpha);
        }
    for (i = 0; i < m; ++i) row_scale[i] = racc[i] > 0.0 ? 1.0 / sqrt(racc[i]) : 1.0;
    for (j = 0; j < n; ++j) col_scale[j] = cacc[j] > 0.0 ? 1.0 / sqrt(cacc[j]) : 1.0;
    free(racc); free(cacc);
}

/* c/src/sk_scale.c:20-72: geometric passes, then rounding to powers of two. */
void orc_pow2_scale(const orc_csr *a, int passes, double *R, double *C)
{
    const int m = a->rows, n = a->cols;
    int i, j, p, it;
    double *rmin, *rmax;
    owned_csr at;
    for (i = 0; i < m; ++i) R[i] = 1.0;
    for (j = 0; j < n; ++j) C[j] = 1.0;
    if (m == 0 || n == 0 || passes <= 0) return;
    make_transpose(a, &at);
    rmin = (double *)calloc((size_t)m, sizeof(double));
    rmax = (double *)calloc((size_t)m, sizeof(double));
    for (it = 0; it < passes; ++it) {
        for (j = 0; j < n; ++j) {
            double mn = 0.0, mx = 0.0;
            for (p = at.ptr[j]; p < at.ptr[j + 1]; ++p) {
                const double v = fabs(at.val[p]) * R[at.idx[p]] * C[j];
                if (v <= 0.0) continue;
                if (mn == 0.0 || v < mn) mn = v;
                if (v > mx) mx = v;
            }
            if (mx > 0.0) C[j] /= sqrt(mn * mx);
        }
        for (i = 0; i < m; ++i) { rmin[i] = 0.0; rmax[i] = 0.0; }
        for (i = 0; i < m; ++i)
            for (p = a->ptr[i]; p < a->ptr[i + 1]; ++p) {
                const double v = fabs(a->val[p]) * R[i] * C[a->idx[p]];
                if (v <= 0.0) continue;
                if (rmin[i] == 0.0 || v < rmin[i]) rmin[i] = v;
                if (v > rmax[i]) rmax[i] = v;
            }
        for (i = 0; i < m; ++i) if (rmax[i] > 0.0) R[i] /= sqrt(rmin[i] * rmax[i]);
    }
    for (i = 0; i < m; ++i) {
        int e;
        if (!(R[i] > 0.0) || !isfinite(R[i])) { R[i] = 1.0; continue; }
        frexp(R[i], &e);
        R[i] = ldexp(1.0, e - 1);
    }
    for (j = 0; j < n; ++j) {
        int e;
        if (!(C[j] > 0.0) || !isfinite(C[j])) { C[j] = 1.0; continue; }
        frexp(C[j], &e);
        C[j] = ldexp(1.0, e - 1);
    }
    free(rmin); free(rmax);
    free_owned(&at);
}
