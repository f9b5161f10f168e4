// TEST INFRASTRUCTURE ONLY. A C entry point onto the reference C++ core's LP driver,
// sihps::solve_lp (src/lp/LpSolver.cpp:126-300: presolve, SIMPLEX / FIRST_ORDER /
// HYBRID, postsolve and the 1e-6 original-space gate), compiled with the core's own
// sources into oracle/_ref by oracle/hooked_lpsolver.py. Two builds use it:
//   libsihps_lp_ref.so     the core as it is (FIRST_ORDER runs the reference's GpuPdlp);
//   libsihps_lp_hooked.so  the core with run_first_order replaced by the integration
//                          block include/integration/lpsolver_run_first_order.inc, so
//                          FIRST_ORDER and HYBRID reach the engine's C ABI.
// The product never links either.
//
// Rows rl <= A x <= ru become the core's A x + s = rhs form the way its MPS reader
// builds ranged rows (src/lp/LpProblem.cpp:29-69): a row with a finite upper bound is
// an 'L' row with rhs = ru and s in [0, ru - rl] ('E' when rl == ru); a row with only
// a lower bound is a 'G' row with rhs = rl and s in (-inf, 0].
#include "lp/LpSolver.hpp"

#include <cmath>
#include <exception>
#include <limits>
#include <vector>

extern "C" {

typedef struct RefLpOptions {
    int method;                       // 0 SIMPLEX, 1 FIRST_ORDER, 2 HYBRID (sihps::LpMethod)
    int use_presolve;
    int hybrid_row_threshold;         // hybrid_first_order_row_threshold
    int pdlp_max_iterations;
    double pdlp_eps;                  // pdlp.eps_optimal (FIRST_ORDER)
    double pdlp_time_limit;           // pdlp.time_limit_seconds (0: none)
    double hybrid_first_order_eps;
    double hybrid_first_order_budget;  // seconds
    double hybrid_simplex_budget;      // seconds
} RefLpOptions;

typedef struct RefLpResult {
    int status;                       // sihps::LpStatus: 0 OPTIMAL, 1 INFEASIBLE, 2 UNBOUNDED, 3 ITERATION_LIMIT, 4 NUMERICAL_FAILURE
    int iterations;
    int used_first_order;
    int first_order_fallback_used;
    int pdlp_converged;
    int pdlp_iterations;
    double objective;
    double primal_residual;           // the original-space gate's residual
    double pdlp_relative_gap;
    double solve_seconds;
} RefLpResult;

void ref_lp_default_options(RefLpOptions* o) {
    const sihps::LpSolverOptions d;
    o->method = static_cast<int>(d.method);
    o->use_presolve = d.use_presolve ? 1 : 0;
    o->hybrid_row_threshold = d.hybrid_first_order_row_threshold;
    o->pdlp_max_iterations = d.pdlp.max_iterations;
    o->pdlp_eps = d.pdlp.eps_optimal;
    o->pdlp_time_limit = d.pdlp.time_limit_seconds;
    o->hybrid_first_order_eps = d.hybrid_first_order_eps;
    o->hybrid_first_order_budget = d.hybrid_first_order_budget_seconds;
    o->hybrid_simplex_budget = d.hybrid_simplex_budget_seconds;
}

// Returns 0 (result filled; x_out, length cols, in the original column space), or -1
// when the core throws.
int ref_solve_lp(int rows, int cols, int nnz, const int* ptr, const int* idx, const double* val, const double* c,
                 const double* cl, const double* cu, const double* rl, const double* ru, const RefLpOptions* o,
                 double* x_out, RefLpResult* r) {
    try {
        const double inf = std::numeric_limits<double>::infinity();
        const auto m = static_cast<std::size_t>(rows);
        sihps::LpProblem p;
        p.A = sihps::CSRMatrix(rows, cols, std::vector<std::int32_t>(ptr, ptr + rows + 1),
                               std::vector<std::int32_t>(idx, idx + nnz), std::vector<double>(val, val + nnz));
        p.obj.assign(c, c + cols);
        p.lower.assign(cl, cl + cols);
        p.upper.assign(cu, cu + cols);
        p.rhs.assign(m, 0.0);
        p.row_types.assign(m, 'L');
        p.slack_lower.assign(m, 0.0);
        p.slack_upper.assign(m, 0.0);
        for (std::size_t i = 0; i < m; ++i) {
            if (std::isfinite(ru[i])) {
                p.rhs[i] = ru[i];
                p.row_types[i] = rl[i] == ru[i] ? 'E' : 'L';
                p.slack_upper[i] = std::isfinite(rl[i]) ? ru[i] - rl[i] : inf;
            } else {
                p.rhs[i] = rl[i];
                p.row_types[i] = 'G';
                p.slack_lower[i] = -inf;
            }
        }
        sihps::LpSolverOptions opt;
        opt.method = static_cast<sihps::LpMethod>(o->method);
        opt.use_presolve = o->use_presolve != 0;
        opt.hybrid_first_order_row_threshold = o->hybrid_row_threshold;
        opt.pdlp.max_iterations = o->pdlp_max_iterations;
        opt.pdlp.eps_optimal = o->pdlp_eps;
        opt.pdlp.time_limit_seconds = o->pdlp_time_limit;
        opt.hybrid_first_order_eps = o->hybrid_first_order_eps;
        opt.hybrid_first_order_budget_seconds = o->hybrid_first_order_budget;
        opt.hybrid_simplex_budget_seconds = o->hybrid_simplex_budget;
        const sihps::LpSolution s = sihps::solve_lp(p, opt);
        r->status = static_cast<int>(s.status);
        r->iterations = s.iterations;
        r->used_first_order = s.used_first_order ? 1 : 0;
        r->first_order_fallback_used = s.first_order_fallback_used ? 1 : 0;
        r->pdlp_converged = s.pdlp.converged ? 1 : 0;
        r->pdlp_iterations = s.pdlp.iterations;
        r->objective = s.objective_value;
        r->primal_residual = s.primal_residual;
        r->pdlp_relative_gap = s.pdlp.relative_gap;
        r->solve_seconds = s.solve_seconds;
        for (int j = 0; j < cols; ++j) x_out[j] = j < static_cast<int>(s.x.size()) ? s.x[static_cast<std::size_t>(j)] : 0.0;
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
