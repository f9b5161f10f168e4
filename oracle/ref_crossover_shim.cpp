// TEST INFRASTRUCTURE ONLY. A C entry point onto the crossover integration source for
// the reference C++ core (include/integration/sihps_crossover.cpp), compiled with it into
// oracle/_ref/libsihps_crossover_ref.so and linked to the core's LP build
// (oracle/_ref/libsihps_lp_ref.so). Rows rl <= A x <= ru become the core's A x + s = rhs
// form exactly as in ref_lpsolver_shim.cpp. The product never links it.
#include "sihps_crossover.hpp"

#include <cmath>
#include <exception>
#include <limits>
#include <vector>

extern "C" {

typedef struct RefCrossoverResult {
    int status;             // sihps::LpStatus: 0 OPTIMAL ... 4 NUMERICAL_FAILURE
    int used_warm_start;
    int dual_iterations;
    int cold_iterations;
    int basic_structurals;
    int repaired;
    double objective;
    double primal_residual;
    double dual_residual;
    double seconds;
} RefCrossoverResult;

// Returns 0 (result, x_out (cols) and y_out (rows, the core's y_dual) filled), or -1 when
// the core throws.
int ref_crossover_lp(int rows, int cols, int nnz, const int* ptr, const int* idx, const double* val,
                     const double* c, const double* cl, const double* cu, const double* rl, const double* ru,
                     const double* x, const double* y, double time_budget, double* x_out, double* y_out,
                     RefCrossoverResult* r) {
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
        sihps_b200::CrossoverStats st;
        const sihps::LpResult s = sihps_b200::crossover(p, std::vector<double>(x, x + cols),
                                                        std::vector<double>(y, y + rows), &st, time_budget);
        r->status = static_cast<int>(s.status);
        r->used_warm_start = st.used_warm_start ? 1 : 0;
        r->dual_iterations = st.dual_iterations;
        r->cold_iterations = st.cold_iterations;
        r->basic_structurals = st.basic_structurals;
        r->repaired = st.repaired;
        r->objective = s.objective_value;
        r->primal_residual = s.primal_residual;
        r->dual_residual = s.dual_residual;
        r->seconds = st.seconds;
        for (int j = 0; j < cols; ++j) x_out[j] = j < static_cast<int>(s.x.size()) ? s.x[static_cast<std::size_t>(j)] : 0.0;
        for (int i = 0; i < rows; ++i)
            y_out[i] = i < static_cast<int>(s.y_dual.size()) ? s.y_dual[static_cast<std::size_t>(i)] : 0.0;
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
