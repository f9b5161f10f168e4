// TEST INFRASTRUCTURE ONLY. C entry points onto the reference C++ core's own GPU PDLP
// (src/cuda/GpuPdlp.cpp and PdlpKernels.cu, over cuSPARSE), compiled with it from the
// reference tree into oracle/_ref by oracle/Makefile, so that the engine's PDLP can be
// compared with the reference's GPU implementation on the same device. The product
// never links it.
//
// With `scale` set, the call follows the reference's first-order driver,
// run_first_order (src/lp/LpSolver.cpp:62-99): Ruiz, then Pock-Chambolle on the
// Ruiz-scaled matrix, composed into one pair of factors (the reference's own
// Scaling.cpp); cost and bounds moved into the scaled space; GpuPdlp; x moved back.
#include "cuda/GpuPdlp.hpp"
#include "lp/Scaling.hpp"

#include <vector>

extern "C" {

typedef struct RefPdlpParams {
    double eps_optimal;
    int max_iterations;
    int restart_period;
    double time_limit_seconds;
    int power_iterations;
    int adaptive_step;
    double eta_min_factor;
    double eta_max_factor;
    int scale;   // 1: Ruiz + Pock-Chambolle as run_first_order does; 0: the model as given
    int reserved;
} RefPdlpParams;

typedef struct RefPdlpStats {
    int converged;
    int iterations;
    int restarts;
    int rejected_steps;
    int host_syncs;
    int reserved;
    double primal_objective;
    double dual_objective;
    double relative_primal_residual;
    double relative_dual_residual;
    double relative_gap;
    double matrix_norm;
    double seconds;
} RefPdlpStats;

// Returns 0 (stats filled, x_out in the caller's space), or -1 when the reference
// throws (invalid matrix, CUDA or cuSPARSE error).
int ref_gpupdlp_solve(int rows, int cols, int nnz, const int* ptr, const int* idx, const double* val,
                      const double* c, const double* cl, const double* cu, const double* rl, const double* ru,
                      const RefPdlpParams* p, double* x_out, RefPdlpStats* st) {
    try {
        const auto n = static_cast<std::size_t>(cols), m = static_cast<std::size_t>(rows);
        sihps::CSRMatrix a(rows, cols, std::vector<std::int32_t>(ptr, ptr + rows + 1),
                           std::vector<std::int32_t>(idx, idx + nnz), std::vector<double>(val, val + nnz));
        sihps::ScaleFactors scale = sihps::ScaleFactors::identity(rows, cols);
        if (p->scale) {
            const sihps::ScaleFactors ruiz = sihps::compute_ruiz_scaling(a);
            const sihps::ScaleFactors pc = sihps::compute_pock_chambolle_scaling(sihps::apply_ruiz_scaling(a, ruiz));
            scale = sihps::compose_scaling(ruiz, pc);
        }
        const sihps::CSRMatrix a_scaled = p->scale ? sihps::apply_ruiz_scaling(a, scale) : a;
        std::vector<double> cost(n), lower(n), upper(n), row_lower(m), row_upper(m);
        for (std::size_t j = 0; j < n; ++j) {
            cost[j] = c[j] * scale.col_scale[j];
            lower[j] = cl[j] / scale.col_scale[j];
            upper[j] = cu[j] / scale.col_scale[j];
        }
        for (std::size_t i = 0; i < m; ++i) {
            row_lower[i] = scale.row_scale[i] * rl[i];
            row_upper[i] = scale.row_scale[i] * ru[i];
        }
        sihps::PdlpParams params;
        params.eps_optimal = p->eps_optimal;
        params.max_iterations = p->max_iterations;
        params.restart_period = p->restart_period;
        params.time_limit_seconds = p->time_limit_seconds;
        params.power_iterations = p->power_iterations;
        params.adaptive_step = p->adaptive_step != 0;
        params.eta_min_factor = p->eta_min_factor;
        params.eta_max_factor = p->eta_max_factor;
        sihps::GpuPdlp pdlp(a_scaled, cost, lower, upper, row_lower, row_upper);
        std::vector<double> xs, ys;
        const sihps::PdlpStats s = pdlp.solve(params, xs, ys);
        for (std::size_t j = 0; j < n; ++j) x_out[j] = xs[j] * scale.col_scale[j];
        st->converged = s.converged ? 1 : 0;
        st->iterations = s.iterations;
        st->restarts = s.restarts;
        st->rejected_steps = s.rejected_steps;
        st->host_syncs = s.host_syncs;
        st->reserved = 0;
        st->primal_objective = s.primal_objective;
        st->dual_objective = s.dual_objective;
        st->relative_primal_residual = s.relative_primal_residual;
        st->relative_dual_residual = s.relative_dual_residual;
        st->relative_gap = s.relative_gap;
        st->matrix_norm = s.matrix_norm;
        st->seconds = s.seconds;
        return 0;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
