// Crossover from a first-order point to an optimal basis for the reference's C++
// core (src/lp): the engine's answer (sankhya_b200_pdlp_solve / _polished, as
// run_first_order returns it) seats a basis in the core's own revised simplex,
// whose warm path (sihps::Simplex::set_warm_start_basis, src/lp/Simplex.hpp:221-228;
// seat_basis then dual simplex, src/lp/Simplex.cpp:457-543, 1508-1533) finishes it
// and holds the answer to the same original-space gate as every other path.
//
// The basis: the nrow columns of the augmented system A x + s = rhs (structurals
// and row slacks) with the smallest reduced cost magnitudes at the first-order dual,
// ties to the ones farthest inside their bounds; positions the core's sparse LU
// (sihps::BasisFactorization) finds dependent take the slack of their unmatched
// row. Each nonbasic column rests at the bound that the sign of its reduced cost at
// the basis's own duals (B' pi = c_B, solved with that LU) makes dual feasible, so
// the dual simplex starts from a dual feasible basis and only repairs the primal
// side. A basis that does not seat, or whose repair fails the gate, leaves the
// solve to the core's cold paths.
#pragma once

#include "lp/LpProblem.hpp"
#include "lp/Simplex.hpp"

#include <vector>

namespace sihps_b200 {

struct CrossoverStats {
    int basic_structurals = 0;  // structurals in the seated basis
    int repaired = 0;           // dependent positions given a slack
    bool used_warm_start = false;
    int dual_iterations = 0;    // pivots of the warm dual simplex
    int cold_iterations = 0;    // phase 1 + phase 2 pivots when the cold path ran
    double seconds = 0.0;
};

// problem: the LP in the core's form; x (n_cols) and y (n_rows): the first-order
// point, y with rc = c + A'y (sk_solve's sign, the engine's; all zero when the caller
// kept only x, as run_first_order does: the basis is then ranked by interiority alone);
// time_budget: seconds for
// the simplex (Simplex::set_time_budget; 0: none), after which it returns
// ITERATION_LIMIT, as HYBRID's budgeted simplex does. Returns the core's LpResult
// (status, x, y_dual, objective and residuals in original units).
sihps::LpResult crossover(const sihps::LpProblem& problem, const std::vector<double>& x,
                          const std::vector<double>& y, CrossoverStats* stats = nullptr,
                          double time_budget = 0.0);

}  // namespace sihps_b200
