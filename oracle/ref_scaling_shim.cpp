// TEST INFRASTRUCTURE ONLY. A C entry point onto the reference's own equilibration
// code (src/lp/Scaling.cpp: compute_ruiz_scaling, compute_pock_chambolle_scaling),
// compiled together with it from the reference tree into oracle/_ref by
// oracle/Makefile. The tests use it to pin the oracle's Ruiz and Pock-Chambolle
// restatements to the reference's results; the product never links it.
#include "lp/Scaling.hpp"

#include <algorithm>
#include <vector>

namespace {

sihps::CSRMatrix make_matrix(int rows, int cols, int nnz, const int* ptr, const int* idx, const double* val) {
    std::vector<std::int32_t> p(ptr, ptr + rows + 1);
    std::vector<std::int32_t> i(idx, idx + nnz);
    std::vector<double> v(val, val + nnz);
    return sihps::CSRMatrix(rows, cols, std::move(p), std::move(i), std::move(v));
}

int copy_out(const sihps::ScaleFactors& f, int rows, int cols, double* row_scale, double* col_scale) {
    if (static_cast<int>(f.row_scale.size()) != rows || static_cast<int>(f.col_scale.size()) != cols) return -1;
    std::copy(f.row_scale.begin(), f.row_scale.end(), row_scale);
    std::copy(f.col_scale.begin(), f.col_scale.end(), col_scale);
    return 0;
}

}  // namespace

// Returns 0, or -1 when the reference rejects the matrix (its constructor throws).
extern "C" int ref_ruiz_scaling(int rows, int cols, int nnz, const int* ptr, const int* idx, const double* val,
                                int max_iters, double tol, double* row_scale, double* col_scale) {
    try {
        const sihps::CSRMatrix a = make_matrix(rows, cols, nnz, ptr, idx, val);
        return copy_out(sihps::compute_ruiz_scaling(a, max_iters, tol), rows, cols, row_scale, col_scale);
    } catch (...) {
        return -1;
    }
}

extern "C" int ref_pock_chambolle_scaling(int rows, int cols, int nnz, const int* ptr, const int* idx,
                                          const double* val, double alpha, double* row_scale, double* col_scale) {
    try {
        const sihps::CSRMatrix a = make_matrix(rows, cols, nnz, ptr, idx, val);
        return copy_out(sihps::compute_pock_chambolle_scaling(a, alpha), rows, cols, row_scale, col_scale);
    } catch (...) {
        return -1;
    }
}
