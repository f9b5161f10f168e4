// Crossover for the reference's C++ core: see sihps_crossover.hpp. Built with the
// core's sources (-I src); it uses the core's public LpProblem, Simplex (its Basis and
// warm start) and BasisFactorization.
#include "sihps_crossover.hpp"

#include "lp/BasisFactorization.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <limits>
#include <numeric>

namespace sihps_b200 {

namespace {

using Status = sihps::Simplex::VarStatus;

// A in CSC form (the basis columns are columns of A)
struct Columns {
    std::vector<std::int32_t> ptr, row;
    std::vector<double> val;
};

Columns by_column(const sihps::CSRMatrix& A) {
    const std::int32_t m = A.rows(), n = A.cols(), nnz = A.nnz();
    Columns c;
    c.ptr.assign(static_cast<std::size_t>(n) + 1, 0);
    c.row.resize(static_cast<std::size_t>(nnz));
    c.val.resize(static_cast<std::size_t>(nnz));
    const std::int32_t* rp = A.row_ptr();
    const std::int32_t* ci = A.col_idx();
    const double* v = A.values();
    for (std::int32_t k = 0; k < nnz; ++k) ++c.ptr[static_cast<std::size_t>(ci[k]) + 1];
    for (std::int32_t j = 0; j < n; ++j) c.ptr[static_cast<std::size_t>(j) + 1] += c.ptr[static_cast<std::size_t>(j)];
    std::vector<std::int32_t> next(c.ptr.begin(), c.ptr.end() - 1);
    for (std::int32_t i = 0; i < m; ++i)
        for (std::int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            const auto q = static_cast<std::size_t>(next[static_cast<std::size_t>(ci[k])]++);
            c.row[q] = i;
            c.val[q] = v[k];
        }
    return c;
}

}  // namespace

sihps::LpResult crossover(const sihps::LpProblem& p, const std::vector<double>& x, const std::vector<double>& y,
                          CrossoverStats* stats, double time_budget) {
    CrossoverStats local;
    CrossoverStats& st = stats ? *stats : local;
    st = CrossoverStats{};
    const auto t0 = std::chrono::steady_clock::now();
    const std::int32_t m = p.n_rows(), n = p.n_cols(), nv = n + m;
    const auto um = static_cast<std::size_t>(m), unv = static_cast<std::size_t>(nv);
    const Columns A = by_column(p.A);

    // values, bounds and reduced costs of the augmented columns: structurals, then the
    // row slacks s = rhs - A x (column e_i, cost 0; reduced cost y_i in rc = c + A'y terms)
    std::vector<double> value(unv), lo(unv), hi(unv), red(unv);
    std::vector<double> ax(um, 0.0);
    p.A.multiply(x.data(), ax.data());
    for (std::int32_t j = 0; j < n; ++j) {
        const auto jj = static_cast<std::size_t>(j);
        value[jj] = x[jj];
        lo[jj] = p.lower[jj];
        hi[jj] = p.upper[jj];
        double r = p.obj[jj];
        for (std::int32_t q = A.ptr[jj]; q < A.ptr[jj + 1]; ++q)
            r += A.val[static_cast<std::size_t>(q)] * y[static_cast<std::size_t>(A.row[static_cast<std::size_t>(q)])];
        red[jj] = r;
    }
    for (std::int32_t i = 0; i < m; ++i) {
        const auto ii = static_cast<std::size_t>(i), v = static_cast<std::size_t>(n + i);
        value[v] = p.rhs[ii] - ax[ii];
        lo[v] = p.slack_lower[ii];
        hi[v] = p.slack_upper[ii];
        red[v] = y[ii];
    }
    std::vector<double> inside(unv);
    for (std::size_t v = 0; v < unv; ++v) {
        double d = std::numeric_limits<double>::infinity();
        if (std::isfinite(lo[v])) d = std::min(d, (value[v] - lo[v]) / (1.0 + std::fabs(lo[v])));
        if (std::isfinite(hi[v])) d = std::min(d, (hi[v] - value[v]) / (1.0 + std::fabs(hi[v])));
        inside[v] = d;
    }

    // the basis: smallest |reduced cost| first, ties to the most interior; a caller with
    // no dual (y all zero, e.g. an answer that kept only x) ranks by interiority alone
    bool have_dual = false;
    for (std::int32_t i = 0; i < m && !have_dual; ++i) have_dual = y[static_cast<std::size_t>(i)] != 0.0;
    std::vector<std::int32_t> order(unv);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](std::int32_t a, std::int32_t b) {
        const auto ua = static_cast<std::size_t>(a), ub = static_cast<std::size_t>(b);
        if (have_dual) {
            const double ra = std::fabs(red[ua]), rb = std::fabs(red[ub]);
            if (ra != rb) return ra < rb;
        }
        return inside[ua] > inside[ub];
    });
    sihps::Simplex::Basis basis;
    basis.n_struct = n;
    basis.n_slack = m;
    basis.n_art = m;
    basis.basic_columns.assign(order.begin(), order.begin() + std::min<std::size_t>(um, unv));
    basis.art_sign.assign(um, 1.0);

    // factorize it with the core's LU; dependent positions take their unmatched row's slack
    const auto column = [&](std::int32_t v) {
        sihps::SparseColumn col;
        if (v < n) {
            const auto vv = static_cast<std::size_t>(v);
            for (std::int32_t q = A.ptr[vv]; q < A.ptr[vv + 1]; ++q)
                col.emplace_back(A.row[static_cast<std::size_t>(q)], A.val[static_cast<std::size_t>(q)]);
        } else {
            col.emplace_back(v - n, 1.0);
        }
        return col;
    };
    sihps::BasisFactorization lu;
    bool factored = false;
    for (int attempt = 0; attempt < 4 && !factored; ++attempt) {
        std::vector<sihps::SparseColumn> cols;
        cols.reserve(um);
        for (std::int32_t v : basis.basic_columns) cols.push_back(column(v));
        const auto fr = lu.factorize(m, cols);
        factored = fr.singular.empty();
        for (const auto& pr : fr.singular) {
            basis.basic_columns[static_cast<std::size_t>(pr.first)] = n + pr.second;
            ++st.repaired;
        }
    }

    std::vector<char> is_basic(unv, 0);
    for (std::int32_t v : basis.basic_columns) {
        if (is_basic[static_cast<std::size_t>(v)]) factored = false;   // a repair repeated a column
        is_basic[static_cast<std::size_t>(v)] = 1;
    }

    // the basis's duals (B' pi = c_B) and the reduced costs they give: d = c - A' pi,
    // slacks -pi; each nonbasic column rests at the bound that d's sign makes dual feasible
    std::vector<double> pi(um, 0.0);
    for (std::size_t k = 0; k < um; ++k) {
        const std::int32_t v = basis.basic_columns[k];
        pi[k] = v < n ? p.obj[static_cast<std::size_t>(v)] : 0.0;
    }
    if (factored) lu.btran(pi);
    basis.nonbasic_status.assign(unv + um, Status::AT_LOWER);   // artificials rest at 0
    for (std::int32_t v = 0; v < nv; ++v) {
        const auto vv = static_cast<std::size_t>(v);
        if (is_basic[vv]) {
            basis.nonbasic_status[vv] = Status::BASIC;
            if (v < n) ++st.basic_structurals;
            continue;
        }
        double d;
        if (v < n) {
            d = p.obj[vv];
            for (std::int32_t q = A.ptr[vv]; q < A.ptr[vv + 1]; ++q)
                d -= A.val[static_cast<std::size_t>(q)] * pi[static_cast<std::size_t>(A.row[static_cast<std::size_t>(q)])];
        } else {
            d = -pi[static_cast<std::size_t>(v - n)];
        }
        const bool lf = std::isfinite(lo[vv]), hf = std::isfinite(hi[vv]);
        if (!lf && !hf) {
            basis.nonbasic_status[vv] = Status::AT_ZERO;
        } else if (lf && hf) {
            const bool low = d > 0.0 ? true : d < 0.0 ? false : value[vv] - lo[vv] <= hi[vv] - value[vv];
            basis.nonbasic_status[vv] = low ? Status::AT_LOWER : Status::AT_UPPER;
        } else {
            basis.nonbasic_status[vv] = lf ? Status::AT_LOWER : Status::AT_UPPER;
        }
    }

    sihps::Simplex simplex(p);
    if (time_budget > 0.0) simplex.set_time_budget(time_budget);
    if (factored) simplex.set_warm_start_basis(&basis);
    sihps::LpResult r = simplex.solve();
    st.used_warm_start = r.used_warm_start;
    st.dual_iterations = r.dual_iterations;
    st.cold_iterations = r.phase1_iterations + r.phase2_iterations;
    st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return r;
}

}  // namespace sihps_b200
