/* Crossover from a first-order point to a certified vertex: see sk_crossover.h.
   Built with the reference's C core (-I c/include, linked with its library);
   it calls only the core's public sk_simplex_solve, sk_verify and sk_solution_*. */
#include "sk_crossover.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "sk_simplex.h"

enum { FREE_COL = 0, AT_LOW = 1, AT_UPP = 2 };

/* rc = c + A'y over the CSC columns of m */
static void reduced_costs(const sk_model* m, const double* y, double* rc)
{
    for (int j = 0; j < m->ncol; ++j) {
        double r = m->c[j];
        for (int p = m->A.p[j]; p < m->A.p[j + 1]; ++p) r += m->A.x[p] * y[m->A.i[p]];
        rc[j] = r;
    }
}

/* The LP over the columns with state FREE_COL, the others held at their bounds. The
   arrays it allocates hang off `red` and `keep` and are released by release_smaller. */
typedef struct smaller_lp {
    sk_model red;
    int* keep;     /* smaller-LP column -> column of m */
    int kept;
} smaller_lp;

static void release_smaller(smaller_lp* s)
{
    free(s->red.A.p); free(s->red.A.i); free(s->red.A.x);
    free(s->red.c); free(s->red.clow); free(s->red.cupp); free(s->red.rlow); free(s->red.rupp);
    free(s->red.vartype); free(s->keep);
    memset(s, 0, sizeof(*s));
}

static sk_status build_smaller(const sk_model* m, const unsigned char* state, smaller_lp* s)
{
    const int n = m->ncol, r = m->nrow;
    int kept = 0, nnz = 0;
    memset(s, 0, sizeof(*s));
    for (int j = 0; j < n; ++j)
        if (state[j] == FREE_COL) { ++kept; nnz += m->A.p[j + 1] - m->A.p[j]; }
    s->keep = (int*)malloc(sizeof(int) * (size_t)(kept + 1));
    s->red.A.p = (int*)malloc(sizeof(int) * (size_t)(kept + 1));
    s->red.A.i = (int*)malloc(sizeof(int) * (size_t)(nnz + 1));
    s->red.A.x = (double*)malloc(sizeof(double) * (size_t)(nnz + 1));
    s->red.c = (double*)malloc(sizeof(double) * (size_t)(kept + 1));
    s->red.clow = (double*)malloc(sizeof(double) * (size_t)(kept + 1));
    s->red.cupp = (double*)malloc(sizeof(double) * (size_t)(kept + 1));
    s->red.vartype = (unsigned char*)calloc((size_t)kept + 1, 1);
    s->red.rlow = (double*)malloc(sizeof(double) * (size_t)(r + 1));
    s->red.rupp = (double*)malloc(sizeof(double) * (size_t)(r + 1));
    double* held = (double*)calloc((size_t)r + 1, sizeof(double));
    if (!s->keep || !s->red.A.p || !s->red.A.i || !s->red.A.x || !s->red.c || !s->red.clow || !s->red.cupp ||
        !s->red.vartype || !s->red.rlow || !s->red.rupp || !held) {
        free(held);
        release_smaller(s);
        return SK_ERR_MEMORY;
    }
    double shift = m->objshift;
    int k = 0, q = 0;
    s->red.A.p[0] = 0;
    for (int j = 0; j < n; ++j) {
        if (state[j] == FREE_COL) {
            s->keep[k] = j;
            s->red.c[k] = m->c[j];
            s->red.clow[k] = m->clow[j];
            s->red.cupp[k] = m->cupp[j];
            for (int p = m->A.p[j]; p < m->A.p[j + 1]; ++p, ++q) {
                s->red.A.i[q] = m->A.i[p];
                s->red.A.x[q] = m->A.x[p];
            }
            s->red.A.p[++k] = q;
        } else {
            const double v = state[j] == AT_LOW ? m->clow[j] : m->cupp[j];
            shift += m->c[j] * v;
            for (int p = m->A.p[j]; p < m->A.p[j + 1]; ++p) held[m->A.i[p]] += m->A.x[p] * v;
        }
    }
    for (int i = 0; i < r; ++i) {
        s->red.rlow[i] = SK_IS_NEG_INF(m->rlow[i]) ? m->rlow[i] : m->rlow[i] - held[i];
        s->red.rupp[i] = SK_IS_INF(m->rupp[i]) ? m->rupp[i] : m->rupp[i] - held[i];
    }
    free(held);
    s->red.nrow = r;
    s->red.ncol = kept;
    s->red.A.nrow = r;
    s->red.A.ncol = kept;
    s->red.A.nzmax = nnz > 0 ? nnz : 1;
    s->red.objshift = shift;
    s->red.objsense = 1.0;
    s->kept = kept;
    return SK_OK;
}

/* The whole model's solution from the smaller LP's: x of the held columns at their
   bounds, y as solved; sk_verify then fills rc, rowact, objective and the residuals. */
static sk_status assemble(const sk_model* m, const unsigned char* state, const smaller_lp* s,
                          const sk_solution* rs, sk_solution* out)
{
    const int n = m->ncol, r = m->nrow;
    out->x = (double*)malloc(sizeof(double) * (size_t)(n + 1));
    out->y = (double*)malloc(sizeof(double) * (size_t)(r + 1));
    out->rc = (double*)malloc(sizeof(double) * (size_t)(n + 1));
    out->rowact = (double*)malloc(sizeof(double) * (size_t)(r + 1));
    if (!out->x || !out->y || !out->rc || !out->rowact) return SK_ERR_MEMORY;
    out->ncol = n;
    out->nrow = r;
    for (int j = 0; j < n; ++j)
        if (state[j] != FREE_COL) out->x[j] = state[j] == AT_LOW ? m->clow[j] : m->cupp[j];
    for (int k = 0; k < s->kept; ++k) out->x[s->keep[k]] = rs->x[k];
    for (int i = 0; i < r; ++i) out->y[i] = rs->y ? rs->y[i] : 0.0;
    return sk_verify(m, out);
}

sk_status sk_b200_crossover(const sk_model* m, const sk_options* o, const double* x, const double* y,
                            double fix_tolerance, int max_rounds, sk_solution* out,
                            sk_b200_crossover_stats* stats)
{
    sk_b200_crossover_stats local;
    if (!stats) stats = &local;
    memset(stats, 0, sizeof(*stats));
    if (!m || !o || !x || !y || !out || !(fix_tolerance > 0.0) || max_rounds < 1 || m->Q || m->objsense != 1.0)
        return SK_ERR_ARG;
    if (sk_model_validate(m) != SK_OK) return SK_ERR_STRUCTURE;
    const double t0 = sk_wall_seconds();
    const int n = m->ncol;
    unsigned char* state = (unsigned char*)calloc((size_t)n + 1, 1);
    double* rc = (double*)malloc(sizeof(double) * (size_t)(n + 1));
    if (!state || !rc) { free(state); free(rc); return SK_ERR_MEMORY; }

    /* the bounds the first-order point selects */
    reduced_costs(m, y, rc);
    const double window = sqrt(fix_tolerance);
    for (int j = 0; j < n; ++j) {
        const int lo = !SK_IS_NEG_INF(m->clow[j]), hi = !SK_IS_INF(m->cupp[j]);
        if (lo && hi && m->clow[j] == m->cupp[j]) state[j] = AT_LOW;
        else if (lo && rc[j] > fix_tolerance && x[j] - m->clow[j] <= window * (1.0 + fabs(m->clow[j])))
            state[j] = AT_LOW;
        else if (hi && rc[j] < -fix_tolerance && m->cupp[j] - x[j] <= window * (1.0 + fabs(m->cupp[j])))
            state[j] = AT_UPP;
    }

    sk_status st = SK_OK;
    int certified = 0;
    for (int round = 0; round < max_rounds && !certified; ++round) {
        smaller_lp s;
        st = build_smaller(m, state, &s);
        if (st != SK_OK) break;
        sk_solution rs;
        sk_spx_stats ss;
        sk_solution_init(&rs);
        memset(&ss, 0, sizeof(ss));
        st = sk_simplex_solve(&s.red, o, &rs, &ss);
        ++stats->rounds;
        stats->simplex_iterations += ss.iterations;
        stats->fixed_columns = n - s.kept;
        int released = 0;
        if (st == SK_OK && rs.result == SK_RESULT_OPTIMAL) {
            sk_solution_free(out);
            st = assemble(m, state, &s, &rs, out);
            if (st == SK_OK && out->primal_infeasibility <= o->primal_tol && out->dual_infeasibility <= o->dual_tol) {
                certified = 1;
            } else if (st == SK_OK) {
                /* release held columns whose reduced cost at the new duals points away from their bound */
                for (int j = 0; j < n; ++j) {
                    if (state[j] == FREE_COL || m->clow[j] == m->cupp[j]) continue;
                    if ((state[j] == AT_LOW && out->rc[j] < -o->dual_tol) ||
                        (state[j] == AT_UPP && out->rc[j] > o->dual_tol)) {
                        state[j] = FREE_COL;
                        ++released;
                    }
                }
            }
        }
        sk_solution_free(&rs);
        release_smaller(&s);
        stats->released_columns += released;
        if (st != SK_OK || (!certified && released == 0)) break;
    }
    free(state);
    free(rc);
    if (!certified && st != SK_ERR_MEMORY) {
        /* the whole model from the simplex's usual start */
        sk_spx_stats ss;
        memset(&ss, 0, sizeof(ss));
        sk_solution_free(out);
        st = sk_simplex_solve(m, o, out, &ss);
        stats->full_fallback = 1;
        stats->simplex_iterations += ss.iterations;
        if (st == SK_OK && out->result == SK_RESULT_OPTIMAL) st = sk_verify(m, out);
    } else if (certified) {
        out->result = SK_RESULT_OPTIMAL;
        out->iterations = stats->simplex_iterations;
    }
    stats->seconds = sk_wall_seconds() - t0;
    out->solve_seconds = stats->seconds;
    return st;
}
