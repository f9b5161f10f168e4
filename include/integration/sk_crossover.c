/* Crossover from a first-order point to a certified vertex: see sk_crossover.h.
   Built with the reference's C core (-I c/include, linked with its library);
   it calls only the core's public sk_simplex_solve, sk_verify and sk_solution_*. */
#include "sk_crossover.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "sk_lu.h"
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

/* The basis the first-order point identifies, taken as it stands: of the ncol + nrow
   columns of [A -I] (structurals, and the row logicals s = A x), the nrow with the
   smallest reduced cost (|rc_j|; a logical's is |y_i|), ties to the farthest inside
   their bounds, factorized with the core's sparse LU; its duals pi (B' pi = c_B) set
   every nonbasic column at the bound that makes it dual feasible, the basic values
   follow from B z_B = -N z_N, and sk_verify certifies the point (y = -pi in sk_solve's
   sign). Returns 1 with out filled when the certificate holds; 0 otherwise (a singular
   basis, or a basic value outside its bounds: the simplex has work to do). */
typedef struct ranked {
    double cost, inside;
    int v;
} ranked;

static int by_rank(const void* a, const void* b)
{
    const ranked* p = (const ranked*)a;
    const ranked* q = (const ranked*)b;
    if (p->cost != q->cost) return p->cost < q->cost ? -1 : 1;
    if (p->inside != q->inside) return p->inside > q->inside ? -1 : 1;
    return p->v - q->v;
}

static int direct_basis(const sk_model* m, const sk_options* o, const double* x, const double* y, const double* rc,
                        sk_solution* out)
{
    const int n = m->ncol, r = m->nrow, nv = n + r;
    int ok = 0;
    double* act = (double*)calloc((size_t)r + 1, sizeof(double));
    double* value = (double*)malloc(sizeof(double) * (size_t)(nv + 1));
    double* lo = (double*)malloc(sizeof(double) * (size_t)(nv + 1));
    double* hi = (double*)malloc(sizeof(double) * (size_t)(nv + 1));
    ranked* rank = (ranked*)malloc(sizeof(ranked) * (size_t)(nv + 1));
    int* pos = (int*)malloc(sizeof(int) * (size_t)(nv + 1));       /* basis position or -1 */
    double* pi = (double*)calloc((size_t)r + 1, sizeof(double));
    double* z = (double*)calloc((size_t)r + 1, sizeof(double));
    sk_csc B;
    memset(&B, 0, sizeof(B));
    B.p = (int*)malloc(sizeof(int) * (size_t)(r + 1));
    B.i = (int*)malloc(sizeof(int) * (size_t)(m->A.p[n] + r + 1));
    B.x = (double*)malloc(sizeof(double) * (size_t)(m->A.p[n] + r + 1));
    sk_lu lu;
    sk_lu_init(&lu);
    if (!act || !value || !lo || !hi || !rank || !pos || !pi || !z || !B.p || !B.i || !B.x) goto done;
    /* a caller with no dual (y all zero) ranks by interiority alone */
    int have_dual = 0;
    for (int i = 0; i < r && !have_dual; ++i) have_dual = y[i] != 0.0;

    for (int j = 0; j < n; ++j)
        for (int p = m->A.p[j]; p < m->A.p[j + 1]; ++p) act[m->A.i[p]] += m->A.x[p] * x[j];
    for (int v = 0; v < nv; ++v) {
        value[v] = v < n ? x[v] : act[v - n];
        lo[v] = v < n ? m->clow[v] : m->rlow[v - n];
        hi[v] = v < n ? m->cupp[v] : m->rupp[v - n];
        double d = INFINITY;
        if (!SK_IS_NEG_INF(lo[v])) d = fmin(d, (value[v] - lo[v]) / (1.0 + fabs(lo[v])));
        if (!SK_IS_INF(hi[v])) d = fmin(d, (hi[v] - value[v]) / (1.0 + fabs(hi[v])));
        rank[v].cost = have_dual ? fabs(v < n ? rc[v] : y[v - n]) : 0.0;
        rank[v].inside = d;
        rank[v].v = v;
        pos[v] = -1;
    }
    qsort(rank, (size_t)nv, sizeof(ranked), by_rank);

    /* B: structural columns of A, logical columns -e_i */
    int nz = 0;
    B.nrow = B.ncol = r;
    B.p[0] = 0;
    for (int k = 0; k < r; ++k) {
        const int v = rank[k].v;
        pos[v] = k;
        if (v < n) {
            for (int p = m->A.p[v]; p < m->A.p[v + 1]; ++p, ++nz) { B.i[nz] = m->A.i[p]; B.x[nz] = m->A.x[p]; }
        } else {
            B.i[nz] = v - n;
            B.x[nz++] = -1.0;
        }
        B.p[k + 1] = nz;
    }
    B.nzmax = nz > 0 ? nz : 1;
    if (sk_lu_factorize(&lu, &B, o->pivot_tol > 0.0 ? o->pivot_tol : 0.1) != SK_OK) goto done;
    for (int k = 0; k < r; ++k) pi[k] = rank[k].v < n ? m->c[rank[k].v] : 0.0;
    if (sk_lu_btran(&lu, pi) != SK_OK) goto done;

    /* nonbasic columns at the bound their reduced cost d (c - A' pi; logicals pi_i) favours */
    for (int v = 0; v < nv; ++v) {
        if (pos[v] >= 0) continue;
        double d;
        if (v < n) {
            d = m->c[v];
            for (int p = m->A.p[v]; p < m->A.p[v + 1]; ++p) d -= m->A.x[p] * pi[m->A.i[p]];
        } else {
            d = pi[v - n];
        }
        const int lf = !SK_IS_NEG_INF(lo[v]), hf = !SK_IS_INF(hi[v]);
        if (lf && hf) value[v] = d > 0.0 ? lo[v] : d < 0.0 ? hi[v] : (value[v] - lo[v] <= hi[v] - value[v] ? lo[v] : hi[v]);
        else if (lf) value[v] = lo[v];
        else if (hf) value[v] = hi[v];
        else value[v] = 0.0;
    }
    /* B z_B = -N z_N over A x - s = 0 */
    for (int v = 0; v < nv; ++v) {
        if (pos[v] >= 0) continue;
        if (v < n) {
            for (int p = m->A.p[v]; p < m->A.p[v + 1]; ++p) z[m->A.i[p]] -= m->A.x[p] * value[v];
        } else {
            z[v - n] += value[v];
        }
    }
    if (sk_lu_ftran(&lu, z) != SK_OK) goto done;
    for (int k = 0; k < r; ++k) value[rank[k].v] = z[k];

    out->x = (double*)malloc(sizeof(double) * (size_t)(n + 1));
    out->y = (double*)malloc(sizeof(double) * (size_t)(r + 1));
    out->rc = (double*)malloc(sizeof(double) * (size_t)(n + 1));
    out->rowact = (double*)malloc(sizeof(double) * (size_t)(r + 1));
    if (!out->x || !out->y || !out->rc || !out->rowact) goto done;
    out->ncol = n;
    out->nrow = r;
    for (int j = 0; j < n; ++j) out->x[j] = value[j];
    for (int i = 0; i < r; ++i) out->y[i] = -pi[i];
    if (sk_verify(m, out) == SK_OK && out->primal_infeasibility <= o->primal_tol &&
        out->dual_infeasibility <= o->dual_tol)
        ok = 1;
done:
    sk_lu_free(&lu);
    free(B.p); free(B.i); free(B.x);
    free(act); free(value); free(lo); free(hi); free(rank); free(pos); free(pi); free(z);
    return ok;
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

    reduced_costs(m, y, rc);
    /* the identified basis as it stands: no simplex when the point was accurate enough */
    sk_solution_free(out);
    if (direct_basis(m, o, x, y, rc, out)) {
        free(state);
        free(rc);
        stats->direct = 1;
        out->result = SK_RESULT_OPTIMAL;
        out->iterations = 0;
        stats->seconds = sk_wall_seconds() - t0;
        out->solve_seconds = stats->seconds;
        return SK_OK;
    }
    sk_solution_free(out);

    /* the bounds the first-order point selects */
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
