/* Crossover from a first-order point of an LP to a vertex certified by the
   reference's sk_verify, for callers of the B200 engine built with the
   reference's C core (c/include/sankhya.h, c/include/sk_simplex.h).

   The reference has no crossover (docs/architecture/PDLP.md:185 lists it as
   not implemented) and its simplex takes no starting basis
   (c/include/sk_simplex.h:39), so the vertex comes from a smaller LP: every
   column whose reduced cost c_j + (A'y)_j at the given dual point selects one
   of its finite bounds by more than fix_tolerance is fixed at that bound,
   the remaining columns are solved by sk_simplex_solve with the row bounds
   shifted by the fixed columns' activity, and the combined point is checked
   by sk_verify on the whole model. A fixed column whose reduced cost at the
   new duals has the wrong sign for its bound is released and the smaller LP
   solved again; when nothing is left to release, or after max_rounds solves,
   the whole model goes to the simplex from its usual start. Before any of that,
   the basis the point identifies (the nrow columns of [A -I] with the smallest
   reduced costs, nonbasic columns at the bounds its own duals favour, factorized
   with the core's sparse LU) is tried as it stands: when sk_verify certifies it,
   no simplex runs. */
#ifndef SK_B200_CROSSOVER_H
#define SK_B200_CROSSOVER_H

#include "sankhya.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sk_b200_crossover_stats {
    int rounds;                   /* smaller-LP simplex solves run                       */
    int fixed_columns;            /* columns fixed in the last smaller LP                */
    int released_columns;         /* fixed columns released over all rounds              */
    int full_fallback;            /* 1: the whole model was solved from the usual start  */
    int direct;                   /* 1: the basis the point identifies was certified as it
                                     stands, without a simplex solve                       */
    long long simplex_iterations; /* over every simplex solve                            */
    double seconds;
} sk_b200_crossover_stats;

/* m: an LP (no Q, objsense 1, as sk_solve's models are); o: the simplex options
   (primal_tol / dual_tol also bound the certificate); x (ncol) and y (nrow): the
   first-order point, y in sk_solve's sign convention (rc = c + A'y, a row at its
   lower bound has y <= 0; all zero when only x is at hand, the identified basis then
   ranked by interiority alone); fix_tolerance > 0: a column is fixed when |rc_j| exceeds
   it and x_j lies within sqrt(fix_tolerance) (1 + |bound|) of the bound its sign
   selects; max_rounds >= 1; out initialised by sk_solution_init. On SK_OK, out holds
   x, y, rc and rowact of the certified vertex (free with sk_solution_free), its
   objective and sk_verify's residuals, and out->result is SK_RESULT_OPTIMAL, or the
   whole-model simplex's result when the fallback ran and did not reach optimality.
   stats may be NULL. */
sk_status sk_b200_crossover(const sk_model* m, const sk_options* o, const double* x, const double* y,
                            double fix_tolerance, int max_rounds, sk_solution* out,
                            sk_b200_crossover_stats* stats);

#ifdef __cplusplus
}
#endif

#endif
