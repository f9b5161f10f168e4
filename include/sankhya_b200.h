/* Extensions of the B200 PDHG engine beyond the reference's C ABI.
 *
 * New symbols only; every reference signature in sankhya_cuda.h is unchanged.
 * Settings structs carry a struct_version so later fields can be appended.
 */
#ifndef SANKHYA_B200_H
#define SANKHYA_B200_H

#include "sankhya_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ timing */

/* Device-side timing of the most recent solve call on this thread, taken with
   CUDA events on the engine's stream. No counterpart in the reference (its
   benchmarks time whole calls on the host, benchmarks/bench_pdlp.cpp:131-281). */
typedef struct SankhyaB200Timing {
    int iterations;          /* PDHG iterations executed on the device          */
    int checkpoints;         /* checkpoint evaluations (host-visible syncs)      */
    int kernel_launches;     /* engine kernels launched by the call              */
    int per_kernel_samples;  /* iterations sampled for the per-kernel averages   */
    double loop_ms;          /* events around all iteration kernels              */
    double checkpoint_ms;    /* events around checkpoint kernels + result copy   */
    double dual_kernel_ms;   /* average duration of one fused A-side launch      */
    double primal_kernel_ms; /* average duration of one fused A'-side launch     */
    double h2d_ms;           /* input upload                                     */
    double d2h_ms;           /* solution download                                */
} SankhyaB200Timing;

/* level 0: none; 1: loop/checkpoint/copy events; 2: also per-kernel events on
   every iteration (adds two event records per launch). Thread-local. */
SANKHYA_CUDA_API void sankhya_b200_set_timing(int level);
SANKHYA_CUDA_API void sankhya_b200_last_timing(SankhyaB200Timing* out);

/* --------------------------------------------------- sk_solve continuous hook */

/* Layout-compatible copies of the reference's public model types
   (c/include/sankhya.h:64-161). Skipped when that header was included first. */
#ifndef SANKHYA_H
typedef struct sk_csc {
    int nrow;
    int ncol;
    int* p;
    int* i;
    double* x;
    int nzmax;
} sk_csc;

typedef struct sk_model {
    int nrow;
    int ncol;
    sk_csc A;
    sk_csc* Q;
    double* c;
    double* rlow;
    double* rupp;
    double* clow;
    double* cupp;
    unsigned char* vartype;
    double objshift;
    double objsense;
    char** rowname;
    char** colname;
    char* name;
} sk_model;

typedef struct sk_options {
    double primal_tol;
    double dual_tol;
    double pivot_tol;
    double time_limit;
    long long iteration_limit;
    long long node_limit;
    int presolve;
    int scaling;
    int refactor_interval;
    int verbosity;
    int threads;
    double mip_gap_abs;
    double mip_gap_rel;
    int mip_cuts;
    int mip_heuristics;
    int dual_simplex;
    int lp_engine;
    unsigned long long random_seed;
} sk_options;
#endif

/* Output of the loop replacement below. */
typedef struct SankhyaB200LoopResult {
    int iterations;   /* iterations executed (the reference's performed_iterations) */
    int converged;    /* all gates passed at a checkpoint                           */
    int numeric_failure;
    double dual_step; /* max |y_new - y| of the last executed iteration            */
    double anorm;     /* sqrt(max column mass * max row mass) of A                 */
    double seconds;
} SankhyaB200LoopResult;

/* Replaces the first-order loop of solve_continuous, c/src/sk_solve.c:849-954:
   diagonal steps tau_j = 0.9/(1 + |A_:j|_1 + |Q_:j|_1), sigma_i = 0.9/(1 + |A_i:|_1),
   x0 = clamp(0), y0 = 0, x_bar = 2 x_new - x, a checkpoint every 20 iterations
   with the reference's gates (row violation <= primal_tol, max|x_bar - x| <=
   primal_tol * max(1, |x|_inf), max|y_new - y| <= dual_tol (1 + anorm), and for
   QP the sk_verify score <= 100 (primal_tol + 2 dual_tol)). x (ncol), y (nrow) and
   activity (nrow) are host outputs with the reference's meaning. The time limit
   is tested after every 20-iteration window instead of after every iteration.
   Returns 0, SK_ERR_ARG (1) on invalid input (including a model that
   sk_model_validate rejects, vartype aside), SK_ERR_MEMORY (2) on allocation
   failure, SK_ERR_NUMERIC (7) on a CUDA error. */
SANKHYA_CUDA_API int sankhya_b200_pdhg_loop(
    const sk_model* model, const sk_options* options, double* x, double* y,
    double* activity, SankhyaB200LoopResult* result);

/* ---------------------------------------------------------- matrix store */

/* The transpose the engine keeps for a matrix made by sankhya_cuda_csr_create,
   i.e. A in CSC form: at_ptr[cols + 1], and for each column its row indices in
   ascending order (at_idx[nnz]) with their values (at_val[nnz]), copied to host
   arrays. The engine builds it on the device (a stable radix sort of the entries
   by column), replacing the host counting sorts the reference uses to move
   between CSR and CSC (c/src/sk_solve.c csc_mv / csc_tmv order). Returns 0 or -1. */
SANKHYA_CUDA_API int sankhya_b200_csr_transpose(const SankhyaCudaCSR* matrix, int* at_ptr, int* at_idx,
                                                double* at_val);

/* ------------------------------------------------------- restarted PDLP */

enum {
    SANKHYA_B200_SCALE_RUIZ = 1,           /* src/lp/Scaling.cpp:11-92              */
    SANKHYA_B200_SCALE_POCK_CHAMBOLLE = 2, /* src/lp/Scaling.cpp:111-145 (alpha=1)  */
    SANKHYA_B200_SCALE_POW2 = 4            /* c/src/sk_scale.c:20-72                */
};

enum {
    SANKHYA_B200_FP64 = 0,       /* FP64 everywhere                                  */
    SANKHYA_B200_FP32_REFINE = 1, /* FP32 inner iterations, FP64 refinement residuals:
                                    with the adaptive step, the iterations run in FP32 on
                                    deviations from an FP64 center that moves to the
                                    restart point at every restart (one refinement: the
                                    problem's residual data b - A x_c and c + A'y_c are
                                    re-formed in FP64 there); restart and KKT decisions
                                    use FP64 residuals of center + deviation. With the
                                    Halpern loop or the fixed step: an FP32 phase to
                                    1e-4, then an FP64 finish.                         */
    SANKHYA_B200_BF16_REFINE = 2 /* as FP32_REFINE (adaptive loop only), with the
                                    scaled matrix values of the FP32 iterations rounded
                                    to bf16 (products accumulate in FP32); the center's
                                    products and all residuals use the FP64 values.    */
};

enum {
    SANKHYA_B200_PDLP_ADAPTIVE = 0, /* GpuPdlp's restarted adaptive PDHG (src/cuda/GpuPdlp.cpp:252-534) */
    SANKHYA_B200_PDLP_HALPERN = 1   /* reflected restarted Halpern PDHG, constant step (no counterpart
                                       in the reference; the method of cuPDLP+, Lu and Yang 2025)      */
};

typedef struct SankhyaB200PdlpSettings {
    int struct_version;   /* 4 (3: without cancel / cancel_context; 2: also without
                             initial_primal_weight; 1: also without algorithm)       */
    int max_iterations;   /* total PDHG iterations (accepted + rejected)          */
    int restart_period;   /* iterations between evaluations (GpuPdlp: 64)         */
    int power_iterations; /* power iterations for ||A||_2 (GpuPdlp: 30)           */
    int adaptive_step;    /* 1: Applegate et al. adaptive step; 0: 0.9/||A||_2    */
    int scaling;          /* bitmask of SANKHYA_B200_SCALE_*                      */
    int ruiz_iterations;  /* 100                                                  */
    int precision;        /* SANKHYA_B200_FP64, _FP32_REFINE or _BF16_REFINE      */
    double eps_optimal;   /* relative KKT tolerance on all three measures         */
    double time_limit;    /* seconds, <= 0 for none                               */
    double eta_min_factor;/* 1e-6 */
    double eta_max_factor;/* 1e4  */
    double ruiz_tolerance;/* 1e-2 */
    int algorithm;        /* SANKHYA_B200_PDLP_ADAPTIVE or SANKHYA_B200_PDLP_HALPERN  (version 2) */
    int reserved;
    double initial_primal_weight; /* > 0: start from this primal weight (e.g. one learned
                                     for an LP family); 0: ||c|| / ||b|| (version 3)      */
    int (*cancel)(void* context); /* non-NULL: called once per restart window, where the
                                     host synchronizes anyway, on the calling thread; a
                                     non-zero return stops the solve with status 3
                                     (GpuPdlp's PdlpParams::cancel, polled the same way,
                                     src/cuda/GpuPdlp.hpp:62-67) (version 4)              */
    void* cancel_context;         /* passed to cancel (version 4)                         */
} SankhyaB200PdlpSettings;

SANKHYA_CUDA_API void sankhya_b200_pdlp_default_settings(SankhyaB200PdlpSettings* settings);

typedef struct SankhyaB200PdlpResult {
    int status;            /* 0 converged, 1 iteration limit, 2 time limit, 3 cancelled,
                              -2 numeric                                              */
    int iterations;
    int restarts;
    int rejected_steps;
    int host_syncs;
    int refinements;       /* FP32_REFINE: FP64 centers formed (the start and one per
                              restart) with the adaptive step; 1 when the FP64 finish
                              ran after an FP32 phase otherwise; 0 for FP64            */
    double primal_objective;
    double dual_objective;
    double relative_primal_residual;
    double relative_dual_residual;
    double relative_gap;
    double matrix_norm;
    double final_step_size;
    double primal_weight;
    double seconds;
} SankhyaB200PdlpResult;

/* Restarted adaptive PDLP (the algorithm of the reference's GpuPdlp,
   src/cuda/GpuPdlp.cpp:252-534) behind the C ABI: optional scaling of the
   model, restarts at the 0.2 / 0.8 / 0.36 criteria, primal-weight smoothing,
   relative-KKT termination. Host arrays; x0 / y0 optional warm start (NULL:
   zeros). x_out (cols) and y_out (rows, may be NULL) are in the caller's
   unscaled space. Bounds with magnitude >= 1e30 are absent. Returns 0, -1 on
   invalid input or CUDA error, -2 on a non-finite iterate. */
SANKHYA_CUDA_API int sankhya_b200_pdlp_solve(
    const SankhyaCudaCSR* matrix, const double* c,
    const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper,
    const SankhyaB200PdlpSettings* settings, const double* x0, const double* y0,
    double* x_out, double* y_out, SankhyaB200PdlpResult* result);

/* The restarted adaptive solve of a convex QP: minimize c'x + x'Q x / 2 subject
   to the same bounds, with Q given either as a full symmetric CSR of size
   cols x cols (hessian, made by sankhya_cuda_csr_create) or as its diagonal
   (quadratic_diagonal, cols entries, finite and >= 0), the two forms of the
   reference's solve_qp (cuda/src/sankhya_cuda_lp.cu:36-52, 236-238; the CPU
   loop's c/src/sk_solve.c:908-923). The diagonal is taken exactly in the
   primal prox, x+ = proj((x - tau (c + A'y)) / (1 + tau q)); a general Q by a
   gradient step with a diagonal majorant, x+ = proj(x - tau (c + Q x + A'y) /
   (1 + tau d)), d_j = sum_k |Q_jk| (Gershgorin, so the step is safe for Q at any
   tau; for a diagonal Q the two forms coincide). Restarts, primal weight,
   precision modes and scaling (of A; Q is scaled by the column factors) are
   those of sankhya_b200_pdlp_solve, and the relative KKT uses the reduced cost
   c + Q x + A'y and the QP objectives (primal c'x + x'Qx/2, dual with -x'Qx/2).
   Needs the adaptive step and algorithm ADAPTIVE. No counterpart in the
   reference's GPU PDLP, which solves LPs only. Both Hessian arguments NULL
   solves the LP. */
SANKHYA_CUDA_API int sankhya_b200_pdlp_solve_qp(
    const SankhyaCudaCSR* matrix, const SankhyaCudaCSR* hessian, const double* quadratic_diagonal,
    const double* c, const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper,
    const SankhyaB200PdlpSettings* settings, const double* x0, const double* y0,
    double* x_out, double* y_out, SankhyaB200PdlpResult* result);

/* ------------------------------------------------- feasibility polishing */

typedef struct SankhyaB200PolishSettings {
    int struct_version;          /* 1                                                    */
    int max_polish_iterations;   /* per polishing solve; 0: as many as the main loop has
                                    run so far                                           */
    double start_tolerance;      /* relative KKT at which the main loop first hands over
                                    (1e-4); each later hand-over is 10x tighter, down to
                                    the smaller of eps_optimal and polish_tolerance      */
    double polish_tolerance;     /* relative primal residual of the polished x and
                                    relative dual residual of the polished y (1e-8)      */
} SankhyaB200PolishSettings;

SANKHYA_CUDA_API void sankhya_b200_polish_default_settings(SankhyaB200PolishSettings* settings);

typedef struct SankhyaB200PolishResult {
    int rounds;                  /* hand-overs from the main loop to polishing          */
    int main_iterations;         /* iterations of the main (restarted adaptive) loop    */
    int primal_iterations;       /* iterations of the primal polishing solves           */
    int dual_iterations;         /* iterations of the dual polishing solves             */
    double main_seconds;
    double polish_seconds;
    double main_relative_primal_residual;  /* the main loop's point at the last hand-over */
    double main_relative_dual_residual;
    double main_relative_gap;
    double pair_relative_primal_residual;  /* the last polished pair, scored on the LP     */
    double pair_relative_dual_residual;
    double pair_relative_gap;
    double pair_primal_objective;
} SankhyaB200PolishResult;

/* Restarted adaptive PDLP with feasibility polishing (no counterpart in the
   reference, which lists crossover and polishing as not implemented,
   docs/architecture/PDLP.md:185; the method is the feasibility polishing of
   PDLP, Applegate et al. 2025). The main loop of sankhya_b200_pdlp_solve runs
   to start_tolerance; then, on the same scaled matrix, two warm-started solves
   of easier problems: the primal feasibility problem (the LP with zero cost)
   from the main loop's x, run until its x meets polish_tolerance in relative
   primal residual, and the dual feasibility problem (every finite bound moved
   to 0, so that its dual feasible set is the original LP's) from the main
   loop's y, run until its y meets polish_tolerance in relative dual residual;
   both are restarted PDHG with the constant step 0.9 / ||A||_2 and the main
   loop's primal weight held, so each stays near its starting point.
   The pair (polished x, polished y) is scored on the original LP (result: its
   relative residuals, gap and objectives); when the pair misses a target (its
   gap above eps_optimal, or a polishing solve out of iterations) the main loop
   resumes to a 10x tighter tolerance and polishing repeats, with budgets that
   grow with the main loop. A polishing solve is skipped when the main loop's
   point already meets polish_tolerance on its measure. The rounds end when the
   pair meets its targets, or at the main loop's iteration limit, time limit or
   cancellation. Status 0: primal and dual residual of the pair <=
   polish_tolerance and gap <= eps_optimal. Otherwise the answer is whichever
   of the scored pairs and the main loop's last point misses its targets by
   the smallest factor (the largest of primal / polish_tolerance, dual /
   polish_tolerance, gap / eps_optimal). Needs precision FP64 and the
   adaptive step of algorithm ADAPTIVE; settings and arrays as for
   sankhya_b200_pdlp_solve; polish NULL takes the defaults; polish_result may
   be NULL. Returns 0, -1 on invalid input or CUDA error, -2 on a non-finite
   iterate. */
SANKHYA_CUDA_API int sankhya_b200_pdlp_solve_polished(
    const SankhyaCudaCSR* matrix, const double* c,
    const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper,
    const SankhyaB200PdlpSettings* settings, const SankhyaB200PolishSettings* polish,
    const double* x0, const double* y0, double* x_out, double* y_out,
    SankhyaB200PdlpResult* result, SankhyaB200PolishResult* polish_result);

/* ------------------------------------------------------- batched LPs */

typedef struct SankhyaB200BatchSettings {
    int struct_version;  /* 1 */
    int max_iterations;  /* per LP (100000, sk_solve's default)              */
    int check_every;     /* 20, as in sk_solve                               */
    int schedule;        /* shared-matrix batch only: 0 = warp shape picked by timing
                            (cached per matrix and batch width), 1..3 = fixed shape
                            (1 x 8, 2 x 4, 4 x 4 slabs x look-ahead); results do not
                            depend on it                                      */
    double primal_tol;   /* 1e-7 */
    double dual_tol;     /* 1e-7 */
    double time_limit;   /* seconds for the whole batch, <= 0 for none        */
} SankhyaB200BatchSettings;

typedef struct SankhyaB200BatchResult {
    int status;          /* 0 gates passed, 1 iteration limit, 2 time limit    */
    int iterations;      /* iterations this LP ran before it was frozen        */
    double objective;    /* c'x over the LP's columns                          */
    double row_violation;/* values of the LP's last checkpoint                 */
    double step;
    double dual_step;
    double anorm;
} SankhyaB200BatchResult;

SANKHYA_CUDA_API void sankhya_b200_batch_default_settings(SankhyaB200BatchSettings* settings);

/* Many independent LPs in one set of launches. No counterpart in the reference:
   it solves LPs one at a time (the node relaxations of c/src/sk_milp.c:431-459
   each call the simplex). The LPs are given as one block-diagonal device matrix:
   LP k owns rows [row_segments[k], row_segments[k+1]) and columns
   [col_segments[k], col_segments[k+1]); a nonzero outside its LP's block is
   rejected. Each LP runs the first-order loop of sk_solve (c/src/sk_solve.c:849-954:
   diagonal steps from its own row/column masses, its own 20-iteration gates and
   its own anorm) and is frozen as soon as its gates pass, so its iterates equal a
   separate solve's. Host arrays are concatenated per LP; bounds use the 1e30
   sentinel. Returns 0 or -1. */
SANKHYA_CUDA_API int sankhya_b200_batch_pdhg(
    const SankhyaCudaCSR* block_matrix, int batch, const int* row_segments, const int* col_segments,
    const double* c, const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper,
    const SankhyaB200BatchSettings* settings, double* x_out, double* y_out,
    SankhyaB200BatchResult* results);

/* Batched PDHG over LPs that share one matrix: the node relaxations of a
   branch-and-bound search, which milp_solve_lp (c/src/sk_milp.c:432-459) solves
   one at a time on the same model with new column bounds. Same loop, gates and
   results as sankhya_b200_batch_pdhg, per LP; the matrix is read once per
   iteration for all LPs. Arrays flagged per_lp hold batch vectors back to back
   (LP-major: batch*n for c and column bounds, batch*m for row bounds); a zero
   flag means one vector shared by every LP. x_out is batch*n, y_out batch*m or
   NULL. Returns 0 or -1. */
SANKHYA_CUDA_API int sankhya_b200_shared_batch_pdhg(
    const SankhyaCudaCSR* matrix, int batch,
    const double* c, int c_per_lp,
    const double* row_lower, const double* row_upper, int row_bounds_per_lp,
    const double* col_lower, const double* col_upper, int col_bounds_per_lp,
    const SankhyaB200BatchSettings* settings, double* x_out, double* y_out,
    SankhyaB200BatchResult* results);

/* ------------------------------------------------- learned warm start */

/* A bipartite message-passing network over the constraint matrix that predicts
   a starting point (x, y) for PDLP on a parametric LP family (fixed matrix,
   varying cost and bounds). No counterpart in the reference, which has no
   learned component and always starts PDLP from zero (src/cuda/GpuPdlp.cpp:278-290);
   the prediction goes to sankhya_b200_pdlp_solve as x0 / y0, cold start stays
   the fallback, and PDLP's own relative-KKT test decides every answer.
   Network: 16 node features, 4 rounds (settable) of width 64, bf16 tensor-core
   dense layers with fp32 accumulation, fp32 aggregation; trained with Adam on
   (instance, solution) pairs, one instance per step. Deterministic. */
typedef struct SankhyaB200GnnSettings {
    int struct_version;          /* 1 */
    int rounds;                  /* message-passing rounds, 4 */
    unsigned long long seed;     /* initialisation stream */
    double learning_rate;        /* Adam step, 1e-3 */
    double y_scale;              /* scale of the dual outputs and of their loss term, 1 */
} SankhyaB200GnnSettings;

typedef struct SankhyaB200Gnn SankhyaB200Gnn;

SANKHYA_CUDA_API void sankhya_b200_gnn_default_settings(SankhyaB200GnnSettings* settings);
SANKHYA_CUDA_API int sankhya_b200_gnn_create(const SankhyaB200GnnSettings* settings, SankhyaB200Gnn** network);
SANKHYA_CUDA_API void sankhya_b200_gnn_destroy(SankhyaB200Gnn* network);
SANKHYA_CUDA_API int sankhya_b200_gnn_parameter_count(const SankhyaB200Gnn* network);
/* fp32 parameters, flat: Ev[16][64], bev, Ec[16][64], bec, per round Wc[128][64], bc,
   Wv[128][64], bv, then wx[64], bx, wy[64], by */
SANKHYA_CUDA_API int sankhya_b200_gnn_get_parameters(SankhyaB200Gnn* network, float* out);
SANKHYA_CUDA_API int sankhya_b200_gnn_set_parameters(SankhyaB200Gnn* network, const float* in);
/* x_out (cols, inside the column bounds) and y_out (rows, may be NULL). */
SANKHYA_CUDA_API int sankhya_b200_gnn_predict(
    SankhyaB200Gnn* network, const SankhyaCudaCSR* matrix, const double* c,
    const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper, double* x_out, double* y_out);
/* Loss against (x_target, y_target) and its gradient (parameter layout above). */
SANKHYA_CUDA_API int sankhya_b200_gnn_gradient(
    SankhyaB200Gnn* network, const SankhyaCudaCSR* matrix, const double* c,
    const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper,
    const double* x_target, const double* y_target, double* loss, float* gradient_out);
/* One Adam step on one instance; loss is the value before the step. */
SANKHYA_CUDA_API int sankhya_b200_gnn_train_step(
    SankhyaB200Gnn* network, const SankhyaCudaCSR* matrix, const double* c,
    const double* row_lower, const double* row_upper,
    const double* col_lower, const double* col_upper,
    const double* x_target, const double* y_target, double* loss);

/* ---------------------------------------------------- allocation-free solve */

/* No counterpart in the reference. The fixed-step solve of sankhya_cuda_lp_pdhg
   (same algorithm, arithmetic and result fields; scalar tau and sigma) for
   callers that cannot allocate device memory while they solve: runtimes that
   hand out all device memory from their own pool, processes with a fixed
   device-memory budget that must not grow after start-up, services that cannot
   take the device-wide synchronisation cudaMalloc/cudaFree can impose. It calls no cudaMalloc, cudaFree or allocating
   library routine: the model (c, bounds) and the solution are device pointers the
   caller owns, and the scratch (iterate buffers, reduction partials) lives in a
   16 MiB array inside the library that every GPU loading the library holds until
   the process exits. Limit: 4*C + 2*R + 128*SMs + 64 doubles must fit in
   2 Mi (2,097,152) doubles, with C = cols and R = rows each rounded up to a
   multiple of 32 and SMs the device's multiprocessor count (148 on a B200, so the
   reduction partials take 18,944 doubles there); larger problems are rejected
   with -1 and a message. The matrix must come from sankhya_cuda_csr_create, with
   its handle unchanged since, and that call's device must be current (-1
   otherwise). The first call on a device
   looks up the array's device address (cudaGetSymbolAddress) and must come before
   any stream capture. All calls share the array and it keeps the last call's
   contents: calls that overlap on the GPU race. Work is queued on the legacy
   default stream; the call returns after the solve. */
SANKHYA_CUDA_API int sankhya_b200_lp_pdhg_device_noalloc(
    const SankhyaCudaCSR* matrix, const double* device_c,
    const double* device_row_lower, const double* device_row_upper,
    const double* device_col_lower, const double* device_col_upper,
    SankhyaCudaLPSettings settings, double* device_solution, SankhyaCudaLPResult* result);

/* Equilibration factors computed on the device, without solving: row_scale
   (rows) and col_scale (cols) such that the scaled matrix is
   diag(row_scale) A diag(col_scale). scaling is a SANKHYA_B200_SCALE_* mask:
   POW2 runs 4 geometric passes rounded to powers of two (c/src/sk_scale.c:20-72),
   RUIZ the infinity-norm equilibration (src/lp/Scaling.cpp:11-92, identity when it
   does not reach ruiz_tolerance in ruiz_iterations), POCK_CHAMBOLLE (alpha = 1,
   Scaling.cpp:111-145) on the result, composed as in src/lp/LpSolver.cpp:62-71. */
SANKHYA_CUDA_API int sankhya_b200_scale_factors(
    const SankhyaCudaCSR* matrix, int scaling, int ruiz_iterations, double ruiz_tolerance,
    double* row_scale, double* col_scale);

#ifdef __cplusplus
}
#endif

#endif
