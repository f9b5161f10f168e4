// Restarted adaptive PDLP behind sankhya_b200_pdlp_solve, in FP64 or with
// FP32 inner iterations inside an FP64 iterative-refinement loop (FP32_REFINE; with
// bf16 matrix values under the FP32 iterations, BF16_REFINE).
//
// The algorithm is the reference's GpuPdlp (src/cuda/GpuPdlp.cpp:179-534,
// src/cuda/PdlpKernels.cu:71-518): power-iteration ||A||_2, eta = 0.9/||A||,
// primal weight omega = ||c||/||b||, Applegate et al. adaptive step with
// accept/reject decided on the device, restart to the better of current and
// average at the 0.2 / 0.8 / 0.36 criteria, log-smoothed omega update,
// relative-KKT termination. Scaling (Ruiz, Pock-Chambolle, power-of-two) is
// computed and applied on the device in FP64.
//
// Per adaptive iteration three launches, all reading eta / omega / the accept
// flag from device memory so a whole window is one CUDA graph:
//   K1  elementwise: commit the previous candidate if accepted (x, y, sums,
//       A x, A x_prev), then y_cand = prox(y + sigma (2 A x - A x_prev))
//   K2  A'-side chunks: x_cand = proj(x - tau (c + A'y_cand)), block sums of |dx|^2
//   K3  A-side chunks:  A x_cand, block sums of |dy|^2 and dy.(A dx); the last
//       block to finish combines all partials in a fixed order and writes the
//       new eta and the accept flag (PdlpKernels.cu:405-494).
// The window ends with a commit, the residual sums of the current and of the
// average iterate (PdlpKernels.cu:101-209, fused into the two products), and
// one small copy to the host, which makes the restart decision.
//
// FP32_REFINE (adaptive step): iterative refinement at every restart. The FP32
// iterations (FP32 matrix values and vectors, FP32 accumulation in the products)
// run on deviations (dx, dy) from an FP64 center (x_c, y_c). At the start and at
// each restart the center moves to the restart point and the FP32 problem is
// re-formed around it in FP64 (the refinement residuals): cost c + A'y_c, column
// bounds minus x_c, row bounds minus A x_c, each rounded once to FP32. Shifting the
// primal box is exact; the dual prox is taken of the absolute dual y_c + v in FP64
// (the row bounds' support function does not move with the shift), so the FP32
// loop solves the same saddle problem as the FP64 one. The window-end residuals
// and the KKT / restart decisions are FP64 sums over center + deviation of the
// scaled FP64 problem. Because the deviations shrink as the solve converges, FP32
// rounding stays relative to the step, not to the iterate, and the loop takes the
// FP64 loop's iterations and reaches its accuracy (plain FP32 iterates stall the
// adaptive step: its interaction term dy'A dx is a difference of O(1) FP32
// products). BF16_REFINE rounds the scaled matrix values of those iterations to
// bf16 (each widened to FP32 as the fused kernel loads it); the center's products
// and the residuals keep the FP64 values. The Halpern loop and the fixed step keep
// an FP32 phase to 1e-4 followed by an FP64 finish.
// (A Gleixner-Steffy-Wolter correction LP with scaled residuals was tried first:
// it re-solves the slow tail of PDLP at every pass and made no progress on boxed
// LPs; re-centering without scaling keeps the restart schedule running instead.)
//
// Feasibility polishing (sankhya_b200_pdlp_solve_polished, run_polished): PDLP's
// published polishing (Applegate et al. 2025) around the FP64 loop, on the same
// scaled matrix and the same Core: a zero-cost primal feasibility solve from the
// loop's x and a dual feasibility solve (finite bounds at 0) from its y, each ended
// by its own residual alone (LoopParams::measure), the pair scored on the LP by the
// window-end residual kernels, and the loop resumed 10x tighter until the pair's
// gap meets the target.
#include "engine.cuh"

#include <cstddef>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <limits>

namespace b200 {

namespace {

constexpr double kStepSafety = 0.9;
constexpr double kMinWeight = 1e-6;
constexpr double kMaxWeight = 1e6;
constexpr double kSmoothing = 0.5;
constexpr double kSufficient = 0.2;
constexpr double kNecessary = 0.8;
constexpr double kArtificial = 0.36;

struct PdlpState {
    double eta;
    double omega;
    double accepted;       // 1 when the last probe accepted its candidate
    double updates;        // probes so far
    double accept_count;   // accepted probes so far
    double accepted_at_restart;
    double eta_min, eta_max;
    double terms_fixed;    // average divisor for the fixed-step path
    double eta_bar, dx_sq, dy_sq, interaction;
    unsigned int ticket;   // last-block election for the probe combine
    unsigned int pad;
    double halpern_k0;     // Halpern path: iterations since the anchor at the window's start
};

template <class T>
__device__ __forceinline__ T clampf(T v, T lo, T hi) {
    return fmin(fmax(v, lo), hi);
}

// ------------------------------------------------------------ iteration kernels

// K1 (PdlpKernels.cu:499-518 commit, then :377-389 dual candidate). With
// y_center (the centered FP32 loop) y, ax, ax_prev are deviations from an FP64
// center and rl / ru the row bounds shifted by A x_center: the prox is taken of
// the absolute dual y_center + v, in FP64, and the candidate stored as a deviation.
template <class T>
__global__ void k_commit_dual(int n, int m, PdlpState* __restrict__ st, T* __restrict__ x,
                              const T* __restrict__ x_cand, T* __restrict__ x_sum, T* __restrict__ y,
                              T* __restrict__ y_cand, T* __restrict__ y_sum, T* __restrict__ ax, T* __restrict__ ax_prev,
                              const T* __restrict__ ax_cand, const T* __restrict__ rl, const T* __restrict__ ru,
                              const double* __restrict__ y_center, T* __restrict__ qx, const T* __restrict__ qx_cand,
                              int make_candidate) {
    const bool acc = st->accepted != 0.0;
    const T sigma = static_cast<T>(st->eta * st->omega);
    const int stride = blockDim.x * gridDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        T yi = y[i], axi = ax[i], axp = ax_prev[i];
        if (acc) {
            const T yc = y_cand[i];
            yi = yc;
            y[i] = yc;
            y_sum[i] += yc;
            axp = axi;
            axi = ax_cand[i];
            ax_prev[i] = axp;
            ax[i] = axi;
        }
        if (make_candidate) {
            const T v = yi + sigma * (T(2) * axi - axp);
            if (y_center) {
                const double s = static_cast<double>(sigma), vd = static_cast<double>(v);
                const double w = (y_center[i] + vd) / s;
                y_cand[i] = static_cast<T>(vd - s * clampf<double>(w, static_cast<double>(rl[i]),
                                                                    static_cast<double>(ru[i])));
            } else {
                y_cand[i] = v - sigma * clampf<T>(v / sigma, rl[i], ru[i]);
            }
        }
    }
    if (acc) {
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
            const T xc = x_cand[j];
            x[j] = xc;
            x_sum[j] += xc;
            if (qx) qx[j] = qx_cand[j];
        }
    }
}

// The adaptive step of Applegate et al., "Practical large-scale linear
// programming using primal-dual hybrid gradient" (NeurIPS 2021, section 3.1).
// For a trial move (dx, dy) made with step `used`, PDHG stays stable while the
// step is at most  |dz|^2_w / (2 |dy' A dx|),  with |dz|^2_w = w |dx|^2 + |dy|^2 / w
// (w the primal weight). The move is kept when `used` is within that limit. The
// next step is min((1 - (k+1)^-0.3) limit, (1 + (k+1)^-0.6) used) for the k-th
// trial: both factors tend to 1, so the step settles just under the limit.
// With no interaction (or no movement) the limit is the largest allowed step;
// a next step that is not a positive finite number keeps `used`; the result is
// clamped to [lo, hi]. The operations, and so the rounding, follow the
// reference's device code (src/cuda/PdlpKernels.cu:454-493).
struct StepRule {
    double limit, next;
    bool keep;
};
__device__ __forceinline__ StepRule step_rule(double used, double w, double dx2, double dy2, double cross, double k,
                                              double lo, double hi) {
    StepRule r;
    const double half_norm = 0.5 * (w * dx2 + dy2 / w);
    r.limit = (cross > 0.0 && half_norm > 0.0) ? half_norm / cross : hi;
    r.keep = used <= r.limit;
    const double damp = 1.0 - pow(k + 1.0, -0.3), boost = 1.0 + pow(k + 1.0, -0.6);
    double next = fmin(damp * r.limit, boost * used);
    if (!(next > 0.0 && isfinite(next))) next = used;
    r.next = fmin(fmax(next, lo), hi);
    return r;
}

// Quadratic objective of the QP entry point: none (LP), a diagonal Hessian taken
// exactly in the primal prox, or a general Hessian taken by a gradient step.
enum QMode { kLp = 0, kQDiag = 1, kQGeneral = 2 };

// K2 (PdlpKernels.cu:391-400 primal candidate + the |dx|^2 part of :405-430). QP:
// diagonal q: x_cand = proj((x - tau (c + A'y)) / (1 + tau q)) (the prox of
// c'x + q x^2 / 2 over the box, the reference's sankhya_cuda_lp.cu:36-52 form);
// general Q: x_cand = proj(x - tau (c + Q x + A'y) / (1 + tau d)), the prox of the
// linearised quadratic plus (x' - x)' D (x' - x) / 2 with the diagonal majorant
// D = diag(d), d_j = sum_k |Q_jk| >= Q (Gershgorin), so the step is safe for Q at any
// tau and only A's coupling limits it. With Q diagonal the two forms coincide.
template <class T, int QM = kLp>
struct PrimalCandEpi {
    const PdlpState* st;
    const T* __restrict__ x;
    const T* __restrict__ c;
    const T* __restrict__ cl;
    const T* __restrict__ cu;
    const T* __restrict__ q;   // QM: the diagonal (kQDiag) or the majorant d (kQGeneral)
    const T* __restrict__ qx;  // kQGeneral: Q x of the committed point
    T* __restrict__ x_cand;
    double* __restrict__ partial;
    using Acc = Slots<1, 1u>;
    struct Row {
        T x, c, lo, hi, q, qx;
    };
    __device__ __forceinline__ Row load(int j) const {
        return Row{x[j], c[j], cl[j], cu[j], QM == kLp ? T(0) : q[j], QM == kQGeneral ? qx[j] : T(0)};
    }
    __device__ __forceinline__ void store(int j, T aty, const Row& r, Acc& acc) const {
        const T tau = static_cast<T>(st->eta / st->omega);
        T xc;
        if (QM == kQDiag) xc = clampf<T>((r.x - tau * (r.c + aty)) / (T(1) + tau * r.q), r.lo, r.hi);
        else if (QM == kQGeneral) xc = clampf<T>(r.x - tau * (r.c + r.qx + aty) / (T(1) + tau * r.q), r.lo, r.hi);
        else xc = clampf<T>(r.x - tau * (r.c + aty), r.lo, r.hi);
        x_cand[j] = xc;
        const double dx = static_cast<double>(xc) - static_cast<double>(r.x);
        acc.add(0, dx * dx);
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

// Row sums of |Q| (the diagonal majorant of a symmetric Q), one warp per row.
__global__ void k_abs_row_sums(int rows, const int* __restrict__ ptr, const double* __restrict__ val,
                               double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int r = warp; r < rows; r += nwarps) {
        double s = 0.0;
        for (int p = ptr[r] + lane; p < ptr[r + 1]; p += 32) s += fabs(val[p]);
        s = warp_sum(s);
        if (lane == 0) out[r] = s;
    }
}

// K3 (A x_cand, |dy|^2, dy.(A x_cand - A x), then PdlpKernels.cu:460-494 in the last block)
template <class T>
struct ProbeEpi {
    PdlpState* st;
    const T* __restrict__ y;
    const T* __restrict__ y_cand;
    const T* __restrict__ ax;
    T* __restrict__ ax_cand;
    double* __restrict__ partial;           // this kernel's [gridDim.x * 2]
    const double* __restrict__ partial_dx;  // K2's [grid_dx]
    int grid_dx;
    using Acc = Slots<2, 3u>;
    struct Row {
        T y, yc, ax;
    };
    __device__ __forceinline__ Row load(int i) const { return Row{y[i], y_cand[i], ax[i]}; }
    __device__ __forceinline__ void store(int i, T axc, const Row& r, Acc& acc) const {
        ax_cand[i] = axc;
        const double dy = static_cast<double>(r.yc) - static_cast<double>(r.y);
        acc.add(0, dy * dy);
        acc.add(1, dy * (static_cast<double>(axc) - static_cast<double>(r.ax)));
    }
    __device__ void finish(Acc& acc, double* smem) const {
        block_store(acc, partial, smem);
        __shared__ bool last;
        if (threadIdx.x == 0) {
            __threadfence();
            const unsigned int t = atomicAdd(&st->ticket, 1u);
            last = (t == gridDim.x - 1);
        }
        __syncthreads();
        if (!last) return;
        __threadfence();
        // fixed-order combine: thread k sums a strided slice, then a fixed tree
        __shared__ double red[3][kThreads];
        double a = 0.0, b = 0.0, d = 0.0;
        for (int g = threadIdx.x; g < grid_dx; g += kThreads) a += __ldcg(partial_dx + g);
        for (int g = threadIdx.x; g < static_cast<int>(gridDim.x); g += kThreads) {
            b += __ldcg(partial + 2 * g);
            d += __ldcg(partial + 2 * g + 1);
        }
        red[0][threadIdx.x] = a;
        red[1][threadIdx.x] = b;
        red[2][threadIdx.x] = d;
        __syncthreads();
        for (int s = kThreads / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) {
                red[0][threadIdx.x] += red[0][threadIdx.x + s];
                red[1][threadIdx.x] += red[1][threadIdx.x + s];
                red[2][threadIdx.x] += red[2][threadIdx.x + s];
            }
            __syncthreads();
        }
        if (threadIdx.x != 0) return;
        const double probe = st->updates + 1.0;
        const StepRule rule = step_rule(st->eta, st->omega, red[0][0], red[1][0], fabs(red[2][0]), probe,
                                        st->eta_min, st->eta_max);
        st->dx_sq = red[0][0];
        st->dy_sq = red[1][0];
        st->interaction = fabs(red[2][0]);
        st->eta_bar = rule.limit;
        st->eta = rule.next;
        st->updates = probe;
        st->accepted = rule.keep ? 1.0 : 0.0;
        st->accept_count += rule.keep ? 1.0 : 0.0;
        st->ticket = 0u;
    }
};

// Fixed-step path (PdlpKernels.cu:71-97): dual on A x_bar, primal on A'y, with sums.
template <class T>
struct DualFixedEpi {
    T* __restrict__ y;
    T* __restrict__ y_sum;
    const T* __restrict__ rl;
    const T* __restrict__ ru;
    T sigma;
    using Acc = NoAcc;
    __device__ __forceinline__ void row(int i, T axb, Acc&) const {
        const T v = y[i] + sigma * axb;
        const T yi = v - sigma * clampf<T>(v / sigma, rl[i], ru[i]);
        y[i] = yi;
        y_sum[i] += yi;
    }
    __device__ __forceinline__ void finish(Acc&, double*) const {}
};

template <class T>
struct PrimalFixedEpi {
    T* __restrict__ x;
    T* __restrict__ x_bar;
    T* __restrict__ x_sum;
    const T* __restrict__ c;
    const T* __restrict__ cl;
    const T* __restrict__ cu;
    T tau;
    using Acc = NoAcc;
    __device__ __forceinline__ void row(int j, T aty, Acc&) const {
        const T xj = x[j];
        const T xn = clampf<T>(xj - tau * (c[j] + aty), cl[j], cu[j]);
        x_bar[j] = T(2) * xn - xj;
        x[j] = xn;
        x_sum[j] += xn;
    }
    __device__ __forceinline__ void finish(Acc&, double*) const {}
};

// Reflected Halpern PDHG (primal first). T(x, y) = (x+, y+) with
// x+ = proj(x - tau (c + A'y)), y+ = prox(y + sigma A (2 x+ - x)); one Halpern step
// z <- lambda (2 T(z) - z) + (1 - lambda) z0, lambda = (k + 1) / (k + 2), k the
// iterations since the anchor z0. 2 x+ - x is also the dual step's point, so the
// primal epilogue writes it to x_bar and the anchored primal update in place.
template <class T>
__device__ __forceinline__ T halpern_lambda(const PdlpState* st, int q) {
    const double k = st->halpern_k0 + static_cast<double>(q);
    return static_cast<T>((k + 1.0) / (k + 2.0));
}

template <class T>
struct PrimalHalpernEpi {
    T* __restrict__ x;
    T* __restrict__ x_bar;
    const T* __restrict__ x0;
    const T* __restrict__ c;
    const T* __restrict__ cl;
    const T* __restrict__ cu;
    const PdlpState* __restrict__ st;
    int q;
    using Acc = NoAcc;
    __device__ __forceinline__ void row(int j, T aty, Acc&) const {
        const T tau = static_cast<T>(st->eta / st->omega);
        const T xj = x[j];
        const T xr = T(2) * clampf<T>(xj - tau * (c[j] + aty), cl[j], cu[j]) - xj;
        const T lam = halpern_lambda<T>(st, q);
        x_bar[j] = xr;
        x[j] = lam * xr + (T(1) - lam) * x0[j];
    }
    __device__ __forceinline__ void finish(Acc&, double*) const {}
};

template <class T>
struct DualHalpernEpi {
    T* __restrict__ y;
    const T* __restrict__ y0;
    const T* __restrict__ rl;
    const T* __restrict__ ru;
    const PdlpState* __restrict__ st;
    int q;
    using Acc = NoAcc;
    __device__ __forceinline__ void row(int i, T axb, Acc&) const {
        const T sigma = static_cast<T>(st->eta * st->omega);
        const T yi = y[i];
        const T v = yi + sigma * axb;
        const T yr = T(2) * (v - sigma * clampf<T>(v / sigma, rl[i], ru[i])) - yi;
        const T lam = halpern_lambda<T>(st, q);
        y[i] = lam * yr + (T(1) - lam) * y0[i];
    }
    __device__ __forceinline__ void finish(Acc&, double*) const {}
};

// One plain application of T at the window's end: x_t = x+ (and x_bar = 2 x+ - x
// for the dual half), y_t = y+, with sums |x+ - x|^2, |x+ - x0|^2 (and the dual
// counterparts) for the fixed-point residual and the primal weight.
template <class T>
struct PrimalTEpi {
    const T* __restrict__ x;
    T* __restrict__ x_bar;
    T* __restrict__ x_t;
    const T* __restrict__ x0;
    const T* __restrict__ c;
    const T* __restrict__ cl;
    const T* __restrict__ cu;
    const PdlpState* __restrict__ st;
    double* __restrict__ partial;
    using Acc = Slots<2, 3u>;
    __device__ __forceinline__ void row(int j, T aty, Acc& acc) const {
        const T tau = static_cast<T>(st->eta / st->omega);
        const T xj = x[j];
        const T xp = clampf<T>(xj - tau * (c[j] + aty), cl[j], cu[j]);
        x_t[j] = xp;
        x_bar[j] = T(2) * xp - xj;
        const double d = static_cast<double>(xp) - static_cast<double>(xj);
        const double e = static_cast<double>(xp) - static_cast<double>(x0[j]);
        acc.add(0, d * d);
        acc.add(1, e * e);
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

template <class T>
struct DualTEpi {
    const T* __restrict__ y;
    T* __restrict__ y_t;
    const T* __restrict__ y0;
    const T* __restrict__ rl;
    const T* __restrict__ ru;
    const PdlpState* __restrict__ st;
    double* __restrict__ partial;
    using Acc = Slots<2, 3u>;
    __device__ __forceinline__ void row(int i, T axb, Acc& acc) const {
        const T sigma = static_cast<T>(st->eta * st->omega);
        const T yi = y[i];
        const T v = yi + sigma * axb;
        const T yp = v - sigma * clampf<T>(v / sigma, rl[i], ru[i]);
        y_t[i] = yp;
        const double d = static_cast<double>(yp) - static_cast<double>(yi);
        const double e = static_cast<double>(yp) - static_cast<double>(y0[i]);
        acc.add(0, d * d);
        acc.add(1, e * e);
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

__global__ void k_set_halpern(PdlpState* st, double k0) { st->halpern_k0 = k0; }

// Restart of the Halpern path: the new anchor and iterate are T(z).
template <class T>
__global__ void k_halpern_restart(int n, int m, const T* __restrict__ x_t, const T* __restrict__ y_t,
                                  T* __restrict__ x, T* __restrict__ x0, T* __restrict__ y, T* __restrict__ y0) {
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) x[j] = x0[j] = x_t[j];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) y[i] = y0[i] = y_t[i];
}

// ----------------------------------------------------------- residual kernels
// PdlpKernels.cu:101-209 split over the two products, accumulated in FP64.
// Row slots: 0 |Ax - proj(Ax)|^2, 1 |y|^2, 2 |y - y_restart|^2, 3 -support(y)
// (sums), 4 max |Ax - proj(Ax)| (max).
template <class T>
struct ResRowsEpi {
    const T* __restrict__ y;
    const T* __restrict__ y_restart;
    const T* __restrict__ rl;
    const T* __restrict__ ru;
    T* __restrict__ ax_out;  // may be null
    double* __restrict__ partial;
    using Acc = Slots<5, 0xFu>;
    __device__ __forceinline__ void row(int i, T axt, Acc& acc) const {
        if (ax_out) ax_out[i] = axt;
        const double axi = axt, lo = rl[i], hi = ru[i], yi = y[i];
        const double pr = axi - fmin(fmax(axi, lo), hi);
        acc.add(0, pr * pr);
        acc.add(1, yi * yi);
        const double dy = yi - static_cast<double>(y_restart[i]);
        acc.add(2, dy * dy);
        double support = 0.0;
        if (yi > 0.0) support = isfinite(hi) ? yi * hi : 0.0;
        else if (yi < 0.0) support = isfinite(lo) ? yi * lo : 0.0;
        acc.add(3, -support);
        acc.max(4, fabs(pr));
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

// Column slots: 0 dual violation^2, 1 dual objective column terms, 2 c'x,
// 3 |x|^2, 4 |x - x_restart|^2 (sums), 5 max |x - proj(x - (c + A'y))| (max;
// the column KKT residual, which sees reduced costs of interior variables even
// when every bound is finite and the dual violation itself is zero).
// QP (QM != kLp): the reduced cost is c + Q x + A'y, slot 2 takes c'x + x'Q x / 2
// and slot 1 the dual objective's -x'Q x / 2 (the QP's Wolfe dual); q is the
// diagonal (kQDiag) or Q x of the evaluated point (kQGeneral).
template <class T, int QM = kLp>
struct ResColsEpi {
    const T* __restrict__ x;
    const T* __restrict__ x_restart;
    const T* __restrict__ c;
    const T* __restrict__ cl;
    const T* __restrict__ cu;
    const T* __restrict__ q;
    T* __restrict__ aty_out;  // may be null
    double* __restrict__ partial;
    using Acc = Slots<6, 0x1Fu>;
    __device__ __forceinline__ void row(int j, T atyt, Acc& acc) const {
        if (aty_out) aty_out[j] = atyt;
        const double xj = x[j], lo = cl[j], hi = cu[j], cj = c[j];
        double r = cj + static_cast<double>(atyt);
        double half_xqx = 0.0;
        if (QM != kLp) {
            const double qxj = QM == kQDiag ? static_cast<double>(q[j]) * xj : static_cast<double>(q[j]);
            r = cj + qxj + static_cast<double>(atyt);
            half_xqx = 0.5 * xj * qxj;
        }
        acc.add(2, QM == kLp ? cj * xj : cj * xj + half_xqx);
        acc.add(3, xj * xj);
        const double dx = xj - static_cast<double>(x_restart[j]);
        acc.add(4, dx * dx);
        const bool lf = isfinite(lo), hf = isfinite(hi);
        double viol = 0.0, term = 0.0;
        if (lf && hf) {
            term = fmin(r * lo, r * hi);
        } else if (lf) {
            viol = fmax(0.0, -r);
            term = fmax(0.0, r) * lo;
        } else if (hf) {
            viol = fmax(0.0, r);
            term = fmin(0.0, r) * hi;
        } else {
            viol = fabs(r);
        }
        acc.add(0, viol * viol);
        acc.add(1, QM == kLp ? term : term - half_xqx);
        acc.max(5, fabs(xj - fmin(fmax(xj - r, lo), hi)));
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

// The same sums for the centered FP32 loop, evaluated in FP64 on the combined point
// (FP64 center + FP32 deviation) against the scaled FP64 problem: A x = ax_center +
// (A dx), A'y = rc_center - c + (A'dy) (rc_center = c + A'y_center), x = x_center + dx,
// y = y_center + dy. The restart reference is the center itself, so the moves since
// the last restart are the deviations.
template <class T>
struct ResRowsCenteredEpi {
    const T* __restrict__ dy;
    const double* __restrict__ y_center;
    const double* __restrict__ ax_center;
    const double* __restrict__ rl;
    const double* __restrict__ ru;
    T* __restrict__ ax_out;  // may be null: receives A dx
    double* __restrict__ partial;
    using Acc = Slots<5, 0xFu>;
    __device__ __forceinline__ void row(int i, T adx, Acc& acc) const {
        if (ax_out) ax_out[i] = adx;
        const double d = static_cast<double>(dy[i]);
        const double axi = ax_center[i] + static_cast<double>(adx), lo = rl[i], hi = ru[i], yi = y_center[i] + d;
        const double pr = axi - fmin(fmax(axi, lo), hi);
        acc.add(0, pr * pr);
        acc.add(1, yi * yi);
        acc.add(2, d * d);
        double support = 0.0;
        if (yi > 0.0) support = isfinite(hi) ? yi * hi : 0.0;
        else if (yi < 0.0) support = isfinite(lo) ? yi * lo : 0.0;
        acc.add(3, -support);
        acc.max(4, fabs(pr));
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

// QP: rc_center includes Q x_center; the deviation's part is q dx (diagonal, FP64
// q) or Q dx (general, the FP32 product dq), and Q x of the combined point is
// q x (diagonal) or qx_center + dq (general).
template <class T, int QM = kLp>
struct ResColsCenteredEpi {
    const T* __restrict__ dx;
    const double* __restrict__ x_center;
    const double* __restrict__ rc_center;
    const double* __restrict__ c;
    const double* __restrict__ cl;
    const double* __restrict__ cu;
    const double* __restrict__ q64;      // kQDiag: the FP64 diagonal; kQGeneral: Q x_center
    const T* __restrict__ dq;            // kQGeneral: Q dx of the evaluated deviation
    double* __restrict__ partial;
    using Acc = Slots<6, 0x1Fu>;
    __device__ __forceinline__ void row(int j, T atdy, Acc& acc) const {
        const double d = static_cast<double>(dx[j]);
        const double xj = x_center[j] + d, lo = cl[j], hi = cu[j], cj = c[j];
        double r = rc_center[j] + static_cast<double>(atdy);
        double half_xqx = 0.0;
        if (QM == kQDiag) {
            r += q64[j] * d;
            half_xqx = 0.5 * xj * (q64[j] * xj);
        } else if (QM == kQGeneral) {
            const double g = static_cast<double>(dq[j]);
            r += g;
            half_xqx = 0.5 * xj * (q64[j] + g);
        }
        acc.add(2, cj * xj + half_xqx);
        acc.add(3, xj * xj);
        acc.add(4, d * d);
        const bool lf = isfinite(lo), hf = isfinite(hi);
        double viol = 0.0, term = 0.0;
        if (lf && hf) {
            term = fmin(r * lo, r * hi);
        } else if (lf) {
            viol = fmax(0.0, -r);
            term = fmax(0.0, r) * lo;
        } else if (hf) {
            viol = fmax(0.0, r);
            term = fmin(0.0, r) * hi;
        } else {
            viol = fabs(r);
        }
        acc.add(0, viol * viol);
        acc.add(1, term - half_xqx);
        acc.max(5, fabs(xj - fmin(fmax(xj - r, lo), hi)));
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

// Re-centering of the FP32 loop: the center moves by the deviation `from` (the
// restart point), x kept inside its bounds.
template <class T>
__global__ void k_recenter(int n, int m, const T* __restrict__ from_x, const T* __restrict__ from_y,
                           double* __restrict__ xc, double* __restrict__ yc, const double* __restrict__ cl,
                           const double* __restrict__ cu) {
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride)
        xc[j] = fmin(fmax(xc[j] + static_cast<double>(from_x[j]), cl[j]), cu[j]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) yc[i] += static_cast<double>(from_y[i]);
}

// FP32 data of the problem around the center (FP64 in, one rounding out):
// c + A'yc, column bounds minus xc, row bounds minus A xc; infinite bounds stay infinite.
// QP: the gradient at the center also holds q x_center (qdiag) or Q x_center (qx_c).
__global__ void k_frame(int n, int m, const double* __restrict__ c, const double* __restrict__ aty_c,
                        const double* __restrict__ cl, const double* __restrict__ cu, const double* __restrict__ xc,
                        const double* __restrict__ rl, const double* __restrict__ ru, const double* __restrict__ ax_c,
                        const double* __restrict__ qdiag, const double* __restrict__ qx_c,
                        double* __restrict__ rc_c, float* __restrict__ c32, float* __restrict__ cl32,
                        float* __restrict__ cu32, float* __restrict__ rl32, float* __restrict__ ru32) {
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        double r = c[j] + aty_c[j];
        if (qdiag) r += qdiag[j] * xc[j];
        else if (qx_c) r += qx_c[j];
        rc_c[j] = r;
        c32[j] = static_cast<float>(r);
        cl32[j] = static_cast<float>(cl[j] - xc[j]);
        cu32[j] = static_cast<float>(cu[j] - xc[j]);
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        rl32[i] = static_cast<float>(rl[i] - ax_c[i]);
        ru32[i] = static_cast<float>(ru[i] - ax_c[i]);
    }
}

// Deviations, running sums and products back to zero after a re-centering; the
// accepted-step count at the restart is recorded as k_restart does.
template <class T>
__global__ void k_zero_deviation(int n, int m, T* __restrict__ x, T* __restrict__ x_sum, T* __restrict__ y,
                                 T* __restrict__ y_sum, T* __restrict__ ax, T* __restrict__ ax_prev, T* __restrict__ qx,
                                 PdlpState* st) {
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        x[j] = x_sum[j] = T(0);
        if (qx) qx[j] = T(0);
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) y[i] = y_sum[i] = ax[i] = ax_prev[i] = T(0);
    if (blockIdx.x == 0 && threadIdx.x == 0) st->accepted_at_restart = st->accept_count;
}

// out[0..7] in the reference's PdlpResiduals order (PdlpKernels.cuh), then the
// step state, then out[12] max primal residual, out[13] max column KKT residual;
// clears the accept flag after the window commit.
__global__ void k_res_combine(const double* __restrict__ prow, int nrow_blocks, const double* __restrict__ pcol,
                              int ncol_blocks, double* __restrict__ out, PdlpState* st, int clear_accept) {
    __shared__ double red[11][kThreads];
    double v[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int g = threadIdx.x; g < nrow_blocks; g += kThreads) {
        for (int k = 0; k < 4; ++k) v[k] += prow[g * 5 + k];
        v[4] = fmax(v[4], prow[g * 5 + 4]);
    }
    for (int g = threadIdx.x; g < ncol_blocks; g += kThreads) {
        for (int k = 0; k < 5; ++k) v[5 + k] += pcol[g * 6 + k];
        v[10] = fmax(v[10], pcol[g * 6 + 5]);
    }
    for (int k = 0; k < 11; ++k) red[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int k = 0; k < 11; ++k)
                red[k][threadIdx.x] = (k == 4 || k == 10) ? fmax(red[k][threadIdx.x], red[k][threadIdx.x + s])
                                                          : red[k][threadIdx.x] + red[k][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // primal_residual_sq, dual_residual_sq, primal_objective, dual_objective,
        // x_norm_sq, y_norm_sq, primal_move_sq, dual_move_sq
        out[0] = red[0][0];
        out[1] = red[5][0];
        out[2] = red[7][0];
        out[3] = red[6][0] + red[3][0];
        out[4] = red[8][0];
        out[5] = red[1][0];
        out[6] = red[9][0];
        out[7] = red[2][0];
        out[8] = st->eta;
        out[9] = st->accept_count;
        out[10] = st->updates;
        out[11] = st->omega;
        out[12] = red[4][0];
        out[13] = red[10][0];
        if (clear_accept) st->accepted = 0.0;
    }
}

// x_avg = (1/terms) x_sum (GpuPdlp.cpp:371-390 with the divisor on the device)
template <class T>
__global__ void k_average(int n, int m, const PdlpState* __restrict__ st, int adaptive, const T* __restrict__ x_sum,
                          const T* __restrict__ y_sum, T* __restrict__ x_avg, T* __restrict__ y_avg) {
    double terms = adaptive ? st->accept_count - st->accepted_at_restart : st->terms_fixed;
    if (terms < 1.0) terms = 1.0;
    const T scale = static_cast<T>(1.0 / terms);
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) x_avg[j] = scale * x_sum[j];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) y_avg[i] = scale * y_sum[i];
}

// Restart (GpuPdlp.cpp:453-497) as one elementwise pass.
template <class T>
__global__ void k_restart(int n, int m, int to_average, int adaptive, T* __restrict__ x, T* __restrict__ y,
                          T* __restrict__ x_bar, const T* __restrict__ x_avg, const T* __restrict__ y_avg,
                          T* __restrict__ ax, T* __restrict__ ax_prev, const T* __restrict__ ax_avg,
                          T* __restrict__ x_sum, T* __restrict__ y_sum, T* __restrict__ x_restart,
                          T* __restrict__ y_restart, T* __restrict__ qx, const T* __restrict__ qx_avg, PdlpState* st) {
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        T xj = x[j];
        if (to_average) {
            xj = x_avg[j];
            x[j] = xj;
            if (qx) qx[j] = qx_avg[j];
        }
        x_bar[j] = xj;
        x_sum[j] = T(0);
        x_restart[j] = xj;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        T yi = y[i];
        if (to_average) { yi = y_avg[i]; y[i] = yi; }
        y_sum[i] = T(0);
        y_restart[i] = yi;
        if (adaptive) {
            T a = ax[i];
            if (to_average) { a = ax_avg[i]; ax[i] = a; }
            ax_prev[i] = a;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && adaptive) st->accepted_at_restart = st->accept_count;
}

__global__ void k_init_state(PdlpState* st, double eta, double omega, double eta_min, double eta_max) {
    st->eta = eta;
    st->omega = omega;
    st->accepted = 0.0;
    st->updates = 0.0;
    st->accept_count = 0.0;
    st->accepted_at_restart = 0.0;
    st->eta_min = eta_min;
    st->eta_max = eta_max;
    st->terms_fixed = 1.0;
    st->eta_bar = eta;
    st->dx_sq = st->dy_sq = st->interaction = 0.0;
    st->ticket = 0u;
    st->pad = 0u;
}

__global__ void k_set_omega(PdlpState* st, double omega, double terms_fixed) {
    st->omega = omega;
    st->terms_fixed = terms_fixed;
}

// ----------------------------------------------------------- norms / power it.

// Sum of squares of v over finite entries below 1e30 in magnitude (block partials).
template <class T>
__global__ void k_sumsq(const T* __restrict__ v, int n, int finite_only, double* __restrict__ partial) {
    __shared__ double smem[kWarps];
    Slots<1, 1u> acc;
    acc.init();
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) {
        const double a = v[j];
        if (!finite_only || (isfinite(a) && fabs(a) < 1e30)) acc.add(0, a * a);
    }
    block_store(acc, partial, smem);
}

__global__ void k_normalize(double* __restrict__ v, int n, const double* __restrict__ norm_sq) {
    const double nrm = sqrt(*norm_sq);
    if (!(nrm > 0.0)) return;
    const double inv = 1.0 / nrm;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) v[j] *= inv;
}

// ----------------------------------------------------------------- scaling

// One warp per CSR row: out[r] = rs[r] * max_p |val[p]| * cs[idx[p]]  (mode 0, Ruiz norms)
//                       out[r] = sum_p |val[p]| * rs[r] * cs[idx[p]]  (mode 1, Pock-Chambolle alpha=1)
//                       out[r] = min, out2[r] = max of |val| rs cs     (mode 2, geometric passes)
__global__ void k_row_stats(int rows, const int* __restrict__ ptr, const int* __restrict__ idx,
                            const double* __restrict__ val, const double* __restrict__ rs,
                            const double* __restrict__ cs, int mode, int transposed, double* __restrict__ out,
                            double* __restrict__ out2) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int r = warp; r < rows; r += nwarps) {
        const double rsr = rs[r];
        double a = mode == 2 ? INFINITY : 0.0, b = 0.0;
        for (int p = ptr[r] + lane; p < ptr[r + 1]; p += 32) {
            if (mode == 0) {
                a = fmax(a, fabs(val[p]) * cs[idx[p]]);
            } else if (mode == 1) {
                const double v = fabs(val[p]);
                if (v != 0.0) a += v * rsr * cs[idx[p]];
            } else {
                // (|a| R_i) C_j in both orientations, as sk_scale.c:41 and :52 form it
                const double v = transposed ? fabs(val[p]) * cs[idx[p]] * rsr : fabs(val[p]) * rsr * cs[idx[p]];
                if (v > 0.0) { a = fmin(a, v); b = fmax(b, v); }
            }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const double oa = __shfl_xor_sync(0xffffffffu, a, off);
            const double ob = __shfl_xor_sync(0xffffffffu, b, off);
            a = mode == 0 ? fmax(a, oa) : (mode == 1 ? a + oa : fmin(a, oa));
            b = fmax(b, ob);
        }
        if (lane == 0) {
            if (mode == 0) out[r] = rsr * a;
            else if (mode == 1) out[r] = a;
            else { out[r] = b > 0.0 ? a : 0.0; out2[r] = b; }
        }
    }
}

// max |norm - 1| over positive norms (Scaling.cpp:64-72), block partials.
__global__ void k_ruiz_dev(const double* __restrict__ rn, int m, const double* __restrict__ cn, int n,
                           double* __restrict__ partial) {
    __shared__ double smem[kWarps];
    Slots<1, 0u> acc;
    acc.init();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m + n; i += blockDim.x * gridDim.x) {
        const double v = i < m ? rn[i] : cn[i - m];
        if (v > 0.0) acc.max(0, fabs(v - 1.0));
    }
    block_store(acc, partial, smem);
}

__global__ void k_div_sqrt(double* __restrict__ s, const double* __restrict__ nrm, int n) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x)
        if (nrm[j] > 0.0) s[j] /= sqrt(nrm[j]);
}

__global__ void k_mul_into(double* __restrict__ s, const double* __restrict__ t, int n) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) s[j] *= t[j];
}

__global__ void k_inv_sqrt_or_one(double* __restrict__ s, const double* __restrict__ acc, int n) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x)
        s[j] = acc[j] > 0.0 ? 1.0 / sqrt(acc[j]) : 1.0;
}

__global__ void k_geo_update(double* __restrict__ s, const double* __restrict__ mn, const double* __restrict__ mx, int n) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x)
        if (mx[j] > 0.0) s[j] /= sqrt(mn[j] * mx[j]);
}

// sk_scale.c:59-70: round to the power of two just below-or-at half the mantissa.
__global__ void k_round_pow2(double* __restrict__ s, int n) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) {
        const double v = s[j];
        if (!(v > 0.0) || !isfinite(v)) { s[j] = 1.0; continue; }
        int e;
        frexp(v, &e);
        s[j] = ldexp(1.0, e - 1);
    }
}

template <class T>
__global__ void k_fill_v(T* __restrict__ v, T value, int n) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) v[j] = value;
}

// Scaled values of a CSR: out[p] = (val[p] * rs[r]) * cs[idx[p]] (Scaling.cpp:94-109)
// transposed = 1 swaps the roles so A^T gets bit-identical values.
__global__ void k_scale_values(int rows, const int* __restrict__ ptr, const int* __restrict__ idx,
                               const double* __restrict__ val, const double* __restrict__ rs,
                               const double* __restrict__ cs, int transposed, double* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int r = warp; r < rows; r += nwarps)
        for (int p = ptr[r] + lane; p < ptr[r + 1]; p += 32)
            out[p] = transposed ? (val[p] * rs[idx[p]]) * cs[r] : (val[p] * rs[r]) * cs[idx[p]];
}

// Scaled model vectors (LpSolver.cpp:74-91); |bound| >= 1e30 becomes +-inf.
__global__ void k_scale_vectors(int n, int m, const double* __restrict__ R, const double* __restrict__ Cs,
                                double* __restrict__ c, double* __restrict__ cl, double* __restrict__ cu,
                                double* __restrict__ rl, double* __restrict__ ru) {
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const double s = Cs[j];
        c[j] = c[j] * s;
        const double lo = cl[j], hi = cu[j];
        cl[j] = lo <= -1e30 ? -INFINITY : lo / s;
        cu[j] = hi >= 1e30 ? INFINITY : hi / s;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const double s = R[i];
        const double lo = rl[i], hi = ru[i];
        rl[i] = lo <= -1e30 ? -INFINITY : s * lo;
        ru[i] = hi >= 1e30 ? INFINITY : s * hi;
    }
}

__global__ void k_unscale(int n, int m, const double* __restrict__ Cs, const double* __restrict__ R,
                          double* __restrict__ x, double* __restrict__ y) {
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) x[j] = x[j] * Cs[j];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) y[i] = y[i] * R[i];
}

// warm start: x' = x / C, y' = y / R
__global__ void k_to_scaled(int n, int m, const double* __restrict__ Cs, const double* __restrict__ R,
                            double* __restrict__ x, double* __restrict__ y) {
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) x[j] = x[j] / Cs[j];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) y[i] = y[i] / R[i];
}

// FP64 point from the FP32 phase: x^ = x, y^ = y (bounds kept exactly).
__global__ void k_widen(int n, int m, const float* __restrict__ x32, const float* __restrict__ y32,
                        const double* __restrict__ cl, const double* __restrict__ cu, double* __restrict__ x,
                        double* __restrict__ y) {
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride)
        x[j] = fmin(fmax(static_cast<double>(x32[j]), cl[j]), cu[j]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) y[i] = static_cast<double>(y32[i]);
}

// The bounds of the dual feasibility problem: every finite bound moved to 0,
// infinite ones kept, so the problem's dual feasible set is the original LP's.
__global__ void k_homogeneous(int len, const double* __restrict__ lo, const double* __restrict__ hi,
                              double* __restrict__ lo0, double* __restrict__ hi0) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += blockDim.x * gridDim.x) {
        lo0[i] = isfinite(lo[i]) ? 0.0 : lo[i];
        hi0[i] = isfinite(hi[i]) ? 0.0 : hi[i];
    }
}

__global__ void k_narrow(long long n, const double* __restrict__ in, float* __restrict__ out) {
    for (long long j = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; j < n;
         j += static_cast<long long>(blockDim.x) * gridDim.x)
        out[j] = static_cast<float>(in[j]);
}

// The scaled matrix values rounded to bf16 (round to nearest even) for the
// BF16_REFINE iterations.
__global__ void k_narrow_bf16(long long n, const double* __restrict__ in, __nv_bfloat16* __restrict__ out) {
    for (long long j = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; j < n;
         j += static_cast<long long>(blockDim.x) * gridDim.x)
        out[j] = __double2bfloat16(in[j]);
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Which relative KKT measures end a loop: all three (the default), or only the
// primal residual / only the dual residual (the polishing solves).
constexpr int kPrimalMeasure = 1, kDualMeasure = 2, kAllMeasures = 7;

struct Kkt {
    double primal = 1, dual = 1, gap = 1, pobj = 0, dobj = 0, pmove = 0, dmove = 0;
    double worst() const { return std::max(std::max(primal, dual), gap); }
    double on(int measure) const {
        return measure == kPrimalMeasure ? primal : measure == kDualMeasure ? dual : worst();
    }
};

Kkt to_kkt(const double* r, double cost_norm, double bound_norm) {
    Kkt k;
    k.primal = std::sqrt(std::max(0.0, r[0])) / (1.0 + bound_norm);
    k.dual = std::sqrt(std::max(0.0, r[1])) / (1.0 + cost_norm);
    k.pobj = r[2];
    k.dobj = r[3];
    k.gap = std::fabs(r[2] - r[3]) / (1.0 + std::fabs(r[2]) + std::fabs(r[3]));
    k.pmove = std::sqrt(std::max(0.0, r[6]));
    k.dmove = std::sqrt(std::max(0.0, r[7]));
    if (!std::isfinite(k.primal) || !std::isfinite(k.dual) || !std::isfinite(k.gap))
        k.primal = k.dual = k.gap = std::numeric_limits<double>::infinity();
    return k;
}

inline int eg(int len) { return elem_grid(std::max(len, 1)); }

// ------------------------------------------------------------- FP64 model

// The scaled FP64 model: factors, scaled values of A and A^T, scaled vectors,
// and scratch for the norms and ||A||_2.
struct Scaled {
    int n = 0, m = 0, sms = 148;
    cudaStream_t stream = nullptr;
    TileCsr A, AT;  // scaled views (values owned here)
    DevBuf blob, vals;
    double *c, *cl, *cu, *rl, *ru, *R, *Cs, *tmp_n, *tmp2_n, *tmp_m, *tmp2_m, *vec_n, *vec_m, *part, *scalar;
    double* host = nullptr;
    int launches = 0;

    int allocate(const Plan& plan) {
        n = plan.a.cols;
        m = plan.a.rows;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, plan.device);
        const size_t nb = (static_cast<size_t>(n) * 8 + 255) / 256 * 256;
        const size_t mb = (static_cast<size_t>(m) * 8 + 255) / 256 * 256;
        const size_t pb = (static_cast<size_t>(sms) * 8 * 8 * 8 + 255) / 256 * 256;
        if (blob.alloc(8 * nb + 7 * mb + 4 * pb + 1024, "cudaMalloc PDLP model")) return -1;
        if (vals.alloc(static_cast<size_t>(plan.a.nnz) * 16 + 1024, "cudaMalloc scaled values")) return -1;
        char* p = blob.as<char>();
        auto take = [&](size_t b) { double* r = reinterpret_cast<double*>(p); p += b; return r; };
        c = take(nb); cl = take(nb); cu = take(nb); Cs = take(nb); tmp_n = take(nb); tmp2_n = take(nb);
        vec_n = take(nb); take(nb);
        rl = take(mb); ru = take(mb); R = take(mb); tmp_m = take(mb); tmp2_m = take(mb); vec_m = take(mb); take(mb);
        part = take(4 * pb);
        scalar = take(1024);
        A = plan.a;
        AT = plan.at;
        A.val = vals.as<double>();
        AT.val = vals.as<double>() + ((static_cast<size_t>(plan.a.nnz) + 63) / 64 * 64);
        return 0;
    }

    double sumsq(const double* v, int len, bool finite_only) {
        const int g = std::min(eg(len), sms * 4);
        k_sumsq<double><<<g, kThreads, 0, stream>>>(v, len, finite_only ? 1 : 0, part);
        k_combine<1, 1u><<<1, kThreads, 0, stream>>>(part, len > 0 ? g : 0, scalar);
        launches += 2;
        cudaMemcpyAsync(host, scalar, sizeof(double), cudaMemcpyDeviceToHost, stream);
        cudaStreamSynchronize(stream);
        return host[0];
    }

    // Ruiz (Scaling.cpp:11-92), then Pock-Chambolle on the Ruiz-scaled matrix,
    // composed (Scaling.cpp:147-152); or the power-of-two passes (sk_scale.c).
    int scale(const Plan& plan, int mode, int ruiz_iters, double ruiz_tol, int* syncs) {
        const int gm = eg(m), gn = eg(n);
        const int wg_m = std::min((m + 7) / 8 + 1, sms * 16), wg_n = std::min((n + 7) / 8 + 1, sms * 16);
        k_fill_v<double><<<gm, kThreads, 0, stream>>>(R, 1.0, m);
        k_fill_v<double><<<gn, kThreads, 0, stream>>>(Cs, 1.0, n);
        const bool any = (mode & 7) != 0;
        if (any && plan.a.nnz > 0 && m > 0 && n > 0) {
            if (mode & SANKHYA_B200_SCALE_POW2) {
                for (int pass = 0; pass < 4; ++pass) {
                    // columns first (sk_scale.c:38-47), then rows (:48-57)
                    k_row_stats<<<wg_n, kThreads, 0, stream>>>(n, plan.at.ptr, plan.at.idx, plan.at.val, Cs, R, 2, 1,
                                                               tmp_n, tmp2_n);
                    k_geo_update<<<gn, kThreads, 0, stream>>>(Cs, tmp_n, tmp2_n, n);
                    k_row_stats<<<wg_m, kThreads, 0, stream>>>(m, plan.a.ptr, plan.a.idx, plan.a.val, R, Cs, 2, 0,
                                                               tmp_m, tmp2_m);
                    k_geo_update<<<gm, kThreads, 0, stream>>>(R, tmp_m, tmp2_m, m);
                    launches += 4;
                }
                k_round_pow2<<<gm, kThreads, 0, stream>>>(R, m);
                k_round_pow2<<<gn, kThreads, 0, stream>>>(Cs, n);
            }
            if (mode & SANKHYA_B200_SCALE_RUIZ) {
                bool converged = false;
                for (int it = 0; it < ruiz_iters; ++it) {
                    k_row_stats<<<wg_m, kThreads, 0, stream>>>(m, plan.a.ptr, plan.a.idx, plan.a.val, R, Cs, 0, 0,
                                                               tmp_m, nullptr);
                    k_row_stats<<<wg_n, kThreads, 0, stream>>>(n, plan.at.ptr, plan.at.idx, plan.at.val, Cs, R, 0, 1,
                                                               tmp_n, nullptr);
                    const int g = std::min(eg(m + n), sms * 4);
                    k_ruiz_dev<<<g, kThreads, 0, stream>>>(tmp_m, m, tmp_n, n, part);
                    k_combine<1, 0u><<<1, kThreads, 0, stream>>>(part, g, scalar);
                    launches += 4;
                    cudaMemcpyAsync(host, scalar, sizeof(double), cudaMemcpyDeviceToHost, stream);
                    B200_TRY(cudaStreamSynchronize(stream), "Ruiz");
                    ++*syncs;
                    if (host[0] < ruiz_tol) { converged = true; break; }
                    k_div_sqrt<<<gm, kThreads, 0, stream>>>(R, tmp_m, m);
                    k_div_sqrt<<<gn, kThreads, 0, stream>>>(Cs, tmp_n, n);
                }
                if (!converged && !(mode & SANKHYA_B200_SCALE_POW2)) {
                    k_fill_v<double><<<gm, kThreads, 0, stream>>>(R, 1.0, m);
                    k_fill_v<double><<<gn, kThreads, 0, stream>>>(Cs, 1.0, n);
                }
            }
            if (mode & SANKHYA_B200_SCALE_POCK_CHAMBOLLE) {
                k_row_stats<<<wg_m, kThreads, 0, stream>>>(m, plan.a.ptr, plan.a.idx, plan.a.val, R, Cs, 1, 0, tmp_m,
                                                           nullptr);
                k_row_stats<<<wg_n, kThreads, 0, stream>>>(n, plan.at.ptr, plan.at.idx, plan.at.val, Cs, R, 1, 1, tmp_n,
                                                           nullptr);
                k_inv_sqrt_or_one<<<gm, kThreads, 0, stream>>>(tmp2_m, tmp_m, m);
                k_inv_sqrt_or_one<<<gn, kThreads, 0, stream>>>(tmp2_n, tmp_n, n);
                k_mul_into<<<gm, kThreads, 0, stream>>>(R, tmp2_m, m);
                k_mul_into<<<gn, kThreads, 0, stream>>>(Cs, tmp2_n, n);
                launches += 6;
            }
        }
        const int wm = std::min((m + 7) / 8 + 1, sms * 16), wn = std::min((n + 7) / 8 + 1, sms * 16);
        k_scale_values<<<wm, kThreads, 0, stream>>>(m, plan.a.ptr, plan.a.idx, plan.a.val, R, Cs, 0,
                                                    const_cast<double*>(A.val));
        k_scale_values<<<wn, kThreads, 0, stream>>>(n, plan.at.ptr, plan.at.idx, plan.at.val, R, Cs, 1,
                                                    const_cast<double*>(AT.val));
        k_scale_vectors<<<eg(std::max(n, m)), kThreads, 0, stream>>>(n, m, R, Cs, c, cl, cu, rl, ru);
        launches += 3;
        B200_TRY(cudaGetLastError(), "scaling launch");
        return 0;
    }

    // GpuPdlp.cpp:179-211 on the device, one sync at the end.
    double power_norm(int iters) {
        const int g = std::min(eg(n), sms * 4);
        k_fill_v<double><<<eg(n), kThreads, 0, stream>>>(vec_n, 1.0, n);
        k_sumsq<double><<<g, kThreads, 0, stream>>>(vec_n, n, 0, part);
        k_combine<1, 1u><<<1, kThreads, 0, stream>>>(part, n > 0 ? g : 0, scalar);
        k_normalize<<<eg(n), kThreads, 0, stream>>>(vec_n, n, scalar);
        const int ga = tiled_grid<StoreEpi>(A), gt = tiled_grid<StoreEpi>(AT);
        for (int k = 0; k < iters; ++k) {
            launch_tiled(A, vec_n, StoreEpi{vec_m}, stream, ga);
            launch_tiled(AT, vec_m, StoreEpi{tmp_n}, stream, gt);
            k_sumsq<double><<<g, kThreads, 0, stream>>>(tmp_n, n, 0, part);
            k_combine<1, 1u><<<1, kThreads, 0, stream>>>(part, n > 0 ? g : 0, scalar);
            k_copy<<<eg(n), kThreads, 0, stream>>>(vec_n, tmp_n, n);
            k_normalize<<<eg(n), kThreads, 0, stream>>>(vec_n, n, scalar);
        }
        launches += 4 + 6 * iters;
        cudaMemcpyAsync(host, scalar, sizeof(double), cudaMemcpyDeviceToHost, stream);
        cudaStreamSynchronize(stream);
        const double lambda = std::sqrt(std::max(0.0, host[0]));
        const double norm = std::sqrt(lambda);
        return (norm > 0.0 && std::isfinite(norm)) ? norm : 1.0;
    }
};

// ------------------------------------------------------------- the iteration

struct LoopParams {
    double eps = 1e-8;
    long long max_iterations = 0;
    int restart_period = 64;
    bool adaptive = true;
    double deadline = 0.0;  // absolute time (now_s() seconds), <= 0 none
    double matrix_norm = 1.0, eta_min_factor = 1e-6, eta_max_factor = 1e4;
    double cost_norm = 0.0, bound_norm = 0.0;
    double omega0 = 0.0;  // > 0: initial primal weight (else ||c|| / ||b||)
    double eta0 = 0.0;    // > 0: initial step size (else 0.9 / ||A||_2)
    bool halpern = false; // reflected restarted Halpern PDHG instead of GpuPdlp's loop
    int (*cancel)(void*) = nullptr;  // polled after each window; non-zero stops the solve
    void* cancel_context = nullptr;
    int measure = kAllMeasures;  // what must reach eps (restarts always use all three)
    bool fixed_weight = false;   // keep omega0 at restarts (the polishing solves)
};

// The FP64 side of the centered FP32 loop: the scaled FP64 problem, the center
// (x_center, y_center: the last restart point, which is also the refinement
// point), its products and the FP32 frame data the iterations run on.
struct Centered {
    TileCsr A, AT;  // scaled FP64 matrix
    TileCsr Q;      // scaled FP64 Hessian (QP, general path; ntiles 0 otherwise)
    const double *c = nullptr, *cl = nullptr, *cu = nullptr, *rl = nullptr, *ru = nullptr;
    const double* qdiag = nullptr;  // scaled FP64 Hessian diagonal (QP, diagonal path)
    double *xc = nullptr, *yc = nullptr, *ax_c = nullptr, *aty_c = nullptr, *rc_c = nullptr;
    double* qx_c = nullptr;         // Q x_center (general path)
    float *c32 = nullptr, *cl32 = nullptr, *cu32 = nullptr, *rl32 = nullptr, *ru32 = nullptr;
    int grid_a = 1, grid_at = 1, grid_q = 1;
};

struct LoopStats {
    long long iterations = 0;
    int restarts = 0, syncs = 0;
    bool converged = false, timed_out = false, numeric = false, cancelled = false;
    double eta = 0.0, accept_count = 0.0, updates = 0.0, omega = 1.0;
    Kkt best;
};

// Restarted PDLP on one problem whose data (c, bounds) have type T and whose matrix
// values have type V (T, or bf16 under fp32 iterates); iterates of type T; reductions
// and decisions in FP64.
template <class T, class V = T>
struct Core {
    int n = 0, m = 0, sms = 148;
    cudaStream_t stream = nullptr;
    TileCsrT<V> A, AT;
    const T *c = nullptr, *cl = nullptr, *cu = nullptr, *rl = nullptr, *ru = nullptr;
    DevBuf blob;
    T *x, *x_cand, *x_sum, *x_avg, *x_restart, *x_bar, *aty;
    T *y, *y_cand, *y_sum, *y_avg, *y_restart, *ax, *ax_prev, *ax_cand, *ax_avg;
    double *part_a, *part_b, *part_c, *part_d, *res;
    PdlpState* st;
    double* host = nullptr;
    int grid_k2 = 1, grid_k3 = 1, grid_rr = 1, grid_rc = 1, grid_df = 1, grid_pf = 1;
    int grid_ph = 1, grid_dh = 1, grid_pt = 1, grid_dt = 1;
    int grid_rrc = 1, grid_rcc = 1;
    int launches = 0;
    std::vector<cudaGraphExec_t> graphs;
    // Quadratic objective (the QP entry point): qmode kQDiag with the diagonal qd,
    // or kQGeneral with the Hessian Q and its diagonal majorant qd, whose products
    // Q x (committed point), Q x_cand and Q x_avg ride along like the A-side ones;
    // kLp otherwise.
    int qmode = kLp;
    const T* qd = nullptr;
    TileCsrT<T> Q;
    DevBuf qblob;
    T *qx = nullptr, *qx_cand = nullptr, *qx_avg = nullptr;
    int grid_qs = 1;
    // Centered mode (FP32 iterations of the FP32_REFINE precision): x, y, ax and the
    // sums are deviations from ctr's FP64 center; the center moves to the restart
    // point at every restart (one refinement), and the window-end residuals are
    // taken in FP64 on center + deviation.
    const Centered* ctr = nullptr;
    int recenters = 0;
    Core() = default;
    Core(const Core&) = delete;
    Core& operator=(const Core&) = delete;
    ~Core() {
        for (auto g : graphs)
            if (g) cudaGraphExecDestroy(g);
    }

    int allocate(int n_, int m_, int sms_) {
        n = n_;
        m = m_;
        sms = sms_;
        const size_t nb = (static_cast<size_t>(n) * sizeof(T) + 255) / 256 * 256;
        const size_t mb = (static_cast<size_t>(m) * sizeof(T) + 255) / 256 * 256;
        const size_t pb = (static_cast<size_t>(sms) * 8 * 8 * 8 + 255) / 256 * 256;
        if (blob.alloc(7 * nb + 9 * mb + 4 * pb + 2048, "cudaMalloc PDLP iterates")) return -1;
        char* p = blob.as<char>();
        auto take = [&](size_t b) { char* r = p; p += b; return r; };
        x = reinterpret_cast<T*>(take(nb)); x_cand = reinterpret_cast<T*>(take(nb));
        x_sum = reinterpret_cast<T*>(take(nb)); x_avg = reinterpret_cast<T*>(take(nb));
        x_restart = reinterpret_cast<T*>(take(nb)); x_bar = reinterpret_cast<T*>(take(nb));
        aty = reinterpret_cast<T*>(take(nb));
        y = reinterpret_cast<T*>(take(mb)); y_cand = reinterpret_cast<T*>(take(mb));
        y_sum = reinterpret_cast<T*>(take(mb)); y_avg = reinterpret_cast<T*>(take(mb));
        y_restart = reinterpret_cast<T*>(take(mb)); ax = reinterpret_cast<T*>(take(mb));
        ax_prev = reinterpret_cast<T*>(take(mb)); ax_cand = reinterpret_cast<T*>(take(mb));
        ax_avg = reinterpret_cast<T*>(take(mb));
        part_a = reinterpret_cast<double*>(take(pb)); part_b = reinterpret_cast<double*>(take(pb));
        part_c = reinterpret_cast<double*>(take(pb)); part_d = reinterpret_cast<double*>(take(pb));
        res = reinterpret_cast<double*>(take(1024));
        st = reinterpret_cast<PdlpState*>(take(1024));
        return 0;
    }

    void set_problem(const TileCsrT<V>& a, const TileCsrT<V>& at, const T* c_, const T* cl_, const T* cu_,
                     const T* rl_, const T* ru_) {
        A = a;
        AT = at;
        c = c_; cl = cl_; cu = cu_; rl = rl_; ru = ru_;
        grid_k2 = qmode == kQDiag ? tiled_grid<PrimalCandEpi<T, kQDiag>, T>(AT)
                  : qmode == kQGeneral ? tiled_grid<PrimalCandEpi<T, kQGeneral>, T>(AT)
                                       : tiled_grid<PrimalCandEpi<T>, T>(AT);
        grid_k3 = tiled_grid<ProbeEpi<T>, T>(A);
        grid_rr = tiled_grid<ResRowsEpi<T>, T>(A);
        grid_rc = qmode == kQDiag ? tiled_grid<ResColsEpi<T, kQDiag>, T>(AT)
                  : qmode == kQGeneral ? tiled_grid<ResColsEpi<T, kQGeneral>, T>(AT)
                                       : tiled_grid<ResColsEpi<T>, T>(AT);
        grid_df = tiled_grid<DualFixedEpi<T>, T>(A);
        grid_pf = tiled_grid<PrimalFixedEpi<T>, T>(AT);
        grid_ph = tiled_grid<PrimalHalpernEpi<T>, T>(AT);
        grid_dh = tiled_grid<DualHalpernEpi<T>, T>(A);
        grid_pt = tiled_grid<PrimalTEpi<T>, T>(AT);
        grid_dt = tiled_grid<DualTEpi<T>, T>(A);
        grid_rrc = tiled_grid<ResRowsCenteredEpi<T>, T>(A);
        grid_rcc = qmode == kQDiag ? tiled_grid<ResColsCenteredEpi<T, kQDiag>, T>(AT)
                   : qmode == kQGeneral ? tiled_grid<ResColsCenteredEpi<T, kQGeneral>, T>(AT)
                                        : tiled_grid<ResColsCenteredEpi<T>, T>(AT);
        for (auto g : graphs)
            if (g) cudaGraphExecDestroy(g);
        graphs.clear();
    }

    // The QP's Hessian: a diagonal (diag, q null) or a general matrix (q, n x n, with
    // diag its majorant row sums |Q|); call after allocate and before set_problem. The
    // general path owns Q x, Q x_cand and Q x_avg.
    int set_hessian(const T* diag, const TileCsrT<T>* q) {
        if (!diag) return 0;
        qd = diag;
        if (!q) {
            qmode = kQDiag;
            return 0;
        }
        qmode = kQGeneral;
        Q = *q;
        const size_t nb = (static_cast<size_t>(n) * sizeof(T) + 255) / 256 * 256;
        if (qblob.alloc(3 * nb, "cudaMalloc Hessian products")) return -1;
        qx = qblob.as<T>();
        qx_cand = reinterpret_cast<T*>(qblob.as<char>() + nb);
        qx_avg = reinterpret_cast<T*>(qblob.as<char>() + 2 * nb);
        grid_qs = tiled_grid<StoreEpiT<T>, T>(Q);
        return 0;
    }

    template <int QM>
    void residuals_q(const T* xv, const T* yv, T* ax_out, T* aty_out, const T* qv, double* out, int clear_accept) {
        const int nbr = A.ntiles ? grid_rr : 0, nbc = AT.ntiles ? grid_rc : 0;
        launch_tiled(A, xv, ResRowsEpi<T>{yv, y_restart, rl, ru, ax_out, part_a}, stream, grid_rr);
        launch_tiled(AT, yv, ResColsEpi<T, QM>{xv, x_restart, c, cl, cu, qv, aty_out, part_b}, stream, grid_rc);
        k_res_combine<<<1, kThreads, 0, stream>>>(part_a, nbr, part_b, nbc, out, st, clear_accept);
        launches += 3;
    }

    template <int QM>
    void residuals_centered(const T* xv, const T* yv, T* ax_out, const T* dq, double* out, int clear_accept) {
        const int nbr = A.ntiles ? grid_rrc : 0, nbc = AT.ntiles ? grid_rcc : 0;
        launch_tiled(A, xv, ResRowsCenteredEpi<T>{yv, ctr->yc, ctr->ax_c, ctr->rl, ctr->ru, ax_out, part_a}, stream,
                     grid_rrc);
        const double* q64 = QM == kQDiag ? ctr->qdiag : ctr->qx_c;
        launch_tiled(AT, yv, ResColsCenteredEpi<T, QM>{xv, ctr->xc, ctr->rc_c, ctr->c, ctr->cl, ctr->cu, q64, dq,
                                                       part_b},
                     stream, grid_rcc);
        k_res_combine<<<1, kThreads, 0, stream>>>(part_a, nbr, part_b, nbc, out, st, clear_accept);
        launches += 3;
    }

    // Residual sums of (xv, yv) into out[0..13]; ax_out / aty_out optional; qv is
    // Q xv (general Hessian) of the evaluated point.
    void residuals(const T* xv, const T* yv, T* ax_out, T* aty_out, double* out, int clear_accept,
                   const T* qv = nullptr) {
        if (ctr) {
            if (qmode == kQDiag) residuals_centered<kQDiag>(xv, yv, ax_out, nullptr, out, clear_accept);
            else if (qmode == kQGeneral) residuals_centered<kQGeneral>(xv, yv, ax_out, qv, out, clear_accept);
            else residuals_centered<kLp>(xv, yv, ax_out, nullptr, out, clear_accept);
            return;
        }
        if (qmode == kQDiag) residuals_q<kQDiag>(xv, yv, ax_out, aty_out, qd, out, clear_accept);
        else if (qmode == kQGeneral) residuals_q<kQGeneral>(xv, yv, ax_out, aty_out, qv, out, clear_accept);
        else residuals_q<kLp>(xv, yv, ax_out, aty_out, nullptr, out, clear_accept);
    }

    void adaptive_iteration(bool make_candidate) {
        const bool general = qmode == kQGeneral;
        k_commit_dual<T><<<eg(std::max(n, m)), kThreads, 0, stream>>>(n, m, st, x, x_cand, x_sum, y, y_cand, y_sum,
                                                                      ax, ax_prev, ax_cand, rl, ru,
                                                                      ctr ? ctr->yc : nullptr, general ? qx : nullptr,
                                                                      qx_cand, make_candidate ? 1 : 0);
        ++launches;
        if (!make_candidate) return;
        if (qmode == kQDiag)
            launch_tiled(AT, y_cand, PrimalCandEpi<T, kQDiag>{st, x, c, cl, cu, qd, nullptr, x_cand, part_c}, stream,
                         grid_k2);
        else if (general)
            launch_tiled(AT, y_cand, PrimalCandEpi<T, kQGeneral>{st, x, c, cl, cu, qd, qx, x_cand, part_c}, stream,
                         grid_k2);
        else
            launch_tiled(AT, y_cand, PrimalCandEpi<T>{st, x, c, cl, cu, nullptr, nullptr, x_cand, part_c}, stream,
                         grid_k2);
        if (general) {
            launch_tiled(Q, x_cand, StoreEpiT<T>{qx_cand}, stream, grid_qs);   // Q x_cand, committed with x_cand
            ++launches;
        }
        launch_tiled(A, x_cand, ProbeEpi<T>{st, y, y_cand, ax, ax_cand, part_d, part_c, AT.ntiles ? grid_k2 : 0},
                     stream, grid_k3);
        launches += 2;
    }

    void fixed_iteration(T tau, T sigma) {
        launch_tiled(A, x_bar, DualFixedEpi<T>{y, y_sum, rl, ru, sigma}, stream, grid_df);
        launch_tiled(AT, y, PrimalFixedEpi<T>{x, x_bar, x_sum, c, cl, cu, tau}, stream, grid_pf);
        launches += 2;
    }

    // One window (period iterations) + window-end evaluation, as a graph.
    int window(int period, bool adaptive, double tau, double sigma, int* graph_slot) {
        cudaGraphExec_t exec = nullptr;
        if (*graph_slot >= 0) exec = graphs[static_cast<size_t>(*graph_slot)];
        if (!exec) {
            const int saved = launches;
            cudaGraph_t g;
            B200_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            for (int k = 0; k < period; ++k) {
                if (adaptive) adaptive_iteration(true);
                else fixed_iteration(static_cast<T>(tau), static_cast<T>(sigma));
            }
            if (adaptive) adaptive_iteration(false);  // commit the last probe
            residuals(x, y, nullptr, nullptr, res, 0, qx);
            k_average<T><<<eg(std::max(n, m)), kThreads, 0, stream>>>(n, m, st, adaptive ? 1 : 0, x_sum, y_sum, x_avg,
                                                                       y_avg);
            if (qmode == kQGeneral) {
                launch_tiled(Q, x_avg, StoreEpiT<T>{qx_avg}, stream, grid_qs);
                ++launches;
            }
            residuals(x_avg, y_avg, ax_avg, nullptr, res + 16, 1, qx_avg);
            cudaMemcpyAsync(host, res, 32 * sizeof(double), cudaMemcpyDeviceToHost, stream);
            B200_TRY(cudaStreamEndCapture(stream, &g), "end capture");
            cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail_cuda("graph instantiate", e);
            if (*graph_slot >= 0) {
                graphs[static_cast<size_t>(*graph_slot)] = exec;
            } else {
                graphs.push_back(exec);
                *graph_slot = static_cast<int>(graphs.size()) - 1;
            }
            launches = saved;
        }
        B200_TRY(cudaGraphLaunch(exec, stream), "graph launch");
        launches += (adaptive ? 3 * period + 1 : 2 * period) + 7;
        return 0;
    }

    // Centered mode: products of the FP64 center and the FP32 frame data around it.
    void build_frame() {
        launch_tiled(ctr->A, ctr->xc, StoreEpi{ctr->ax_c}, stream, ctr->grid_a);
        launch_tiled(ctr->AT, ctr->yc, StoreEpi{ctr->aty_c}, stream, ctr->grid_at);
        const bool general = qmode == kQGeneral;
        if (general) {
            launch_tiled(ctr->Q, ctr->xc, StoreEpi{ctr->qx_c}, stream, ctr->grid_q);
            ++launches;
        }
        k_frame<<<eg(std::max(n, m)), kThreads, 0, stream>>>(n, m, ctr->c, ctr->aty_c, ctr->cl, ctr->cu, ctr->xc,
                                                             ctr->rl, ctr->ru, ctr->ax_c,
                                                             qmode == kQDiag ? ctr->qdiag : nullptr,
                                                             general ? ctr->qx_c : nullptr, ctr->rc_c, ctr->c32,
                                                             ctr->cl32, ctr->cu32, ctr->rl32, ctr->ru32);
        launches += 3;
        ++recenters;
    }

    // Centered mode: the center moves by the deviation (fx, fy); with rebuild the
    // frame follows and the deviations restart at zero (a restart), else the
    // center alone is updated (the final point).
    void recenter(const T* fx, const T* fy, bool rebuild) {
        k_recenter<T><<<eg(std::max(n, m)), kThreads, 0, stream>>>(n, m, fx, fy, ctr->xc, ctr->yc, ctr->cl, ctr->cu);
        ++launches;
        if (!rebuild) return;
        build_frame();
        k_zero_deviation<T><<<eg(std::max(n, m)), kThreads, 0, stream>>>(n, m, x, x_sum, y, y_sum, ax, ax_prev,
                                                                          qmode == kQGeneral ? qx : nullptr, st);
        ++launches;
    }

    // One Halpern window: `period` anchored steps, then T at the window's end
    // (into x_cand / y_cand), its residual sums (res[32..35]) and the relative KKT of
    // T(z) (res[0..13]); x_restart / y_restart hold the anchor. A graph per (period,
    // tau, sigma); the anchor offset comes from the device state.
    int halpern_window(int period, int* graph_slot) {
        cudaGraphExec_t exec = nullptr;
        if (*graph_slot >= 0) exec = graphs[static_cast<size_t>(*graph_slot)];
        if (!exec) {
            const int saved = launches;
            cudaGraph_t g;
            B200_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            for (int q = 0; q < period; ++q) {
                launch_tiled(AT, y, PrimalHalpernEpi<T>{x, x_bar, x_restart, c, cl, cu, st, q}, stream, grid_ph);
                launch_tiled(A, x_bar, DualHalpernEpi<T>{y, y_restart, rl, ru, st, q}, stream, grid_dh);
            }
            launch_tiled(AT, y, PrimalTEpi<T>{x, x_bar, x_cand, x_restart, c, cl, cu, st, part_c}, stream, grid_pt);
            k_combine<2, 3u><<<1, kThreads, 0, stream>>>(part_c, AT.ntiles ? grid_pt : 0, res + 32);
            launch_tiled(A, x_bar, DualTEpi<T>{y, y_cand, y_restart, rl, ru, st, part_d}, stream, grid_dt);
            k_combine<2, 3u><<<1, kThreads, 0, stream>>>(part_d, A.ntiles ? grid_dt : 0, res + 34);
            residuals(x_cand, y_cand, nullptr, nullptr, res, 0);
            cudaMemcpyAsync(host, res, 40 * sizeof(double), cudaMemcpyDeviceToHost, stream);
            B200_TRY(cudaStreamEndCapture(stream, &g), "end capture");
            cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail_cuda("graph instantiate", e);
            if (*graph_slot >= 0) {
                graphs[static_cast<size_t>(*graph_slot)] = exec;
            } else {
                graphs.push_back(exec);
                *graph_slot = static_cast<int>(graphs.size()) - 1;
            }
            launches = saved;
        }
        B200_TRY(cudaGraphLaunch(exec, stream), "graph launch");
        launches += 2 * period + 7;
        return 0;
    }

    // Reflected restarted Halpern PDHG (the method of cuPDLP+, Lu and Yang 2025,
    // restated): constant step eta = 0.9 / ||A||_2 split by the primal weight,
    // restarts to T(z) when the fixed-point residual r = sqrt(omega |dx|^2 +
    // |dy|^2 / omega) falls to 0.2 of its value at the last restart, or to 0.8
    // and rises again, or after 0.36 of all iterations; at a restart the primal
    // weight moves halfway (in log) to |y+ - y0| / |x+ - x0|. Termination on the
    // relative KKT of T(z) at each window's end.
    int run_halpern(const LoopParams& lp, LoopStats* out) {
        const size_t nb = sizeof(T) * static_cast<size_t>(std::max(n, 1));
        const size_t mb = sizeof(T) * static_cast<size_t>(std::max(m, 1));
        for (T* v : {x_sum, x_cand, x_avg, aty}) cudaMemsetAsync(v, 0, nb, stream);
        for (T* v : {y_sum, y_cand, y_avg, ax_cand, ax_avg}) cudaMemsetAsync(v, 0, mb, stream);
        B200_TRY(cudaMemcpyAsync(x_restart, x, nb, cudaMemcpyDeviceToDevice, stream), "copy");
        B200_TRY(cudaMemcpyAsync(y_restart, y, mb, cudaMemcpyDeviceToDevice, stream), "copy");
        const double eta = kStepSafety / lp.matrix_norm;
        double omega = 1.0;
        if (lp.cost_norm > 0.0 && lp.bound_norm > 0.0)
            omega = std::min(kMaxWeight, std::max(kMinWeight, lp.cost_norm / lp.bound_norm));
        if (lp.omega0 > 0.0) omega = lp.omega0;
        k_init_state<<<1, 1, 0, stream>>>(st, eta, omega, eta, eta);
        B200_TRY(cudaGetLastError(), "Halpern setup");
        long long iteration = 0, since_restart = 0;
        double r_restart = std::numeric_limits<double>::infinity(), r_previous = r_restart;
        int slot_full = -1, slot_tail = -1;
        while (iteration < lp.max_iterations) {
            const int period = static_cast<int>(std::min<long long>(lp.restart_period, lp.max_iterations - iteration));
            if (period <= 0) break;
            int* slot = period == lp.restart_period ? &slot_full : &slot_tail;
            k_set_omega<<<1, 1, 0, stream>>>(st, omega, 0.0);
            k_set_halpern<<<1, 1, 0, stream>>>(st, static_cast<double>(since_restart));
            if (halpern_window(period, slot)) return -1;
            B200_TRY(cudaStreamSynchronize(stream), "Halpern window");
            ++out->syncs;
            iteration += period;
            since_restart += period;
            const double* h = host;
            const Kkt kkt = to_kkt(h, lp.cost_norm, lp.bound_norm);
            out->best = kkt;
            const double dx2 = h[32], dx0 = h[33], dy2 = h[34], dy0 = h[35];
            if (!std::isfinite(kkt.primal) || !std::isfinite(dx2) || !std::isfinite(dy2)) {
                out->numeric = true;
                break;
            }
            if (kkt.primal <= lp.eps && kkt.dual <= lp.eps && kkt.gap <= lp.eps) {
                B200_TRY(cudaMemcpyAsync(x, x_cand, nb, cudaMemcpyDeviceToDevice, stream), "copy");
                B200_TRY(cudaMemcpyAsync(y, y_cand, mb, cudaMemcpyDeviceToDevice, stream), "copy");
                out->converged = true;
                break;
            }
            if (lp.deadline > 0.0 && now_s() > lp.deadline) {
                out->timed_out = true;
                break;
            }
            if (lp.cancel && lp.cancel(lp.cancel_context) != 0) {
                out->cancelled = true;
                break;
            }
            const double r = std::sqrt(omega * dx2 + dy2 / omega);
            const bool sufficient = r <= kSufficient * r_restart;
            const bool necessary = r <= kNecessary * r_restart && r > r_previous;
            const bool artificial = static_cast<double>(since_restart) >= kArtificial * static_cast<double>(iteration);
            r_previous = r;
            if (!(sufficient || necessary || artificial)) continue;
            k_halpern_restart<T><<<eg(std::max(n, m)), kThreads, 0, stream>>>(n, m, x_cand, y_cand, x, x_restart, y,
                                                                               y_restart);
            ++launches;
            since_restart = 0;
            r_restart = r;
            r_previous = std::numeric_limits<double>::infinity();
            ++out->restarts;
            if (dx0 > 1e-28 && dy0 > 1e-28) {
                const double target = std::sqrt(dy0 / dx0);
                const double updated = std::exp(kSmoothing * std::log(target) + (1.0 - kSmoothing) * std::log(omega));
                if (std::isfinite(updated)) omega = std::min(kMaxWeight, std::max(kMinWeight, updated));
            }
        }
        out->iterations += iteration;
        out->omega = omega;
        out->eta = eta;
        return 0;
    }

    // Starting point already in x, y (T). Sets up A x, the restart reference
    // and the step state, then runs restarted windows (GpuPdlp.cpp:252-534).
    int run(const LoopParams& lp, LoopStats* out) {
        if (lp.halpern) return run_halpern(lp, out);
        const size_t nb = sizeof(T) * static_cast<size_t>(std::max(n, 1));
        const size_t mb = sizeof(T) * static_cast<size_t>(std::max(m, 1));
        if (ctr) {
            // the start point is the center (its products and frame); deviations zero
            if (!lp.adaptive) return fail_msg("the centered FP32 loop needs the adaptive step");
            build_frame();
            B200_TRY(cudaMemsetAsync(x, 0, nb, stream), "zero");
            B200_TRY(cudaMemsetAsync(y, 0, mb, stream), "zero");
        }
        for (T* v : {x_sum, x_cand, x_avg, aty}) cudaMemsetAsync(v, 0, nb, stream);
        for (T* v : {y_sum, y_cand, y_avg, ax_cand, ax_avg}) cudaMemsetAsync(v, 0, mb, stream);
        B200_TRY(cudaMemcpyAsync(x_restart, x, nb, cudaMemcpyDeviceToDevice, stream), "copy");
        B200_TRY(cudaMemcpyAsync(x_bar, x, nb, cudaMemcpyDeviceToDevice, stream), "copy");
        B200_TRY(cudaMemcpyAsync(y_restart, y, mb, cudaMemcpyDeviceToDevice, stream), "copy");
        if (m) launch_tiled(A, x, StoreEpiT<T>{ax}, stream, tiled_grid<StoreEpiT<T>, T>(A));
        if (qmode == kQGeneral) launch_tiled(Q, x, StoreEpiT<T>{qx}, stream, grid_qs);
        B200_TRY(cudaMemcpyAsync(ax_prev, ax, mb, cudaMemcpyDeviceToDevice, stream), "copy");
        const double eta_global = kStepSafety / lp.matrix_norm;
        const double eta_min = lp.eta_min_factor / lp.matrix_norm, eta_max = lp.eta_max_factor / lp.matrix_norm;
        double omega = 1.0;
        if (lp.cost_norm > 0.0 && lp.bound_norm > 0.0)
            omega = std::min(kMaxWeight, std::max(kMinWeight, lp.cost_norm / lp.bound_norm));
        if (lp.omega0 > 0.0) omega = lp.omega0;
        const double eta_start = lp.eta0 > 0.0 ? std::min(std::max(lp.eta0, eta_min), eta_max) : eta_global;
        k_init_state<<<1, 1, 0, stream>>>(st, eta_start, omega, eta_min, eta_max);
        B200_TRY(cudaGetLastError(), "PDLP setup");

        long long iteration = 0;
        int windows_since_restart = 0;
        long long iterations_since_restart = 0;
        double mu_at_restart = std::numeric_limits<double>::infinity(), mu_previous = mu_at_restart;
        int slot_full = -1, slot_tail = -1;
        double omega_full = -1.0, omega_tail = -1.0;
        while (iteration < lp.max_iterations) {
            const int period = static_cast<int>(std::min<long long>(lp.restart_period, lp.max_iterations - iteration));
            if (period <= 0) break;
            const double terms_fixed = static_cast<double>((windows_since_restart + 1) * lp.restart_period);
            k_set_omega<<<1, 1, 0, stream>>>(st, omega, terms_fixed);
            const double tau = eta_global / omega, sigma = eta_global * omega;
            const bool full = period == lp.restart_period;
            int* slot = full ? &slot_full : &slot_tail;
            double* baked = full ? &omega_full : &omega_tail;
            if (!lp.adaptive && *slot >= 0 && omega != *baked) {
                // the fixed path bakes tau/sigma into the graph: rebuild it when omega moved
                cudaGraphExecDestroy(graphs[static_cast<size_t>(*slot)]);
                graphs[static_cast<size_t>(*slot)] = nullptr;
            }
            *baked = omega;
            if (window(period, lp.adaptive, tau, sigma, slot)) return -1;
            B200_TRY(cudaStreamSynchronize(stream), "PDLP window");
            ++out->syncs;
            iteration += period;
            iterations_since_restart += period;
            ++windows_since_restart;
            const double* h = host;
            const Kkt current = to_kkt(h, lp.cost_norm, lp.bound_norm);
            const Kkt average = to_kkt(h + 16, lp.cost_norm, lp.bound_norm);
            out->eta = h[16 + 8];
            out->accept_count = h[16 + 9];
            out->updates = h[16 + 10];
            const bool average_better = lp.measure == kAllMeasures ? average.worst() < current.worst()
                                                                   : average.on(lp.measure) < current.on(lp.measure);
            out->best = average_better ? average : current;
            const Kkt best = out->best;
            if (!std::isfinite(current.primal) && !std::isfinite(average.primal)) {
                out->numeric = true;
                break;
            }
            if (lp.measure == kAllMeasures ? best.primal <= lp.eps && best.dual <= lp.eps && best.gap <= lp.eps
                                           : best.on(lp.measure) <= lp.eps) {
                if (average_better) {
                    B200_TRY(cudaMemcpyAsync(x, x_avg, nb, cudaMemcpyDeviceToDevice, stream), "copy");
                    B200_TRY(cudaMemcpyAsync(y, y_avg, mb, cudaMemcpyDeviceToDevice, stream), "copy");
                }
                out->converged = true;
                if (ctr) recenter(x, y, false);
                break;
            }
            if (lp.deadline > 0.0 && now_s() > lp.deadline) {
                out->timed_out = true;
                if (ctr) recenter(x, y, false);
                break;
            }
            if (lp.cancel && lp.cancel(lp.cancel_context) != 0) {
                out->cancelled = true;
                if (ctr) recenter(x, y, false);
                break;
            }
            const double mu = best.worst();
            const bool sufficient = mu <= kSufficient * mu_at_restart;
            const bool necessary = mu <= kNecessary * mu_at_restart && mu > mu_previous;
            const bool artificial =
                static_cast<double>(iterations_since_restart) >= kArtificial * static_cast<double>(iteration);
            mu_previous = mu;
            if (!(sufficient || necessary || artificial)) continue;
            if (ctr) {
                // restart = refinement: the center moves to the restart point, the FP32
                // problem is re-formed around it in FP64, the deviations restart at zero
                recenter(average_better ? x_avg : x, average_better ? y_avg : y, true);
            } else {
                k_restart<T><<<eg(std::max(n, m)), kThreads, 0, stream>>>(
                    n, m, average_better ? 1 : 0, lp.adaptive ? 1 : 0, x, y, x_bar, x_avg, y_avg, ax, ax_prev,
                    ax_avg, x_sum, y_sum, x_restart, y_restart, qmode == kQGeneral ? qx : nullptr, qx_avg, st);
                ++launches;
            }
            windows_since_restart = 0;
            iterations_since_restart = 0;
            mu_at_restart = mu;
            mu_previous = std::numeric_limits<double>::infinity();
            ++out->restarts;
            if (!lp.fixed_weight && best.pmove > 1e-14 && best.dmove > 1e-14) {
                const double target = best.dmove / best.pmove;
                const double updated = std::exp(kSmoothing * std::log(target) + (1.0 - kSmoothing) * std::log(omega));
                if (std::isfinite(updated)) omega = std::min(kMaxWeight, std::max(kMinWeight, updated));
            }
        }
        if (ctr && !out->converged && !out->timed_out && !out->cancelled && !out->numeric)
            recenter(x, y, false);  // iteration limit: the center takes the last point
        out->iterations += iteration;
        out->omega = omega;
        return 0;
    }
};

struct HostSlot {
    double* p = nullptr;
    ~HostSlot() { if (p) cudaFreeHost(p); }
};

}  // namespace

}  // namespace b200

using namespace b200;

extern "C" void sankhya_b200_pdlp_default_settings(SankhyaB200PdlpSettings* s) {
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->struct_version = 4;
    s->max_iterations = 500000;
    s->restart_period = 64;
    s->power_iterations = 30;
    s->adaptive_step = 1;
    s->scaling = SANKHYA_B200_SCALE_RUIZ | SANKHYA_B200_SCALE_POCK_CHAMBOLLE;
    s->ruiz_iterations = 100;
    s->precision = SANKHYA_B200_FP64;
    s->eps_optimal = 1e-8;
    s->time_limit = 0.0;
    s->eta_min_factor = 1e-6;
    s->eta_max_factor = 1e4;
    s->ruiz_tolerance = 1e-2;
}

namespace b200 {
namespace {

__global__ void k_scale_diag(int n, const double* __restrict__ q, const double* __restrict__ Cs,
                             double* __restrict__ out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x)
        out[j] = (q[j] * Cs[j]) * Cs[j];
}

// Feasibility polishing around the FP64 main loop (sankhya_b200_pdlp_solve_polished).
// hi holds the start point on entry and the answer on return (scaled space); lp is the
// main loop's parameters with the scaled problem's norms; stats receives the loop
// counters of every solve and the answer's relative KKT on the original problem.
int run_polished(const Scaled& sc, Core<double>& hi, const LoopParams& lp, const SankhyaB200PdlpSettings& s,
                 const SankhyaB200PolishSettings& ps, double* host, LoopStats* stats, SankhyaB200PolishResult* pr,
                 int* launches) {
    cudaStream_t stream = hi.stream;
    const int n = hi.n, m = hi.m;
    const size_t nb = sizeof(double) * static_cast<size_t>(std::max(n, 1));
    const size_t mb = sizeof(double) * static_cast<size_t>(std::max(m, 1));
    const size_t nd = (nb + 255) / 256 * 256, md = (mb + 255) / 256 * 256;
    DevBuf buf;
    if (buf.alloc(5 * nd + 4 * md, "cudaMalloc polishing data")) return -1;
    char* base = buf.as<char>();
    double* zero_c = reinterpret_cast<double*>(base);
    double* cl0 = reinterpret_cast<double*>(base + nd);
    double* cu0 = reinterpret_cast<double*>(base + 2 * nd);
    double* xp = reinterpret_cast<double*>(base + 3 * nd);   // the pair being scored
    double* xb = reinterpret_cast<double*>(base + 4 * nd);   // the best pair so far
    double* rl0 = reinterpret_cast<double*>(base + 5 * nd);
    double* ru0 = reinterpret_cast<double*>(base + 5 * nd + md);
    double* yd = reinterpret_cast<double*>(base + 5 * nd + 2 * md);
    double* yb = reinterpret_cast<double*>(base + 5 * nd + 3 * md);
    B200_TRY(cudaMemsetAsync(zero_c, 0, nb, stream), "zero");
    k_homogeneous<<<eg(n), kThreads, 0, stream>>>(n, sc.cl, sc.cu, cl0, cu0);
    k_homogeneous<<<eg(m), kThreads, 0, stream>>>(m, sc.rl, sc.ru, rl0, ru0);
    *launches += 2;
    Core<double> pol;
    pol.stream = stream;
    pol.host = host;
    if (pol.allocate(n, m, sc.sms)) return -1;
    const auto d2d = cudaMemcpyDeviceToDevice;

    // how far a point misses the targets (<= 1: met)
    const auto miss = [&](const Kkt& k) {
        return std::max(std::max(k.primal, k.dual) / ps.polish_tolerance, k.gap / s.eps_optimal);
    };
    LoopStats& acc = *stats;
    double tol = std::max(ps.start_tolerance, s.eps_optimal);
    long long main_used = 0;
    bool have_pair = false, met = false;
    Kkt best_pair;
    for (;;) {
        // the main loop, resumed from its own last point with its step and weight
        const double t_main = now_s();
        LoopParams ml = lp;
        ml.eps = tol;
        ml.max_iterations = s.max_iterations - main_used;
        if (main_used > 0) {
            ml.omega0 = acc.omega;
            ml.eta0 = acc.eta;
        }
        LoopStats ms;
        if (hi.run(ml, &ms)) return -1;
        pr->main_seconds += now_s() - t_main;
        main_used += ms.iterations;
        pr->main_iterations = static_cast<int>(std::min<long long>(main_used, 2147483647LL));
        acc.iterations += ms.iterations;
        acc.restarts += ms.restarts;
        acc.syncs += ms.syncs;
        acc.updates += ms.updates;
        acc.accept_count += ms.accept_count;
        acc.eta = ms.eta;
        acc.omega = ms.omega;
        acc.best = ms.best;
        acc.numeric = ms.numeric;
        acc.timed_out = ms.timed_out;
        acc.cancelled = ms.cancelled;
        if (ms.numeric || ms.timed_out || ms.cancelled) break;
        ++pr->rounds;
        pr->main_relative_primal_residual = ms.best.primal;
        pr->main_relative_dual_residual = ms.best.dual;
        pr->main_relative_gap = ms.best.gap;

        const double t_pol = now_s();
        const long long budget = ps.max_polish_iterations > 0
                                     ? ps.max_polish_iterations
                                     : std::max<long long>(main_used, lp.restart_period);
        // Both polishing solves run restarted PDHG with the safe constant step 0.9 / ||A||_2
        // and the main loop's primal weight held: such PDHG started at z0 stays within the
        // weighted distance from z0 to the solution set, so the polished point stays near
        // the main loop's (and near its objective). The adaptive step loses that bound on
        // a zero-cost problem, where its interaction term starts near zero and lets the
        // step grow to its cap.
        LoopParams pl = lp;
        pl.eps = ps.polish_tolerance;
        pl.max_iterations = budget;
        pl.omega0 = ms.omega;
        pl.adaptive = false;
        pl.fixed_weight = true;
        // primal feasibility problem (zero cost) from the main loop's x, dual at zero
        B200_TRY(cudaMemcpyAsync(xp, hi.x, nb, d2d, stream), "copy");
        if (!(ms.best.primal <= ps.polish_tolerance)) {
            pol.set_problem(sc.A, sc.AT, zero_c, sc.cl, sc.cu, sc.rl, sc.ru);
            B200_TRY(cudaMemcpyAsync(pol.x, hi.x, nb, d2d, stream), "copy");
            B200_TRY(cudaMemsetAsync(pol.y, 0, mb, stream), "zero");
            pl.cost_norm = 0.0;
            pl.bound_norm = lp.bound_norm;
            pl.measure = kPrimalMeasure;
            LoopStats fs;
            if (pol.run(pl, &fs)) return -1;
            pr->primal_iterations += static_cast<int>(fs.iterations);
            acc.iterations += fs.iterations;
            acc.syncs += fs.syncs;
            acc.timed_out = acc.timed_out || fs.timed_out;
            acc.cancelled = acc.cancelled || fs.cancelled;
            if (fs.numeric) {
                acc.numeric = true;
                break;
            }
            B200_TRY(cudaMemcpyAsync(xp, pol.x, nb, d2d, stream), "copy");
        }
        // dual feasibility problem (finite bounds at zero) from the main loop's y, primal at zero
        B200_TRY(cudaMemcpyAsync(yd, hi.y, mb, d2d, stream), "copy");
        if (!(ms.best.dual <= ps.polish_tolerance) && !acc.timed_out && !acc.cancelled) {
            pol.set_problem(sc.A, sc.AT, sc.c, cl0, cu0, rl0, ru0);
            B200_TRY(cudaMemsetAsync(pol.x, 0, nb, stream), "zero");
            B200_TRY(cudaMemcpyAsync(pol.y, hi.y, mb, d2d, stream), "copy");
            pl.cost_norm = lp.cost_norm;
            pl.bound_norm = 0.0;
            pl.measure = kDualMeasure;
            LoopStats fs;
            if (pol.run(pl, &fs)) return -1;
            pr->dual_iterations += static_cast<int>(fs.iterations);
            acc.iterations += fs.iterations;
            acc.syncs += fs.syncs;
            acc.timed_out = acc.timed_out || fs.timed_out;
            acc.cancelled = acc.cancelled || fs.cancelled;
            if (fs.numeric) {
                acc.numeric = true;
                break;
            }
            B200_TRY(cudaMemcpyAsync(yd, pol.y, mb, d2d, stream), "copy");
        }
        pr->polish_seconds += now_s() - t_pol;
        // the pair, scored on the original problem
        pol.set_problem(sc.A, sc.AT, sc.c, sc.cl, sc.cu, sc.rl, sc.ru);
        B200_TRY(cudaMemcpyAsync(pol.x, xp, nb, d2d, stream), "copy");
        B200_TRY(cudaMemcpyAsync(pol.x_restart, xp, nb, d2d, stream), "copy");
        B200_TRY(cudaMemcpyAsync(pol.y, yd, mb, d2d, stream), "copy");
        B200_TRY(cudaMemcpyAsync(pol.y_restart, yd, mb, d2d, stream), "copy");
        k_init_state<<<1, 1, 0, stream>>>(pol.st, ms.eta, ms.omega, ms.eta, ms.eta);
        ++pol.launches;
        pol.residuals(pol.x, pol.y, nullptr, nullptr, pol.res, 0);
        B200_TRY(cudaMemcpyAsync(host, pol.res, 16 * sizeof(double), cudaMemcpyDeviceToHost, stream), "copy");
        B200_TRY(cudaStreamSynchronize(stream), "polishing");
        ++acc.syncs;
        const Kkt pair = to_kkt(host, lp.cost_norm, lp.bound_norm);
        pr->pair_relative_primal_residual = pair.primal;
        pr->pair_relative_dual_residual = pair.dual;
        pr->pair_relative_gap = pair.gap;
        pr->pair_primal_objective = pair.pobj;
        if (!have_pair || miss(pair) < miss(best_pair)) {
            B200_TRY(cudaMemcpyAsync(xb, xp, nb, d2d, stream), "copy");
            B200_TRY(cudaMemcpyAsync(yb, yd, mb, d2d, stream), "copy");
            best_pair = pair;
            have_pair = true;
        }
        met = pair.primal <= ps.polish_tolerance && pair.dual <= ps.polish_tolerance && pair.gap <= s.eps_optimal;
        if (met) break;
        // not yet: the main loop resumes to a tighter tolerance (at the floor its own
        // point meets both polishing measures and the gap, and the pair is that point)
        if (acc.timed_out || acc.cancelled || !ms.converged || main_used >= s.max_iterations) break;
        tol = std::max(tol * 0.1, std::min(s.eps_optimal, ps.polish_tolerance));
    }
    *launches += pol.launches;
    acc.converged = met;
    // the answer: the pair that met the targets, else the closer of the best pair and
    // the main loop's last point (hi.x / hi.y, scored acc.best)
    if (have_pair && (met || acc.numeric || miss(best_pair) < miss(acc.best))) {
        B200_TRY(cudaMemcpyAsync(hi.x, xb, nb, d2d, stream), "copy");
        B200_TRY(cudaMemcpyAsync(hi.y, yb, mb, d2d, stream), "copy");
        acc.best = best_pair;
        acc.numeric = false;
    }
    B200_TRY(cudaStreamSynchronize(stream), "polishing");
    return 0;
}

// The LP and QP solve: minimize c'x (+ x'Q x / 2) over rl <= A x <= ru, cl <= x <= cu,
// with Q a general symmetric Hessian (hessian, full CSR) or a diagonal (qdiag).
int pdlp_solve(const SankhyaCudaCSR* matrix, const SankhyaCudaCSR* hessian, const double* qdiag, const double* c,
               const double* row_lower, const double* row_upper, const double* col_lower, const double* col_upper,
               const SankhyaB200PdlpSettings* settings, const double* x0, const double* y0, double* x_out,
               double* y_out, SankhyaB200PdlpResult* result, bool polishing = false,
               const SankhyaB200PolishSettings* polish = nullptr, SankhyaB200PolishResult* polish_result = nullptr) {
    clear_error();
    (void)cudaGetLastError();  // a caller's earlier non-sticky error is not ours
    SankhyaB200PolishResult local_pr;
    if (!polish_result) polish_result = &local_pr;
    std::memset(polish_result, 0, sizeof(*polish_result));
    if (!result) return fail_msg("null result");
    std::memset(result, 0, sizeof(*result));
    result->status = -1;
    SankhyaB200PdlpSettings s;
    sankhya_b200_pdlp_default_settings(&s);
    if (settings) {
        if (settings->struct_version == 1) {
            std::memcpy(&s, settings, offsetof(SankhyaB200PdlpSettings, algorithm));
        } else if (settings->struct_version == 2) {
            std::memcpy(&s, settings, offsetof(SankhyaB200PdlpSettings, initial_primal_weight));
        } else if (settings->struct_version == 3) {
            std::memcpy(&s, settings, offsetof(SankhyaB200PdlpSettings, cancel));
        } else if (settings->struct_version == 4) {
            s = *settings;
        } else {
            return fail_msg("unsupported settings struct_version");
        }
    }
    s.struct_version = 4;
    if (s.algorithm != SANKHYA_B200_PDLP_ADAPTIVE && s.algorithm != SANKHYA_B200_PDLP_HALPERN)
        return fail_msg("invalid PDLP settings");
    if (!(s.initial_primal_weight >= 0.0) || !std::isfinite(s.initial_primal_weight))
        return fail_msg("invalid PDLP settings");
    if (!matrix || !c || !row_lower || !row_upper || !col_lower || !col_upper || !x_out)
        return fail_msg("null model or output pointer");
    if (s.max_iterations <= 0 || s.restart_period <= 0 || s.power_iterations < 0 || !(s.eps_optimal > 0.0) ||
        s.time_limit < 0.0 || !(s.eta_min_factor > 0.0) || !(s.eta_max_factor >= s.eta_min_factor) ||
        s.ruiz_iterations < 0 ||
        (s.precision != SANKHYA_B200_FP64 && s.precision != SANKHYA_B200_FP32_REFINE &&
         s.precision != SANKHYA_B200_BF16_REFINE))
        return fail_msg("invalid PDLP settings");
    const int n = matrix->cols, m = matrix->rows;
    const bool quadratic = hessian != nullptr || qdiag != nullptr;
    if (hessian && qdiag) return fail_msg("give either a Hessian or its diagonal, not both");
    if (hessian && (hessian->rows != n || hessian->cols != n)) return fail_msg("the Hessian must be cols x cols");
    if (qdiag)
        for (int j = 0; j < n; ++j)
            if (!std::isfinite(qdiag[j]) || qdiag[j] < 0.0) return fail_msg("invalid quadratic diagonal");
    if (quadratic && (s.algorithm != SANKHYA_B200_PDLP_ADAPTIVE || !s.adaptive_step))
        return fail_msg("the QP solve runs the adaptive step of the restarted loop");
    if (s.precision == SANKHYA_B200_BF16_REFINE && (s.algorithm != SANKHYA_B200_PDLP_ADAPTIVE || !s.adaptive_step))
        return fail_msg("BF16_REFINE runs the adaptive step of the restarted loop");
    SankhyaB200PolishSettings ps;
    sankhya_b200_polish_default_settings(&ps);
    if (polishing) {
        if (polish) {
            if (polish->struct_version != 1) return fail_msg("unsupported polishing settings struct_version");
            ps = *polish;
        }
        if (!(ps.start_tolerance > 0.0) || !(ps.polish_tolerance > 0.0) || ps.max_polish_iterations < 0)
            return fail_msg("invalid polishing settings");
        if (quadratic || s.precision != SANKHYA_B200_FP64 || s.algorithm != SANKHYA_B200_PDLP_ADAPTIVE ||
            !s.adaptive_step)
            return fail_msg("polishing runs the FP64 adaptive loop of an LP");
    }
    for (int j = 0; j < n; ++j)
        if (!std::isfinite(c[j]) || std::isnan(col_lower[j]) || std::isnan(col_upper[j]) || col_lower[j] > col_upper[j])
            return fail_msg("invalid cost or column bound");
    for (int i = 0; i < m; ++i)
        if (std::isnan(row_lower[i]) || std::isnan(row_upper[i]) || row_lower[i] > row_upper[i])
            return fail_msg("invalid row bound");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) return fail_msg("no CUDA device available");
    const double t_start = now_s();
    std::shared_ptr<Plan> plan;
    if (get_plan(matrix, &plan)) return -1;
    HostSlot hs;
    B200_TRY(cudaMallocHost(reinterpret_cast<void**>(&hs.p), 64 * sizeof(double)), "cudaMallocHost");
    cudaStream_t stream = engine_stream();
    Scaled sc;
    sc.stream = stream;
    sc.host = hs.p;
    if (sc.allocate(*plan)) return -1;
    const size_t nb = sizeof(double) * static_cast<size_t>(n), mb = sizeof(double) * static_cast<size_t>(m);
    if (n) {
        B200_TRY(cudaMemcpyAsync(sc.c, c, nb, cudaMemcpyHostToDevice, stream), "upload c");
        B200_TRY(cudaMemcpyAsync(sc.cl, col_lower, nb, cudaMemcpyHostToDevice, stream), "upload col_lower");
        B200_TRY(cudaMemcpyAsync(sc.cu, col_upper, nb, cudaMemcpyHostToDevice, stream), "upload col_upper");
    }
    if (m) {
        B200_TRY(cudaMemcpyAsync(sc.rl, row_lower, mb, cudaMemcpyHostToDevice, stream), "upload row_lower");
        B200_TRY(cudaMemcpyAsync(sc.ru, row_upper, mb, cudaMemcpyHostToDevice, stream), "upload row_upper");
    }
    int syncs = 0;
    if (sc.scale(*plan, s.scaling, s.ruiz_iterations, s.ruiz_tolerance, &syncs)) return -1;
    // norms of the scaled data (GpuPdlp.cpp:94-99), finite entries only
    const double cost_norm = std::sqrt(sc.sumsq(sc.c, n, true));
    const double bound_norm = std::sqrt(sc.sumsq(sc.rl, m, true) + sc.sumsq(sc.ru, m, true));
    syncs += 3;
    const double matrix_norm = sc.power_norm(s.power_iterations);
    ++syncs;

    TimingState& ts = timing();
    ts.last = SankhyaB200Timing{};
    LoopStats stats;
    LoopParams lp;
    lp.restart_period = s.restart_period;
    lp.adaptive = s.adaptive_step != 0;
    lp.halpern = s.algorithm == SANKHYA_B200_PDLP_HALPERN;
    if (s.initial_primal_weight > 0.0) lp.omega0 = std::min(kMaxWeight, std::max(kMinWeight, s.initial_primal_weight));
    lp.deadline = s.time_limit > 0.0 ? t_start + s.time_limit : 0.0;
    lp.cancel = s.cancel;
    lp.cancel_context = s.cancel_context;
    lp.matrix_norm = matrix_norm;
    lp.eta_min_factor = s.eta_min_factor;
    lp.eta_max_factor = s.eta_max_factor;
    int refinements = 0;
    int launches = sc.launches;

    // QP: the Hessian in the scaled space, Q' = C Q C (a diagonal q' = C^2 q); for a
    // general Q also its diagonal majorant d_j = sum_k |Q'_jk|
    std::shared_ptr<Plan> qplan;
    DevBuf qbuf;
    TileCsr Qs;
    double* qd_s = nullptr;
    if (hessian) {
        if (get_plan(hessian, &qplan)) return -1;
        const size_t qv = (static_cast<size_t>(qplan->a.nnz) * 8 + 255) / 256 * 256;
        if (qbuf.alloc(qv + static_cast<size_t>(n) * 8 + 256, "cudaMalloc scaled Hessian")) return -1;
        Qs = qplan->a;
        Qs.val = qbuf.as<double>();
        qd_s = reinterpret_cast<double*>(qbuf.as<char>() + qv);
        const int wg = std::min((n + 7) / 8 + 1, sc.sms * 16);
        k_scale_values<<<wg, kThreads, 0, stream>>>(n, qplan->a.ptr, qplan->a.idx, qplan->a.val, sc.Cs, sc.Cs, 0,
                                                    qbuf.as<double>());
        k_abs_row_sums<<<wg, kThreads, 0, stream>>>(n, qplan->a.ptr, Qs.val, qd_s);
        launches += 2;
    } else if (qdiag) {
        if (qbuf.alloc(static_cast<size_t>(n) * 8 + 256, "cudaMalloc scaled Hessian diagonal")) return -1;
        qd_s = qbuf.as<double>();
        if (n) B200_TRY(cudaMemcpyAsync(qd_s, qdiag, nb, cudaMemcpyHostToDevice, stream), "upload diagonal");
        k_scale_diag<<<eg(n), kThreads, 0, stream>>>(n, qd_s, sc.Cs, qd_s);
        ++launches;
    }

    // FP64 point of the scaled problem (x^, y^): starts at zeros or the warm start
    Core<double> hi;
    hi.stream = stream;
    hi.host = hs.p;
    if (hi.allocate(n, m, sc.sms)) return -1;
    if (hi.set_hessian(qd_s, hessian ? &Qs : nullptr)) return -1;
    hi.set_problem(sc.A, sc.AT, sc.c, sc.cl, sc.cu, sc.rl, sc.ru);
    B200_TRY(cudaMemsetAsync(hi.x, 0, std::max<size_t>(nb, 1), stream), "zero");
    B200_TRY(cudaMemsetAsync(hi.y, 0, std::max<size_t>(mb, 1), stream), "zero");
    if (x0 && n) B200_TRY(cudaMemcpyAsync(hi.x, x0, nb, cudaMemcpyHostToDevice, stream), "upload x0");
    if (y0 && m) B200_TRY(cudaMemcpyAsync(hi.y, y0, mb, cudaMemcpyHostToDevice, stream), "upload y0");
    if (x0 || y0) k_to_scaled<<<eg(std::max(n, m)), kThreads, 0, stream>>>(n, m, sc.Cs, sc.R, hi.x, hi.y);

    if (s.precision == SANKHYA_B200_FP64) {
        lp.eps = s.eps_optimal;
        lp.max_iterations = s.max_iterations;
        lp.cost_norm = cost_norm;
        lp.bound_norm = bound_norm;
        if (polishing) {
            if (run_polished(sc, hi, lp, s, ps, hs.p, &stats, polish_result, &launches)) return -1;
        } else if (hi.run(lp, &stats)) {
            return -1;
        }
        launches += hi.launches;
    } else if (lp.adaptive && !lp.halpern) {
        // ------------------------- FP32 iterations around an FP64 center, refined at restarts
        // (matrix values in FP32, or in bf16 for BF16_REFINE; the center's products and
        // every residual use the FP64 values)
        DevBuf vals32, blob32, cbuf;
        const size_t nnz = static_cast<size_t>(plan->a.nnz);
        const bool bf16 = s.precision == SANKHYA_B200_BF16_REFINE;
        const size_t vbytes = bf16 ? 2 : 4;
        if (vals32.alloc(nnz * 2 * vbytes + 1024, "cudaMalloc narrowed values")) return -1;
        float* a32 = nullptr;
        float* at32 = nullptr;
        __nv_bfloat16* a16 = nullptr;
        __nv_bfloat16* at16 = nullptr;
        if (bf16) {
            a16 = vals32.as<__nv_bfloat16>();
            at16 = a16 + (nnz + 127) / 128 * 128;
            k_narrow_bf16<<<sc.sms * 8, kThreads, 0, stream>>>(static_cast<long long>(nnz), sc.A.val, a16);
            k_narrow_bf16<<<sc.sms * 8, kThreads, 0, stream>>>(static_cast<long long>(nnz), sc.AT.val, at16);
        } else {
            a32 = vals32.as<float>();
            at32 = a32 + (nnz + 63) / 64 * 64;
            k_narrow<<<sc.sms * 8, kThreads, 0, stream>>>(static_cast<long long>(nnz), sc.A.val, a32);
            k_narrow<<<sc.sms * 8, kThreads, 0, stream>>>(static_cast<long long>(nnz), sc.AT.val, at32);
        }
        const size_t nf = (static_cast<size_t>(n) * 4 + 255) / 256 * 256;
        const size_t mf = (static_cast<size_t>(m) * 4 + 255) / 256 * 256;
        const size_t nd = (static_cast<size_t>(n) * 8 + 255) / 256 * 256;
        const size_t md = (static_cast<size_t>(m) * 8 + 255) / 256 * 256;
        if (blob32.alloc(3 * nf + 2 * mf + 256, "cudaMalloc FP32 frame")) return -1;
        if (cbuf.alloc(3 * nd + md + 256, "cudaMalloc FP64 center products")) return -1;
        char* base = blob32.as<char>();
        Centered ctr;
        ctr.A = sc.A;
        ctr.AT = sc.AT;
        ctr.c = sc.c; ctr.cl = sc.cl; ctr.cu = sc.cu; ctr.rl = sc.rl; ctr.ru = sc.ru;
        ctr.xc = hi.x;
        ctr.yc = hi.y;
        ctr.aty_c = cbuf.as<double>();
        ctr.rc_c = reinterpret_cast<double*>(cbuf.as<char>() + nd);
        ctr.ax_c = reinterpret_cast<double*>(cbuf.as<char>() + 2 * nd);
        ctr.c32 = reinterpret_cast<float*>(base);
        ctr.cl32 = reinterpret_cast<float*>(base + nf);
        ctr.cu32 = reinterpret_cast<float*>(base + 2 * nf);
        ctr.rl32 = reinterpret_cast<float*>(base + 3 * nf);
        ctr.ru32 = reinterpret_cast<float*>(base + 3 * nf + mf);
        ctr.grid_a = tiled_grid<StoreEpi>(sc.A);
        ctr.grid_at = tiled_grid<StoreEpi>(sc.AT);
        // QP: the FP64 Hessian for the center's gradient and residuals, FP32 copies for
        // the deviations' products
        DevBuf q32buf;
        TileCsrT<float> Q32;
        float* qd32 = nullptr;
        ctr.qdiag = qd_s;
        if (hessian) {
            ctr.Q = Qs;
            ctr.qdiag = nullptr;   // the centered residuals take Q x_center, not a diagonal
            ctr.qx_c = reinterpret_cast<double*>(cbuf.as<char>() + 2 * nd + md);
            ctr.grid_q = tiled_grid<StoreEpi>(Qs);
            const size_t qnnz = static_cast<size_t>(Qs.nnz);
            const size_t qv32 = (qnnz * 4 + 255) / 256 * 256;
            if (q32buf.alloc(qv32 + static_cast<size_t>(n) * 4 + 256, "cudaMalloc FP32 Hessian")) return -1;
            k_narrow<<<sc.sms * 8, kThreads, 0, stream>>>(static_cast<long long>(qnnz), Qs.val, q32buf.as<float>());
            Q32 = Qs.with_values<float>(q32buf.as<float>());
            qd32 = reinterpret_cast<float*>(q32buf.as<char>() + qv32);
            k_narrow<<<eg(n), kThreads, 0, stream>>>(n, qd_s, qd32);
        } else if (qdiag) {
            if (q32buf.alloc(static_cast<size_t>(n) * 4 + 256, "cudaMalloc FP32 Hessian diagonal")) return -1;
            qd32 = q32buf.as<float>();
            k_narrow<<<eg(n), kThreads, 0, stream>>>(n, qd_s, qd32);
        }
        lp.eps = s.eps_optimal;
        lp.max_iterations = s.max_iterations;
        lp.cost_norm = cost_norm;
        lp.bound_norm = bound_norm;
        auto run_lo = [&](auto& lo, const auto& av, const auto& atv) -> int {
            lo.stream = stream;
            lo.host = hs.p;
            if (lo.allocate(n, m, sc.sms)) return -1;
            if (lo.set_hessian(qd32, hessian ? &Q32 : nullptr)) return -1;
            lo.set_problem(av, atv, ctr.c32, ctr.cl32, ctr.cu32, ctr.rl32, ctr.ru32);
            lo.ctr = &ctr;
            if (lo.run(lp, &stats)) return -1;
            refinements = lo.recenters;
            launches += hi.launches + lo.launches;
            return 0;
        };
        if (bf16) {
            Core<float, __nv_bfloat16> lo;
            if (run_lo(lo, sc.A.with_values<__nv_bfloat16>(a16), sc.AT.with_values<__nv_bfloat16>(at16))) return -1;
        } else {
            Core<float> lo;
            if (run_lo(lo, sc.A.with_values<float>(a32), sc.AT.with_values<float>(at32))) return -1;
        }
    } else {
        // ------------- Halpern or fixed-step loop: FP32 iterations, then an FP64 finish
        DevBuf vals32, blob32;
        const size_t nnz = static_cast<size_t>(plan->a.nnz);
        if (vals32.alloc(nnz * 8 + 1024, "cudaMalloc FP32 values")) return -1;
        float* a32 = vals32.as<float>();
        float* at32 = a32 + (nnz + 63) / 64 * 64;
        k_narrow<<<sc.sms * 8, kThreads, 0, stream>>>(static_cast<long long>(nnz), sc.A.val, a32);
        k_narrow<<<sc.sms * 8, kThreads, 0, stream>>>(static_cast<long long>(nnz), sc.AT.val, at32);
        const size_t nf = (static_cast<size_t>(n) * 4 + 255) / 256 * 256;
        const size_t mf = (static_cast<size_t>(m) * 4 + 255) / 256 * 256;
        if (blob32.alloc(3 * nf + 2 * mf + 256, "cudaMalloc FP32 model")) return -1;
        char* base = blob32.as<char>();
        float* c32 = reinterpret_cast<float*>(base);
        float* cl32 = reinterpret_cast<float*>(base + nf);
        float* cu32 = reinterpret_cast<float*>(base + 2 * nf);
        float* rl32 = reinterpret_cast<float*>(base + 3 * nf);
        float* ru32 = reinterpret_cast<float*>(base + 3 * nf + mf);
        const int gv = eg(std::max(n, m));
        k_narrow<<<gv, kThreads, 0, stream>>>(n, sc.c, c32);
        k_narrow<<<gv, kThreads, 0, stream>>>(n, sc.cl, cl32);
        k_narrow<<<gv, kThreads, 0, stream>>>(n, sc.cu, cu32);
        k_narrow<<<gv, kThreads, 0, stream>>>(m, sc.rl, rl32);
        k_narrow<<<gv, kThreads, 0, stream>>>(m, sc.ru, ru32);
        Core<float> lo;
        lo.stream = stream;
        lo.host = hs.p;
        if (lo.allocate(n, m, sc.sms)) return -1;
        lo.set_problem(sc.A.with_values<float>(a32), sc.AT.with_values<float>(at32), c32, cl32, cu32, rl32, ru32);
        k_narrow<<<gv, kThreads, 0, stream>>>(n, hi.x, lo.x);
        k_narrow<<<gv, kThreads, 0, stream>>>(m, hi.y, lo.y);
        LoopParams flp = lp;
        flp.eps = std::max(s.eps_optimal, 1e-4);
        flp.max_iterations = s.max_iterations;
        flp.cost_norm = cost_norm;
        flp.bound_norm = bound_norm;
        LoopStats fs;
        if (lo.run(flp, &fs)) return -1;
        stats = fs;
        k_widen<<<gv, kThreads, 0, stream>>>(n, m, lo.x, lo.y, sc.cl, sc.cu, hi.x, hi.y);
        const long long left = s.max_iterations - fs.iterations;
        if (!fs.numeric && !fs.timed_out && !fs.cancelled && left > 0 && (!fs.converged || s.eps_optimal < flp.eps)) {
            lp.eps = s.eps_optimal;
            lp.max_iterations = left;
            lp.cost_norm = cost_norm;
            lp.bound_norm = bound_norm;
            lp.omega0 = fs.omega;
            lp.eta0 = fs.eta;
            LoopStats fin;
            if (hi.run(lp, &fin)) return -1;
            ++refinements;
            stats.iterations += fin.iterations;
            stats.restarts += fin.restarts;
            stats.updates += fin.updates;
            stats.accept_count += fin.accept_count;
            stats.syncs += fin.syncs;
            stats.eta = fin.eta;
            stats.omega = fin.omega;
            stats.best = fin.best;
            stats.converged = fin.converged;
            stats.timed_out = fin.timed_out;
            stats.numeric = fin.numeric;
            stats.cancelled = fin.cancelled;
        }
        launches += hi.launches + lo.launches;
    }

    // back to the caller's space
    k_unscale<<<eg(std::max(n, m)), kThreads, 0, stream>>>(n, m, sc.Cs, sc.R, hi.x, hi.y);
    if (n) B200_TRY(cudaMemcpyAsync(x_out, hi.x, nb, cudaMemcpyDeviceToHost, stream), "download x");
    if (y_out && m) B200_TRY(cudaMemcpyAsync(y_out, hi.y, mb, cudaMemcpyDeviceToHost, stream), "download y");
    B200_TRY(cudaStreamSynchronize(stream), "download");
    ++syncs;
    syncs += stats.syncs;
    const Kkt& best = stats.best;
    result->status = stats.numeric ? -2 : stats.converged ? 0 : stats.cancelled ? 3 : stats.timed_out ? 2 : 1;
    result->iterations = static_cast<int>(std::min<long long>(stats.iterations, 2147483647LL));
    result->restarts = stats.restarts;
    result->rejected_steps = (lp.adaptive && !lp.halpern)
                                 ? static_cast<int>(std::max(0.0, stats.updates - stats.accept_count)) : 0;
    result->host_syncs = syncs;
    result->refinements = refinements;
    result->primal_objective = best.pobj;
    result->dual_objective = best.dobj;
    result->relative_primal_residual = best.primal;
    result->relative_dual_residual = best.dual;
    result->relative_gap = best.gap;
    result->matrix_norm = matrix_norm;
    result->final_step_size = (lp.adaptive && !lp.halpern) ? stats.eta : kStepSafety / matrix_norm;
    result->primal_weight = stats.omega;
    result->seconds = now_s() - t_start;
    ts.last.iterations = result->iterations;
    ts.last.checkpoints = syncs;
    ts.last.kernel_launches = launches;
    return stats.numeric ? -2 : 0;
}

}  // namespace
}  // namespace b200

extern "C" int sankhya_b200_pdlp_solve(const SankhyaCudaCSR* matrix, const double* c, const double* row_lower,
                                       const double* row_upper, const double* col_lower, const double* col_upper,
                                       const SankhyaB200PdlpSettings* settings, const double* x0, const double* y0,
                                       double* x_out, double* y_out, SankhyaB200PdlpResult* result) {
    return b200::pdlp_solve(matrix, nullptr, nullptr, c, row_lower, row_upper, col_lower, col_upper, settings, x0,
                            y0, x_out, y_out, result);
}

extern "C" int sankhya_b200_pdlp_solve_qp(const SankhyaCudaCSR* matrix, const SankhyaCudaCSR* hessian,
                                          const double* quadratic_diagonal, const double* c, const double* row_lower,
                                          const double* row_upper, const double* col_lower, const double* col_upper,
                                          const SankhyaB200PdlpSettings* settings, const double* x0, const double* y0,
                                          double* x_out, double* y_out, SankhyaB200PdlpResult* result) {
    return b200::pdlp_solve(matrix, hessian, quadratic_diagonal, c, row_lower, row_upper, col_lower, col_upper,
                            settings, x0, y0, x_out, y_out, result);
}

extern "C" void sankhya_b200_polish_default_settings(SankhyaB200PolishSettings* s) {
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->struct_version = 1;
    s->max_polish_iterations = 0;
    s->start_tolerance = 1e-4;
    s->polish_tolerance = 1e-8;
}

extern "C" int sankhya_b200_pdlp_solve_polished(const SankhyaCudaCSR* matrix, const double* c,
                                                const double* row_lower, const double* row_upper,
                                                const double* col_lower, const double* col_upper,
                                                const SankhyaB200PdlpSettings* settings,
                                                const SankhyaB200PolishSettings* polish, const double* x0,
                                                const double* y0, double* x_out, double* y_out,
                                                SankhyaB200PdlpResult* result, SankhyaB200PolishResult* polish_result) {
    return b200::pdlp_solve(matrix, nullptr, nullptr, c, row_lower, row_upper, col_lower, col_upper, settings, x0,
                            y0, x_out, y_out, result, true, polish, polish_result);
}

extern "C" int sankhya_b200_scale_factors(const SankhyaCudaCSR* matrix, int scaling, int ruiz_iterations,
                                          double ruiz_tolerance, double* row_scale, double* col_scale) {
    clear_error();
    (void)cudaGetLastError();
    if (!matrix || (matrix->rows > 0 && !row_scale) || (matrix->cols > 0 && !col_scale) || ruiz_iterations < 0 ||
        !(ruiz_tolerance > 0.0) || (scaling & ~7))
        return fail_msg("invalid scaling arguments");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) return fail_msg("no CUDA device available");
    std::shared_ptr<Plan> plan;
    if (get_plan(matrix, &plan)) return -1;
    Scaled sc;
    sc.stream = engine_stream();
    HostSlot hs;
    B200_TRY(cudaMallocHost(reinterpret_cast<void**>(&hs.p), 64 * sizeof(double)), "cudaMallocHost");
    sc.host = hs.p;
    if (sc.allocate(*plan)) return -1;
    const int n = matrix->cols, m = matrix->rows;
    const size_t nb = sizeof(double) * static_cast<size_t>(n), mb = sizeof(double) * static_cast<size_t>(m);
    B200_TRY(cudaMemsetAsync(sc.blob.p, 0, sc.blob.bytes, sc.stream), "clear workspace");
    int syncs = 0;
    if (sc.scale(*plan, scaling, ruiz_iterations, ruiz_tolerance, &syncs)) return -1;
    if (n) B200_TRY(cudaMemcpyAsync(col_scale, sc.Cs, nb, cudaMemcpyDeviceToHost, sc.stream), "download C");
    if (m) B200_TRY(cudaMemcpyAsync(row_scale, sc.R, mb, cudaMemcpyDeviceToHost, sc.stream), "download R");
    B200_TRY(cudaStreamSynchronize(sc.stream), "scaling");
    return 0;
}
