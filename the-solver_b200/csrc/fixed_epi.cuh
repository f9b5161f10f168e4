// Epilogues and small kernels of the CUDA-prototype arithmetic contract
// (cuda/src/sankhya_cuda_lp.cu), shared by the fixed-step solvers.
#pragma once

#include "engine.cuh"

namespace b200 {

// cuda/src/sankhya_cuda_lp.cu:26-34
struct DualCudaEpi {
    const double* __restrict__ y;
    const double* __restrict__ rl;
    const double* __restrict__ ru;
    const double* __restrict__ sig;  // per-row steps or null
    double sigma;
    double* __restrict__ y_new;
    using Acc = NoAcc;
    struct Row {
        double y, lo, hi, s;
    };
    __device__ __forceinline__ Row load(int i) const { return Row{y[i], rl[i], ru[i], sig ? sig[i] : sigma}; }
    __device__ __forceinline__ void store(int i, double act, const Row& r, Acc&) const {
        const double trial = dadd(r.y, dmul(r.s, act));
        y_new[i] = dsub(trial, dmul(r.s, box_ieee(ddiv(trial, r.s), r.lo, r.hi)));
    }
    __device__ __forceinline__ void finish(Acc&, double*) const {}
};

// cuda/src/sankhya_cuda_lp.cu:36-52
struct PrimalCudaEpi {
    const double* __restrict__ x;
    const double* __restrict__ c;
    const double* __restrict__ tauv;  // per-column steps or null
    const double* __restrict__ qgrad; // Q x (explicit Hessian) or null
    const double* __restrict__ qdiag; // diagonal Q or null
    const double* __restrict__ cl;
    const double* __restrict__ cu;
    double tau, theta;
    double* __restrict__ x_new;
    double* __restrict__ x_bar;
    using Acc = NoAcc;
    struct Row {
        double x, c, t, lo, hi, curvature, qg;
    };
    __device__ __forceinline__ Row load(int j) const {
        return Row{x[j], c[j], tauv ? tauv[j] : tau, cl[j], cu[j], qdiag ? qdiag[j] : 0.0, qgrad ? qgrad[j] : 0.0};
    }
    __device__ __forceinline__ void store(int j, double g, const Row& r, Acc&) const {
        const double trial = ddiv(dsub(r.x, dmul(r.t, dadd(dadd(r.c, g), r.qg))), dadd(1.0, dmul(r.t, r.curvature)));
        const double next = box_ieee(trial, r.lo, r.hi);
        x_new[j] = next;
        x_bar[j] = dadd(next, dmul(theta, dsub(next, r.x)));
    }
    __device__ __forceinline__ void finish(Acc&, double*) const {}
};

// Checkpoint, rows of A (cuda/src/sankhya_cuda_lp.cu:258-263, 290-297, 337-360).
// Slots: 0 non-finite flag, 1 row violation, 2 KKT, 3 dual residual, 4 complementarity.
struct CheckRowsCudaEpi {
    const double* __restrict__ y;
    const double* __restrict__ rl;
    const double* __restrict__ ru;
    double* __restrict__ partial;
    using Acc = Slots<5, 0u>;
    __device__ __forceinline__ void row(int i, double act, Acc& acc) const {
        const double mult = y[i], lo = rl[i], hi = ru[i];
        if (!isfinite(act) || !isfinite(mult)) acc.max(0, 1.0);
        if (isfinite(lo)) acc.max(1, lo - act);
        if (isfinite(hi)) acc.max(1, act - hi);
        acc.max(2, fabs(act - box_ieee(act + mult, lo, hi)));
        const bool at_lower = has_lower_gate(lo) && fabs(act - lo) <= 1e-9;
        const bool at_upper = has_upper_gate(hi) && fabs(act - hi) <= 1e-9;
        if (at_lower && at_upper) {
        } else if (at_lower) {
            acc.max(3, mult);
        } else if (at_upper) {
            acc.max(3, -mult);
        } else {
            acc.max(3, fabs(mult));
        }
        if (mult < 0.0 && has_lower_gate(lo)) acc.max(4, -mult * fabs(act - lo));
        else if (mult > 0.0 && has_upper_gate(hi)) acc.max(4, mult * fabs(hi - act));
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

// Checkpoint, columns (cuda/src/sankhya_cuda_lp.cu:258-260, 273-289, 298-336).
// Slots: 0 non-finite, 1 objective (sum), 2 step, 3 scale, 4 KKT, 5 dual residual,
// 6 complementarity. Also advances x_prev to x.
struct CheckColsCudaEpi {
    const double* __restrict__ x;
    double* __restrict__ x_prev;
    const double* __restrict__ c;
    const double* __restrict__ qdiag;
    const double* __restrict__ qx;
    const double* __restrict__ cl;
    const double* __restrict__ cu;
    double* __restrict__ partial;
    using Acc = Slots<7, 1u << 1>;
    __device__ __forceinline__ void row(int j, double aty, Acc& acc) const {
        const double xj = x[j], lo = cl[j], hi = cu[j], cj = c[j];
        const double qxj = qx ? qx[j] : 0.0;
        if (!isfinite(xj) || !isfinite(aty) || !isfinite(qxj)) acc.max(0, 1.0);
        double obj = cj * xj;
        if (qdiag) obj += 0.5 * qdiag[j] * xj * xj;
        else if (qx) obj += 0.5 * xj * qxj;
        acc.add(1, obj);
        acc.max(2, fabs(xj - x_prev[j]));
        x_prev[j] = xj;
        acc.max(3, fabs(xj));
        const double qg = qdiag ? qdiag[j] * xj : qxj;
        const double residual = cj + aty + qg;
        acc.max(4, fabs(xj - box_ieee(xj - residual, lo, hi)));
        const bool at_lower = has_lower_gate(lo) && fabs(xj - lo) <= 1e-9;
        const bool at_upper = has_upper_gate(hi) && fabs(xj - hi) <= 1e-9;
        if (at_lower && at_upper) {
        } else if (at_lower) {
            acc.max(5, -residual);
        } else if (at_upper) {
            acc.max(5, residual);
        } else {
            acc.max(5, fabs(residual));
        }
        if (residual > 0.0 && has_lower_gate(lo)) acc.max(6, residual * fabs(xj - lo));
        else if (residual < 0.0 && has_upper_gate(hi)) acc.max(6, -residual * fabs(hi - xj));
    }
    __device__ __forceinline__ void finish(Acc& acc, double* smem) const { block_store(acc, partial, smem); }
};

// Per-element input checks of cuda/src/sankhya_cuda_lp.cu:136-153 on the
// uploaded arrays; failure classes are or-ed into *flags (1 cost / column bound,
// 2 row bound, 4 primal step, 8 dual step, 16 quadratic diagonal).
__device__ __forceinline__ bool dev_valid_lower(double v) { return !isnan(v) && !(isinf(v) && v > 0.0); }
__device__ __forceinline__ bool dev_valid_upper(double v) { return !isnan(v) && !(isinf(v) && v < 0.0); }

static __global__ void k_validate_fixed(int n, int m, const double* __restrict__ c, const double* __restrict__ cl,
                                 const double* __restrict__ cu, const double* __restrict__ rl,
                                 const double* __restrict__ ru, const double* __restrict__ tauv,
                                 const double* __restrict__ sigv, const double* __restrict__ qd,
                                 unsigned int* __restrict__ flags) {
    unsigned int f = 0;
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        if (!isfinite(c[j]) || !dev_valid_lower(cl[j]) || !dev_valid_upper(cu[j]) || cl[j] > cu[j]) f |= 1u;
        if (tauv && (!isfinite(tauv[j]) || tauv[j] <= 0.0)) f |= 4u;
        if (qd && (!isfinite(qd[j]) || qd[j] < 0.0)) f |= 16u;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        if (!dev_valid_lower(rl[i]) || !dev_valid_upper(ru[i]) || rl[i] > ru[i]) f |= 2u;
        if (sigv && (!isfinite(sigv[i]) || sigv[i] <= 0.0)) f |= 8u;
    }
    f = __reduce_or_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && f) atomicOr(flags, f);
}

static __global__ void k_init_box_ieee(int n, const double* __restrict__ lo, const double* __restrict__ hi,
                                double* __restrict__ x, double* __restrict__ x_bar) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) {
        const double v = box_ieee(0.0, lo[j], hi[j]);
        x[j] = v;
        x_bar[j] = v;
    }
}

}  // namespace b200
