// Warm-start network for a parametric LP family: bipartite message passing over
// the constraint matrix (variable nodes = columns, constraint nodes = rows), 4
// rounds of hidden width 64, predicting a primal / dual starting point for PDLP.
// The reference has no learned component; this file defines the network, its
// forward and backward kernels and its training step.
//
//   Hv0 = relu(Fv Ev + bev), Hc0 = relu(Fc Ec + bec)                (features: 16)
//   round t: Hc = relu([Hc, D_r A Hv] Wc_t + bc_t)
//            Hv = relu([Hv, D_c A' Hc] Wv_t + bv_t)                   (D: 1 / degree)
//   x_hat = lo + (hi - lo) sigmoid(Hv wx + bx) (boxed), clamp(bs (Hv wx + bx)) otherwise
//   y_hat = ys (Hc wy + by)
//   loss  = mean ((x_hat - x*) / width)^2 + mean ((y_hat - y*) / ys)^2
//
// Dense layers run on the tensor cores with bf16 operands and fp32 accumulation
// (inputs rounded to bf16 when staged in shared memory): the layer products and
// the input gradients (K = 16, 64 or 128; N = 64 or 128) on the 5th-generation
// tensor cores, tcgen05.mma with a TMEM accumulator (tc_gemm.cuh), and so are
// the weight gradients of the 128-wide layers, which reduce over all nodes in
// fixed node slices; the 16-wide input layers' weight gradients and any operand
// that is not 16-byte aligned take an mma.sync m16n8k16 kernel. They are
// HBM-bound streams of the activations, not tensor-throughput-bound. Aggregations are fp32 gathers over the stored A
// and A' (warp per node, 64 channels, entries in stored order). Every reduction
// (weight gradients split over K, bias sums, head sums, loss) has a fixed order,
// so a training run is reproducible bit for bit.
#include "batch_common.cuh"
#include "tc_gemm.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

namespace b200 {

namespace {

using batch::atomic_max_nonneg;
using batch::k_abs_sums;
using batch::slot_value;

constexpr int kH = 64;          // hidden width
constexpr int kF = 16;          // input features per node
constexpr int kX = 2 * kH;      // row width of a layer input [H | aggregation]
constexpr int kGemmThreads = 128;
constexpr int kRedBlocks = 296; // partial sums per reduction (2 per SM)

// ----------------------------------------------------------------- GEMM

template <class TB>
struct Gemm {
    int M, N, K;                  // C[M x N] = A[M x K] B[K x N]
    const float* A;
    long long sam, sak;           // element (m, k) at A[m sam + k sak]
    const TB* B;
    long long sbk, sbn;           // element (k, n) at B[k sbk + n sbn]
    float* C;
    long long scm, scn, scz;      // element (m, n) of K-slice z at C[z scz + m scm + n scn]
    int kchunk;                   // K extent of one grid.z slice
    const float* bias;            // per output column, or null
    int relu;
};

__device__ __forceinline__ __nv_bfloat16 to_bf16(float v) { return __float2bfloat16_rn(v); }
__device__ __forceinline__ __nv_bfloat16 to_bf16(__nv_bfloat16 v) { return v; }

__device__ __forceinline__ unsigned ld_pair(const __nv_bfloat16* p) { return *reinterpret_cast<const unsigned*>(p); }

__device__ __forceinline__ void mma_bf16(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0,
                                         unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Stages a 64 x 32 tile, element (r, k) = src[(r0 + r) sr + (k0 + k) sk] (zero
// outside r0 + r < rlim, k0 + k < kend), into dst[r][k] as bf16. When k is the
// contiguous index, a warp reads 32 consecutive k of one row. Otherwise each
// thread takes two consecutive k of one row (lanes 0-7: eight consecutive rows,
// lane bits 3-4: the k pair), so the global reads fill whole sectors and the
// 4-byte shared stores of a warp fall in 32 different banks (row stride 20 words).
template <class T>
__device__ __forceinline__ void stage_tile(__nv_bfloat16 (*dst)[40], const T* src, long long sr, long long sk, int r0,
                                           int rlim, int k0, int kend) {
    if (sk == 1) {
        for (int i = threadIdx.x; i < 64 * 32; i += kGemmThreads) {
            const int r = i >> 5, k = i & 31;
            const int gr = r0 + r, gk = k0 + k;
            dst[r][k] = (gr < rlim && gk < kend) ? to_bf16(src[gr * sr + gk]) : to_bf16(0.f);
        }
    } else {
        for (int q = threadIdx.x; q < 64 * 16; q += kGemmThreads) {
            const int r = (q & 7) + 8 * ((q >> 5) & 7);
            const int k = 2 * (((q >> 3) & 3) + 4 * (q >> 8));
            const int gr = r0 + r, gk = k0 + k;
            const bool live = gr < rlim;
            __nv_bfloat162 v;
            v.x = (live && gk < kend) ? to_bf16(src[gr * sr + gk * sk]) : to_bf16(0.f);
            v.y = (live && gk + 1 < kend) ? to_bf16(src[gr * sr + (gk + 1) * sk]) : to_bf16(0.f);
            *reinterpret_cast<__nv_bfloat162*>(&dst[r][k]) = v;
        }
    }
}

// One block = a 64 x 64 tile of C (4 warps x 16 rows, 8 n8 tiles each); K in
// steps of 32 staged as bf16 in shared memory (A row-major, B transposed so both
// fragments are pairs of consecutive k).
template <class TB>
__global__ void __launch_bounds__(kGemmThreads) k_gemm_bf16(Gemm<TB> g) {
    __shared__ __align__(16) __nv_bfloat16 As[64][40];
    __shared__ __align__(16) __nv_bfloat16 Bt[64][40];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int m0 = blockIdx.x * 64, n0 = blockIdx.y * 64;
    const int kb = blockIdx.z * g.kchunk;
    const int ke = min(g.K, kb + g.kchunk);
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[j][e] = 0.f;
    const int g4 = lane >> 2, t4 = lane & 3;
    for (int k0 = kb; k0 < ke; k0 += 32) {
        stage_tile(As, g.A, g.sam, g.sak, m0, g.M, k0, ke);
        stage_tile(Bt, g.B, g.sbn, g.sbk, n0, g.N, k0, ke);
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 32; kk += 16) {
            const int r = warp * 16 + g4;
            const unsigned a0 = ld_pair(&As[r][kk + 2 * t4]), a1 = ld_pair(&As[r + 8][kk + 2 * t4]);
            const unsigned a2 = ld_pair(&As[r][kk + 2 * t4 + 8]), a3 = ld_pair(&As[r + 8][kk + 2 * t4 + 8]);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const unsigned b0 = ld_pair(&Bt[8 * j + g4][kk + 2 * t4]);
                const unsigned b1 = ld_pair(&Bt[8 * j + g4][kk + 2 * t4 + 8]);
                mma_bf16(acc[j], a0, a1, a2, a3, b0, b1);
            }
        }
        __syncthreads();
    }
    float* C = g.C + blockIdx.z * g.scz;
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int row = m0 + warp * 16 + g4 + 8 * h, col = n0 + 8 * j + 2 * t4 + e;
                if (row < g.M && col < g.N) {
                    float v = acc[j][2 * h + e];
                    if (g.bias) v += g.bias[col];
                    if (g.relu) v = fmaxf(v, 0.f);
                    C[row * g.scm + col * g.scn] = v;
                }
            }
}

// out[i] = sum over z of part[z stride + i]. A block covers 64 consecutive
// outputs with sixteen slice phases (z = q mod 16); each thread keeps eight
// accumulators (z = q + 16 u mod 128), summed by a fixed tree, and the phases are
// combined by a fixed tree: a fixed order for every output, and eight independent
// loads in flight per thread.
constexpr int kSumPhases = 16;

__global__ void __launch_bounds__(kSumPhases * kH) k_sum_slices(int count, int slices, long long stride,
                                                                const float* __restrict__ part,
                                                                float* __restrict__ out) {
    __shared__ float red[kSumPhases][kH];
    const int i = threadIdx.x & (kH - 1), q = threadIdx.x >> 6;
    const int c = blockIdx.x * kH + i;
    float a[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (c < count)
        for (int z0 = q; z0 < slices; z0 += 8 * kSumPhases)
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (z0 + kSumPhases * u < slices) a[u] += part[(z0 + kSumPhases * u) * stride + c];
    red[q][i] = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
    __syncthreads();
    if (q == 0 && c < count) {
        float r[8];
#pragma unroll
        for (int h = 0; h < 8; ++h) r[h] = red[2 * h][i] + red[2 * h + 1][i];
        out[c] = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    }
}

void sum_slices(int count, int slices, long long stride, const float* part, float* out, cudaStream_t st) {
    k_sum_slices<<<(count + kH - 1) / kH, kSumPhases * kH, 0, st>>>(count, slices, stride, part, out);
}

// --------------------------------------------------------- aggregation

// out[r][c] (+)= post[r] sum_p a_p pre[col_p] in[col_p][c], c < 64: one warp per
// row, two channels per lane, entries in stored order.
__global__ void __launch_bounds__(kThreads) k_spmm64(int rows, const int* __restrict__ ptr, const int* __restrict__ idx,
                                                     const double* __restrict__ val, const float* __restrict__ in,
                                                     int sin, const float* __restrict__ pre,
                                                     const float* __restrict__ post, float* __restrict__ out, int sout,
                                                     int accumulate) {
    const int lane = threadIdx.x & 31;
    for (long long r = static_cast<long long>(blockIdx.x) * kWarps + (threadIdx.x >> 5); r < rows;
         r += static_cast<long long>(gridDim.x) * kWarps) {
        float2 acc = make_float2(0.f, 0.f);
        const int p1 = ptr[r + 1];
        for (int p = ptr[r]; p < p1; ++p) {
            const int col = idx[p];
            float a = static_cast<float>(val[p]);
            if (pre) a *= pre[col];
            const float2 v = *reinterpret_cast<const float2*>(in + static_cast<long long>(col) * sin + 2 * lane);
            acc.x += a * v.x;
            acc.y += a * v.y;
        }
        if (post) {
            acc.x *= post[r];
            acc.y *= post[r];
        }
        float2* o = reinterpret_cast<float2*>(out + r * sout + 2 * lane);
        if (accumulate) {
            const float2 prev = *o;
            acc.x += prev.x;
            acc.y += prev.y;
        }
        *o = acc;
    }
}

// dz[i][c] = dh[i][c] where h[i][c] > 0, else 0 (relu backward).
__global__ void k_relu_mask(int rows, const float* __restrict__ dh, int sdh, const float* __restrict__ h, int sh,
                            float* __restrict__ dz) {
    const long long total = static_cast<long long>(rows) * kH;
    for (long long e = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; e < total;
         e += static_cast<long long>(blockDim.x) * gridDim.x) {
        const long long i = e / kH;
        const int c = static_cast<int>(e % kH);
        dz[e] = h[i * sh + c] > 0.f ? dh[i * sdh + c] : 0.f;
    }
}

// Per-block column sums of dz [rows x 64] (block b: rows b, b + gridDim.x, ...,
// four row phases reduced in order): part[b][c].
__global__ void k_colsum64(int rows, const float* __restrict__ dz, float* __restrict__ part) {
    __shared__ float s[4][kH];
    const int c = threadIdx.x & (kH - 1), q = threadIdx.x >> 6;
    float acc = 0.f;
    for (long long i = blockIdx.x * 4LL + q; i < rows; i += 4LL * gridDim.x) acc += dz[i * kH + c];
    s[q][c] = acc;
    __syncthreads();
    if (q == 0) part[blockIdx.x * kH + c] = ((s[0][c] + s[1][c]) + s[2][c]) + s[3][c];
}

// ------------------------------------------------------------ features

struct FeatureSlots {
    unsigned long long cmax, bmax, rmax, anorm, cdeg, rdeg;
    unsigned int bany, rany;
};

__device__ __forceinline__ bool present(double v) { return fabs(v) < 1.0e30; }

// Block maxima first (shared-memory tree), then one atomic per block and slot.
__global__ void __launch_bounds__(kThreads) k_feature_maxima(int m, int n, const double* __restrict__ c,
                                                             const double* __restrict__ cl, const double* __restrict__ cu,
                                                             const double* __restrict__ rl, const double* __restrict__ ru,
                                                             const double* __restrict__ rnorm,
                                                             const double* __restrict__ cnorm,
                                                             const int* __restrict__ aptr, const int* __restrict__ tptr,
                                                             FeatureSlots* __restrict__ s) {
    __shared__ double red[6][kThreads];
    __shared__ unsigned int any[2];
    if (threadIdx.x < 2) any[threadIdx.x] = 0u;
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};   // cmax, bmax, rmax, anorm, cdeg, rdeg
    bool bany = false, rany = false;
    const int stride = blockDim.x * gridDim.x;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        v[0] = fmax(v[0], fabs(c[j]));
        if (present(cl[j])) { v[1] = fmax(v[1], fabs(cl[j])); bany = true; }
        if (present(cu[j])) { v[1] = fmax(v[1], fabs(cu[j])); bany = true; }
        v[3] = fmax(v[3], cnorm[j]);
        v[4] = fmax(v[4], static_cast<double>(tptr[j + 1] - tptr[j]));
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        if (present(rl[i])) { v[2] = fmax(v[2], fabs(rl[i])); rany = true; }
        if (present(ru[i])) { v[2] = fmax(v[2], fabs(ru[i])); rany = true; }
        v[3] = fmax(v[3], rnorm[i]);
        v[5] = fmax(v[5], static_cast<double>(aptr[i + 1] - aptr[i]));
    }
    for (int k = 0; k < 6; ++k) red[k][threadIdx.x] = v[k];
    __syncthreads();
    if (bany) any[0] = 1u;
    if (rany) any[1] = 1u;
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 6; ++k) red[k][threadIdx.x] = fmax(red[k][threadIdx.x], red[k][threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&s->cmax, red[0][0]);
        atomic_max_nonneg(&s->bmax, red[1][0]);
        atomic_max_nonneg(&s->rmax, red[2][0]);
        atomic_max_nonneg(&s->anorm, red[3][0]);
        atomic_max_nonneg(&s->cdeg, red[4][0]);
        atomic_max_nonneg(&s->rdeg, red[5][0]);
        if (any[0]) atomicOr(&s->bany, 1u);
        if (any[1]) atomicOr(&s->rany, 1u);
    }
}

__global__ void k_features(int m, int n, const double* __restrict__ c, const double* __restrict__ cl,
                           const double* __restrict__ cu, const double* __restrict__ rl, const double* __restrict__ ru,
                           const double* __restrict__ rnorm, const double* __restrict__ cnorm,
                           const int* __restrict__ aptr, const int* __restrict__ tptr,
                           const FeatureSlots* __restrict__ s, float* __restrict__ fv, float* __restrict__ fc,
                           float* __restrict__ inv_row, float* __restrict__ inv_col, double* __restrict__ bs_out) {
    const double cs = fmax(slot_value(s->cmax), 1e-300);
    const double bs = s->bany ? fmax(slot_value(s->bmax), 1e-300) : 1.0;
    const double rs = s->rany ? fmax(slot_value(s->rmax), 1e-300) : 1.0;
    const double an = fmax(slot_value(s->anorm), 1e-300);
    const double cdeg = fmax(slot_value(s->cdeg), 1.0), rdeg = fmax(slot_value(s->rdeg), 1.0);
    const int stride = blockDim.x * gridDim.x;
    if (blockIdx.x == 0 && threadIdx.x == 0) *bs_out = bs;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        float* f = fv + static_cast<long long>(j) * kF;
        const bool hl = present(cl[j]), hu = present(cu[j]);
        const double deg = static_cast<double>(tptr[j + 1] - tptr[j]);
        f[0] = static_cast<float>(c[j] / cs);
        f[1] = static_cast<float>(hl ? cl[j] / bs : 0.0);
        f[2] = static_cast<float>(hu ? cu[j] / bs : 0.0);
        f[3] = hl ? 1.f : 0.f;
        f[4] = hu ? 1.f : 0.f;
        f[5] = static_cast<float>(cnorm[j] / an);
        f[6] = static_cast<float>(deg / cdeg);
        f[7] = 1.f;
        for (int k = 8; k < kF; ++k) f[k] = 0.f;
        inv_col[j] = static_cast<float>(1.0 / fmax(deg, 1.0));
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        float* f = fc + static_cast<long long>(i) * kF;
        const bool gl = present(rl[i]), gu = present(ru[i]);
        const double deg = static_cast<double>(aptr[i + 1] - aptr[i]);
        f[0] = static_cast<float>(gl ? rl[i] / rs : 0.0);
        f[1] = static_cast<float>(gu ? ru[i] / rs : 0.0);
        f[2] = gl ? 1.f : 0.f;
        f[3] = gu ? 1.f : 0.f;
        f[4] = static_cast<float>(rnorm[i] / an);
        f[5] = static_cast<float>(deg / rdeg);
        f[6] = 1.f;
        for (int k = 7; k < kF; ++k) f[k] = 0.f;
        inv_row[i] = static_cast<float>(1.0 / fmax(deg, 1.0));
    }
}

// ---------------------------------------------------------------- heads

// Warp per node. s = h . w + b (fp32, lanes' two channels then an xor tree).
// With a target: loss term, dh = ds w into dh (row stride sdh), and per-block
// partials part[b][0..63] = sum ds h, part[b][64] = sum ds, part[b][65] = loss.
struct HeadArgs {
    int rows;
    const float* h;
    int sh;
    const float* w;         // 64 weights followed by the bias
    const double* lo;       // x head only
    const double* hi;
    const double* bs;       // x head only: scale for unboxed columns
    double ys;              // y head only
    int is_x;
    double* out;
    const double* target;
    float* dh;
    int sdh;
    float* part;
};

__global__ void __launch_bounds__(kThreads) k_head(HeadArgs a) {
    __shared__ float red[kWarps][kH + 2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float w0 = a.w[2 * lane], w1 = a.w[2 * lane + 1], wb = a.w[kH];
    float g0 = 0.f, g1 = 0.f, gb = 0.f, gl = 0.f;
    const double inv_count = 1.0 / static_cast<double>(max(a.rows, 1));
    const double bs = a.is_x ? *a.bs : 1.0;
    for (long long r = static_cast<long long>(blockIdx.x) * kWarps + warp; r < a.rows;
         r += static_cast<long long>(gridDim.x) * kWarps) {
        const float2 hv = *reinterpret_cast<const float2*>(a.h + r * a.sh + 2 * lane);
        float s = hv.x * w0 + hv.y * w1;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        const double sd = static_cast<double>(s + wb);
        double pred, ds_dpred = 1.0, width = 1.0;
        if (a.is_x) {
            const double lo = a.lo[r], hi = a.hi[r];
            const bool hl = present(lo), hu = present(hi);
            if (hl && hu) {
                const double sig = 1.0 / (1.0 + exp(-sd));
                pred = lo + (hi - lo) * sig;
                ds_dpred = (hi - lo) * sig * (1.0 - sig);
                width = fmax(hi - lo, 1e-12);
            } else {
                const double lin = bs * sd;
                pred = lin;
                bool inside = true;
                if (hl && lin <= lo) { pred = lo; inside = false; }
                if (hu && lin >= hi) { pred = hi; inside = false; }
                ds_dpred = inside ? bs : 0.0;
                width = bs;
            }
        } else {
            pred = a.ys * sd;
            ds_dpred = a.ys;
            width = a.ys;
        }
        if (lane == 0) a.out[r] = pred;
        if (a.target) {
            const double e = (pred - a.target[r]) / width;
            const double ds = 2.0 * e / width * inv_count * ds_dpred;
            const float dsf = static_cast<float>(ds);
            *reinterpret_cast<float2*>(a.dh + r * a.sdh + 2 * lane) = make_float2(dsf * w0, dsf * w1);
            g0 += dsf * hv.x;
            g1 += dsf * hv.y;
            if (lane == 0) {
                gb += dsf;
                gl += static_cast<float>(e * e * inv_count);
            }
        }
    }
    if (!a.target) return;
    red[warp][2 * lane] = g0;
    red[warp][2 * lane + 1] = g1;
    if (lane == 0) {
        red[warp][kH] = gb;
        red[warp][kH + 1] = gl;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kH + 2; i += blockDim.x) {
        float t = 0.f;
        for (int w = 0; w < kWarps; ++w) t += red[w][i];
        a.part[blockIdx.x * (kH + 2) + i] = t;
    }
}

// ----------------------------------------------------------- optimiser

__global__ void k_adam(int count, float lr, float b1, float b2, float eps, float c1, float c2, float* __restrict__ p,
                       const float* __restrict__ g, float* __restrict__ mo, float* __restrict__ vo,
                       __nv_bfloat16* __restrict__ ph) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += blockDim.x * gridDim.x) {
        const float gi = g[i];
        const float mi = b1 * mo[i] + (1.f - b1) * gi;
        const float vi = b2 * vo[i] + (1.f - b2) * gi * gi;
        mo[i] = mi;
        vo[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        ph[i] = __float2bfloat16_rn(pi);
    }
}

__global__ void k_to_bf16(int count, const float* __restrict__ p, __nv_bfloat16* __restrict__ ph) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += blockDim.x * gridDim.x)
        ph[i] = __float2bfloat16_rn(p[i]);
}

__global__ void k_clamp_to_bounds(int n, const double* __restrict__ lo, const double* __restrict__ hi,
                                  double* __restrict__ x) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += blockDim.x * gridDim.x) {
        double v = x[j];
        if (present(lo[j]) && v < lo[j]) v = lo[j];
        if (present(hi[j]) && v > hi[j]) v = hi[j];
        x[j] = v;
    }
}

// ------------------------------------------------------------- layout

struct Offsets {
    long long Ev, bev, Ec, bec, wx, wy, total;
    std::vector<long long> Wc, bc, Wv, bv;
};

Offsets param_offsets(int rounds) {
    Offsets o;
    long long p = 0;
    o.Ev = p; p += kF * kH;
    o.bev = p; p += kH;
    o.Ec = p; p += kF * kH;
    o.bec = p; p += kH;
    for (int t = 0; t < rounds; ++t) {
        o.Wc.push_back(p); p += kX * kH;
        o.bc.push_back(p); p += kH;
        o.Wv.push_back(p); p += kX * kH;
        o.bv.push_back(p); p += kH;
    }
    o.wx = p; p += kH + 1;
    o.wy = p; p += kH + 1;
    o.total = p;
    return o;
}

uint64_t splitmix(uint64_t& s) {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

}  // namespace b200

using namespace b200;

struct SankhyaB200Gnn {
    SankhyaB200GnnSettings settings{};
    int device = 0;
    Offsets off;
    DevBuf model;                     // params, grad, adam m, v (fp32) + bf16 params
    float *params = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    __nv_bfloat16* params_h = nullptr;
    long long step = 0;
    // per-instance workspace, sized for (m, n)
    int m = -1, n = -1;
    DevBuf ws;
    double *c = nullptr, *rl = nullptr, *ru = nullptr, *cl = nullptr, *cu = nullptr, *rnorm = nullptr, *cnorm = nullptr;
    double *x_hat = nullptr, *y_hat = nullptr, *x_t = nullptr, *y_t = nullptr, *bs = nullptr;
    float *fv = nullptr, *fc = nullptr, *inv_row = nullptr, *inv_col = nullptr;
    std::vector<float*> xv, xc;       // rounds + 1 layer inputs [n|m x 128]
    float *gv = nullptr, *gc = nullptr, *zv = nullptr, *zc = nullptr, *part = nullptr, *lossf = nullptr;
    FeatureSlots* slots = nullptr;
    DevBuf tc_flag;                   // set by a tensor-core GEMM whose bounded wait gave up
    int sms = 148;
};

namespace b200 {
namespace {

int elem_blocks(long long count) {
    const long long b = (count + kThreads - 1) / kThreads;
    return static_cast<int>(std::max<long long>(1, std::min<long long>(b, 148LL * 16)));
}

int ensure_workspace(SankhyaB200Gnn* g, int m, int n) {
    if (g->m == m && g->n == n) return 0;
    const int R = g->settings.rounds;
    auto al = [](long long bytes) { return (bytes + 255) / 256 * 256; };
    const long long nd = al(8LL * n), md = al(8LL * m);
    const long long nx = al(4LL * n * kX), mx = al(4LL * m * kX);
    const long long nh = al(4LL * n * kH), mh = al(4LL * m * kH);
    const long long nf = al(4LL * n * kF), mf = al(4LL * m * kF);
    const long long part_floats = std::max<long long>(148LL * 2 * kX * kH, static_cast<long long>(kRedBlocks) * (kH + 2));
    const long long total = 6 * nd + 5 * md + 256 + nf + mf + al(4LL * n) + al(4LL * m) + (R + 1) * (nx + mx) + nx +
                            mx + nh + mh + al(4 * part_floats) + 256 + al(sizeof(FeatureSlots));
    g->m = g->n = -1;
    if (g->ws.alloc(static_cast<size_t>(total), "cudaMalloc network workspace")) return -1;
    char* p = g->ws.as<char>();
    auto take = [&](long long b) { char* r = p; p += b; return r; };
    g->c = reinterpret_cast<double*>(take(nd));
    g->cl = reinterpret_cast<double*>(take(nd));
    g->cu = reinterpret_cast<double*>(take(nd));
    g->cnorm = reinterpret_cast<double*>(take(nd));
    g->x_hat = reinterpret_cast<double*>(take(nd));
    g->x_t = reinterpret_cast<double*>(take(nd));
    g->rl = reinterpret_cast<double*>(take(md));
    g->ru = reinterpret_cast<double*>(take(md));
    g->rnorm = reinterpret_cast<double*>(take(md));
    g->y_hat = reinterpret_cast<double*>(take(md));
    g->y_t = reinterpret_cast<double*>(take(md));
    g->bs = reinterpret_cast<double*>(take(256));
    g->fv = reinterpret_cast<float*>(take(nf));
    g->fc = reinterpret_cast<float*>(take(mf));
    g->inv_col = reinterpret_cast<float*>(take(al(4LL * n)));
    g->inv_row = reinterpret_cast<float*>(take(al(4LL * m)));
    g->xv.assign(R + 1, nullptr);
    g->xc.assign(R + 1, nullptr);
    for (int t = 0; t <= R; ++t) {
        g->xv[t] = reinterpret_cast<float*>(take(nx));
        g->xc[t] = reinterpret_cast<float*>(take(mx));
    }
    g->gv = reinterpret_cast<float*>(take(nx));
    g->gc = reinterpret_cast<float*>(take(mx));
    g->zv = reinterpret_cast<float*>(take(nh));
    g->zc = reinterpret_cast<float*>(take(mh));
    g->part = reinterpret_cast<float*>(take(al(4 * part_floats)));
    g->lossf = reinterpret_cast<float*>(take(256));
    g->slots = reinterpret_cast<FeatureSlots*>(take(al(sizeof(FeatureSlots))));
    g->m = m;
    g->n = n;
    return 0;
}

// The tensor-core (tcgen05) GEMM where its layout conditions hold: 16-byte
// aligned rows of A and C (row strides multiples of 4 floats). One CTA per SM-share
// of TMEM (512 columns per SM, N per CTA), persistent over the 128-row tiles.
bool tc_fits(const void* a, int lda, const void* c, int ldc) {
    return (reinterpret_cast<uintptr_t>(a) & 15u) == 0 && (reinterpret_cast<uintptr_t>(c) & 15u) == 0 &&
           lda % 4 == 0 && ldc % 4 == 0;
}

// K = 64 / 128: the cp.async-pipelined kernel, one CTA per SM (its shared memory).
template <int N, int K, int ST>
void gemm_tc_pipe(SankhyaB200Gnn* s, cudaStream_t st, int M, const float* A, int lda, const __nv_bfloat16* B, int sbk,
                  int sbn, const float* bias, int relu, float* C, int ldc) {
    using S = tc::TcPipeShape<N, K, ST>;
    const void* fn = reinterpret_cast<const void*>(&tc::k_gemm_tc_pipe<N, K, ST>);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kSmem);
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, S::kThreads, S::kSmem);
    const int tiles = (M + S::kM - 1) / S::kM;
    const int grid = std::max(1, std::min(tiles, s->sms * std::max(1, per_sm)));
    tc::k_gemm_tc_pipe<N, K, ST><<<grid, S::kThreads, S::kSmem, st>>>(M, A, lda, B, sbk, sbn, bias, relu, C, ldc,
                                                                       s->tc_flag.as<unsigned int>());
}

template <int N, int K>
void gemm_tc(SankhyaB200Gnn* s, cudaStream_t st, int M, const float* A, int lda, const __nv_bfloat16* B, int sbk,
             int sbn, const float* bias, int relu, float* C, int ldc) {
    if constexpr (K == 128) {
        gemm_tc_pipe<N, K, 4>(s, st, M, A, lda, B, sbk, sbn, bias, relu, C, ldc);
        return;
    } else if constexpr (K == 64) {
        gemm_tc_pipe<N, K, 3>(s, st, M, A, lda, B, sbk, sbn, bias, relu, C, ldc);
        return;
    }
    using S = tc::TcShape<N, K>;
    const void* fn = reinterpret_cast<const void*>(&tc::k_gemm_tc<N, K>);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, S::kSmem);
    const int tiles = (M + S::kM - 1) / S::kM;
    const int grid = std::max(1, std::min(tiles, s->sms * std::min(4, 512 / S::kCols)));
    tc::k_gemm_tc<N, K><<<grid, 128, S::kSmem, st>>>(M, A, lda, B, sbk, sbn, bias, relu, C, ldc,
                                                     s->tc_flag.as<unsigned int>());
}

// C = A B (+ bias, relu) with A fp32 [M x K] (row-major, lda) and B bf16 [K x 64] row-major.
void gemm_forward(SankhyaB200Gnn* s, cudaStream_t st, int M, int K, const float* A, int lda,
                  const __nv_bfloat16* W, const float* bias, float* C, int ldc) {
    if (M == 0) return;
    if (tc_fits(A, lda, C, ldc) && (K == kF || K == kX)) {
        if (K == kF) gemm_tc<kH, kF>(s, st, M, A, lda, W, kH, 1, bias, 1, C, ldc);
        else gemm_tc<kH, kX>(s, st, M, A, lda, W, kH, 1, bias, 1, C, ldc);
        return;
    }
    Gemm<__nv_bfloat16> g{M, kH, K, A, lda, 1, W, kH, 1, C, ldc, 1, 0, K, bias, 1};
    k_gemm_bf16<__nv_bfloat16><<<dim3((M + 63) / 64, 1, 1), kGemmThreads, 0, st>>>(g);
}

// dX [M x K] = dZ [M x 64] W^T, W bf16 [K x 64] row-major; K = 128.
void gemm_input_grad(SankhyaB200Gnn* s, cudaStream_t st, int M, const float* dz, const __nv_bfloat16* W, int K,
                     float* dx, int ldx) {
    if (M == 0) return;
    if (tc_fits(dz, kH, dx, ldx) && K == kX && (reinterpret_cast<uintptr_t>(W) & 15u) == 0) {
        gemm_tc<kX, kH>(s, st, M, dz, kH, W, 1, kH, nullptr, 0, dx, ldx);
        return;
    }
    Gemm<__nv_bfloat16> g{M, K, kH, dz, kH, 1, W, 1, kH, dx, ldx, 1, 0, kH, nullptr, 0};
    k_gemm_bf16<__nv_bfloat16><<<dim3((M + 63) / 64, (K + 63) / 64, 1), kGemmThreads, 0, st>>>(g);
}

// Fails the call when a tensor-core GEMM's bounded wait gave up (the flag is cleared).
int check_tc(SankhyaB200Gnn* s, cudaStream_t st) {
    unsigned int flag = 0;
    B200_TRY(cudaMemcpyAsync(&flag, s->tc_flag.p, sizeof(flag), cudaMemcpyDeviceToHost, st), "read GEMM flag");
    B200_TRY(cudaStreamSynchronize(st), "network");
    if (!flag) return 0;
    cudaMemsetAsync(s->tc_flag.p, 0, sizeof(flag), st);
    return fail_msg("a tensor-core GEMM's wait for its MMAs gave up");
}

// dW [K x 64] = X^T dZ over `rows` nodes (X fp32 [rows x K] with row stride ldx),
// split over nodes into fixed slices, summed in slice order into out.
void gemm_weight_grad(SankhyaB200Gnn* s, cudaStream_t st, int rows, const float* X, int ldx, int K, const float* dz,
                      float* out) {
    if (rows == 0) {
        cudaMemsetAsync(out, 0, sizeof(float) * K * kH, st);
        return;
    }
    if (K == kX && tc_fits(X, ldx, dz, kH)) {
        // tensor-core path: one slice (a whole number of 64-node stages) per resident CTA
        using W = tc::WgPipeShape<3>;
        const void* fn = reinterpret_cast<const void*>(&tc::k_wgrad_tc_pipe<kX, 3>);
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, W::kSmem);
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, W::kThreads, W::kSmem);
        const int want = std::max(1, std::min({148 * 2, s->sms * std::max(1, per_sm), (rows + W::kNodes - 1) / W::kNodes}));
        const int chunk = ((rows + want - 1) / want + W::kNodes - 1) / W::kNodes * W::kNodes;
        const int slices = (rows + chunk - 1) / chunk;
        tc::k_wgrad_tc_pipe<kX, 3><<<slices, W::kThreads, W::kSmem, st>>>(rows, chunk, X, ldx, dz, s->part,
                                                                           s->tc_flag.as<unsigned int>());
        sum_slices(K * kH, slices, static_cast<long long>(K) * kH, s->part, out, st);
        return;
    }
    const int slices = std::max(1, std::min(148 * 2, (rows + 255) / 256));
    const int chunk = (rows + slices - 1) / slices;
    Gemm<float> g{K, kH, rows, X, 1, ldx, dz, kH, 1, s->part, kH, 1, static_cast<long long>(K) * kH, chunk, nullptr, 0};
    k_gemm_bf16<float><<<dim3((K + 63) / 64, 1, slices), kGemmThreads, 0, st>>>(g);
    sum_slices(K * kH, slices, static_cast<long long>(K) * kH, s->part, out, st);
}

void bias_grad(SankhyaB200Gnn* s, cudaStream_t st, int rows, const float* dz, float* out) {
    const int blocks = kRedBlocks;
    k_colsum64<<<blocks, 4 * kH, 0, st>>>(rows, dz, s->part);
    sum_slices(kH, blocks, kH, s->part, out, st);
}

void spmm(cudaStream_t st, const TileCsr& M, const float* in, int sin, const float* pre, const float* post, float* out,
          int sout, int accumulate) {
    if (M.rows == 0) return;
    const int blocks = static_cast<int>(std::min<long long>((M.rows + kWarps - 1) / kWarps, 148LL * 8));
    k_spmm64<<<blocks, kThreads, 0, st>>>(M.rows, M.ptr, M.idx, M.val, in, sin, pre, post, out, sout, accumulate);
}

int upload_instance(SankhyaB200Gnn* g, const Plan& plan, const double* c, const double* rl, const double* ru,
                    const double* cl, const double* cu, cudaStream_t st) {
    const int m = plan.a.rows, n = plan.a.cols;
    B200_TRY(cudaMemcpyAsync(g->c, c, 8LL * n, cudaMemcpyHostToDevice, st), "upload c");
    B200_TRY(cudaMemcpyAsync(g->cl, cl, 8LL * n, cudaMemcpyHostToDevice, st), "upload col bounds");
    B200_TRY(cudaMemcpyAsync(g->cu, cu, 8LL * n, cudaMemcpyHostToDevice, st), "upload col bounds");
    if (m) {
        B200_TRY(cudaMemcpyAsync(g->rl, rl, 8LL * m, cudaMemcpyHostToDevice, st), "upload row bounds");
        B200_TRY(cudaMemcpyAsync(g->ru, ru, 8LL * m, cudaMemcpyHostToDevice, st), "upload row bounds");
    }
    B200_TRY(cudaMemsetAsync(g->slots, 0, sizeof(FeatureSlots), st), "zero slots");
    if (m) k_abs_sums<<<elem_blocks(m), kThreads, 0, st>>>(m, plan.a.ptr, plan.a.val, g->rnorm);
    k_abs_sums<<<elem_blocks(n), kThreads, 0, st>>>(n, plan.at.ptr, plan.at.val, g->cnorm);
    k_feature_maxima<<<elem_blocks(std::max(m, n)), kThreads, 0, st>>>(m, n, g->c, g->cl, g->cu, g->rl, g->ru,
                                                                       g->rnorm, g->cnorm, plan.a.ptr, plan.at.ptr,
                                                                       g->slots);
    k_features<<<elem_blocks(std::max(m, n)), kThreads, 0, st>>>(m, n, g->c, g->cl, g->cu, g->rl, g->ru, g->rnorm,
                                                                 g->cnorm, plan.a.ptr, plan.at.ptr, g->slots, g->fv,
                                                                 g->fc, g->inv_row, g->inv_col, g->bs);
    B200_TRY(cudaGetLastError(), "network features");
    return 0;
}

void forward(SankhyaB200Gnn* g, const Plan& plan, cudaStream_t st) {
    const int m = plan.a.rows, n = plan.a.cols, R = g->settings.rounds;
    const Offsets& o = g->off;
    gemm_forward(g, st, n, kF, g->fv, kF, g->params_h + o.Ev, g->params + o.bev, g->xv[0], kX);
    gemm_forward(g, st, m, kF, g->fc, kF, g->params_h + o.Ec, g->params + o.bec, g->xc[0], kX);
    for (int t = 0; t < R; ++t) {
        spmm(st, plan.a, g->xv[t], kX, nullptr, g->inv_row, g->xc[t] + kH, kX, 0);
        gemm_forward(g, st, m, kX, g->xc[t], kX, g->params_h + o.Wc[t], g->params + o.bc[t], g->xc[t + 1], kX);
        spmm(st, plan.at, g->xc[t + 1], kX, nullptr, g->inv_col, g->xv[t] + kH, kX, 0);
        gemm_forward(g, st, n, kX, g->xv[t], kX, g->params_h + o.Wv[t], g->params + o.bv[t], g->xv[t + 1], kX);
    }
}

// Heads (+ loss and head gradients when targets are on the device).
void heads(SankhyaB200Gnn* g, const Plan& plan, cudaStream_t st, bool with_target) {
    const int m = plan.a.rows, n = plan.a.cols, R = g->settings.rounds;
    const Offsets& o = g->off;
    const int blocks = kRedBlocks;
    HeadArgs hx{n, g->xv[R], kX, g->params + o.wx, g->cl, g->cu, g->bs, 1.0, 1, g->x_hat,
                with_target ? g->x_t : nullptr, g->gv, kX, g->part};
    k_head<<<blocks, kThreads, 0, st>>>(hx);
    if (with_target) {
        sum_slices(kH + 1, blocks, kH + 2, g->part, g->grad + o.wx, st);
        sum_slices(1, blocks, kH + 2, g->part + kH + 1, g->lossf, st);
    }
    if (m) {
        HeadArgs hy{m, g->xc[R], kX, g->params + o.wy, nullptr, nullptr, nullptr, g->settings.y_scale, 0, g->y_hat,
                    with_target ? g->y_t : nullptr, g->gc, kX, g->part};
        k_head<<<blocks, kThreads, 0, st>>>(hy);
        if (with_target) {
            sum_slices(kH + 1, blocks, kH + 2, g->part, g->grad + o.wy, st);
            sum_slices(1, blocks, kH + 2, g->part + kH + 1, g->lossf + 1, st);
        }
    } else if (with_target) {
        cudaMemsetAsync(g->grad + o.wy, 0, sizeof(float) * (kH + 1), st);
        cudaMemsetAsync(g->lossf + 1, 0, sizeof(float), st);
    }
}

void backward(SankhyaB200Gnn* g, const Plan& plan, cudaStream_t st) {
    const int m = plan.a.rows, n = plan.a.cols, R = g->settings.rounds;
    const Offsets& o = g->off;
    for (int t = R - 1; t >= 0; --t) {
        k_relu_mask<<<elem_blocks(static_cast<long long>(n) * kH), kThreads, 0, st>>>(n, g->gv, kX, g->xv[t + 1], kX,
                                                                                     g->zv);
        gemm_weight_grad(g, st, n, g->xv[t], kX, kX, g->zv, g->grad + o.Wv[t]);
        bias_grad(g, st, n, g->zv, g->grad + o.bv[t]);
        gemm_input_grad(g, st, n, g->zv, g->params_h + o.Wv[t], kX, g->gv, kX);
        spmm(st, plan.a, g->gv + kH, kX, g->inv_col, nullptr, g->gc, kX, 1);
        if (m) {
            k_relu_mask<<<elem_blocks(static_cast<long long>(m) * kH), kThreads, 0, st>>>(m, g->gc, kX, g->xc[t + 1],
                                                                                         kX, g->zc);
        }
        gemm_weight_grad(g, st, m, g->xc[t], kX, kX, g->zc, g->grad + o.Wc[t]);
        if (m) {
            bias_grad(g, st, m, g->zc, g->grad + o.bc[t]);
            gemm_input_grad(g, st, m, g->zc, g->params_h + o.Wc[t], kX, g->gc, kX);
        } else {
            cudaMemsetAsync(g->grad + o.bc[t], 0, sizeof(float) * kH, st);
        }
        spmm(st, plan.at, g->gc + kH, kX, g->inv_row, nullptr, g->gv, kX, 1);
    }
    k_relu_mask<<<elem_blocks(static_cast<long long>(n) * kH), kThreads, 0, st>>>(n, g->gv, kX, g->xv[0], kX, g->zv);
    gemm_weight_grad(g, st, n, g->fv, kF, kF, g->zv, g->grad + o.Ev);
    bias_grad(g, st, n, g->zv, g->grad + o.bev);
    if (m) {
        k_relu_mask<<<elem_blocks(static_cast<long long>(m) * kH), kThreads, 0, st>>>(m, g->gc, kX, g->xc[0], kX,
                                                                                     g->zc);
        bias_grad(g, st, m, g->zc, g->grad + o.bec);
    } else {
        cudaMemsetAsync(g->grad + o.bec, 0, sizeof(float) * kH, st);
    }
    gemm_weight_grad(g, st, m, g->fc, kF, kF, g->zc, g->grad + o.Ec);
}

int check_model(SankhyaB200Gnn* g) {
    if (!g) return fail_msg("null network");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != g->device) return fail_msg("network used on another device");
    return 0;
}

int prepare(SankhyaB200Gnn* g, const SankhyaCudaCSR* matrix, const double* c, const double* rl, const double* ru,
            const double* cl, const double* cu, std::shared_ptr<Plan>* plan) {
    clear_error();
    (void)cudaGetLastError();
    if (check_model(g)) return -1;
    if (!matrix || !c || !cl || !cu || ((!rl || !ru) && matrix->rows > 0)) return fail_msg("invalid network arguments");
    if (matrix->cols <= 0 || matrix->rows < 0) return fail_msg("invalid matrix dimensions");
    // the checks of sankhya_b200_pdlp_solve: a NaN would poison the features and,
    // through a training step, the parameters
    for (int j = 0; j < matrix->cols; ++j)
        if (!std::isfinite(c[j]) || std::isnan(cl[j]) || std::isnan(cu[j]) || cl[j] > cu[j])
            return fail_msg("invalid cost or column bound");
    for (int i = 0; i < matrix->rows; ++i)
        if (std::isnan(rl[i]) || std::isnan(ru[i]) || rl[i] > ru[i]) return fail_msg("invalid row bound");
    if (get_plan(matrix, plan)) return -1;
    if (ensure_workspace(g, matrix->rows, matrix->cols)) return -1;
    return upload_instance(g, **plan, c, rl, ru, cl, cu, engine_stream());
}

int upload_targets(SankhyaB200Gnn* g, int m, int n, const double* x_t, const double* y_t, cudaStream_t st) {
    if (!x_t || (m > 0 && !y_t)) return fail_msg("missing training targets");
    for (int j = 0; j < n; ++j)
        if (!std::isfinite(x_t[j])) return fail_msg("non-finite training target");
    for (int i = 0; i < m; ++i)
        if (!std::isfinite(y_t[i])) return fail_msg("non-finite training target");
    B200_TRY(cudaMemcpyAsync(g->x_t, x_t, 8LL * n, cudaMemcpyHostToDevice, st), "upload x target");
    if (m) B200_TRY(cudaMemcpyAsync(g->y_t, y_t, 8LL * m, cudaMemcpyHostToDevice, st), "upload y target");
    return 0;
}

int read_loss(SankhyaB200Gnn* g, cudaStream_t st, double* loss) {
    float l[2] = {0.f, 0.f};
    B200_TRY(cudaMemcpyAsync(l, g->lossf, sizeof(l), cudaMemcpyDeviceToHost, st), "read loss");
    if (check_tc(g, st)) return -1;
    if (loss) *loss = static_cast<double>(l[0]) + static_cast<double>(l[1]);
    return 0;
}

}  // namespace
}  // namespace b200

extern "C" void sankhya_b200_gnn_default_settings(SankhyaB200GnnSettings* s) {
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    s->struct_version = 1;
    s->rounds = 4;
    s->seed = 1;
    s->learning_rate = 1e-3;
    s->y_scale = 1.0;
}

extern "C" int sankhya_b200_gnn_create(const SankhyaB200GnnSettings* settings, SankhyaB200Gnn** out) {
    clear_error();
    (void)cudaGetLastError();
    if (!out) return fail_msg("null output handle");
    *out = nullptr;
    SankhyaB200GnnSettings s;
    sankhya_b200_gnn_default_settings(&s);
    if (settings) {
        if (settings->struct_version != 1) return fail_msg("unsupported settings struct_version");
        s = *settings;
    }
    if (s.rounds < 1 || s.rounds > 16 || !(s.learning_rate > 0.0) || !(s.y_scale > 0.0))
        return fail_msg("invalid network settings");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) return fail_msg("no CUDA device available");
    SankhyaB200Gnn* g = new (std::nothrow) SankhyaB200Gnn();
    if (!g) return fail_msg("out of host memory");
    g->settings = s;
    cudaGetDevice(&g->device);
    g->off = param_offsets(s.rounds);
    const long long P = g->off.total;
    const long long fb = (4 * P + 255) / 256 * 256, hb = (2 * P + 255) / 256 * 256;
    if (g->model.alloc(static_cast<size_t>(4 * fb + hb), "cudaMalloc network parameters") ||
        g->tc_flag.alloc(256, "cudaMalloc GEMM flag") ||
        cudaMemset(g->tc_flag.p, 0, 256) != cudaSuccess) {
        delete g;
        return -1;
    }
    cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, g->device);
    char* p = g->model.as<char>();
    g->params = reinterpret_cast<float*>(p);
    g->grad = reinterpret_cast<float*>(p + fb);
    g->adam_m = reinterpret_cast<float*>(p + 2 * fb);
    g->adam_v = reinterpret_cast<float*>(p + 3 * fb);
    g->params_h = reinterpret_cast<__nv_bfloat16*>(p + 4 * fb);
    // uniform(-a, a), a = sqrt(6 / fan_in) for matrices, heads uniform(-0.1, 0.1) / sqrt(H), zero biases
    std::vector<float> init(static_cast<size_t>(P), 0.f);
    uint64_t state = s.seed;
    auto fill = [&](long long at, int rows, int cols, double a) {
        for (long long i = 0; i < static_cast<long long>(rows) * cols; ++i) {
            const double u = static_cast<double>(splitmix(state) >> 11) * (1.0 / 9007199254740992.0);
            init[static_cast<size_t>(at + i)] = static_cast<float>((2.0 * u - 1.0) * a);
        }
    };
    fill(g->off.Ev, kF, kH, std::sqrt(6.0 / kF));
    fill(g->off.Ec, kF, kH, std::sqrt(6.0 / kF));
    for (int t = 0; t < s.rounds; ++t) {
        fill(g->off.Wc[t], kX, kH, std::sqrt(6.0 / kX));
        fill(g->off.Wv[t], kX, kH, std::sqrt(6.0 / kX));
    }
    fill(g->off.wx, 1, kH, 0.1 / std::sqrt(static_cast<double>(kH)));
    fill(g->off.wy, 1, kH, 0.1 / std::sqrt(static_cast<double>(kH)));
    cudaStream_t st = engine_stream();
    if (cudaMemcpyAsync(g->params, init.data(), 4 * P, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(g->adam_m, 0, 2 * fb, st) != cudaSuccess || cudaMemsetAsync(g->grad, 0, fb, st) != cudaSuccess) {
        delete g;
        return fail_msg("network initialisation failed");
    }
    k_to_bf16<<<elem_blocks(P), kThreads, 0, st>>>(static_cast<int>(P), g->params, g->params_h);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        delete g;
        return fail_msg("network initialisation failed");
    }
    *out = g;
    return 0;
}

extern "C" void sankhya_b200_gnn_destroy(SankhyaB200Gnn* g) { delete g; }

extern "C" int sankhya_b200_gnn_parameter_count(const SankhyaB200Gnn* g) {
    return g ? static_cast<int>(g->off.total) : -1;
}

extern "C" int sankhya_b200_gnn_get_parameters(SankhyaB200Gnn* g, float* out) {
    clear_error();
    if (check_model(g)) return -1;
    if (!out) return fail_msg("null output");
    cudaStream_t st = engine_stream();
    B200_TRY(cudaMemcpyAsync(out, g->params, 4 * g->off.total, cudaMemcpyDeviceToHost, st), "read parameters");
    B200_TRY(cudaStreamSynchronize(st), "read parameters");
    return 0;
}

extern "C" int sankhya_b200_gnn_set_parameters(SankhyaB200Gnn* g, const float* in) {
    clear_error();
    if (check_model(g)) return -1;
    if (!in) return fail_msg("null input");
    for (long long i = 0; i < g->off.total; ++i)
        if (!std::isfinite(in[i])) return fail_msg("non-finite parameter");
    cudaStream_t st = engine_stream();
    B200_TRY(cudaMemcpyAsync(g->params, in, 4 * g->off.total, cudaMemcpyHostToDevice, st), "write parameters");
    k_to_bf16<<<elem_blocks(g->off.total), kThreads, 0, st>>>(static_cast<int>(g->off.total), g->params, g->params_h);
    B200_TRY(cudaStreamSynchronize(st), "write parameters");
    return 0;
}

extern "C" int sankhya_b200_gnn_predict(SankhyaB200Gnn* g, const SankhyaCudaCSR* matrix, const double* c,
                                        const double* rl, const double* ru, const double* cl, const double* cu,
                                        double* x_out, double* y_out) {
    std::shared_ptr<Plan> plan;
    if (prepare(g, matrix, c, rl, ru, cl, cu, &plan)) return -1;
    if (!x_out) return fail_msg("null output");
    cudaStream_t st = engine_stream();
    forward(g, *plan, st);
    heads(g, *plan, st, false);
    const int m = plan->a.rows, n = plan->a.cols;
    k_clamp_to_bounds<<<elem_blocks(n), kThreads, 0, st>>>(n, g->cl, g->cu, g->x_hat);
    B200_TRY(cudaGetLastError(), "network forward");
    B200_TRY(cudaMemcpyAsync(x_out, g->x_hat, 8LL * n, cudaMemcpyDeviceToHost, st), "read prediction");
    if (y_out && m) B200_TRY(cudaMemcpyAsync(y_out, g->y_hat, 8LL * m, cudaMemcpyDeviceToHost, st), "read prediction");
    return check_tc(g, st);
}

extern "C" int sankhya_b200_gnn_gradient(SankhyaB200Gnn* g, const SankhyaCudaCSR* matrix, const double* c,
                                         const double* rl, const double* ru, const double* cl, const double* cu,
                                         const double* x_target, const double* y_target, double* loss,
                                         float* grad_out) {
    std::shared_ptr<Plan> plan;
    if (prepare(g, matrix, c, rl, ru, cl, cu, &plan)) return -1;
    cudaStream_t st = engine_stream();
    if (upload_targets(g, plan->a.rows, plan->a.cols, x_target, y_target, st)) return -1;
    forward(g, *plan, st);
    heads(g, *plan, st, true);
    backward(g, *plan, st);
    B200_TRY(cudaGetLastError(), "network backward");
    if (grad_out)
        B200_TRY(cudaMemcpyAsync(grad_out, g->grad, 4 * g->off.total, cudaMemcpyDeviceToHost, st), "read gradient");
    return read_loss(g, st, loss);
}

extern "C" int sankhya_b200_gnn_train_step(SankhyaB200Gnn* g, const SankhyaCudaCSR* matrix, const double* c,
                                           const double* rl, const double* ru, const double* cl, const double* cu,
                                           const double* x_target, const double* y_target, double* loss) {
    std::shared_ptr<Plan> plan;
    if (prepare(g, matrix, c, rl, ru, cl, cu, &plan)) return -1;
    cudaStream_t st = engine_stream();
    if (upload_targets(g, plan->a.rows, plan->a.cols, x_target, y_target, st)) return -1;
    forward(g, *plan, st);
    heads(g, *plan, st, true);
    backward(g, *plan, st);
    g->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, static_cast<float>(g->step)), c2 = 1.f - std::pow(b2, static_cast<float>(g->step));
    k_adam<<<elem_blocks(g->off.total), kThreads, 0, st>>>(static_cast<int>(g->off.total),
                                                           static_cast<float>(g->settings.learning_rate), b1, b2, 1e-8f,
                                                           c1, c2, g->params, g->grad, g->adam_m, g->adam_v,
                                                           g->params_h);
    B200_TRY(cudaGetLastError(), "network training step");
    return read_loss(g, st, loss);
}
