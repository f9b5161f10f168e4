// Dense layers of the warm-start network on the 5th-generation tensor cores:
// tcgen05.mma (kind::f16, bf16 x bf16 -> fp32) with the accumulator in tensor
// memory, issued by one thread per CTA.
//
//   C[M x N] = A[M x K] B (+ bias, relu),  A fp32 row-major (lda), B bf16 with
//   element (k, n) at B[k sbk + n sbn], C fp32 row-major (ldc), N in {64, 128},
//   K in {16, 64, 128}.
//
// A CTA of 128 threads owns a 128 x N accumulator in TMEM (N columns) and walks
// 128-row tiles of A (persistent). B is staged once per CTA. Each tile: the
// threads round A to bf16 into shared memory in the canonical K-major layout
// without swizzle (8 x 16-byte core matrices; core (row block i, k block j) at
// (i K/8 + j) 128 bytes, so the K-adjacent core is 128 bytes away (leading byte
// offset) and the next 8-row block K/8 * 128 bytes (stride byte offset)); thread
// 0 issues K/16 MMAs of 128 x N x 16 and commits them to an mbarrier; after the
// wait each warp reads its 32 rows (TMEM lanes 32w..32w+31) with tcgen05.ld and
// applies bias / relu. The operands are rounded to bf16 exactly as the mma.sync
// kernel rounds them; only the fp32 accumulation order inside the tensor core
// differs.
//
// Descriptor bitfields follow CUTLASS's cute/arch/mma_sm100_desc.hpp
// (SmemDescriptor, InstrDescriptor); tests/test_tc_descriptors.py checks them on
// the host against those unions.
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace b200 {
namespace tc {

// Shared-memory matrix descriptor: start address, leading / stride byte offsets
// (16-byte units), version 1 (Blackwell), base offset 0, SWIZZLE_NONE.
__host__ __device__ constexpr uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: fp32 accumulator, bf16 A and B, both
// K-major, N / 8 and M / 16.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
           (static_cast<uint32_t>(M >> 4) << 24);
}

// Byte offset of element (r, k) in the canonical K-major tile with K columns.
template <int K>
__host__ __device__ constexpr uint32_t kmajor_offset(int r, int k) {
    return static_cast<uint32_t>(((r >> 3) * (K / 8) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Bounded wait for the mbarrier phase; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, long long limit) {
    for (long long i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

constexpr long long kWaitLimit = 1ll << 22;

template <int N, int K>
struct TcShape {
    static_assert(N == 64 || N == 128, "N is 64 or 128");
    static_assert(K == 16 || K == 64 || K == 128, "K is 16, 64 or 128");
    static constexpr int kM = 128;
    static constexpr int kABytes = kM * K * 2;
    static constexpr int kBBytes = N * K * 2;
    static constexpr int kSmem = kABytes + kBBytes + 64 + 128;  // + mbarrier, TMEM address slot, alignment
    static constexpr int kCols = N;                              // TMEM columns (a power of 2 >= 32)
};

template <int N, int K>
__global__ void __launch_bounds__(128) k_gemm_tc(int M, const float* __restrict__ A, int lda,
                                                 const __nv_bfloat16* __restrict__ B, int sbk, int sbn,
                                                 const float* __restrict__ bias, int relu, float* __restrict__ C,
                                                 int ldc, unsigned int* __restrict__ err) {
    using S = TcShape<N, K>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    unsigned char* sA = smem;
    unsigned char* sB = smem + S::kABytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + S::kBBytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    for (int e = tid; e < N * K; e += 128) {
        const int n = e / K, k = e - n * K;
        *reinterpret_cast<__nv_bfloat16*>(sB + kmajor_offset<K>(n, k)) = B[static_cast<long long>(k) * sbk + n * sbn];
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(S::kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;
    const uint32_t idesc = instr_desc_bf16(S::kM, N);
    const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB), bar = smem_u32(mbar);
    uint32_t phase = 0;
    bool failed = false;
    for (int tile = blockIdx.x; tile * S::kM < M && !failed; tile += gridDim.x) {
        const int m0 = tile * S::kM;
        // A tile: fp32 -> bf16, four consecutive k per thread step (8 bytes into one core row)
        for (int q = tid; q < S::kM * (K / 4); q += 128) {
            const int r = q / (K / 4), k4 = (q - r * (K / 4)) * 4;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (m0 + r < M) v = *reinterpret_cast<const float4*>(A + static_cast<long long>(m0 + r) * lda + k4);
            __nv_bfloat162 lo = __floats2bfloat162_rn(v.x, v.y), hi = __floats2bfloat162_rn(v.z, v.w);
            uint2 packed;
            packed.x = *reinterpret_cast<uint32_t*>(&lo);
            packed.y = *reinterpret_cast<uint32_t*>(&hi);
            *reinterpret_cast<uint2*>(sA + kmajor_offset<K>(r, k4)) = packed;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int s = 0; s < K / 16; ++s) {
                const uint64_t da = smem_desc(a_base + s * 256, 128, (K / 8) * 128);
                const uint64_t db = smem_desc(b_base + s * 256, 128, (K / 8) * 128);
                const uint32_t accumulate = s > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        const bool ok = mbar_wait(bar, phase, kWaitLimit);
        failed = __syncthreads_or(!ok) != 0;
        phase ^= 1u;
        if (failed) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int row = m0 + warp * 32 + lane;
#pragma unroll
        for (int c0 = 0; c0 < N; c0 += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
                float* out = C + static_cast<long long>(row) * ldc + c0;
#pragma unroll
                for (int j = 0; j < 16; j += 4) {
                    float4 o;
                    float* f = &o.x;
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        float t = __uint_as_float(v[j + e]);
                        if (bias) t += bias[c0 + j + e];
                        if (relu) t = fmaxf(t, 0.f);
                        f[e] = t;
                    }
                    *reinterpret_cast<float4*>(out + j) = o;
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (failed) {
        // the MMA may still be writing TMEM: wait for it (bounded) before freeing
        if (tid == 0) atomicOr(err, 1u);
        mbar_wait(bar, phase ^ 1u, kWaitLimit);
        __syncthreads();
    }
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::kCols));
}

}  // namespace tc
}  // namespace b200
