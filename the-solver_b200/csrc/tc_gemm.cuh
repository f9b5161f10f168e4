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
// offset) and the next 8-row block K/8 * 128 bytes (stride byte offset)). The
// staging is by 32-byte pieces (8 k of one row) numbered so that piece u lands at
// byte 16 u: each thread keeps up to 8 pieces (16 float4 loads) in flight, and the
// first pieces of its next tile are loaded while the current tile's MMAs and
// epilogue run. Thread 0 issues K/16 MMAs of 128 x N x 16 and commits them to an
// mbarrier; after the wait each warp reads its 32 rows (TMEM lanes 32w..32w+31)
// with tcgen05.ld, applies bias / relu and transposes 32 x 16 blocks through shared
// memory so that its stores cover 64 contiguous bytes of 8 rows at a time. The
// operands are rounded to bf16 exactly as the mma.sync kernel rounds them; only
// the fp32 accumulation order inside the tensor core differs.
//
// k_gemm_tc_pipe (below) is the same product for K = 64 and 128 fed by cp.async stages,
// and k_wgrad_tc_pipe computes the weight gradients X^T dZ with both operands
// MN-major, summed over node slices in a fixed order.
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

// The same with A and B both MN-major (bits 15 and 16): A's M and B's N index is the
// contiguous one inside a 16-byte core row.
__host__ __device__ constexpr uint32_t instr_desc_bf16_mn(int M, int N) {
    return instr_desc_bf16(M, N) | (1u << 15) | (1u << 16);
}

// Byte offset of element (mn, k) in the canonical MN-major layout without swizzle used
// by the weight-gradient kernel: a core matrix is 8 k-rows of 16 bytes (8 consecutive
// mn), the next 8 mn are 128 bytes away (stride byte offset) and the next 8 k are
// (MN / 8) * 128 bytes away (leading byte offset).
template <int MN>
__host__ __device__ constexpr uint32_t mnmajor_offset(int mn, int k) {
    return static_cast<uint32_t>((k >> 3) * (MN / 8) * 128 + (mn >> 3) * 128 + (k & 7) * 16 + (mn & 7) * 2);
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

// 8 fp32 -> 8 bf16 (16 bytes), round to nearest even.
__device__ __forceinline__ uint4 pack8(const float4& a, const float4& b) {
    __nv_bfloat162 p0 = __floats2bfloat162_rn(a.x, a.y), p1 = __floats2bfloat162_rn(a.z, a.w);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(b.x, b.y), p3 = __floats2bfloat162_rn(b.z, b.w);
    uint4 r;
    r.x = *reinterpret_cast<uint32_t*>(&p0);
    r.y = *reinterpret_cast<uint32_t*>(&p1);
    r.z = *reinterpret_cast<uint32_t*>(&p2);
    r.w = *reinterpret_cast<uint32_t*>(&p3);
    return r;
}

// Staging unit u of a 128 x K tile of A: 8 consecutive k (32 bytes of fp32) of one
// row. With t = u / 8, the unit is k-block t mod (K/8) of row 8 (t div (K/8)) + u mod 8,
// which puts it at byte u * 16 of the canonical K-major layout: a warp's 32 units fill
// 512 contiguous bytes of shared memory (no bank conflicts) and read 128 contiguous
// bytes from each of 8 rows (whole sectors) when K >= 32.
template <int K>
__device__ __forceinline__ void unit_row_k(int u, int& r, int& k) {
    const int t = u >> 3;
    r = (t / (K / 8)) * 8 + (u & 7);
    k = (t % (K / 8)) * 8;
}

template <int K>
__device__ __forceinline__ void load_unit(const float* __restrict__ A, int lda, int M, int m0, int u, float4& lo,
                                          float4& hi) {
    int r, k;
    unit_row_k<K>(u, r, k);
    if (m0 + r < M) {
        const float4* p = reinterpret_cast<const float4*>(A + static_cast<long long>(m0 + r) * lda + k);
        lo = __ldg(p);
        hi = __ldg(p + 1);
    } else {
        lo = hi = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

template <int N, int K>
struct TcShape {
    static_assert(N == 64 || N == 128, "N is 64 or 128");
    static_assert(K == 16 || K == 64 || K == 128, "K is 16, 64 or 128");
    static constexpr int kM = 128;
    static constexpr int kABytes = kM * K * 2;
    static constexpr int kBBytes = N * K * 2;
    // epilogue staging (4 warps x 32 rows x 16 floats) in the A buffer, or after B when
    // the A buffer is smaller
    static constexpr int kStageBytes = 4 * 32 * 16 * 4;
    static constexpr int kStageOffset = kABytes >= kStageBytes ? 0 : kABytes + kBBytes;
    static constexpr int kExtra = kABytes >= kStageBytes ? 0 : kStageBytes;
    static constexpr int kSmem = kABytes + kBBytes + kExtra + 64 + 128;  // + mbarrier, TMEM slot, alignment
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
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + S::kBBytes + S::kExtra);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // B in pieces of 8 consecutive k of one column n (16 bytes at kmajor_offset(n, k)):
    // lanes take consecutive n, so the loads are contiguous when n is the contiguous
    // index (sbn == 1) and each piece is one 16-byte load when k is (sbk == 1).
#pragma unroll 4
    for (int e = tid; e < N * (K / 8); e += 128) {
        const int n = e % N, k = (e / N) * 8;
        uint4 piece;
        if (sbk == 1) {
            piece = *reinterpret_cast<const uint4*>(B + static_cast<long long>(n) * sbn + k);
        } else {
            uint32_t w[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const __nv_bfloat16 lo = B[static_cast<long long>(k + 2 * j) * sbk + static_cast<long long>(n) * sbn];
                const __nv_bfloat16 hi = B[static_cast<long long>(k + 2 * j + 1) * sbk + static_cast<long long>(n) * sbn];
                w[j] = static_cast<uint32_t>(__bfloat16_as_ushort(lo)) | (static_cast<uint32_t>(__bfloat16_as_ushort(hi)) << 16);
            }
            piece = make_uint4(w[0], w[1], w[2], w[3]);
        }
        *reinterpret_cast<uint4*>(sB + kmajor_offset<K>(n, k)) = piece;
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
    // A tile staging: each thread owns units tid + 128 i (i < K/8), loaded in batches of
    // kUB units; the first batch of the next tile is loaded while this tile's MMAs and
    // epilogue run.
    constexpr int kPer = K / 8, kUB = kPer < 8 ? kPer : 8;
    float4 buf[2 * kUB];
    if (blockIdx.x * S::kM < M) {
#pragma unroll
        for (int i = 0; i < kUB; ++i) load_unit<K>(A, lda, M, blockIdx.x * S::kM, tid + 128 * i, buf[2 * i], buf[2 * i + 1]);
    }
    for (int tile = blockIdx.x; tile * S::kM < M && !failed; tile += gridDim.x) {
        const int m0 = tile * S::kM;
#pragma unroll
        for (int b = 0; b < kPer / kUB; ++b) {
            if (b > 0) {
#pragma unroll
                for (int i = 0; i < kUB; ++i)
                    load_unit<K>(A, lda, M, m0, tid + 128 * (b * kUB + i), buf[2 * i], buf[2 * i + 1]);
            }
#pragma unroll
            for (int i = 0; i < kUB; ++i)
                *reinterpret_cast<uint4*>(sA + (tid + 128 * (b * kUB + i)) * 16) = pack8(buf[2 * i], buf[2 * i + 1]);
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
        const int next = tile + gridDim.x;
        if (next * S::kM < M) {
#pragma unroll
            for (int i = 0; i < kUB; ++i) load_unit<K>(A, lda, M, next * S::kM, tid + 128 * i, buf[2 * i], buf[2 * i + 1]);
        }
        const bool ok = mbar_wait(bar, phase, kWaitLimit);
        failed = __syncthreads_or(!ok) != 0;
        phase ^= 1u;
        if (failed) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // Epilogue: each warp takes its 32 rows 16 columns at a time from TMEM (one row
        // per lane), applies bias / relu and passes them through shared memory (the A
        // buffer, free once the MMAs are done; 16-float rows with the float4 slots XOR-ed
        // by (row / 2) mod 4, which keeps both the row-wise writes and the column-wise
        // reads free of bank conflicts), so that a store instruction writes 64 contiguous
        // bytes of each of 8 rows instead of 16 bytes of each of 32.
        float* stg = reinterpret_cast<float*>(sA + S::kStageOffset) + warp * 32 * 16;
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
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float4 o;
                float* f = &o.x;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    float t = __uint_as_float(v[4 * q + e]);
                    if (bias) t += bias[c0 + 4 * q + e];
                    if (relu) t = fmaxf(t, 0.f);
                    f[e] = t;
                }
                *reinterpret_cast<float4*>(stg + lane * 16 + 4 * (q ^ ((lane >> 1) & 3))) = o;
            }
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int rr = 8 * i + (lane >> 2), q = lane & 3;
                const float4 o = *reinterpret_cast<const float4*>(stg + rr * 16 + 4 * (q ^ ((rr >> 1) & 3)));
                const int row = m0 + warp * 32 + rr;
                if (row < M) *reinterpret_cast<float4*>(C + static_cast<long long>(row) * ldc + c0 + 4 * q) = o;
            }
            __syncwarp();
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

// ------------------------------------------------------ layer GEMM, pipelined
//
// The same product for K in {64, 128}, fed by cp.async instead of register-staged
// loads. A stage is a 64-column K-slice of a tile (32 KB of fp32), so that a CTA keeps
// ST - 1 slices (1.5 to 2 tiles) in flight while it converts, multiplies and writes
// back the current tile:
//   - a slice's 16-byte chunks (row r, chunk c) are copied to row r of an fp32 stage
//     at chunk position c XOR (r mod 8) (rows past M are zero-filled by a source size
//     of 0 and read nothing);
//   - the threads convert the stage to bf16 in the canonical K-major layout, piece u
//     (8 k of one row, as in k_gemm_tc) at byte 16 u: the 8 rows a warp phase reads
//     sit at 8 different chunk positions, so the reads are free of bank conflicts,
//     and so are the linear writes;
//   - thread 0 issues the K/16 MMAs, and 8 warps run the epilogue: warp w reads TMEM
//     lanes 32 (w mod 4) (the quarter a warp may access) for column half w / 4.
// One CTA per SM (its shared memory), persistent over the 128-row tiles.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int Pending>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(Pending) : "memory");
}

template <int N, int K, int ST>
struct TcPipeShape {
    static_assert(N == 64 || N == 128, "N is 64 or 128");
    static_assert(K == 64 || K == 128, "K is 64 or 128");
    static_assert(ST >= 2 && ST <= 4, "2 to 4 stages");
    static constexpr int kThreads = 256;
    static constexpr int kM = 128;
    static constexpr int kKS = 64;                        // k columns per stage (a K-slice)
    static constexpr int kSlices = K / kKS;               // stages per tile
    static constexpr int kChunks = kKS / 4;               // 16-byte chunks per fp32 slice row
    static constexpr int kStageBytes = kM * kKS * 4;      // one fp32 K-slice of a tile
    static constexpr int kABytes = kM * K * 2;            // bf16 canonical A
    static constexpr int kBBytes = N * K * 2;             // bf16 canonical B
    static constexpr int kEpiBytes = 8 * 32 * 16 * 4;     // 8 warps x 32 rows x 16 floats
    static constexpr int kSmem = ST * kStageBytes + kABytes + kBBytes + kEpiBytes + 64 + 128;
    static constexpr int kCols = N;
};

template <int N, int K, int ST>
__global__ void __launch_bounds__(256, 1) k_gemm_tc_pipe(int M, const float* __restrict__ A, int lda,
                                                      const __nv_bfloat16* __restrict__ B, int sbk, int sbn,
                                                      const float* __restrict__ bias, int relu, float* __restrict__ C,
                                                      int ldc, unsigned int* __restrict__ err) {
    using S = TcPipeShape<N, K, ST>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    unsigned char* stages = smem;
    unsigned char* sA = smem + ST * S::kStageBytes;
    unsigned char* sB = sA + S::kABytes;
    float* sE = reinterpret_cast<float*>(sB + S::kBBytes);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(sB + S::kBBytes + S::kEpiBytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tiles = (M + S::kM - 1) / S::kM;

    // Unit j of this CTA is K-slice j mod kSlices of its tile j / kSlices; it goes to
    // stage j mod ST (an empty group past the last tile keeps the group count uniform).
    const int t0 = blockIdx.x;
    auto issue = [&](int j) {
        const int tile = t0 + (j / S::kSlices) * gridDim.x, k0 = (j % S::kSlices) * S::kKS;
        if (tile < tiles) {
            const int m0 = tile * S::kM;
            const uint32_t base = smem_u32(stages + (j % ST) * S::kStageBytes);
#pragma unroll 4
            for (int q = tid; q < S::kM * S::kChunks; q += S::kThreads) {
                const int r = q / S::kChunks, c = q - r * S::kChunks;
                const bool live = m0 + r < M;
                const float* src = A + static_cast<long long>(live ? m0 + r : 0) * lda + k0 + c * 4;
                cp_async16(base + r * (S::kKS * 4) + ((c ^ (r & 7)) << 4), src, live ? 16 : 0);
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int j = 0; j < ST - 1; ++j) issue(j);

    // B pieces as in k_gemm_tc
#pragma unroll 4
    for (int e = tid; e < N * (K / 8); e += S::kThreads) {
        const int n = e % N, k = (e / N) * 8;
        uint4 piece;
        if (sbk == 1) {
            piece = *reinterpret_cast<const uint4*>(B + static_cast<long long>(n) * sbn + k);
        } else {
            uint32_t w[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const __nv_bfloat16 lo = B[static_cast<long long>(k + 2 * j) * sbk + static_cast<long long>(n) * sbn];
                const __nv_bfloat16 hi = B[static_cast<long long>(k + 2 * j + 1) * sbk + static_cast<long long>(n) * sbn];
                w[j] = static_cast<uint32_t>(__bfloat16_as_ushort(lo)) | (static_cast<uint32_t>(__bfloat16_as_ushort(hi)) << 16);
            }
            piece = make_uint4(w[0], w[1], w[2], w[3]);
        }
        *reinterpret_cast<uint4*>(sB + kmajor_offset<K>(n, k)) = piece;
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
    const int quarter = warp & 3, half = warp >> 2;
    float* stg = sE + warp * 32 * 16;
    int i = 0;
    for (int tile = t0; tile < tiles; tile += gridDim.x, ++i) {
        const int m0 = tile * S::kM;
#pragma unroll
        for (int sl = 0; sl < S::kSlices; ++sl) {
            const int j = i * S::kSlices + sl;
            // the stage converted last takes unit j + ST - 1
            issue(j + ST - 1);
            cp_async_wait<ST - 1>();
            __syncthreads();
            const unsigned char* st = stages + (j % ST) * S::kStageBytes;
            // slice pieces (8 k of one row) numbered as in unit_row_k over the slice's
            // kKS columns; piece (r, k) of the tile lands at kmajor_offset<K>(r, k)
#pragma unroll
            for (int v = 0; v < S::kKS / 16; ++v) {
                const int u = tid + S::kThreads * v;
                int r, k;
                unit_row_k<S::kKS>(u, r, k);
                const unsigned char* row = st + r * (S::kKS * 4);
                const float4 lo = *reinterpret_cast<const float4*>(row + (((k >> 2) ^ (r & 7)) << 4));
                const float4 hi = *reinterpret_cast<const float4*>(row + ((((k >> 2) + 1) ^ (r & 7)) << 4));
                *reinterpret_cast<uint4*>(sA + kmajor_offset<K>(r, sl * S::kKS + k)) = pack8(lo, hi);
            }
            // the next slice's issue reuses the stage just read
            if (sl + 1 < S::kSlices) __syncthreads();
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int k16 = 0; k16 < K / 16; ++k16) {
                const uint64_t da = smem_desc(a_base + k16 * 256, 128, (K / 8) * 128);
                const uint64_t db = smem_desc(b_base + k16 * 256, 128, (K / 8) * 128);
                const uint32_t accumulate = k16 > 0 ? 1u : 0u;
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
#pragma unroll
        for (int c0 = half * (N / 2); c0 < (half + 1) * (N / 2); c0 += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + static_cast<uint32_t>(c0)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float4 o;
                float* f = &o.x;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    float t = __uint_as_float(v[4 * q + e]);
                    if (bias) t += bias[c0 + 4 * q + e];
                    if (relu) t = fmaxf(t, 0.f);
                    f[e] = t;
                }
                *reinterpret_cast<float4*>(stg + lane * 16 + 4 * (q ^ ((lane >> 1) & 3))) = o;
            }
            __syncwarp();
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int rr = 8 * j + (lane >> 2), q = lane & 3;
                const float4 o = *reinterpret_cast<const float4*>(stg + rr * 16 + 4 * (q ^ ((rr >> 1) & 3)));
                const int row = m0 + quarter * 32 + rr;
                if (row < M) *reinterpret_cast<float4*>(C + static_cast<long long>(row) * ldc + c0 + 4 * q) = o;
            }
            __syncwarp();
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (failed) {
        // the MMA may still be writing TMEM: wait for it (bounded) before freeing
        if (tid == 0) atomicOr(err, 1u);
        mbar_wait(bar, phase ^ 1u, kWaitLimit);
    }
    cp_async_wait<0>();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::kCols));
}

// ------------------------------------------------------------ weight gradient
//
// part[z][f * 64 + n] = sum over the nodes k of slice z of X[k][f] dZ[k][n]: the
// weight gradient dW = X^T dZ of a 128-wide layer input (f < 128) against the 64
// channels of dZ, over the node slice [z chunk, min(rows, (z + 1) chunk)). The fixed
// slices are summed afterwards in slice order, so the result does not depend on
// timing.
//
// The node index is the MMA's K: A = X^T (128 x nodes) and B = dZ (nodes x 64) are
// both MN-major, so one 32-byte piece of a row of X or dZ (8 features or channels of
// one node) becomes one 16-byte core row. A 64-node bf16 buffer holds A in 16 KB (core
// (feature block i, node block j) at j 2048 + i 128) and B in 8 KB (j 1024 + i 128);
// with unit u = thread + 256 v, piece u lands at byte u * 16 (linear, no bank
// conflicts): X piece u is node block u / 128, feature block (u / 8) mod 16, node u mod
// 8; dZ piece u is node block u / 64, channel block (u / 8) mod 8, node u mod 8.
// Each 64-node stage of X (32 KB) and dZ (16 KB) is copied by cp.async as 16-byte
// chunks into one of ST fp32 stages (chunk c of node row k at position c XOR (k mod 8);
// nodes past the slice are zero-filled), converted into one of two bf16 MN-major
// buffers (the layout above) and multiplied; ST - 1
// stages are in flight while the current one is converted. 256 threads, one CTA per
// SM; the epilogue splits TMEM by lane quarter (warp mod 4) and column half (warp / 4).
template <int ST>
struct WgPipeShape {
    static constexpr int kThreads = 256;
    static constexpr int kNodes = 64;
    static constexpr int kXBytes = kNodes * 128 * 4;      // fp32 X rows of a stage
    static constexpr int kZBytes = kNodes * 64 * 4;       // fp32 dZ rows of a stage
    static constexpr int kStage = kXBytes + kZBytes;
    static constexpr int kABytes = 128 * kNodes * 2;      // bf16 X^T
    static constexpr int kBBytes = kNodes * 64 * 2;       // bf16 dZ
    static constexpr int kBuf = kABytes + kBBytes;
    static constexpr int kSmem = ST * kStage + 2 * kBuf + 64 + 128;
    static constexpr int kCols = 64;
};

template <int F, int ST>
__global__ void __launch_bounds__(256) k_wgrad_tc_pipe(int rows, int chunk, const float* __restrict__ X, int ldx,
                                                       const float* __restrict__ dZ, float* __restrict__ part,
                                                       unsigned int* __restrict__ err) {
    static_assert(F == 128, "the layer input is 128 wide");
    using S = WgPipeShape<ST>;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    unsigned char* stages = smem;
    unsigned char* bufs = smem + ST * S::kStage;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(bufs + 2 * S::kBuf);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int k0 = blockIdx.x * chunk, k1 = min(rows, k0 + chunk);
    const int nst = k1 > k0 ? (k1 - k0 + S::kNodes - 1) / S::kNodes : 0;
    float* out = part + static_cast<long long>(blockIdx.x) * (128 * 64);
    if (nst == 0) {
        for (int e = tid; e < 128 * 64; e += S::kThreads) out[e] = 0.f;
        return;
    }
    auto issue = [&](int st) {
        if (st < nst) {
            const int nb = k0 + st * S::kNodes;
            const uint32_t xs = smem_u32(stages + (st % ST) * S::kStage), zs = xs + S::kXBytes;
#pragma unroll 4
            for (int q = tid; q < S::kNodes * 32; q += S::kThreads) {   // X: 32 chunks per node
                const int k = q >> 5, c = q & 31;
                const bool live = nb + k < k1;
                const float* src = X + static_cast<long long>(live ? nb + k : 0) * ldx + c * 4;
                cp_async16(xs + k * 512 + ((c ^ (k & 7)) << 4), src, live ? 16 : 0);
            }
#pragma unroll 4
            for (int q = tid; q < S::kNodes * 16; q += S::kThreads) {   // dZ: 16 chunks per node
                const int k = q >> 4, c = q & 15;
                const bool live = nb + k < k1;
                const float* src = dZ + static_cast<long long>(live ? nb + k : 0) * 64 + c * 4;
                cp_async16(zs + k * 256 + ((c ^ (k & 7)) << 4), src, live ? 16 : 0);
            }
        }
        cp_async_commit();
    };
#pragma unroll
    for (int st = 0; st < ST - 1; ++st) issue(st);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(S::kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar + 1)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;
    const uint32_t idesc = instr_desc_bf16_mn(128, 64);
    bool failed = false;
    int issued = 0;
    for (int st = 0; st < nst; ++st) {
        const int b = st & 1;
        issue(st + ST - 1);
        cp_async_wait<ST - 1>();
        // the MMAs of stage st - 2 read buffer b: wait for their commit
        bool ok = true;
        if (st >= 2) ok = mbar_wait(smem_u32(mbar + b), static_cast<uint32_t>(((st - 2) >> 1) & 1), kWaitLimit);
        failed = __syncthreads_or(!ok) != 0;
        if (failed) break;
        const unsigned char* xs = stages + (st % ST) * S::kStage;
        const unsigned char* zs = xs + S::kXBytes;
        unsigned char* sA = bufs + b * S::kBuf;
        unsigned char* sB = sA + S::kABytes;
#pragma unroll
        for (int v = 0; v < 4; ++v) {   // X^T pieces
            const int u = tid + S::kThreads * v, k = (u >> 7) * 8 + (u & 7), c = ((u >> 3) & 15) * 2;
            const unsigned char* row = xs + k * 512;
            const float4 lo = *reinterpret_cast<const float4*>(row + ((c ^ (k & 7)) << 4));
            const float4 hi = *reinterpret_cast<const float4*>(row + (((c + 1) ^ (k & 7)) << 4));
            *reinterpret_cast<uint4*>(sA + u * 16) = pack8(lo, hi);
        }
#pragma unroll
        for (int v = 0; v < 2; ++v) {   // dZ pieces
            const int u = tid + S::kThreads * v, k = (u >> 6) * 8 + (u & 7), c = ((u >> 3) & 7) * 2;
            const unsigned char* row = zs + k * 256;
            const float4 lo = *reinterpret_cast<const float4*>(row + ((c ^ (k & 7)) << 4));
            const float4 hi = *reinterpret_cast<const float4*>(row + (((c + 1) ^ (k & 7)) << 4));
            *reinterpret_cast<uint4*>(sB + u * 16) = pack8(lo, hi);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
#pragma unroll
            for (int s = 0; s < S::kNodes / 16; ++s) {
                const uint64_t da = smem_desc(a0 + s * 2 * 2048, 2048, 128);
                const uint64_t db = smem_desc(b0 + s * 2 * 1024, 1024, 128);
                const uint32_t accumulate = (st > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(mbar + b))
                         : "memory");
        }
        issued = st + 1;
    }
    if (!failed) {
        const int last = nst - 1;
        const bool ok = mbar_wait(smem_u32(mbar + (last & 1)), static_cast<uint32_t>((last >> 1) & 1), kWaitLimit);
        failed = __syncthreads_or(!ok) != 0;
    }
    if (!failed) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int quarter = warp & 3, half = warp >> 2;
        float* row = out + (quarter * 32 + lane) * 64;
#pragma unroll
        for (int c0 = half * 32; c0 < half * 32 + 32; c0 += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + static_cast<uint32_t>(c0)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 4; ++q)
                *reinterpret_cast<float4*>(row + c0 + 4 * q) =
                    make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]), __uint_as_float(v[4 * q + 2]),
                                __uint_as_float(v[4 * q + 3]));
        }
    } else {
        if (tid == 0) atomicOr(err, 1u);
        for (int b = 0; b < 2; ++b) {
            const int st = issued - 1 - ((issued - 1 - b) & 1);   // last stage committed on buffer b
            if (st >= 0 && (st & 1) == b) mbar_wait(smem_u32(mbar + b), static_cast<uint32_t>((st >> 1) & 1), kWaitLimit);
        }
    }
    cp_async_wait<0>();
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::kCols));
}

}  // namespace tc
}  // namespace b200
