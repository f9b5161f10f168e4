// Stable transpose of a device CSR matrix on the device: the row of A^T for
// column j lists the entries of column j in ascending row order (ascending
// source position), which is the order of the host counting sort the reference
// uses to convert between its CSC model and CSR (c/src/sk_solve.c csc_mv /
// csc_tmv visit entries in that order). Applied to a CSC matrix (= the CSR of
// A^T) it yields A's CSR with each row's columns ascending, the order of the
// reference's scatter loops.
//
// Method: an LSD radix sort of the entry positions keyed by column (8-bit
// digits, as many passes as the column count needs). Each pass counts digits
// per warp tile of 2048 entries, turns the (digit, tile) counts into offsets with
// a device exclusive scan, and scatters each tile in order, ranking equal digits
// inside a group of 32 with __match_any_sync, so equal keys keep their order.
// Row indices come from a binary search of the entry position in the row
// offsets. Everything is O(nnz) device work; the host sees only the result.
#include "engine.cuh"

namespace b200 {

namespace {

constexpr int kRadixTile = 2048;   // entries per warp tile
constexpr int kScanChunk = 2048;   // elements per scan block (8 per thread)

// Exclusive scan, phase 1: per block of kScanChunk, local exclusive prefixes
// and the block total.
__global__ void k_scan_local(const int* __restrict__ in, int count, int* __restrict__ out, int* __restrict__ sums) {
    __shared__ int warp_tot[kThreads / 32];
    const int base = blockIdx.x * kScanChunk + threadIdx.x * 8;
    int v[8], s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        v[k] = base + k < count ? in[base + k] : 0;
        s += v[k];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    int before = 0;
    for (int i = 0; i < w; ++i) before += warp_tot[i];
    int run = before + incl - s;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        if (base + k < count) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == kThreads - 1) sums[blockIdx.x] = before + incl;
}

// Phase 2: exclusive scan of the block totals in one block (chunks with carry);
// total written to *total.
__global__ void k_scan_sums(int* __restrict__ sums, int nblocks, int* __restrict__ total) {
    __shared__ int buf[1024];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nblocks; b0 += 1024) {
        const int i = b0 + threadIdx.x;
        const int v = i < nblocks ? sums[i] : 0;
        buf[threadIdx.x] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            const int t = threadIdx.x >= o ? buf[threadIdx.x - o] : 0;
            __syncthreads();
            buf[threadIdx.x] += t;
            __syncthreads();
        }
        if (i < nblocks) sums[i] = carry + buf[threadIdx.x] - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += buf[1023];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan_add(int* __restrict__ out, int count, const int* __restrict__ sums) {
    const int add = sums[blockIdx.x];
    const int base = blockIdx.x * kScanChunk;
    for (int i = threadIdx.x; i < kScanChunk; i += blockDim.x)
        if (base + i < count) out[base + i] += add;
}

// out[0..count) = exclusive prefix sums of in, out[count] = the total.
// tmp holds at least ceil(count / kScanChunk) ints.
void exclusive_scan(const int* in, int count, int* out, int* tmp, cudaStream_t st) {
    const int nblocks = std::max(1, (count + kScanChunk - 1) / kScanChunk);
    k_scan_local<<<nblocks, kThreads, 0, st>>>(in, count, out, tmp);
    k_scan_sums<<<1, 1024, 0, st>>>(tmp, nblocks, out + count);
    k_scan_add<<<nblocks, kThreads, 0, st>>>(out, count, tmp);
}

// Row of every entry: the r with ptr[r] <= p < ptr[r + 1].
__global__ void k_entry_rows(int rows, int nnz, const int* __restrict__ ptr, int* __restrict__ rowid) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += blockDim.x * gridDim.x) {
        int lo = 0, hi = rows;   // ptr[lo] <= p < ptr[hi]
        while (hi - lo > 1) {
            const int mid = lo + (hi - lo) / 2;
            if (ptr[mid] <= p) lo = mid; else hi = mid;
        }
        rowid[p] = lo;
    }
}

// Column counts and the initial (key, position) arrays; an index outside
// [0, cols) sets *bad and is not counted.
__global__ void k_count_keys(int nnz, int cols, const int* __restrict__ idx, int* __restrict__ cnt,
                             int* __restrict__ keys, int* __restrict__ pos, unsigned int* __restrict__ bad) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += blockDim.x * gridDim.x) {
        const int j = idx[p];
        if (j < 0 || j >= cols) {
            atomicOr(bad, 1u);
            keys[p] = 0;
        } else {
            atomicAdd(&cnt[j], 1);
            keys[p] = j;
        }
        pos[p] = p;
    }
}

__global__ void k_radix_hist(int nnz, const int* __restrict__ keys, int shift, int ntiles, int* __restrict__ hist) {
    __shared__ int cnt[kWarps][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int tile = blockIdx.x * kWarps + w;
    for (int d = lane; d < 256; d += 32) cnt[w][d] = 0;
    __syncwarp();
    if (tile >= ntiles) return;
    const int begin = tile * kRadixTile, end = min(nnz, begin + kRadixTile);
    for (int p = begin + lane; p < end; p += 32) atomicAdd(&cnt[w][(keys[p] >> shift) & 255], 1);
    __syncwarp();
    for (int d = lane; d < 256; d += 32) hist[d * ntiles + tile] = cnt[w][d];
}

// Stable scatter of one tile: groups of 32 in order; equal digits in a group
// ranked by lane, after the counts of earlier groups of the same tile.
__global__ void k_radix_scatter(int nnz, const int* __restrict__ kin, const int* __restrict__ vin, int shift,
                                int ntiles, const int* __restrict__ offs, int* __restrict__ kout,
                                int* __restrict__ vout) {
    __shared__ int run[kWarps][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int tile = blockIdx.x * kWarps + w;
    for (int d = lane; d < 256; d += 32) run[w][d] = 0;
    __syncwarp();
    if (tile >= ntiles) return;
    const int begin = tile * kRadixTile, end = min(nnz, begin + kRadixTile);
    const unsigned below = (1u << lane) - 1u;
    for (int g = begin; g < end; g += 32) {
        const int p = g + lane;
        const bool live = p < end;
        int key = 0, v = 0, d = 256;
        if (live) {
            key = kin[p];
            v = vin[p];
            d = (key >> shift) & 255;
        }
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & below);
        int at = 0;
        if (live) at = offs[d * ntiles + tile] + run[w][d] + rank;
        __syncwarp();
        if (live && rank == 0) run[w][d] += __popc(peers);
        __syncwarp();
        if (live) {
            kout[at] = key;
            vout[at] = v;
        }
    }
}

__global__ void k_gather_transpose(int nnz, const int* __restrict__ perm, const int* __restrict__ rowid,
                                   const double* __restrict__ val, int* __restrict__ tidx, double* __restrict__ tval) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += blockDim.x * gridDim.x) {
        const int p = perm[k];
        tidx[k] = rowid[p];
        tval[k] = val[p];
    }
}

int blocks_for(long long count) {
    return static_cast<int>(std::max<long long>(1, std::min<long long>((count + kThreads - 1) / kThreads, 148LL * 32)));
}

}  // namespace

int device_transpose(int rows, int cols, int nnz, const int* ptr, const int* idx, const double* val, int* tptr,
                     int* tidx, double* tval, cudaStream_t st) {
    if (rows < 0 || cols < 0 || nnz < 0) return fail_msg("invalid matrix dimensions");
    const int ntiles = std::max(1, (nnz + kRadixTile - 1) / kRadixTile);
    const long long hist_len = 256LL * ntiles;
    const long long scan_tmp = std::max<long long>(cols + 1, hist_len) / kScanChunk + 2;
    auto al = [](long long b) { return (b + 255) / 256 * 256; };
    const long long n4 = al(4LL * std::max(nnz, 1));
    DevBuf buf;
    if (buf.alloc(static_cast<size_t>(5 * n4 + al(4LL * (cols + 1)) + 2 * al(4LL * (hist_len + 1)) + al(4 * scan_tmp) +
                                      256),
                  "cudaMalloc transpose scratch"))
        return -1;
    char* p = buf.as<char>();
    auto take = [&](long long b) { char* r = p; p += b; return reinterpret_cast<int*>(r); };
    int *rowid = take(n4), *k0 = take(n4), *v0 = take(n4), *k1 = take(n4), *v1 = take(n4);
    int* cnt = take(al(4LL * (cols + 1)));
    int* hist = take(al(4LL * (hist_len + 1)));
    int* offs = take(al(4LL * (hist_len + 1)));
    int* tmp = take(al(4 * scan_tmp));
    unsigned int* bad = reinterpret_cast<unsigned int*>(take(256));
    B200_TRY(cudaMemsetAsync(cnt, 0, 4LL * (cols + 1), st), "transpose counts");
    B200_TRY(cudaMemsetAsync(bad, 0, 4, st), "transpose flag");
    if (nnz > 0) {
        k_entry_rows<<<blocks_for(nnz), kThreads, 0, st>>>(rows, nnz, ptr, rowid);
        k_count_keys<<<blocks_for(nnz), kThreads, 0, st>>>(nnz, cols, idx, cnt, k0, v0, bad);
    }
    exclusive_scan(cnt, cols, tptr, tmp, st);
    unsigned int h_bad = 0;
    B200_TRY(cudaMemcpyAsync(&h_bad, bad, 4, cudaMemcpyDeviceToHost, st), "transpose check");
    B200_TRY(cudaStreamSynchronize(st), "transpose check");
    if (h_bad) return fail_msg("matrix index out of range");
    if (nnz == 0) return 0;
    int bits = 0;
    while (bits < 31 && (1LL << bits) < cols) ++bits;
    const int passes = std::max(1, (bits + 7) / 8);
    const int grid = (ntiles + kWarps - 1) / kWarps;
    int *ki = k0, *vi = v0, *ko = k1, *vo = v1;
    for (int pass = 0; pass < passes; ++pass) {
        const int shift = 8 * pass;
        k_radix_hist<<<grid, kThreads, 0, st>>>(nnz, ki, shift, ntiles, hist);
        exclusive_scan(hist, static_cast<int>(hist_len), offs, tmp, st);
        k_radix_scatter<<<grid, kThreads, 0, st>>>(nnz, ki, vi, shift, ntiles, offs, ko, vo);
        std::swap(ki, ko);
        std::swap(vi, vo);
    }
    k_gather_transpose<<<blocks_for(nnz), kThreads, 0, st>>>(nnz, vi, rowid, val, tidx, tval);
    B200_TRY(cudaGetLastError(), "device transpose");
    B200_TRY(cudaStreamSynchronize(st), "device transpose");
    return 0;
}

}  // namespace b200
