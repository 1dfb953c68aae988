// Reduced-precision centroid probe (the precision form of GetClustersAccessOrderIVF,
// searcher.hpp:181-215, for flat and two-level indexes).
//
// The centroid scores come from one tensor-core GEMM per batch (pdxg_gemm.cu, BF16 or
// FP8-E4M3 operands, FP32 accumulation, epilogue |c|^2 - 2 q.c: the squared L2 distance up to
// the query's own |q|^2). Per query, probe_select_kernel takes the m' = ceil(1.1 nprobe)
// centroids with the smallest scores (the probe list widened by 10%), rescores them in FP32
// with the reference's own probe arithmetic (Horizontal, avx2_computers.hpp:47-98: 8 FMA lanes,
// pairwise double reduction) and keeps the nprobe nearest by (distance, id). A centroid the
// reduced-precision score pushes out of the widened list is the probe-set error of this form;
// whenever the exact nprobe nearest are all inside it, the visit order equals the reference's.
#include <cstdint>
#include <cuda_runtime.h>

#include "pdxg_block.cuh"
#include "pdxg_common.cuh"

namespace pdxg {

// |c|^2 of each row (FP32 result of an FP64 sum); one warp per row.
__global__ void row_sq_kernel(const float* __restrict__ x, uint32_t n, uint32_t d, float* __restrict__ out) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (row >= n) return;
    double s = 0.0;
    for (uint32_t i = lane; i < d; i += 32) {
        const double v = x[(size_t)row * d + i];
        s += v * v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[row] = (float)s;
}

constexpr int kSelectThreads = 128;

// Shared memory of one probe CTA: query, one key per centroid, candidates, sort keys.
size_t probe_select_smem(uint32_t d, uint32_t n1, uint32_t cand_cap, uint32_t sort_cap) {
    return ((size_t)d * 4 + 15) / 16 * 16 + (size_t)((n1 + 3) & ~3u) * 4 + (size_t)cand_cap * 4 + (size_t)sort_cap * 8;
}

// Order-preserving map of a float onto uint32 (negative scores included).
__device__ __forceinline__ uint32_t float_key(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// One CTA per query: widened candidate list from the approximate scores, FP32 rescore, the
// nprobe nearest sorted by (distance, id) into order[q * stride ..], count[q].
__global__ void __launch_bounds__(kSelectThreads) probe_select_kernel(const __grid_constant__ ProbeParams pp) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ Scalars s;
    const uint32_t q = blockIdx.x;
    const uint32_t n1 = pp.nclusters, d = pp.d;
    float* qf = reinterpret_cast<float*>(smem);                                         // [d]
    uint32_t* keys = reinterpret_cast<uint32_t*>(smem + ((size_t)d * 4 + 15) / 16 * 16);  // [n1]
    uint32_t* cand = keys + ((n1 + 3) & ~3u);                                            // [cand_cap]
    uint64_t* sortb = reinterpret_cast<uint64_t*>(cand + pp.cand_cap);                   // [sort_cap]
    const uint32_t np = pp.q_nprobe ? __ldg(pp.q_nprobe + q) : pp.nprobe;
    const uint32_t m = np < n1 ? np : n1;
    uint32_t mw = (uint32_t)ceilf(__fmul_rn(1.1f, (float)m));
    if (mw > n1) mw = n1;
    const float* src = pp.queries + (size_t)q * d;
    for (uint32_t i = threadIdx.x; i < d; i += kSelectThreads) qf[i] = __ldg(src + i);
    const float* sc = pp.scores + (size_t)q * pp.ld_scores;
    for (uint32_t c = threadIdx.x; c < n1; c += kSelectThreads) keys[c] = float_key(__ldg(sc + c));
    __syncthreads();
    // the mw smallest approximate scores: below the mw-th key, then ties in id order
    uint32_t kth, less;
    block_radix_select<kSelectThreads>(keys, n1, mw, s, kth, less);
    const uint32_t nl = block_compact<kSelectThreads>(
        n1, [&](uint32_t, uint32_t v) { return keys[v] < kth; }, [](uint32_t i) { return i; }, cand, s);
    const uint32_t nt = block_compact<kSelectThreads>(
        n1, [&](uint32_t, uint32_t v) { return keys[v] == kth; }, [](uint32_t i) { return i; }, cand + nl, s);
    (void)nt;
    // FP32 rescore of the candidates, 8 threads each (LevelOps::probe's arithmetic)
    const uint32_t N = next_pow2(mw);
    const uint32_t sub = threadIdx.x & 7;
    for (uint32_t base = 0; base < N; base += kSelectThreads / 8) {
        const uint32_t i = base + (threadIdx.x >> 3);
        const bool active = i < mw;
        const uint32_t c = active ? cand[i] : 0u;
        const float dd = horiz_f32_group8(qf, pp.centroids + (size_t)c * d, d, sub, active);
        if (sub == 0 && i < N) sortb[i] = active ? (((uint64_t)__float_as_uint(dd) << 32) | c) : ~0ull;
    }
    __syncthreads();
    block_bitonic_sort<kSelectThreads>(sortb, N);
    for (uint32_t i = threadIdx.x; i < m; i += kSelectThreads) pp.order[(size_t)q * pp.stride + i] = (uint32_t)sortb[i];
    if (threadIdx.x == 0) {
        pp.count[q] = m;
        if (pp.stats) {
            // the approximate scores read each centroid once per query (score_bytes per
            // centroid), the rescore the widened list in FP32
            const unsigned long long b = (unsigned long long)n1 * pp.score_bytes + (unsigned long long)mw * d * 4u;
            atomicAdd(pp.stats + 8, b);
            atomicAdd(pp.stats, b);
        }
    }
}

// Exact probe of a flat index for a whole batch, ahead of the scan (LevelOps::probe's result,
// searcher.hpp:181-215): FP32 distances to every centroid in the AVX2 Horizontal order, the
// nprobe nearest by (distance, id), ascending. One CTA per query. The scan kernel then needs no
// per-centroid arrays in shared memory, only per-vector ones.
template <int T>
__global__ void __launch_bounds__(T) probe_exact_kernel(const __grid_constant__ ProbeParams pp) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ Scalars s;
    const uint32_t q = blockIdx.x;
    const uint32_t n1 = pp.nclusters, d = pp.d;
    float* qf = reinterpret_cast<float*>(smem);                                         // [d]
    uint32_t* keys = reinterpret_cast<uint32_t*>(smem + ((size_t)d * 4 + 15) / 16 * 16);  // [n1]
    uint32_t* cand = keys + ((n1 + 3) & ~3u);                                            // [cand_cap]
    uint64_t* sortb = reinterpret_cast<uint64_t*>(cand + pp.cand_cap);                   // [sort_cap]
    const uint32_t np = pp.q_nprobe ? __ldg(pp.q_nprobe + q) : pp.nprobe;
    const uint32_t m = np < n1 ? np : n1;
    const float* src = pp.queries + (size_t)q * d;
    for (uint32_t i = threadIdx.x; i < d; i += T) qf[i] = __ldg(src + i);
    __syncthreads();
    const uint32_t sub = threadIdx.x & 7;
    for (uint32_t base = 0; base < n1; base += T / 8) {
        const uint32_t c = base + (threadIdx.x >> 3);
        const bool active = c < n1;
        const float dd = horiz_f32_group8(qf, pp.centroids + (size_t)(active ? c : 0) * d, d, sub, active);
        if (active && sub == 0) keys[c] = __float_as_uint(dd);
    }
    __syncthreads();
    if (m < n1) {
        uint32_t kth, less;
        block_radix_select<T>(keys, n1, m, s, kth, less);
        const uint32_t nl = block_compact<T>(
            n1, [&](uint32_t, uint32_t v) { return keys[v] < kth; }, [](uint32_t i) { return i; }, cand, s);
        block_compact<T>(n1, [&](uint32_t, uint32_t v) { return keys[v] == kth; }, [](uint32_t i) { return i; },
                         cand + nl, s);
    } else {
        for (uint32_t i = threadIdx.x; i < n1; i += T) cand[i] = i;  // every centroid: sort them all
        __syncthreads();
    }
    const uint32_t N = next_pow2(m);
    for (uint32_t i = threadIdx.x; i < N; i += T)
        sortb[i] = (i < m) ? (((uint64_t)keys[cand[i]] << 32) | cand[i]) : ~0ull;
    __syncthreads();
    block_bitonic_sort<T>(sortb, N);
    for (uint32_t i = threadIdx.x; i < m; i += T) pp.order[(size_t)q * pp.stride + i] = (uint32_t)sortb[i];
    if (threadIdx.x == 0) {
        pp.count[q] = m;
        if (pp.stats) {
            const unsigned long long b = (unsigned long long)n1 * d * 4u;
            atomicAdd(pp.stats + 8, b);
            atomicAdd(pp.stats, b);
        }
    }
}

cudaError_t launch_probe_exact(const ProbeParams& pp, cudaStream_t st) {
    const size_t smem = probe_select_smem(pp.d, pp.nclusters, pp.cand_cap, pp.sort_cap);
    // large levels sort thousands of keys per query: more threads per CTA
    if (pp.nclusters > 2048) {
        cudaError_t e = cudaFuncSetAttribute(probe_exact_kernel<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        probe_exact_kernel<512><<<pp.nq, 512, smem, st>>>(pp);
    } else {
        cudaError_t e = cudaFuncSetAttribute(probe_exact_kernel<kSelectThreads>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        probe_exact_kernel<kSelectThreads><<<pp.nq, kSelectThreads, smem, st>>>(pp);
    }
    return cudaGetLastError();
}

cudaError_t launch_row_sq(const float* x, uint32_t n, uint32_t d, float* out, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    row_sq_kernel<<<(n * 32 + 255) / 256, 256, 0, st>>>(x, n, d, out);
    return cudaGetLastError();
}


cudaError_t launch_probe_select(const ProbeParams& pp, cudaStream_t st) {
    const size_t smem = probe_select_smem(pp.d, pp.nclusters, pp.cand_cap, pp.sort_cap);
    cudaError_t e = cudaFuncSetAttribute(probe_select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    probe_select_kernel<<<pp.nq, kSelectThreads, smem, st>>>(pp);
    return cudaGetLastError();
}

}  // namespace pdxg
