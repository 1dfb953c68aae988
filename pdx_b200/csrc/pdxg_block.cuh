// Block-level primitives shared by the search kernels: per-CTA scalars, block sum,
// order-preserving ballot compaction, exact radix select, bitonic sort, and the F32 distance
// helpers that reproduce the reference's AVX2 reduction order.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "pdxg_common.cuh"

namespace pdxg {

struct Scalars {
    uint32_t warp[32];
    uint32_t hist[256];
    uint32_t sc[4];
    uint32_t hsize;
    uint32_t top_slot;
    float top;
    uint32_t query;
    uint32_t n_order;
    unsigned long long bytes[6];  // algorithmic bytes of the current query by phase (stats only)
    unsigned long long visits;
    unsigned long long merged;
    unsigned long long cycles[3];  // stats only: top-level search, L1 Start, rest of the query
};

// Phases of the algorithmic-byte accounting (stats[3 + phase]).
enum Phase { kTopLevel = 0, kStart = 1, kWarmup = 2, kSurvivorH = 3, kSurvivorV = 4, kProbe = 5 };

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ uint32_t warp_id() { return threadIdx.x >> 5; }

template <int T>
__device__ __forceinline__ uint32_t block_sum(uint32_t x, Scalars& s) {
    constexpr int NW = T / 32;
    x = __reduce_add_sync(0xffffffffu, x);
    if (lane_id() == 0) s.warp[warp_id()] = x;
    __syncthreads();
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) tot += s.warp[w];
    __syncthreads();
    return tot;
}

// Order-preserving compaction of i in [0, n) with pred(i): out[rank] = val(i).
// In-place use (out aliasing the array val() reads) is safe: every element of a chunk is
// read before the chunk's writes, and writes never reach past the current chunk.
template <int T, class Pred, class Val>
__device__ uint32_t block_compact(uint32_t n, Pred pred, Val val, uint32_t* out, Scalars& s) {
    constexpr int NW = T / 32;
    const uint32_t lane = lane_id(), warp = warp_id();
    uint32_t total = 0;
    for (uint32_t c0 = 0; c0 < n; c0 += T) {
        const uint32_t i = c0 + threadIdx.x;
        const bool in = i < n;
        const uint32_t v = in ? val(i) : 0u;
        const bool p = in && pred(i, v);
        const unsigned b = __ballot_sync(0xffffffffu, p);
        if (lane == 0) s.warp[warp] = __popc(b);
        __syncthreads();
        uint32_t off = total, ctot = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const uint32_t c = s.warp[w];
            off += (w < (int)warp) ? c : 0u;
            ctot += c;
        }
        if (p) out[off + __popc(b & ((1u << lane) - 1u))] = v;
        total += ctot;
        __syncthreads();
    }
    return total;
}

// Exact selection: kth = the m-th smallest key (1 <= m <= n), less = #keys < kth.
template <int T>
__device__ void block_radix_select(const uint32_t* keys, uint32_t n, uint32_t m, Scalars& s,
                                   uint32_t& kth, uint32_t& less) {
    uint32_t prefix = 0, mask = 0, rem = m, acc_less = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += T) s.hist[i] = 0;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += T) {
            const uint32_t k = keys[i];
            if ((k & mask) == prefix) atomicAdd(&s.hist[(k >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            const uint32_t lane = lane_id();
            uint32_t loc[8], sum = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                loc[j] = s.hist[lane * 8 + j];
                sum += loc[j];
            }
            uint32_t incl = sum;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= (uint32_t)off) incl += t;
            }
            const uint32_t excl = incl - sum;
            const bool mine = excl < rem && rem <= incl;
            const unsigned bm = __ballot_sync(0xffffffffu, mine);
            if (lane == (uint32_t)(__ffs(bm) - 1)) {
                uint32_t c = excl;
                int b = 0;
                for (; b < 7; ++b) {
                    if (c + loc[b] >= rem) break;
                    c += loc[b];
                }
                s.sc[0] = lane * 8 + b;
                s.sc[1] = c;
            }
        }
        __syncthreads();
        const uint32_t bin = s.sc[0], cum = s.sc[1];
        prefix |= bin << shift;
        mask |= 0xFFu << shift;
        rem -= cum;
        acc_less += cum;
        __syncthreads();
    }
    kth = prefix;
    less = acc_less;
}

// Ascending bitonic sort of N (power of two) u64 keys in shared memory.
template <int T>
__device__ void block_bitonic_sort(uint64_t* a, uint32_t N) {
    for (uint32_t size = 2; size <= N; size <<= 1) {
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t i = threadIdx.x; i < (N >> 1); i += T) {
                const uint32_t lo = 2u * stride * (i / stride) + (i % stride);
                const uint32_t hi = lo + stride;
                const bool asc = (lo & size) == 0;
                const uint64_t x = a[lo], y = a[hi];
                if ((x > y) == asc) {
                    a[lo] = y;
                    a[hi] = x;
                }
            }
            __syncthreads();
        }
    }
}

__device__ __forceinline__ uint32_t next_pow2(uint32_t x) {
    return x <= 1 ? 1u : 1u << (32 - __clz(x - 1));
}

// ------------------------------------------------------------------------------------------
// Warp-level primitives (one warp per query in the replay kernels).

// Ascending bitonic sort of N (power of two) u64 keys by one warp.
__device__ __forceinline__ void warp_sort_u64(uint64_t* a, uint32_t N) {
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t size = 2; size <= N; size <<= 1) {
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t i = lane; i < (N >> 1); i += 32) {
                const uint32_t lo = 2u * stride * (i / stride) + (i % stride);
                const uint32_t hi = lo + stride;
                const bool asc = (lo & size) == 0;
                const uint64_t x = a[lo], y = a[hi];
                if ((x > y) == asc) {
                    a[lo] = y;
                    a[hi] = x;
                }
            }
            __syncwarp();
        }
    }
}

// Largest heap distance and its lowest slot (LevelOps::recompute_top), on every lane. The
// distances are non-negative floats, ordered as their bit patterns.
__device__ __forceinline__ void warp_heap_top(const float* hd, uint32_t hsize, float& top, uint32_t& slot) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t best = 0, bs = 0xFFFFFFFFu;
    for (uint32_t j = lane; j < hsize; j += 32) {
        const uint32_t x = __float_as_uint(hd[j]);
        if (bs == 0xFFFFFFFFu || x > best) {
            best = x;
            bs = j;
        }
    }
    const uint32_t gmax = __reduce_max_sync(0xffffffffu, best);
    slot = __reduce_min_sync(0xffffffffu, (best == gmax) ? bs : 0xFFFFFFFFu);
    top = __uint_as_float(gmax);
}

// Exclusive prefix of x over the warp's lanes; *total receives the sum.
__device__ __forceinline__ uint32_t warp_exclusive_scan(uint32_t x, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    total = __shfl_sync(0xffffffffu, incl, 31);
    return incl - x;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// ------------------------------------------------------------------------------------------
// Distances.

// avx2_computers.hpp:47-98 over one 64-dim row, 8 threads per row (sub = lane & 7): lane j
// accumulates dims j, j+8, ..., j+56 with FMA; lanes 0 of each 8-group return the f32 result.
__device__ __forceinline__ float horiz64_f32_group8(const float* q, const float* x, uint32_t sub,
                                                    bool active) {
    float acc = 0.0f;
    if (active) {
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const float d = __fsub_rn(q[sub + 8 * t], __ldg(x + sub + 8 * t));
            acc = __fmaf_rn(d, d, acc);
        }
    }
    double s = (double)acc + (double)__shfl_down_sync(0xffffffffu, acc, 4, 8);
    s = s + __shfl_down_sync(0xffffffffu, s, 2, 8);
    s = s + __shfl_down_sync(0xffffffffu, s, 1, 8);
    return (float)s;
}

// Full-length avx2 Horizontal(q, x, d) for centroid probing, 8 threads per vector.
__device__ __forceinline__ float horiz_f32_group8(const float* q, const float* x, uint32_t d,
                                                  uint32_t sub, bool active) {
    float acc = 0.0f;
    const uint32_t full = d & ~7u;
    if (active) {
        for (uint32_t i = 0; i < full; i += 8) {
            const float t = __fsub_rn(q[i + sub], __ldg(x + i + sub));
            acc = __fmaf_rn(t, t, acc);
        }
    }
    double s = (double)acc + (double)__shfl_down_sync(0xffffffffu, acc, 4, 8);
    s = s + __shfl_down_sync(0xffffffffu, s, 2, 8);
    s = s + __shfl_down_sync(0xffffffffu, s, 1, 8);
    if (active && sub == 0) {
        for (uint32_t i = full; i < d; ++i) {
            const float t = __fsub_rn(q[i], __ldg(x + i));
            s += (double)__fmul_rn(t, t);
        }
    }
    return (float)s;
}

// QuantizeEmbedding (scalar.hpp:76-94) of one packed 32-bit word of a U8 level's query: words
// [0, qw_hoff) hold the vertical dims 4 w .. 4 w + 3 (zero past d_v), words from qw_hoff the
// horizontal dims in 64-dim blocks.
__device__ __forceinline__ uint32_t quantize_word(const float* qf, const DevLevel& lv, uint32_t w) {
    uint32_t word = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        uint32_t dim;
        bool valid;
        if (w < lv.qw_hoff) {
            dim = w * 4 + b;
            valid = dim < lv.dv;
        } else {
            dim = lv.dv + (w - lv.qw_hoff) * 4 + b;
            valid = true;
        }
        uint32_t byte = 0;
        if (valid) {
            const float v = __fmul_rn(__fsub_rn(qf[dim], lv.base), lv.scale);
            const int r = (int)roundf(v);
            byte = r > 255 ? 255u : (r < 0 ? 0u : (uint32_t)r);
        }
        word |= byte << (8 * b);
    }
    return word;
}

}  // namespace pdxg
