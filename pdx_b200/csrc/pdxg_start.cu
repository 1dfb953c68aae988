// Batched Start for U8 levels (PDXearch::Start, searcher.hpp:217-281), ahead of the scan.
//
// A query's first Start computes the full distance from the query to every vector of the first
// cluster it visits, then keeps the best k. In a batch many queries start in the same cluster,
// and the reference reads that whole cluster once per query. Here the queries of a batch are
// grouped by their first visited cluster and each cluster is read once per group of up to
// kStartQ queries, with the query-vector dot products on the integer tensor cores. U8
// distances are exact integer sums (no rounding): |q - x|^2 = |q|^2 + |x|^2 - 2 q.x holds
// exactly, so the values equal those of the per-query Start. The search kernel then runs
// push_smallest on them (searcher.hpp:256-280) instead of recomputing.
//
//   start_count_kernel : first non-empty cluster of each unfiltered query, counted per cluster
//   start_plan_kernel  : one CTA -- per-cluster offsets, each query's row, work items
//   start_dist_kernel  : persistent CTAs over (cluster, <= kStartQ queries, 256 vectors) items,
//                        mma.sync m16n8k32 u8 x u8 -> s32 (a 16 x 8 x 32 tile per instruction)
#include <cstdint>
#include <cuda_runtime.h>

#include "pdxg_block.cuh"
#include "pdxg_common.cuh"

namespace pdxg {

constexpr int kStartQ = 16;        // queries per work item
constexpr int kStartV = 256;       // vectors per work item (one per thread)
constexpr int kPlanThreads = 1024;

__global__ void start_count_kernel(const __grid_constant__ StartParams sp) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= sp.nq) return;
    sp.row_of[q] = -1;
    sp.first_cl[q] = 0xFFFFFFFFu;
    if (sp.filter_of && sp.filter_of[q] != -1) return;
    const uint32_t cnt = sp.q_order_count[q];
    const uint32_t* ord = sp.q_order + (size_t)q * sp.q_order_stride;
    for (uint32_t i = 0; i < cnt; ++i) {
        const uint32_t c = ord[i];
        if (sp.l1.clusters[c].live == 0) continue;  // num_embeddings == 0 (searcher.hpp:662)
        sp.first_cl[q] = c;
        sp.slot_of[q] = atomicAdd(sp.cl_count + c, 1u);
        return;
    }
}

// Exclusive scan of n values in place with one CTA; returns the total.
__device__ uint32_t cta_exclusive_scan(uint32_t* a, uint32_t n, uint32_t* warp_tot) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < n; b0 += kPlanThreads) {
        const uint32_t i = b0 + threadIdx.x;
        const uint32_t x = i < n ? a[i] : 0u;
        uint32_t incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += t;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint32_t v = warp_tot[lane];
            uint32_t wi = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= (uint32_t)o) wi += t;
            }
            warp_tot[lane] = wi - v;  // exclusive prefix of the warp totals
            if (lane == 31) warp_tot[32] = wi;
        }
        __syncthreads();
        if (i < n) a[i] = carry + warp_tot[warp] + incl - x;
        carry += warp_tot[32];
        __syncthreads();
    }
    return carry;
}

__global__ void __launch_bounds__(kPlanThreads) start_plan_kernel(const __grid_constant__ StartParams sp) {
    __shared__ uint32_t warp_tot[33];
    const uint32_t n1 = sp.l1.nclusters;
    // cl_off[c] = first row of cluster c; cl_items[c] = first work item of cluster c
    for (uint32_t c = threadIdx.x; c < n1; c += kPlanThreads) {
        const uint32_t L = sp.cl_count[c];
        sp.cl_off[c] = L;
        const uint32_t nv = sp.l1.clusters[c].n;
        sp.cl_items[c] = L ? ((L + kStartQ - 1) / kStartQ) * ((nv + kStartV - 1) / kStartV) : 0u;
    }
    __syncthreads();
    cta_exclusive_scan(sp.cl_off, n1, warp_tot);
    const uint32_t total_items = cta_exclusive_scan(sp.cl_items, n1, warp_tot);
    for (uint32_t q = threadIdx.x; q < sp.nq; q += kPlanThreads) {
        const uint32_t c = sp.first_cl[q];
        if (c == 0xFFFFFFFFu) continue;
        const uint32_t row = sp.cl_off[c] + sp.slot_of[q];
        sp.row_of[q] = (int32_t)row;
        sp.sorted_q[row] = q;
    }
    for (uint32_t c = threadIdx.x; c < n1; c += kPlanThreads) {
        const uint32_t L = sp.cl_count[c];
        if (!L) continue;
        const uint32_t nv = sp.l1.clusters[c].n;
        const uint32_t nqc = (L + kStartQ - 1) / kStartQ, nvc = (nv + kStartV - 1) / kStartV;
        uint32_t it = sp.cl_items[c];
        for (uint32_t a = 0; a < nqc; ++a)
            for (uint32_t b = 0; b < nvc; ++b, ++it) {
                sp.items[2 * it] = c;
                sp.items[2 * it + 1] = (a << 16) | b;
            }
    }
    if (threadIdx.x == 0) {
        sp.n_items[0] = total_items;
        sp.queue[0] = 0;
    }
}

// u8 x u8 -> s32 tensor-core product of a 16 x 32 query tile and a 32 x 8 vector tile,
// accumulated into c (exact: every product and partial sum is an integer below 2^31).
__device__ __forceinline__ void mma_u8_16x8x32(int (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+r"(c[0]), "+r"(c[1]), "+r"(c[2]), "+r"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// CTA = one work item: up to 16 queries x 256 vectors of one cluster. Warp w takes vectors
// [32 w, 32 w + 32) in four 8-vector tiles. The squared distance of an integer query q and
// vector x is |q|^2 + |x|^2 - 2 q.x exactly; q.x runs on the tensor cores, |x|^2 with dp4a on
// the same loaded words, |q|^2 once per query.
__global__ void __launch_bounds__(kStartV) start_dist_kernel(const __grid_constant__ StartParams sp) {
    extern __shared__ __align__(16) uint32_t qw[];  // [kStartQ][qs] packed query words
    __shared__ uint32_t item;
    __shared__ uint32_t qsq[kStartQ];
    const DevLevel& lv = sp.l1;
    const uint32_t nwords = lv.qw_hoff + lv.n_hblocks * 16;
    const uint32_t qs = nwords + 4;  // row stride: fragment loads of 8 rows hit distinct banks
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t gq = lane >> 2, gk = lane & 3;  // fragment row / k-group of this lane
    for (;;) {
        if (threadIdx.x == 0) item = atomicAdd(sp.queue, 1u);
        __syncthreads();
        const uint32_t it = item;
        __syncthreads();
        if (it >= sp.n_items[0]) break;
        const uint32_t c = sp.items[2 * it];
        const uint32_t ab = sp.items[2 * it + 1];
        const uint32_t qa = ab >> 16, vb = ab & 0xFFFFu;
        const uint32_t L = sp.cl_count[c];
        const uint32_t r0 = sp.cl_off[c] + qa * kStartQ;
        const uint32_t nqc = (L - qa * kStartQ) < (uint32_t)kStartQ ? (L - qa * kStartQ) : (uint32_t)kStartQ;
        // QuantizeEmbedding of the item's queries, packed as the search kernel packs them;
        // rows past nqc are zero
        for (uint32_t e = threadIdx.x; e < kStartQ * nwords; e += kStartV) {
            const uint32_t j = e / nwords, w = e % nwords;
            qw[j * qs + w] = j < nqc ? quantize_word(sp.queries + (size_t)sp.sorted_q[r0 + j] * lv.d, lv, w) : 0u;
        }
        __syncthreads();
        if (warp < kStartQ / 2) {
            // |q|^2: warp w sums queries 2 w and 2 w + 1
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t j = 2 * warp + h;
                uint32_t acc = 0;
                for (uint32_t w = lane; w < nwords; w += 32) acc = __dp4a(qw[j * qs + w], qw[j * qs + w], acc);
                acc = __reduce_add_sync(0xffffffffu, acc);
                if (lane == 0) qsq[j] = acc;
            }
        }
        __syncthreads();
        const DevCluster cl = lv.clusters[c];
        const uint32_t* vert = reinterpret_cast<const uint32_t*>(sp.arena + cl.vert_off);
        const uint8_t* hor = sp.arena + cl.hor_off;
        // four 8-vector tiles per warp, all in flight at once; tiles past the cluster load
        // in-bounds padding (n_pad) and are not stored
        const uint32_t vw = vb * kStartV + warp * 32;  // first vector of this warp
        if (vw < cl.n) {
            int acc[4][4];
            uint32_t xsq[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                xsq[t] = 0;
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[t][e] = 0;
            }
            const bool tile_in[4] = {true, vw + 8 < cl.n_pad, vw + 16 < cl.n_pad, vw + 24 < cl.n_pad};
            // vertical words: k step of 8 words (32 dims); lane holds words gk and gk + 4
#pragma unroll 2
            for (uint32_t g = 0; g < lv.qw_hoff; g += 8) {
                const uint32_t w0 = g + gk, w1 = g + 4 + gk;
                uint32_t b0[4], b1[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const uint32_t v = vw + 8 * t + gq;
                    b0[t] = (tile_in[t] && w0 < lv.n_vwords) ? __ldg(vert + (size_t)w0 * cl.n_pad + v) : 0u;
                    b1[t] = (tile_in[t] && w1 < lv.n_vwords) ? __ldg(vert + (size_t)w1 * cl.n_pad + v) : 0u;
                }
                uint32_t a[4];
                a[0] = w0 < lv.qw_hoff ? qw[gq * qs + w0] : 0u;
                a[1] = w0 < lv.qw_hoff ? qw[(gq + 8) * qs + w0] : 0u;
                a[2] = w1 < lv.qw_hoff ? qw[gq * qs + w1] : 0u;
                a[3] = w1 < lv.qw_hoff ? qw[(gq + 8) * qs + w1] : 0u;
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    xsq[t] = __dp4a(b0[t], b0[t], xsq[t]);
                    xsq[t] = __dp4a(b1[t], b1[t], xsq[t]);
                    mma_u8_16x8x32(acc[t], a, b0[t], b1[t]);
                }
            }
            // horizontal blocks: 16 words per vector row, two k steps per block
            for (uint32_t b = 0; b < lv.n_hblocks; ++b) {
                uint4 x[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const uint32_t v = vw + 8 * t + gq;
                    const uint32_t* row = reinterpret_cast<const uint32_t*>(hor + ((size_t)b * cl.n_pad + v) * kHDim);
                    // words gk, 4 + gk, 8 + gk, 12 + gk of the row
                    x[t] = tile_in[t] ? make_uint4(__ldg(row + gk), __ldg(row + 4 + gk), __ldg(row + 8 + gk),
                                                   __ldg(row + 12 + gk))
                                      : make_uint4(0u, 0u, 0u, 0u);
                }
                const uint32_t qo = lv.qw_hoff + b * 16;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    uint32_t a[4];
                    a[0] = qw[gq * qs + qo + 8 * h + gk];
                    a[1] = qw[(gq + 8) * qs + qo + 8 * h + gk];
                    a[2] = qw[gq * qs + qo + 8 * h + 4 + gk];
                    a[3] = qw[(gq + 8) * qs + qo + 8 * h + 4 + gk];
#pragma unroll
                    for (int t = 0; t < 4; ++t) {
                        const uint32_t b0 = h ? x[t].z : x[t].x, b1 = h ? x[t].w : x[t].y;
                        xsq[t] = __dp4a(b0, b0, xsq[t]);
                        xsq[t] = __dp4a(b1, b1, xsq[t]);
                        mma_u8_16x8x32(acc[t], a, b0, b1);
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                // |x|^2 of vector vw + 8 t + gq: the four lanes of its k-groups hold a quarter each
                uint32_t xs4 = xsq[t];
                xs4 += __shfl_xor_sync(0xffffffffu, xs4, 1);
                xs4 += __shfl_xor_sync(0xffffffffu, xs4, 2);
                // accumulator layout: acc[0..1] = (row gq, cols 2 gk, 2 gk + 1), acc[2..3] = row gq + 8
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const uint32_t j = gq + (e >> 1) * 8;
                    const uint32_t col = 2 * gk + (e & 1);
                    const uint32_t vx = vw + 8 * t + col;
                    const uint32_t xs = __shfl_sync(0xffffffffu, xs4, col * 4);  // lane of vector col
                    if (j < nqc && vx < cl.n)
                        sp.dist[(size_t)(r0 + j) * sp.stride + vx] = qsq[j] + xs - 2u * (uint32_t)acc[t][e];
                }
            }
        }
        __syncthreads();
    }
}

size_t start_dist_smem(const DevLevel& lv) {
    return (size_t)kStartQ * (lv.qw_hoff + lv.n_hblocks * 16 + 4) * 4;
}

cudaError_t launch_start_batched(const StartParams& sp, int grid, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(sp.cl_count, 0, sizeof(uint32_t) * sp.l1.nclusters, st);
    if (e != cudaSuccess) return e;
    start_count_kernel<<<(sp.nq + 255) / 256, 256, 0, st>>>(sp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    start_plan_kernel<<<1, kPlanThreads, 0, st>>>(sp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t smem = start_dist_smem(sp.l1);
    e = cudaFuncSetAttribute(start_dist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    start_dist_kernel<<<grid, kStartV, smem, st>>>(sp);
    return cudaGetLastError();
}

int start_dist_occupancy(size_t smem) {
    int blocks = 0;
    cudaFuncSetAttribute(start_dist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, start_dist_kernel, kStartV, smem);
    return blocks;
}

uint64_t start_item_bound(uint32_t nq, uint32_t n1, uint32_t max_n) {
    return ((uint64_t)(nq + kStartQ - 1) / kStartQ + n1) * ((max_n + kStartV - 1) / kStartV);
}

}  // namespace pdxg
