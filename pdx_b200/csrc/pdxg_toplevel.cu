// Tree top level for a whole batch (PDXTreeIndex::Search, index.hpp:545-566), tiled.
//
// The top-level search is a pruned F32 PDXearch over the meso clusters, whose "vectors" are
// the L1 centroids, with k = the L1 nprobe. On IVF2 indexes every query reads about half of
// all L1 centroids there (k is large against the few vectors per meso cluster, so the
// ADSampling bound prunes little), and thousands of queries of a batch read the same meso
// clusters. One CTA per query re-reads those centroids from L2 once per query and is bound by
// its load pipe. This form computes the exact per-pair quantities once, with reuse across
// queries, and then replays the reference's decisions on them:
//
//   1. meso_probe_kernel: exact centroid distances in the AVX2 order of Horizontal
//      (searcher.hpp:181-215), the `top` nearest meso clusters per query sorted by (distance,
//      id), and per meso cluster the list of queries that probe it.
//   2. meso_partials_kernel: one CTA per (meso cluster, 128 of its queries, 32 of its
//      vectors). Query rows and cluster blocks are staged in shared memory with cp.async;
//      each thread keeps 4 queries x 4 vectors of FP32 chains in registers, so a staged
//      element feeds four chains. It writes, per (query, vector):
//        * the vertical chain (one fused multiply-add per dimension in dimension order,
//          Vertical of avx2_computers.hpp) at every warmup checkpoint: the cumulative
//          DIMENSIONS_FETCHING_SIZES steps from 0, capped at d_v, the last being d_v;
//        * the sum of every 64-dim horizontal block in the AVX2 order of Horizontal
//          (avx2_computers.hpp:47-98: 8 FMA lanes, lanes j and j + 4 added in double, then
//          pairs, then the total, rounded to float).
//   3. top_replay_kernel: one warp per query replays Start / Warmup / Prune / MergeIntoHeap
//      (searcher.hpp:217-566) on those values, so it takes the same decisions on the same
//      floats as the per-query kernel. A warmup that stops before d_v leaves vertical dims
//      for the vectors that survive every horizontal block; their chains continue from the
//      running distance and are recomputed here from the centroid data, in dimension order.
//      The sorted L1 visit order goes to l1_order for the search kernel.
#include <cfloat>
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

#include "pdxg_block.cuh"
#include "pdxg_common.cuh"

namespace pdxg {

// -------------------------------------------------------------------------------- probe
// CTA = up to kProbeQ queries; thread (centroid c of a group of 32, lane sub of 8) runs lane
// `sub` of Horizontal (avx2_computers.hpp:47-98: dims sub, sub + 8, ... with FMA) for every
// query of the CTA, so each centroid element is loaded once per CTA. The 8 lanes then combine
// in double exactly as horiz_f32_group8 does; the d % 8 tail is added by lane 0 in double.
constexpr int kProbeThreads = 256;
constexpr int kProbeQ = 8;

__global__ void __launch_bounds__(kProbeThreads) meso_probe_kernel(const __grid_constant__ TopLevelParams tp) {
    extern __shared__ __align__(16) uint8_t smem[];
    const DevLevel& l0 = tp.l0;
    const uint32_t d = l0.d, nc = l0.nclusters, qp = tp.probe_q;
    const uint32_t q0 = blockIdx.x * qp;
    const uint32_t nqc = (tp.nq - q0) < qp ? (tp.nq - q0) : qp;  // queries of this CTA
    const uint32_t N = next_pow2(nc);
    float* qs = reinterpret_cast<float*>(smem);                              // [qp][d]
    uint64_t* keys = reinterpret_cast<uint64_t*>(smem + ((size_t)qp * d * 4 + 15) / 16 * 16);  // [qp][N]
    for (uint32_t i = threadIdx.x; i < nqc * d; i += kProbeThreads) qs[i] = __ldg(tp.queries + (size_t)q0 * d + i);
    __syncthreads();
    const uint32_t sub = threadIdx.x & 7;
    const uint32_t full = d & ~7u;
    for (uint32_t c0 = 0; c0 < nc; c0 += kProbeThreads / 8) {
        const uint32_t c = c0 + (threadIdx.x >> 3);
        const bool active = c < nc;
        const float* x = l0.centroids + (size_t)(active ? c : 0) * d;
        float acc[kProbeQ];
#pragma unroll
        for (int j = 0; j < kProbeQ; ++j) acc[j] = 0.0f;
        if (active) {
            for (uint32_t i = 0; i < full; i += 8) {
                const float xv = __ldg(x + i + sub);
#pragma unroll
                for (int j = 0; j < kProbeQ; ++j) {
                    if (j < (int)nqc) {
                        const float t = __fsub_rn(qs[j * d + i + sub], xv);
                        acc[j] = __fmaf_rn(t, t, acc[j]);
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kProbeQ; ++j) {
            double sm = (double)acc[j] + (double)__shfl_down_sync(0xffffffffu, acc[j], 4, 8);
            sm = sm + __shfl_down_sync(0xffffffffu, sm, 2, 8);
            sm = sm + __shfl_down_sync(0xffffffffu, sm, 1, 8);
            if (active && sub == 0 && j < (int)nqc) {
                for (uint32_t i = full; i < d; ++i) {
                    const float t = __fsub_rn(qs[j * d + i], __ldg(x + i));
                    sm += (double)__fmul_rn(t, t);
                }
                keys[(size_t)j * N + c] = ((uint64_t)__float_as_uint((float)sm) << 32) | c;
            }
        }
    }
    for (uint32_t i = threadIdx.x; i < nqc * N; i += kProbeThreads)
        if (i % N >= nc) keys[i] = ~0ull;
    __syncthreads();
    // warp j: query q0 + j -- the `m` smallest (distance, id) pairs, ascending (the list of
    // LevelOps::probe)
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (uint32_t j = warp; j < nqc; j += kProbeThreads / 32) {
        const uint32_t q = q0 + j;
        if (tp.filter_of && __ldg(tp.filter_of + q) != -1) {
            if (lane == 0) tp.ntop[q] = 0;
            continue;
        }
        uint64_t* kq = keys + (size_t)j * N;
        warp_sort_u64(kq, N);
        const uint32_t topq = tp.q_top ? __ldg(tp.q_top + q) : tp.top;
        const uint32_t m = topq < nc ? topq : nc;
        // offsets: exclusive prefix of nvals * stride over the probe list
        uint32_t carry = 0;
        for (uint32_t r0 = 0; r0 < m; r0 += 32) {
            const uint32_t r = r0 + lane;
            const uint32_t c = r < m ? (uint32_t)kq[r] : 0u;
            const uint32_t sz = r < m ? tp.nvals * ((l0.clusters[c].n + 3u) & ~3u) : 0u;
            uint32_t incl = sz;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (uint32_t)o) incl += t;
            }
            if (r < m) {
                tp.order[(size_t)q * tp.top + r] = c;
                tp.off[(size_t)q * tp.top + r] = carry + incl - sz;
                const uint32_t slot = atomicAdd(tp.list_count + c, 1u);
                tp.lists[(size_t)c * tp.nq + slot] = q * tp.top + r;
            }
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) tp.ntop[q] = m;
    }
}

// -------------------------------------------------------------------------------- partials
constexpr int kTQ = 128;          // queries per CTA
constexpr int kTV = 32;           // vectors per CTA
constexpr int kTD = 64;           // dimensions per stage
constexpr int kRow = kTD + 4;     // floats per staged row (16-byte aligned; conflict-free columns)
constexpr int kPartialsThreads = 256;

struct PartialsSmem {
    float q[2][kTQ * kRow];       // query rows [slot][dim]
    float x[2][kTV * kRow];       // vertical: [dim][32 vectors]; horizontal: [vector][dim]
    unsigned long long qoff[kTQ]; // float offset of each slot's partials (vals + qoff)
    uint32_t qrow[kTQ];           // query index of each slot
    uint32_t cp[kMaxCheckpoints]; // warmup checkpoints
};

// Packed FP32 pairs (sm_100): each half rounds exactly as the scalar sub.rn / fma.rn.
__device__ __forceinline__ uint64_t f32x2_dup(float a) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(a));
    return r;
}
__device__ __forceinline__ uint64_t f32x2_sub(uint64_t a, uint64_t b) {
    uint64_t r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ uint64_t f32x2_fma(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ void f32x2_unpack(uint64_t v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}


__global__ void __launch_bounds__(kPartialsThreads, 2) meso_partials_kernel(const __grid_constant__ TopLevelParams tp) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    PartialsSmem& S = *reinterpret_cast<PartialsSmem*>(smem_raw);
    const uint32_t m = blockIdx.y;
    const uint32_t cnt = tp.list_count[m];
    const uint32_t first = blockIdx.x * kTQ;
    if (first >= cnt) return;
    const DevLevel& l0 = tp.l0;
    const DevCluster c = l0.clusters[m];
    const uint32_t v0 = blockIdx.z * kTV;
    if (v0 >= c.n) return;
    const uint32_t n_pad = c.n_pad, stride = (c.n + 3u) & ~3u;
    const uint32_t d = l0.d, dv = l0.dv, nb = l0.n_hblocks, ncp = tp.ncp;
    const uint32_t ntile = (cnt - first) < (uint32_t)kTQ ? (cnt - first) : (uint32_t)kTQ;
    const uint32_t tid = threadIdx.x;
    if (tid < (uint32_t)kMaxCheckpoints) S.cp[tid] = tp.cp[tid];
    if (tid < kTQ) {
        if (tid < ntile) {
            const uint32_t e = tp.lists[(size_t)m * tp.nq + first + tid];
            const uint32_t q = e / tp.top;
            S.qrow[tid] = q;
            S.qoff[tid] = (unsigned long long)q * tp.per_query + tp.off[e];
        } else {
            S.qrow[tid] = 0;
            S.qoff[tid] = 0;
        }
    }
    __syncthreads();

    const float* vert = reinterpret_cast<const float*>(tp.arena + c.vert_off);
    const float* hor = reinterpret_cast<const float*>(tp.arena + c.hor_off);
    const uint32_t nvc = (dv + kTD - 1) / kTD;  // vertical stages
    const uint32_t nst = nvc + nb;

    // stage s: query dims and the cluster block it covers, into buffer s & 1
    auto issue = [&](uint32_t st) {
        const uint32_t buf = st & 1;
        uint32_t j0, len;
        if (st < nvc) {
            j0 = st * kTD;
            len = (dv - j0) < (uint32_t)kTD ? (dv - j0) : (uint32_t)kTD;
        } else {
            j0 = dv + (st - nvc) * kTD;
            len = kTD;
        }
        const uint32_t n4 = len >> 2;  // float4 per row
        // query rows: 128 slots x 16 float4
#pragma unroll
        for (int t = 0; t < (kTQ * kTD / 4) / kPartialsThreads; ++t) {
            const uint32_t e = tid + t * kPartialsThreads;
            const uint32_t s = e >> 4, c4 = e & 15;
            if (s < ntile && c4 < n4)
                cp_async16(&S.q[buf][s * kRow + c4 * 4], tp.queries + (size_t)S.qrow[s] * d + j0 + c4 * 4);
        }
        if (st < nvc) {
            // vertical rows: len dims x 32 vectors (row stride n_pad: in bounds)
#pragma unroll
            for (int t = 0; t < (kTD * kTV / 4) / kPartialsThreads; ++t) {
                const uint32_t e = tid + t * kPartialsThreads;
                const uint32_t jj = e >> 3, c4 = e & 7;
                if (jj < len) cp_async16(&S.x[buf][jj * kTV + c4 * 4], vert + (size_t)(j0 + jj) * n_pad + v0 + c4 * 4);
            }
        } else {
            // horizontal block rows of the 32 vectors: 32 x 64 floats, contiguous in memory
            const float* hb = hor + ((size_t)(st - nvc) * n_pad + v0) * kHDim;
#pragma unroll
            for (int t = 0; t < (kTV * kTD / 4) / kPartialsThreads; ++t) {
                const uint32_t e = tid + t * kPartialsThreads;
                const uint32_t vv = e >> 4, c4 = e & 15;
                cp_async16(&S.x[buf][vv * kRow + c4 * 4], hb + (size_t)vv * kHDim + c4 * 4);
            }
        }
    };

    const uint32_t lane = tid & 31, warp = tid >> 5;
    const uint32_t vg = lane & 7, qg = lane >> 3;
    // thread tile: query slots slot0 + 4 i (i = 0..3; 4 consecutive rows per warp and load, so
    // distinct banks)
    const uint32_t slot0 = warp * 16 + qg;
    auto slot_ok = [&](int i) { return slot0 + 4 * i < ntile; };
    auto out_row = [&](int i, uint32_t row) { return tp.vals + S.qoff[slot0 + 4 * i] + (size_t)row * stride; };

    issue(0);
    cp_async_commit();
    // Stage st is in buffer st & 1 once this returns; st + 1 is in flight.
    auto begin_stage = [&](uint32_t st) {
        if (st + 1 < nst) issue(st + 1);
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
    };

    // vertical dims: one chain per (query, vector), stored at every checkpoint. Vectors
    // 2 vg + {0, 1} and 2 vg + 16 + {0, 1}, each adjacent pair in one packed register; a tile
    // with at most 16 vectors left (a cluster's tail) runs the first half only (NB = 1), as it
    // stores nothing from the second.
    auto vertical = [&](auto nb_tag) {
        constexpr int NB = decltype(nb_tag)::value;
        uint64_t acc[4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[i][0] = acc[i][1] = 0ull;
        uint32_t ck = 0;
        for (uint32_t st = 0; st < nvc; ++st) {
            begin_stage(st);
            const float* qs = S.q[st & 1];
            const float* xs = S.x[st & 1];
            const uint32_t j0 = st * kTD;
            const uint32_t len = (dv - j0) < (uint32_t)kTD ? (dv - j0) : (uint32_t)kTD;
            for (uint32_t jj = 0; jj < len; jj += 4) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    uint64_t qv[4], xv[2];
#pragma unroll
                    for (int i = 0; i < 4; ++i) qv[i] = f32x2_dup(qs[(slot0 + 4 * i) * kRow + jj + u]);
#pragma unroll
                    for (int b = 0; b < NB; ++b)
                        xv[b] = *reinterpret_cast<const uint64_t*>(xs + (jj + u) * kTV + 2 * vg + 16 * b);
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int b = 0; b < NB; ++b) {
                            const uint64_t t = f32x2_sub(qv[i], xv[b]);
                            acc[i][b] = f32x2_fma(t, t, acc[i][b]);
                        }
                }
                if (ck < ncp && j0 + jj + 4 == S.cp[ck]) {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int b = 0; b < NB; ++b) {
                            const uint32_t v = v0 + 2 * vg + 16 * b;
                            if (slot_ok(i) && v < stride)
                                *reinterpret_cast<uint64_t*>(out_row(i, ck) + v) = acc[i][b];
                        }
                    ++ck;
                }
            }
            __syncthreads();
        }
    };
    const bool tail = c.n - v0 <= 16u;
    if (tail) vertical(std::integral_constant<int, 1>());
    else vertical(std::integral_constant<int, 2>());

    // horizontal blocks: per (query, vector) the AVX2 Horizontal sum of each block. Lanes
    // (j, j + 1) of Horizontal run as one packed chain: dims j + 8 t and j + 1 + 8 t are
    // adjacent in both staged rows. Passes of 4 queries x NB vectors (vg + 16 h, vg + 16 h + 8):
    // a tail tile with at most 16 vectors left runs pass 0 only, with at most 8 left one vector
    // per thread; it stores nothing from the rest.
    auto horizontal = [&](auto nb_tag, int passes) {
        constexpr int NB = decltype(nb_tag)::value;
        for (uint32_t st = nvc; st < nst; ++st) {
            begin_stage(st);
            const float* qs = S.q[st & 1];
            const float* xs = S.x[st & 1];
            const uint32_t row = ncp + (st - nvc);
#pragma unroll 1
            for (int h = 0; h < passes; ++h) {
                const uint32_t xo0 = (vg + 16 * h) * kRow, xo1 = (vg + 16 * h + 8) * kRow;
                double D0[4][2], D1[4][2], E0[4][2], E1[4][2];
                // lane pairs in the order they combine: (0,1) + (4,5) -> s0, s1; (2,3) + (6,7) -> s2, s3
#pragma unroll 1
                for (int cp2 = 0; cp2 < 4; ++cp2) {
                    const int c2 = ((cp2 & 1) << 2) | ((cp2 >> 1) << 1);  // 0, 4, 2, 6
                    uint64_t a[4][2];
#pragma unroll
                    for (int i = 0; i < 4; ++i) a[i][0] = a[i][1] = 0ull;
#pragma unroll
                    for (int t = 0; t < 8; ++t) {
                        const int dim = c2 + 8 * t;
                        const uint64_t x0 = *reinterpret_cast<const uint64_t*>(xs + xo0 + dim);
                        uint64_t x1 = 0ull;
                        if constexpr (NB == 2) x1 = *reinterpret_cast<const uint64_t*>(xs + xo1 + dim);
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const uint64_t qv = *reinterpret_cast<const uint64_t*>(qs + (slot0 + 4 * i) * kRow + dim);
                            uint64_t tt = f32x2_sub(qv, x0);
                            a[i][0] = f32x2_fma(tt, tt, a[i][0]);
                            if constexpr (NB == 2) {
                                tt = f32x2_sub(qv, x1);
                                a[i][1] = f32x2_fma(tt, tt, a[i][1]);
                            }
                        }
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int b = 0; b < NB; ++b) {
                            float lo, hi;
                            f32x2_unpack(a[i][b], lo, hi);
                            if (cp2 == 0) {          // lanes 0, 1
                                D0[i][b] = (double)lo;
                                D1[i][b] = (double)hi;
                            } else if (cp2 == 1) {   // lanes 4, 5: s0, s1
                                D0[i][b] = D0[i][b] + (double)lo;
                                D1[i][b] = D1[i][b] + (double)hi;
                            } else if (cp2 == 2) {   // lanes 2, 3
                                E0[i][b] = (double)lo;
                                E1[i][b] = (double)hi;
                            } else {                 // lanes 6, 7: s2, s3
                                E0[i][b] = E0[i][b] + (double)lo;
                                E1[i][b] = E1[i][b] + (double)hi;
                            }
                        }
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int b = 0; b < NB; ++b) {
                        const uint32_t v = v0 + vg + 16 * h + 8 * b;
                        if (slot_ok(i) && v < stride)
                            out_row(i, row)[v] = (float)((D0[i][b] + E0[i][b]) + (D1[i][b] + E1[i][b]));
                    }
            }
            __syncthreads();
        }
    };
    if (c.n - v0 <= 8u) horizontal(std::integral_constant<int, 1>(), 1);
    else horizontal(std::integral_constant<int, 2>(), tail ? 1 : 2);
}

// -------------------------------------------------------------------------------- replay

// Shared memory of the replay: the ratio table (d floats) for the CTA, then per warp
//   sortbuf [r_sort_cap] u64 | pre [2][r_pre_floats] | hd, hid [r_heap_cap] | dist, pos [r_work_cap]
//   | meta [top] x {cluster, partials offset}
__global__ void top_replay_kernel(const __grid_constant__ TopLevelParams tp) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const DevLevel& l0 = tp.l0;
    const uint32_t d = l0.d, dv = l0.dv, nb = l0.n_hblocks, ncp = tp.ncp;
    float* ratios = reinterpret_cast<float*>(smem);
    for (uint32_t i = threadIdx.x; i < d; i += blockDim.x) ratios[i] = __ldg(tp.ratios + i);
    __syncthreads();  // the only block-wide barrier
    const uint32_t q = blockIdx.x * (blockDim.x >> 5) + warp;
    if (q >= tp.nq) return;  // whole warp
    if (tp.filter_of && __ldg(tp.filter_of + q) != -1) {
        if (lane == 0) tp.l1_count[q] = 0;
        return;
    }
    uint8_t* base = smem + ((size_t)d * 4 + 15) / 16 * 16 + (size_t)warp * tp.r_warp_bytes;
    uint64_t* sortbuf = reinterpret_cast<uint64_t*>(base);
    float* prebuf = reinterpret_cast<float*>(sortbuf + tp.r_sort_cap);
    float* hd = prebuf + 2 * tp.r_pre_floats;
    uint32_t* hid = reinterpret_cast<uint32_t*>(hd + tp.r_heap_cap);
    float* dist = reinterpret_cast<float*>(hid + tp.r_heap_cap);
    uint32_t* pos = reinterpret_cast<uint32_t*>(dist + tp.r_work_cap);
    uint32_t* meta_c = pos + tp.r_work_cap;   // [top] probed meso cluster
    uint32_t* meta_o = meta_c + tp.top;       // [top] offset of its partials

    const uint32_t k = tp.q_nprobe ? __ldg(tp.q_nprobe + q) : tp.k1;
    const uint32_t m_top = tp.ntop[q];
    const float* qf = tp.queries + (size_t)q * d;
    const float* qvals = tp.vals + (size_t)q * tp.per_query;
    unsigned long long bytes = (unsigned long long)l0.nclusters * d * 4u;  // centroid probe
    unsigned long long visits = 0;
    auto thr_at = [&](uint32_t cur, float top) {
        const float r = (cur == d) ? 1.0f : ratios[cur];
        return __fmul_rn(top, r);
    };
    for (uint32_t r = lane; r < m_top; r += 32) {
        meta_c[r] = tp.order[(size_t)q * tp.top + r];
        meta_o[r] = tp.off[(size_t)q * tp.top + r];
    }
    __syncwarp();
    // next probed cluster with vectors at or after r (m_top if none)
    auto next_nonempty = [&](uint32_t r) {
        while (r < m_top && l0.clusters[meta_c[r]].n == 0) ++r;
        return r;
    };
    // all partial rows of probed cluster r into buffer `buf`, asynchronously
    auto fetch = [&](uint32_t r, int buf) {
        const uint32_t n = l0.clusters[meta_c[r]].n;
        const uint32_t n4 = tp.nvals * ((n + 3u) & ~3u) / 4;
        const float4* src = reinterpret_cast<const float4*>(qvals + meta_o[r]);
        float* dst = prebuf + (size_t)buf * tp.r_pre_floats;
        for (uint32_t i = lane; i < n4; i += 32) cp_async16(dst + 4 * i, src + i);
        cp_async_commit();
    };

    uint32_t hsize = 0, slot = 0;
    float top = 0.0f;
    uint32_t r = next_nonempty(0);
    int buf = 0;
    if (r < m_top) fetch(r, 0);
    while (r < m_top) {
        const uint32_t rn = next_nonempty(r + 1);
        if (rn < m_top) {
            fetch(rn, buf ^ 1);
            cp_async_wait1();
        } else {
            cp_async_wait0();
        }
        __syncwarp();
        const float* pre = prebuf + (size_t)buf * tp.r_pre_floats;
        const DevCluster c = l0.clusters[meta_c[r]];
        const uint32_t n = c.n;
        ++visits;
        const uint32_t stride = (n + 3u) & ~3u;
        // the loop body runs once per non-empty probed cluster; `continue` is not used below
        do {
        const uint32_t* ids = reinterpret_cast<const uint32_t*>(tp.arena + c.ids_off);
        if (hsize < k) {
            // Start (searcher.hpp:217-281): full distances, push the best k - |heap| in the
            // order LevelOps::push_smallest uses (below the m-th key by position, then ties)
            bytes += (unsigned long long)n * d * 4u;
            const uint32_t N = next_pow2(n);
            for (uint32_t v = lane; v < N; v += 32) {
                if (v < n) {
                    float a = pre[(size_t)(ncp - 1) * stride + v];
                    for (uint32_t b = 0; b < nb; ++b) a = __fadd_rn(a, pre[(size_t)(ncp + b) * stride + v]);
                    dist[v] = a;
                    sortbuf[v] = ((uint64_t)__float_as_uint(a) << 32) | v;
                } else {
                    sortbuf[v] = ~0ull;
                }
            }
            __syncwarp();
            warp_sort_u64(sortbuf, N);
            const uint32_t mm = (k - hsize) < n ? (k - hsize) : n;
            const uint32_t kth = (uint32_t)(sortbuf[mm - 1] >> 32);
            uint32_t cntp = 0;
            for (int pass = 0; pass < 2; ++pass) {
                for (uint32_t b0 = 0; b0 < n; b0 += 32) {
                    const uint32_t v = b0 + lane;
                    const uint32_t key = v < n ? __float_as_uint(dist[v]) : 0u;
                    const bool sel = v < n && (pass == 0 ? key < kth : key == kth);
                    const unsigned bal = __ballot_sync(0xffffffffu, sel);
                    const uint32_t at = cntp + __popc(bal & ((1u << lane) - 1u));
                    if (sel && at < mm) {
                        hd[hsize + at] = dist[v];
                        hid[hsize + at] = __ldg(ids + v);
                    }
                    cntp += __popc(bal);
                }
            }
            hsize += mm;
            __syncwarp();
            warp_heap_top(hd, hsize, top, slot);
            break;
        }
        // Warmup (searcher.hpp:374-435): vertical checkpoints until >= ceil(0.8 n) fail the bound
        const uint32_t needed = (uint32_t)ceilf(__fmul_rn(kSelectivity, (float)n));
        uint32_t cur = 0, step = 0, n_pruned = 0;
        while (n_pruned < needed && cur < dv) {
            const uint32_t last = tp.cp[step];
            const float thr = thr_at(last, top);
            bytes += (unsigned long long)n * (last - cur) * 4u;
            uint32_t cntp = 0;
            const float* row = pre + (size_t)step * stride;
            for (uint32_t v = lane; v < n; v += 32) cntp += row[v] >= thr ? 1u : 0u;
            n_pruned = __reduce_add_sync(0xffffffffu, cntp);
            cur = last;
            ++step;
        }
        // Prune (searcher.hpp:437-540). The bound's heap top is fixed until the merge, so each
        // vector's way through the horizontal blocks and the remaining vertical dims depends on
        // that vector alone: each lane follows its own vectors, and the survivors of every
        // step are the same, in the same order, as with the step-by-step compaction.
        const float* erow = pre + (size_t)(step - 1) * stride;
        const float* vert = reinterpret_cast<const float*>(tp.arena + c.vert_off);
        unsigned long long lane_bytes = 0;
        for (uint32_t c0 = 0; c0 < n; c0 += 32) {
            const uint32_t v = c0 + lane;
            bool alive = v < n;
            float dd = alive ? erow[v] : 0.0f;
            uint32_t cv = cur;
            alive = alive && dd < thr_at(cv, top);
            for (uint32_t b = 0; alive && b < nb; ++b) {
                lane_bytes += kHDim * 4u;
                dd = __fadd_rn(dd, pre[(size_t)(ncp + b) * stride + v]);
                cv += kHDim;
                alive = dd < thr_at(cv, top);
            }
            uint32_t cur_v = cur;
            while (alive && cur_v < dv) {
                const uint32_t last = (cur_v + kHDim < dv) ? cur_v + kHDim : dv;
                lane_bytes += (unsigned long long)(last - cur_v) * 4u;
                for (uint32_t j = cur_v; j < last; ++j) {
                    const float t = __fsub_rn(__ldg(qf + j), __ldg(vert + (size_t)j * c.n_pad + v));
                    dd = __fmaf_rn(t, t, dd);
                }
                cv = (cv + kHDim < d) ? cv + kHDim : d;
                cur_v = last;
                alive = dd < thr_at(cv, top);
                if (cv == d) break;
            }
            if (v < n) {
                dist[v] = dd;
                pos[v] = alive ? 1u : 0u;
            }
        }
        bytes += __reduce_add_sync(0xffffffffu, (uint32_t)lane_bytes);
        __syncwarp();
        // MergeIntoHeap (searcher.hpp:542-566): sequential, strict-<, in position order
        for (uint32_t c0 = 0; c0 < n; c0 += 32) {
            const uint32_t v = c0 + lane;
            const bool alive = v < n && pos[v] != 0u;
            const float dd = alive ? dist[v] : 0.0f;
            const uint32_t idv = alive ? __ldg(ids + v) : 0u;
            unsigned bal = __ballot_sync(0xffffffffu, alive);
            while (bal) {
                const int i = __ffs(bal) - 1;
                bal &= bal - 1;
                const float ddi = __shfl_sync(0xffffffffu, dd, i);
                const uint32_t idi = __shfl_sync(0xffffffffu, idv, i);
                if (hsize < k || ddi < top) {
                    if (lane == 0) {
                        const uint32_t at = (hsize >= k) ? slot : hsize;
                        hd[at] = ddi;
                        hid[at] = idi;
                    }
                    if (hsize < k) ++hsize;
                    __syncwarp();
                    warp_heap_top(hd, hsize, top, slot);
                }
            }
        }
        } while (false);
        __syncwarp();  // every lane is done with `pre` before the next fetch overwrites it
        r = rn;
        buf ^= 1;
    }
    // BuildResultSetFromHeap (searcher.hpp:568-585): the L1 clusters, nearest first
    const uint32_t N = next_pow2(hsize ? hsize : 1);
    for (uint32_t i = lane; i < N; i += 32)
        sortbuf[i] = (i < hsize) ? (((uint64_t)__float_as_uint(hd[i]) << 32) | hid[i]) : ~0ull;
    __syncwarp();
    warp_sort_u64(sortbuf, N);
    uint32_t cnt = hsize;
    if (cnt && __uint_as_float((uint32_t)(sortbuf[cnt - 1] >> 32)) == FLT_MAX) --cnt;
    if (cnt > k) cnt = k;
    for (uint32_t i = lane; i < cnt; i += 32) tp.l1_order[(size_t)q * tp.k1 + i] = (uint32_t)sortbuf[i];
    if (lane == 0) {
        tp.l1_count[q] = cnt;
        if (tp.stats) {
            atomicAdd(tp.stats + 3, bytes);
            atomicAdd(tp.stats, bytes);
            atomicAdd(tp.stats + 1, visits);
        }
    }
}

// -------------------------------------------------------------------------------- launch
size_t partials_smem_bytes() { return sizeof(PartialsSmem); }

// ev (optional, 2 events): recorded after the meso probe and after the partials.
cudaError_t launch_top_level_tiled(const TopLevelParams& tp, uint32_t vtiles, int replay_warps,
                                   cudaStream_t st, const cudaEvent_t* ev) {
    cudaError_t e = cudaMemsetAsync(tp.list_count, 0, sizeof(uint32_t) * tp.l0.nclusters, st);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(meso_probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tp.probe_smem);
    if (e != cudaSuccess) return e;
    meso_probe_kernel<<<(tp.nq + tp.probe_q - 1) / tp.probe_q, kProbeThreads, tp.probe_smem, st>>>(tp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (ev && (e = cudaEventRecord(ev[0], st)) != cudaSuccess) return e;
    const int psmem = (int)sizeof(PartialsSmem);
    e = cudaFuncSetAttribute(meso_partials_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, psmem);
    if (e != cudaSuccess) return e;
    dim3 grid((tp.nq + kTQ - 1) / kTQ, tp.l0.nclusters, vtiles);
    meso_partials_kernel<<<grid, kPartialsThreads, psmem, st>>>(tp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (ev && (e = cudaEventRecord(ev[1], st)) != cudaSuccess) return e;
    const size_t rsmem = tp.r_smem;
    e = cudaFuncSetAttribute(top_replay_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsmem);
    if (e != cudaSuccess) return e;
    top_replay_kernel<<<(tp.nq + replay_warps - 1) / replay_warps, 32 * replay_warps, rsmem, st>>>(tp);
    return cudaGetLastError();
}

}  // namespace pdxg
