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
#include <cuda_runtime.h>

#include "pdxg_block.cuh"
#include "pdxg_common.cuh"

namespace pdxg {

// -------------------------------------------------------------------------------- probe
constexpr int kProbeThreads = 128;

__global__ void __launch_bounds__(kProbeThreads) meso_probe_kernel(const __grid_constant__ TopLevelParams tp) {
    extern __shared__ __align__(16) uint8_t smem[];
    const DevLevel& l0 = tp.l0;
    const uint32_t q = blockIdx.x;
    if (tp.filter_of && __ldg(tp.filter_of + q) != -1) {
        if (threadIdx.x == 0) tp.ntop[q] = 0;
        return;
    }
    const uint32_t d = l0.d, nc = l0.nclusters;
    float* qf = reinterpret_cast<float*>(smem);
    uint64_t* keys = reinterpret_cast<uint64_t*>(smem + ((d * 4 + 15) / 16) * 16);
    const float* src = tp.queries + (size_t)q * d;
    for (uint32_t i = threadIdx.x; i < d; i += kProbeThreads) qf[i] = __ldg(src + i);
    __syncthreads();
    const uint32_t sub = threadIdx.x & 7;
    for (uint32_t base = 0; base < nc; base += kProbeThreads / 8) {
        const uint32_t c = base + (threadIdx.x >> 3);
        const bool active = c < nc;
        const float dd = horiz_f32_group8(qf, l0.centroids + (size_t)(active ? c : 0) * d, d, sub, active);
        if (active && sub == 0) keys[c] = ((uint64_t)__float_as_uint(dd) << 32) | c;
    }
    const uint32_t N = next_pow2(nc);
    for (uint32_t i = nc + threadIdx.x; i < N; i += kProbeThreads) keys[i] = ~0ull;
    __syncthreads();
    // the `m` smallest (distance, id) pairs, ascending: the same list as LevelOps::probe
    block_bitonic_sort<kProbeThreads>(keys, N);
    const uint32_t topq = tp.q_top ? __ldg(tp.q_top + q) : tp.top;
    const uint32_t m = topq < nc ? topq : nc;
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (uint32_t r = 0; r < m; ++r) {
            const uint32_t c = (uint32_t)keys[r];
            tp.order[(size_t)q * tp.top + r] = c;
            tp.off[(size_t)q * tp.top + r] = acc;
            acc += tp.nvals * ((l0.clusters[c].n + 3u) & ~3u);
        }
        tp.ntop[q] = m;
    }
    for (uint32_t r = threadIdx.x; r < m; r += kProbeThreads) {
        const uint32_t c = (uint32_t)keys[r];
        const uint32_t slot = atomicAdd(tp.list_count + c, 1u);
        tp.lists[(size_t)c * tp.nq + slot] = q * tp.top + r;
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

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

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
    // thread tile: query slots warp * 16 + qg + 4 i (4 distinct rows per warp and load: distinct
    // banks) and vectors vg + 8 i, i = 0..3
    const uint32_t slot0 = warp * 16 + qg;
    auto store = [&](uint32_t row, uint32_t i, uint32_t b, float val) {
        const uint32_t sl = slot0 + 4 * i, v = v0 + vg + 8 * b;
        if (sl < ntile && v < stride) tp.vals[S.qoff[sl] + (size_t)row * stride + v] = val;
    };

    issue(0);
    cp_async_commit();
    // Stage st is in buffer st & 1 once this returns; st + 1 is in flight.
    auto begin_stage = [&](uint32_t st) {
        if (st + 1 < nst) issue(st + 1);
        cp_async_commit();
        cp_async_wait1();
        __syncthreads();
    };

    // vertical dims: one chain per (query, vector), stored at every checkpoint
    {
        float acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[i][b] = 0.0f;
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
                    float qv[4], xv[4];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        qv[i] = qs[(slot0 + 4 * i) * kRow + jj + u];
                        xv[i] = xs[(jj + u) * kTV + vg + 8 * i];
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int b = 0; b < 4; ++b) {
                            const float t = __fsub_rn(qv[i], xv[b]);
                            acc[i][b] = __fmaf_rn(t, t, acc[i][b]);
                        }
                }
                if (ck < ncp && j0 + jj + 4 == S.cp[ck]) {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int b = 0; b < 4; ++b) store(ck, i, b, acc[i][b]);
                    ++ck;
                }
            }
            __syncthreads();
        }
    }

    // horizontal blocks: per (query, vector) the AVX2 Horizontal sum of each block
    for (uint32_t st = nvc; st < nst; ++st) {
        begin_stage(st);
        const float* qs = S.q[st & 1];
        const float* xs = S.x[st & 1];
        const uint32_t row = ncp + (st - nvc);
        // two passes of 4 queries x 2 vectors keep the double sums in registers
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
            const uint32_t xo0 = (vg + 16 * h) * kRow, xo1 = (vg + 16 * h + 8) * kRow;
            // lane `sub` of Horizontal: dims sub, sub + 8, ..., sub + 56 with FMA
            auto chain = [&](int sub, float (&a)[4][2]) {
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i][0] = a[i][1] = 0.0f;
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const int dim = sub + 8 * t;
                    const float x0 = xs[xo0 + dim], x1 = xs[xo1 + dim];
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const float qv = qs[(slot0 + 4 * i) * kRow + dim];
                        float tt = __fsub_rn(qv, x0);
                        a[i][0] = __fmaf_rn(tt, tt, a[i][0]);
                        tt = __fsub_rn(qv, x1);
                        a[i][1] = __fmaf_rn(tt, tt, a[i][1]);
                    }
                }
            };
            float a[4][2];
            double D[4][2], E[4][2], F[4][2];
            // lanes in the order they combine: (0 + 4) + (2 + 6), then (1 + 5) + (3 + 7)
#pragma unroll 1
            for (int sp = 0; sp < 8; ++sp) {
                const int sub = ((sp >> 2) & 1) + ((sp >> 1) & 1) * 2 + (sp & 1) * 4;
                chain(sub, a);
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int b = 0; b < 2; ++b) {
                        const double av = (double)a[i][b];
                        if (sp == 0) D[i][b] = av;                                   // lane 0
                        else if (sp == 1) D[i][b] = D[i][b] + av;                     // s0
                        else if (sp == 2) E[i][b] = av;                               // lane 2
                        else if (sp == 3) D[i][b] = D[i][b] + (E[i][b] + av);         // s0 + s2
                        else if (sp == 4) E[i][b] = av;                               // lane 1
                        else if (sp == 5) E[i][b] = E[i][b] + av;                     // s1
                        else if (sp == 6) F[i][b] = av;                               // lane 3
                        else D[i][b] = D[i][b] + (E[i][b] + (F[i][b] + av));          // + (s1 + s3)
                    }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int b = 0; b < 2; ++b) store(row, i, 2 * h + b, (float)D[i][b]);
        }
        __syncthreads();
    }
}

// -------------------------------------------------------------------------------- replay
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

// Largest heap distance and its lowest slot (LevelOps::recompute_top), on every lane.
__device__ __forceinline__ void warp_heap_top(const float* hd, uint32_t hsize, float& top, uint32_t& slot) {
    const uint32_t lane = threadIdx.x & 31;
    float best = -1.0f;
    uint32_t bs = 0xFFFFFFFFu;
    for (uint32_t j = lane; j < hsize; j += 32) {
        const float x = hd[j];
        if (x > best || (x == best && j < bs)) {
            best = x;
            bs = j;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, o);
        const uint32_t os = __shfl_xor_sync(0xffffffffu, bs, o);
        if (ob > best || (ob == best && os < bs)) {
            best = ob;
            bs = os;
        }
    }
    top = best;
    slot = bs;
}

// Order-preserving in-place compaction of pos[0, count) to the entries with dist < thr.
__device__ __forceinline__ uint32_t warp_keep_below(uint32_t* pos, uint32_t count, const float* dist, float thr) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t total = 0;
    for (uint32_t b0 = 0; b0 < count; b0 += 32) {
        const uint32_t i = b0 + lane;
        const bool in = i < count;
        const uint32_t v = in ? pos[i] : 0u;
        const bool keep = in && dist[v] < thr;
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        __syncwarp();
        if (keep) pos[total + __popc(bal & ((1u << lane) - 1u))] = v;
        total += __popc(bal);
        __syncwarp();
    }
    return total;
}

__global__ void top_replay_kernel(const __grid_constant__ TopLevelParams tp) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t q = blockIdx.x * (blockDim.x >> 5) + warp;
    if (q >= tp.nq) return;  // whole warp; no block-wide barriers below
    if (tp.filter_of && __ldg(tp.filter_of + q) != -1) {
        if (lane == 0) tp.l1_count[q] = 0;
        return;
    }
    uint8_t* base = smem + (size_t)warp * tp.r_warp_bytes;
    uint64_t* sortbuf = reinterpret_cast<uint64_t*>(base);
    float* pre = reinterpret_cast<float*>(sortbuf + tp.r_sort_cap);
    float* hd = pre + tp.r_pre_floats;
    uint32_t* hid = reinterpret_cast<uint32_t*>(hd + tp.r_heap_cap);
    float* dist = reinterpret_cast<float*>(hid + tp.r_heap_cap);
    uint32_t* pos = reinterpret_cast<uint32_t*>(dist + tp.r_work_cap);

    const DevLevel& l0 = tp.l0;
    const uint32_t d = l0.d, dv = l0.dv, dh = l0.dh, nb = l0.n_hblocks, ncp = tp.ncp;
    const uint32_t k = tp.q_nprobe ? __ldg(tp.q_nprobe + q) : tp.k1;
    const uint32_t m_top = tp.ntop[q];
    const float* qf = tp.queries + (size_t)q * d;
    const float* qvals = tp.vals + (size_t)q * tp.per_query;
    unsigned long long bytes = (unsigned long long)l0.nclusters * d * 4u;  // centroid probe
    unsigned long long visits = 0;
    auto thr_at = [&](uint32_t cur, float top) {
        const float r = (cur == d) ? 1.0f : __ldg(tp.ratios + cur);
        return __fmul_rn(top, r);
    };

    uint32_t hsize = 0, slot = 0;
    float top = 0.0f;
    for (uint32_t r = 0; r < m_top; ++r) {
        const uint32_t mc = tp.order[(size_t)q * tp.top + r];
        const DevCluster c = l0.clusters[mc];
        const uint32_t n = c.n;
        if (n == 0) continue;
        ++visits;
        const uint32_t stride = (n + 3u) & ~3u;
        // this cluster's partials, all rows at once (one memory round trip)
        {
            const float4* src = reinterpret_cast<const float4*>(qvals + tp.off[(size_t)q * tp.top + r]);
            float4* dst = reinterpret_cast<float4*>(pre);
            const uint32_t n4 = tp.nvals * stride / 4;
            for (uint32_t i = lane; i < n4; i += 32) dst[i] = __ldg(src + i);
            __syncwarp();
        }
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
            continue;
        }
        // Warmup (searcher.hpp:374-435)
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
        // Prune (searcher.hpp:437-540)
        float thr = thr_at(cur, top);
        uint32_t nsurv = 0;
        {
            const float* row = pre + (size_t)(step - 1) * stride;
            for (uint32_t b0 = 0; b0 < n; b0 += 32) {
                const uint32_t v = b0 + lane;
                const float val = v < n ? row[v] : 0.0f;
                if (v < n) dist[v] = val;
                const bool keep = v < n && val < thr;
                const unsigned bal = __ballot_sync(0xffffffffu, keep);
                if (keep) pos[nsurv + __popc(bal & ((1u << lane) - 1u))] = v;
                nsurv += __popc(bal);
            }
            __syncwarp();
        }
        uint32_t cur_v = cur, cur_h = 0;
        while (dh && nsurv && cur_h < dh) {
            bytes += (unsigned long long)nsurv * kHDim * 4u;
            const float* hrow = pre + (size_t)(ncp + cur_h / kHDim) * stride;
            for (uint32_t i = lane; i < nsurv; i += 32) {
                const uint32_t v = pos[i];
                dist[v] = __fadd_rn(dist[v], hrow[v]);
            }
            __syncwarp();
            cur_h += kHDim;
            cur += kHDim;
            thr = thr_at(cur, top);
            nsurv = warp_keep_below(pos, nsurv, dist, thr);
        }
        const float* vert = reinterpret_cast<const float*>(tp.arena + c.vert_off);
        while (nsurv && cur_v < dv) {
            const uint32_t last = (cur_v + kHDim < dv) ? cur_v + kHDim : dv;
            bytes += (unsigned long long)nsurv * (last - cur_v) * 4u;
            for (uint32_t i = lane; i < nsurv; i += 32) {
                const uint32_t v = pos[i];
                float a = dist[v];
                for (uint32_t j = cur_v; j < last; ++j) {
                    const float t = __fsub_rn(__ldg(qf + j), __ldg(vert + (size_t)j * c.n_pad + v));
                    a = __fmaf_rn(t, t, a);
                }
                dist[v] = a;
            }
            __syncwarp();
            cur = (cur + kHDim < d) ? cur + kHDim : d;
            cur_v = last;
            thr = thr_at(cur, top);
            nsurv = warp_keep_below(pos, nsurv, dist, thr);
            if (cur == d) break;
        }
        // MergeIntoHeap (searcher.hpp:542-566): sequential, strict-<, survivor order
        for (uint32_t i = 0; i < nsurv; ++i) {
            const uint32_t v = pos[i];
            const float dd = dist[v];
            if (hsize < k || dd < top) {
                if (lane == 0) {
                    const uint32_t at = (hsize >= k) ? slot : hsize;
                    hd[at] = dd;
                    hid[at] = __ldg(ids + v);
                }
                if (hsize < k) ++hsize;
                __syncwarp();
                warp_heap_top(hd, hsize, top, slot);
            }
        }
        __syncwarp();
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

cudaError_t launch_top_level_tiled(const TopLevelParams& tp, uint32_t vtiles, int replay_warps,
                                   cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(tp.list_count, 0, sizeof(uint32_t) * tp.l0.nclusters, st);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(meso_probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tp.probe_smem);
    if (e != cudaSuccess) return e;
    meso_probe_kernel<<<tp.nq, kProbeThreads, tp.probe_smem, st>>>(tp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int psmem = (int)sizeof(PartialsSmem);
    e = cudaFuncSetAttribute(meso_partials_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, psmem);
    if (e != cudaSuccess) return e;
    dim3 grid((tp.nq + kTQ - 1) / kTQ, tp.l0.nclusters, vtiles);
    meso_partials_kernel<<<grid, kPartialsThreads, psmem, st>>>(tp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t rsmem = (size_t)tp.r_warp_bytes * replay_warps;
    e = cudaFuncSetAttribute(top_replay_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsmem);
    if (e != cudaSuccess) return e;
    top_replay_kernel<<<(tp.nq + replay_warps - 1) / replay_warps, 32 * replay_warps, rsmem, st>>>(tp);
    return cudaGetLastError();
}

}  // namespace pdxg
