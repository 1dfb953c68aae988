// Batched first half of the two-level (tree) search: the exact per-query quantities that the
// top-level PDXearch over the meso clusters (PDXTreeIndex::Search, index.hpp:545-566) bases its
// decisions on, computed for a whole batch with data reuse across queries.
//
// The top-level search is a pruned F32 PDXearch whose "vectors" are the L1 centroids, grouped
// in small meso clusters that every query of the batch reads. Instead of one CTA per query
// walking those clusters with one load per fused multiply-add, this stage
//   1. ranks each query's meso clusters by centroid distance (meso_probe_kernel), and
//   2. computes, for every (query, L1 centroid) pair the query will visit, the vertical
//      distance chain at each warmup checkpoint (one FMA per dimension, dimension order) and the
//      sum of every 64-dim horizontal block in the reference's AVX2 order (8 FMA lanes,
//      pairwise double reduction) -- meso_partials_kernel, 32 queries per CTA, each centroid
//      element loaded once per 4 queries.
// The search kernel then replays the reference's Start / Warmup / Prune / Merge on these
// values, so the resulting L1 visit order is bit-identical to the reference's.
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "pdxg_block.cuh"
#include "pdxg_common.cuh"

namespace pdxg {

// -------------------------------------------------------------------------------- probe
// One CTA per query: exact distances to every meso centroid, the `top` nearest sorted
// ascending (ties by id), their offsets in the partials buffer, and the per-cluster lists of
// probing queries for meso_partials_kernel.
template <int T>
__global__ void __launch_bounds__(T) meso_probe_kernel(const __grid_constant__ TopLevelParams tp) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ Scalars s;
    const DevLevel& l0 = tp.l0;
    const uint32_t q = blockIdx.x;
    float* qf = reinterpret_cast<float*>(smem);
    uint32_t* dist = reinterpret_cast<uint32_t*>(smem + tp.smem_dist);
    uint32_t* pos = dist + tp.n0_cap;
    uint64_t* sortbuf = reinterpret_cast<uint64_t*>(smem + tp.smem_sort);
    const float* src = tp.queries + (size_t)q * l0.d;
    for (uint32_t i = threadIdx.x; i < l0.d; i += T) qf[i] = __ldg(src + i);
    __syncthreads();
    const uint32_t nc = l0.nclusters;
    const uint32_t sub = threadIdx.x & 7;
    for (uint32_t base = 0; base < nc; base += T / 8) {
        const uint32_t c = base + (threadIdx.x >> 3);
        const bool active = c < nc;
        const float dd = horiz_f32_group8(qf, l0.centroids + (size_t)(active ? c : 0) * l0.d, l0.d, sub, active);
        if (active && sub == 0) dist[c] = __float_as_uint(dd);
    }
    __syncthreads();
    const uint32_t m = tp.top < nc ? tp.top : nc;
    uint32_t kth, less;
    block_radix_select<T>(dist, nc, m, s, kth, less);
    const uint32_t nl = block_compact<T>(
        nc, [&](uint32_t, uint32_t v) { return dist[v] < kth; }, [](uint32_t i) { return i; }, pos, s);
    block_compact<T>(nc, [&](uint32_t, uint32_t v) { return dist[v] == kth; },
                     [](uint32_t i) { return i; }, pos + nl, s);
    uint32_t N = 1;
    while (N < m) N <<= 1;
    for (uint32_t i = threadIdx.x; i < N; i += T)
        sortbuf[i] = (i < m) ? (((uint64_t)dist[pos[i]] << 32) | pos[i]) : ~0ull;
    __syncthreads();
    block_bitonic_sort<T>(sortbuf, N);
    if (threadIdx.x == 0) {
        unsigned long long off = (unsigned long long)q * tp.per_query_floats;
        for (uint32_t r = 0; r < m; ++r) {
            const uint32_t c = (uint32_t)sortbuf[r];
            tp.order[(size_t)q * tp.top + r] = c;
            tp.offsets[(size_t)q * tp.top + r] = off;
            off += (unsigned long long)l0.clusters[c].n * tp.nvals;
        }
    }
    for (uint32_t r = threadIdx.x; r < m; r += T) {
        const uint32_t c = (uint32_t)sortbuf[r];
        const uint32_t slot = atomicAdd(tp.list_count + c, 1u);
        tp.lists[(size_t)c * tp.nq + slot] = q * tp.top + r;
    }
}

// -------------------------------------------------------------------------------- partials
constexpr int kPQ = 32;       // queries per CTA
constexpr int kPChunk = 64;   // dimensions staged per step
constexpr int kPStride = 36;  // floats per staged query row (32 queries + pad, 16B aligned)
constexpr int kHStride = 68;  // floats per staged horizontal row (64 + pad, 16B aligned)

// CTA = (meso cluster, 32 probing queries); 8 warps x 4 queries, lane = vector. Query and
// vector tiles are staged in shared memory with coalesced loads; every staged vector element
// feeds 4 queries' FMA chains from registers.
__global__ void __launch_bounds__(256) meso_partials_kernel(const __grid_constant__ TopLevelParams tp) {
    __shared__ __align__(16) float qs[kPChunk * kPStride];          // [dim][query]
    __shared__ __align__(16) float xs[32 * kHStride];               // vertical [dim][vec] / rows
    __shared__ unsigned long long offs[kPQ];
    __shared__ uint32_t qids[kPQ];
    const uint32_t m = blockIdx.x;
    const uint32_t cnt = tp.list_count[m];
    const uint32_t first = blockIdx.y * kPQ;
    if (first >= cnt) return;
    const DevLevel& l0 = tp.l0;
    const DevCluster c = l0.clusters[m];
    const uint32_t n = c.n, np = c.n_pad, d = l0.d, dv = l0.dv;
    if (n == 0) return;
    const uint32_t ntile = (cnt - first) < (uint32_t)kPQ ? (cnt - first) : (uint32_t)kPQ;
    if (threadIdx.x < kPQ) {
        if (threadIdx.x < ntile) {
            const uint32_t e = tp.lists[(size_t)m * tp.nq + first + threadIdx.x];
            qids[threadIdx.x] = e / tp.top;
            offs[threadIdx.x] = tp.offsets[e];
        } else {
            qids[threadIdx.x] = 0xFFFFFFFFu;
            offs[threadIdx.x] = 0;
        }
    }
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t qi0 = warp * 4;  // this warp's 4 queries of the tile
    const float* vert = reinterpret_cast<const float*>(tp.arena + c.vert_off);
    const float* hor = reinterpret_cast<const float*>(tp.arena + c.hor_off);
    const uint32_t nck = tp.n_ckpt;

    // dims [j0, j0 + len) of the tile's queries, transposed to [dim][query]
    auto stage_q = [&](uint32_t j0, uint32_t len) {
        for (uint32_t e = threadIdx.x; e < kPChunk * kPQ; e += 256) {
            const uint32_t qi = e / kPChunk, jj = e % kPChunk;
            float v = 0.0f;
            if (jj < len && qi < ntile) v = __ldg(tp.queries + (size_t)qids[qi] * d + j0 + jj);
            qs[jj * kPStride + qi] = v;
        }
    };
    __syncthreads();

    for (uint32_t vc = 0; vc < n; vc += 32) {
        const uint32_t v = vc + lane;
        const bool active = v < n;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        uint32_t ck = 0;
        for (uint32_t j0 = 0; j0 < dv; j0 += kPChunk) {
            const uint32_t len = (dv - j0) < (uint32_t)kPChunk ? (dv - j0) : (uint32_t)kPChunk;
            __syncthreads();
            stage_q(j0, len);
            // vertical tile [len dims][32 vectors] (rows are n_pad-padded: in bounds)
            for (uint32_t e = threadIdx.x; e < (uint32_t)kPChunk * 32; e += 256) {
                const uint32_t jj = e >> 5, vv = e & 31;
                xs[jj * 32 + vv] = (jj < len) ? __ldg(vert + (size_t)(j0 + jj) * np + vc + vv) : 0.0f;
            }
            __syncthreads();
#pragma unroll 4
            for (uint32_t jj = 0; jj < len; ++jj) {
                const float x = xs[jj * 32 + lane];
                const float4 q4 = *reinterpret_cast<const float4*>(qs + jj * kPStride + qi0);
                float t = __fsub_rn(q4.x, x);
                acc[0] = __fmaf_rn(t, t, acc[0]);
                t = __fsub_rn(q4.y, x);
                acc[1] = __fmaf_rn(t, t, acc[1]);
                t = __fsub_rn(q4.z, x);
                acc[2] = __fmaf_rn(t, t, acc[2]);
                t = __fsub_rn(q4.w, x);
                acc[3] = __fmaf_rn(t, t, acc[3]);
                if (j0 + jj + 1 == tp.ckpt[ck]) {
                    if (active) {
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            if (qi0 + i < ntile) tp.vals[offs[qi0 + i] + (size_t)ck * n + v] = acc[i];
                    }
                    ++ck;
                }
            }
        }
        for (uint32_t b = 0; b < l0.n_hblocks; ++b) {
            __syncthreads();
            stage_q(dv + b * kHDim, kHDim);
            // 32 horizontal rows of this block: contiguous 32 x 256 B in global memory
            const float4* src = reinterpret_cast<const float4*>(hor + ((size_t)b * np + vc) * kHDim);
            for (uint32_t e = threadIdx.x; e < 32 * 16; e += 256) {
                const uint32_t r = e >> 4, c4 = e & 15;
                const float4 val = (vc + r < np) ? __ldg(src + e) : make_float4(0.f, 0.f, 0.f, 0.f);
                *reinterpret_cast<float4*>(xs + r * kHStride + c4 * 4) = val;
            }
            __syncthreads();
            float h[4][8];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) h[i][j] = 0.0f;
            const float* row = xs + lane * kHStride;
#pragma unroll 2
            for (int t8 = 0; t8 < 8; ++t8) {
                const float4 a = *reinterpret_cast<const float4*>(row + t8 * 8);
                const float4 bq = *reinterpret_cast<const float4*>(row + t8 * 8 + 4);
                const float x8[8] = {a.x, a.y, a.z, a.w, bq.x, bq.y, bq.z, bq.w};
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float4 q4 = *reinterpret_cast<const float4*>(qs + (t8 * 8 + j) * kPStride + qi0);
                    float dd = __fsub_rn(q4.x, x8[j]);
                    h[0][j] = __fmaf_rn(dd, dd, h[0][j]);
                    dd = __fsub_rn(q4.y, x8[j]);
                    h[1][j] = __fmaf_rn(dd, dd, h[1][j]);
                    dd = __fsub_rn(q4.z, x8[j]);
                    h[2][j] = __fmaf_rn(dd, dd, h[2][j]);
                    dd = __fsub_rn(q4.w, x8[j]);
                    h[3][j] = __fmaf_rn(dd, dd, h[3][j]);
                }
            }
            if (active) {
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    // avx2_computers.hpp:62-83: (lo+hi) pairwise in double
                    const double s0 = (double)h[i][0] + (double)h[i][4];
                    const double s1 = (double)h[i][1] + (double)h[i][5];
                    const double s2 = (double)h[i][2] + (double)h[i][6];
                    const double s3 = (double)h[i][3] + (double)h[i][7];
                    const float r = (float)((s0 + s2) + (s1 + s3));
                    if (qi0 + i < ntile) tp.vals[offs[qi0 + i] + (size_t)(nck + b) * n + v] = r;
                }
            }
        }
    }
}

// -------------------------------------------------------------------------------- replay
// One warp per query replays the reference's top-level PDXearch (searcher.hpp:217-585 on the
// meso level, k = L1 nprobe) on the exact values of meso_partials_kernel: Start, the warmup
// checkpoints, the horizontal blocks and the strict-< merge take the same decisions on the
// same float values. Survivors of every horizontal block continue the vertical chain from
// their running distance (not from the pure vertical chain), so those few values are
// recomputed from the centroid data here, in dimension order.

__device__ __forceinline__ uint32_t warp_compact_inplace(uint32_t* arr, uint32_t count,
                                                         const uint32_t* dist, uint32_t thr) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t total = 0;
    for (uint32_t base = 0; base < count; base += 32) {
        const uint32_t i = base + lane;
        const bool in = i < count;
        const uint32_t v = in ? arr[i] : 0u;
        const bool pred = in && __uint_as_float(dist[v]) < __uint_as_float(thr);
        const unsigned b = __ballot_sync(0xffffffffu, pred);
        if (pred) arr[total + __popc(b & ((1u << lane) - 1u))] = v;
        total += __popc(b);
        __syncwarp();
    }
    return total;
}

__device__ __forceinline__ void warp_bitonic_sort(uint64_t* a, uint32_t N) {
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

// max of hd[0, hsize) and its lowest slot, on every lane
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
    for (int off = 16; off > 0; off >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, off);
        const uint32_t os = __shfl_xor_sync(0xffffffffu, bs, off);
        if (ob > best || (ob == best && os < bs)) {
            best = ob;
            bs = os;
        }
    }
    top = best;
    slot = bs;
}

__global__ void __launch_bounds__(256) top_replay_kernel(const __grid_constant__ TopLevelParams tp) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t q = blockIdx.x * (blockDim.x >> 5) + warp;
    if (q >= tp.nq) return;  // whole warp
    uint8_t* base = smem + (size_t)warp * tp.r_warp_bytes;
    uint64_t* sortbuf = reinterpret_cast<uint64_t*>(base);
    float* hd = reinterpret_cast<float*>(base + (size_t)tp.r_sort_cap * 8);
    uint32_t* hid = reinterpret_cast<uint32_t*>(hd + tp.r_heap_cap);
    uint32_t* dist = hid + tp.r_heap_cap;
    uint32_t* pos = dist + tp.r_dist_cap;
    const DevLevel& l0 = tp.l0;
    const uint32_t d = l0.d, dv = l0.dv, k = tp.k1, nck = tp.n_ckpt;
    const float* qf = tp.queries + (size_t)q * d;
    const uint32_t m_top = tp.top < l0.nclusters ? tp.top : l0.nclusters;
    uint32_t hsize = 0, slot = 0;
    float top = 0.0f;
    for (uint32_t r = 0; r < m_top; ++r) {
        const uint32_t mc = tp.order[(size_t)q * tp.top + r];
        const DevCluster c = l0.clusters[mc];
        const uint32_t n = c.n;
        if (n == 0) continue;
        const float* pre = tp.vals + tp.offsets[(size_t)q * tp.top + r];
        const uint32_t* ids = reinterpret_cast<const uint32_t*>(tp.arena + c.ids_off);
        if (hsize < k) {
            // Start (searcher.hpp:217-281): full distances, push the best k - |heap|
            uint32_t N = 1;
            while (N < n) N <<= 1;
            for (uint32_t v = lane; v < N; v += 32) {
                if (v < n) {
                    float a = pre[(size_t)(nck - 1) * n + v];
                    for (uint32_t b = 0; b < l0.n_hblocks; ++b) a = __fadd_rn(a, pre[(size_t)(nck + b) * n + v]);
                    sortbuf[v] = ((uint64_t)__float_as_uint(a) << 32) | v;
                } else {
                    sortbuf[v] = ~0ull;
                }
            }
            __syncwarp();
            warp_bitonic_sort(sortbuf, N);
            const uint32_t m = (k - hsize) < n ? (k - hsize) : n;
            for (uint32_t j = lane; j < m; j += 32) {
                hd[hsize + j] = __uint_as_float((uint32_t)(sortbuf[j] >> 32));
                hid[hsize + j] = __ldg(ids + (uint32_t)sortbuf[j]);
            }
            hsize += m;
            __syncwarp();
            warp_heap_top(hd, hsize, top, slot);
            continue;
        }
        // Warmup (searcher.hpp:374-435)
        const uint32_t needed = (uint32_t)ceilf(__fmul_rn(kSelectivity, (float)n));
        uint32_t cur = 0, step = 0, n_pruned = 0;
        while (n_pruned < needed && cur < dv) {
            const uint32_t last = tp.ckpt[step];
            const float ratio = (last == d) ? 1.0f : __ldg(tp.ratios + last);
            const float thr = __fmul_rn(top, ratio);
            uint32_t cnt = 0;
            const float* vs = pre + (size_t)step * n;
            for (uint32_t v = lane; v < n; v += 32) {
                const float val = vs[v];
                dist[v] = __float_as_uint(val);
                cnt += val >= thr ? 1u : 0u;
            }
            n_pruned = __reduce_add_sync(0xffffffffu, cnt);
            cur = last;
            ++step;
        }
        __syncwarp();
        // Prune (searcher.hpp:437-540)
        auto thr_at = [&](uint32_t cc) {
            const float ratio = (cc == d) ? 1.0f : __ldg(tp.ratios + cc);
            return __float_as_uint(__fmul_rn(top, ratio));
        };
        uint32_t thr = thr_at(cur);
        uint32_t nsurv = 0;
        for (uint32_t b0 = 0; b0 < n; b0 += 32) {
            const uint32_t v = b0 + lane;
            const bool pred = v < n && __uint_as_float(dist[v]) < __uint_as_float(thr);
            const unsigned bal = __ballot_sync(0xffffffffu, pred);
            if (pred) pos[nsurv + __popc(bal & ((1u << lane) - 1u))] = v;
            nsurv += __popc(bal);
        }
        __syncwarp();
        uint32_t cur_v = cur, cur_h = 0;
        while (l0.dh && nsurv && cur_h < l0.dh) {
            const float* hs = pre + (size_t)(nck + cur_h / kHDim) * n;
            for (uint32_t i = lane; i < nsurv; i += 32) {
                const uint32_t v = pos[i];
                dist[v] = __float_as_uint(__fadd_rn(__uint_as_float(dist[v]), hs[v]));
            }
            __syncwarp();
            cur_h += kHDim;
            cur += kHDim;
            thr = thr_at(cur);
            nsurv = warp_compact_inplace(pos, nsurv, dist, thr);
        }
        const float* vert = reinterpret_cast<const float*>(tp.arena + c.vert_off);
        while (nsurv && cur_v < dv) {
            const uint32_t last = (cur_v + kHDim < dv) ? cur_v + kHDim : dv;
            for (uint32_t i = lane; i < nsurv; i += 32) {
                const uint32_t v = pos[i];
                float acc = __uint_as_float(dist[v]);
                for (uint32_t j = cur_v; j < last; ++j) {
                    const float t = __fsub_rn(__ldg(qf + j), __ldg(vert + (size_t)j * c.n_pad + v));
                    acc = __fmaf_rn(t, t, acc);
                }
                dist[v] = __float_as_uint(acc);
            }
            __syncwarp();
            cur = (cur + kHDim < d) ? cur + kHDim : d;
            cur_v = last;
            thr = thr_at(cur);
            nsurv = warp_compact_inplace(pos, nsurv, dist, thr);
            if (cur == d) break;
        }
        // MergeIntoHeap (searcher.hpp:542-566)
        for (uint32_t i = 0; i < nsurv; ++i) {
            const uint32_t v = pos[i];
            const float dd = __uint_as_float(dist[v]);
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
    // BuildResultSetFromHeap (searcher.hpp:568-585): ascending order of the L1 clusters
    uint32_t N = 1;
    while (N < hsize) N <<= 1;
    for (uint32_t i = lane; i < N; i += 32)
        sortbuf[i] = (i < hsize) ? (((uint64_t)__float_as_uint(hd[i]) << 32) | hid[i]) : ~0ull;
    __syncwarp();
    warp_bitonic_sort(sortbuf, N);
    uint32_t cnt = hsize;
    if (cnt && __uint_as_float((uint32_t)(sortbuf[cnt - 1] >> 32)) == FLT_MAX) --cnt;
    if (cnt > k) cnt = k;
    for (uint32_t i = lane; i < cnt; i += 32) tp.l1_order[(size_t)q * k + i] = (uint32_t)sortbuf[i];
    if (lane == 0) tp.l1_count[q] = cnt;
}

// -------------------------------------------------------------------------------- launch
cudaError_t launch_top_level(const TopLevelParams& tp, cudaStream_t st) {
    const size_t smem = tp.smem_total;
    cudaError_t e = cudaFuncSetAttribute(meso_probe_kernel<128>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(tp.list_count, 0, sizeof(uint32_t) * tp.l0.nclusters, st);
    if (e != cudaSuccess) return e;
    meso_probe_kernel<128><<<tp.nq, 128, smem, st>>>(tp);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 grid(tp.l0.nclusters, (tp.nq + kPQ - 1) / kPQ);
    meso_partials_kernel<<<grid, 256, 0, st>>>(tp);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const uint32_t wpb = tp.r_warps_per_block;
    const size_t rsmem = (size_t)tp.r_warp_bytes * wpb;
    e = cudaFuncSetAttribute(top_replay_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsmem);
    if (e != cudaSuccess) return e;
    top_replay_kernel<<<(tp.nq + wpb - 1) / wpb, 32 * wpb, rsmem, st>>>(tp);
    return cudaGetLastError();
}

}  // namespace pdxg
