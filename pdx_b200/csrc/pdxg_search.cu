// PDXearch on B200: one CTA per query, persistent over a batch of queries.
//
// Each CTA walks one query's clusters in probe order with the reference's sequential
// semantics, so results are identical to PDXearch::Search / FilteredSearch
// (searcher.hpp:596-856) on the same prepared query:
//   * probe order: exact F32 centroid distances in the reference's AVX2 reduction order,
//     block radix-select of the nprobe nearest, bitonic sort (searcher.hpp:181-215);
//   * Start for clusters met while the heap holds fewer than k entries: full distances,
//     only the best k - |heap| are pushed (searcher.hpp:217-281);
//   * Warmup: vertical dims in the DIMENSIONS_FETCHING_SIZES steps until >= ceil(0.8 n)
//     vectors fail the ADSampling bound (searcher.hpp:374-435);
//   * Prune: survivors compacted with __ballot_sync/__popc, gathered 64-dim horizontal
//     blocks, then the remaining vertical dims in 64-dim steps, re-pruning after each block
//     (searcher.hpp:437-540);
//   * MergeIntoHeap with strict-< admission in survivor order (searcher.hpp:542-566).
// Distances: U8 uses __vabsdiffu4 + __dp4a into exact uint32 (the exact scalar semantics of
// scalar_computers.hpp:137-194); F32 vertical is one fused multiply-add per dimension and F32
// horizontal reproduces avx2_computers.hpp:47-98 (8 FMA lanes, pairwise double reduction).
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <tuple>

#include "pdxg_block.cuh"
#include "pdxg_common.cuh"

namespace pdxg {

__constant__ uint32_t c_fetch_sizes[kNumFetchSizes] = {16,  16,  32,  32,  32,   32,   64,
                                                       64,  64,  64,  128, 128,  128,  128,
                                                       256, 256, 512, 1024, 2048, 16384};

constexpr uint32_t kMaskU8 = 0x7FFFFFFFu;                 // numeric_limits<u32>::max() / 2
#define PDXG_MASK_F32 (FLT_MAX / 2.0f)                     // numeric_limits<float>::max() / 2

// ------------------------------------------------------------------------------------------
// Per-CTA state in shared memory.
struct Shared {
    float* qf;          // prepared query, f32 [d]
    uint32_t* qw;       // U8 query words: [n_vwords] vertical groups, then [n_hblocks*16]
    uint32_t* dist;     // [work_cap] partial distances (u32, or f32 bits)
    uint32_t* pos;      // [work_cap] survivor positions
    float* hd;          // [heap_cap] heap distances
    uint32_t* hid;      // [heap_cap] heap row ids
    uint32_t* order;    // [order_cap] cluster visit order
    uint32_t* bits;     // [bits_cap] survivor bitmap of the last warmup step, then its prefix
    uint64_t* sortw;    // work region viewed as u64 [work_cap]
    uint64_t* sorth;    // heap region viewed as u64 [heap_cap]
};




// ------------------------------------------------------------------------------------------
// Distances.

__device__ __forceinline__ uint32_t sqdiff4(uint32_t a, uint32_t b, uint32_t acc) {
    const uint32_t d = __vabsdiffu4(a, b);
    return __dp4a(d, d, acc);
}

// ------------------------------------------------------------------------------------------
// Per-level search state and operations (T threads, one query). TOMB: the level may hold
// tombstoned slots (Append / Delete); the instantiations without it are the read-only scan.
template <int T, bool U8, bool TOMB = false>
struct LevelOps {
    static constexpr bool u8 = U8;
    const SearchParams& p;
    const DevLevel& lv;
    Shared& sh;
    Scalars& s;
    const uint32_t* fsel;   // this query's selection bitmap over the level (null = unfiltered)
    const uint32_t* fpass;  // this query's passing count per cluster
    bool top_level;         // the tree's meso-cluster search
    int32_t pre_row = -1;   // row of this query's batched first-cluster distances (U8), or -1
    uint32_t pre_cluster = 0xFFFFFFFFu;  // the cluster they belong to

    __device__ LevelOps(const SearchParams& p_, const DevLevel& lv_, Shared& sh_, Scalars& s_,
                        int filter, bool top_level_ = false)
        : p(p_), lv(lv_), sh(sh_), s(s_), fsel(nullptr), fpass(nullptr), top_level(top_level_) {
        if (filter >= 0) {
            fsel = p.sel_bits + (size_t)filter * lv.sel_words;
            fpass = p.passing + (size_t)filter * lv.nclusters;
        } else if (filter <= -2) {
            fsel = p.reg_sel + (size_t)(-2 - filter) * lv.sel_words;
            fpass = p.reg_pass + (size_t)(-2 - filter) * lv.nclusters;
        }
    }

    __device__ __forceinline__ const uint32_t* vert(const DevCluster& c) const {
        return reinterpret_cast<const uint32_t*>(p.arena + c.vert_off);
    }
    __device__ __forceinline__ const uint32_t* ids(const DevCluster& c) const {
        return reinterpret_cast<const uint32_t*>(p.arena + c.ids_off);
    }
    __device__ __forceinline__ float reported(uint32_t raw) const {
        return u8 ? __fmul_rn(__uint2float_rn(raw), lv.inv_scale_sq) : __uint_as_float(raw);
    }
    __device__ __forceinline__ float thr_f(uint32_t cur) const {
        const float r = (cur == lv.d) ? 1.0f : __ldg(p.ratios + cur);
        return __fmul_rn(s.top, r);
    }
    // Pruning threshold in the raw distance domain, as u32 bits (searcher.hpp:75-91).
    __device__ __forceinline__ uint32_t thr_raw(uint32_t cur) const {
        const float f = thr_f(cur);
        if (!u8) return __float_as_uint(f);
        const float scaled = __fmul_rn(f, lv.scale_sq);
        return scaled >= 4294967296.0f ? 0xFFFFFFFFu : __float2uint_rz(scaled);
    }
    // dist < threshold, in the level's distance domain (F32 compares as floats).
    __device__ __forceinline__ bool below(uint32_t raw, uint32_t thr) const {
        return u8 ? raw < thr : __uint_as_float(raw) < __uint_as_float(thr);
    }
    __device__ __forceinline__ bool selected(const DevCluster& c, uint32_t v) const {
        if (!fsel) return true;
        const uint32_t* bits = fsel + c.sel_word;
        return (__ldg(bits + (v >> 5)) >> (v & 31)) & 1u;
    }
    // Cluster with tombstoned slots (uniform across the block).
    __device__ __forceinline__ bool has_tombstones(const DevCluster& c) const { return TOMB && c.live < c.n; }
    __device__ __forceinline__ bool tombstone(const DevCluster& c, uint32_t v) const {
        return (__ldg(lv.tomb + c.sel_word + (v >> 5)) >> (v & 31)) & 1u;
    }
    // MaskDistancesWithTombstones (searcher.hpp:169-179): the raw distance of every tombstoned
    // slot becomes the mask value (from_zero: every other slot becomes 0).
    __device__ void mask_tombstones(const DevCluster& c, bool from_zero) {
        const uint32_t mask = mask_raw();
        for (uint32_t v = threadIdx.x; v < c.n; v += T) {
            if (tombstone(c, v)) sh.dist[v] = mask;
            else if (from_zero) sh.dist[v] = 0u;
        }
        __syncthreads();
    }
    // Algorithmic-traffic accounting (only when p.stats is set; values are block-uniform).
    __device__ __forceinline__ void count_bytes(unsigned long long b, Phase ph) const {
        if (p.stats && threadIdx.x == 0) s.bytes[top_level ? kTopLevel : ph] += b;
    }
    static constexpr uint32_t kElem = U8 ? 1u : 4u;

    __device__ __forceinline__ uint32_t mask_raw() const {
        return u8 ? kMaskU8 : __float_as_uint(PDXG_MASK_F32);
    }

    // Vertical dims [d0, d1) for all vectors; returns #vectors with dist >= thr (counted only
    // when count is set, and then sh.bits receives the bitmap of the vectors below thr, one
    // word per 32 positions). Distances start from 0 with from_zero, else from sh.dist. For U8,
    // d0 is a multiple of 4; a trailing partial group is reached only with d1 == dv and its
    // padding bytes are zero in both query and data.
    // Each thread keeps kVPT vectors (v, v + T, ...) and issues a whole batch of rows for all of
    // them before consuming any, so one step costs one memory round trip, not one per vector.
    // The loop runs per warp (base is warp-uniform), so every lane reaches each ballot.
    // U8 with up to 128 threads: one batch covers 1024 vectors (one L2 round trip per warmup step
    // for clusters up to that size; measured faster on B200)
    static constexpr int kVPT = (U8 && T <= 128) ? 1024 / T : 4;
    __device__ uint32_t vertical_all(const DevCluster& c, uint32_t d0, uint32_t d1, bool count,
                                     uint32_t thr, bool from_zero = false) {
        const uint32_t* base = vert(c);
        const uint32_t n = c.n, np = c.n_pad;
        const uint32_t lane = lane_id();
        uint32_t pruned = 0;
        for (uint32_t wb = threadIdx.x - lane; wb < n; wb += T * kVPT) {
            const uint32_t v0 = wb + lane;
            bool act[kVPT];
#pragma unroll
            for (int k = 0; k < kVPT; ++k) act[k] = v0 + k * T < n;
            bool keep[kVPT];
            if constexpr (U8) {
                constexpr int GB = 4;  // groups per batch
                const uint32_t g0 = d0 >> 2, g1 = (d1 + 3) >> 2;
                uint32_t acc[kVPT];
#pragma unroll
                for (int k = 0; k < kVPT; ++k) acc[k] = (act[k] && !from_zero) ? sh.dist[v0 + k * T] : 0u;
                for (uint32_t g = g0; g < g1; g += GB) {
                    uint32_t x[kVPT][GB];
#pragma unroll
                    for (int j = 0; j < GB; ++j)
#pragma unroll
                        for (int k = 0; k < kVPT; ++k)
                            x[k][j] = (act[k] && g + j < g1) ? __ldg(base + (size_t)(g + j) * np + v0 + k * T) : 0u;
#pragma unroll
                    for (int j = 0; j < GB; ++j) {
                        if (g + j < g1) {
                            const uint32_t qv = sh.qw[g + j];
#pragma unroll
                            for (int k = 0; k < kVPT; ++k) acc[k] = sqdiff4(qv, x[k][j], acc[k]);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < kVPT; ++k) {
                    keep[k] = act[k] && acc[k] < thr;
                    if (act[k]) {
                        sh.dist[v0 + k * T] = acc[k];
                        pruned += (count && acc[k] >= thr) ? 1u : 0u;
                    }
                }
            } else {
                constexpr int DB = 8;  // dims per batch
                const float* fb = reinterpret_cast<const float*>(base);
                float acc[kVPT];
#pragma unroll
                for (int k = 0; k < kVPT; ++k) acc[k] = (act[k] && !from_zero) ? __uint_as_float(sh.dist[v0 + k * T]) : 0.0f;
                for (uint32_t j = d0; j < d1; j += DB) {
                    float x[kVPT][DB];
#pragma unroll
                    for (int t = 0; t < DB; ++t)
#pragma unroll
                        for (int k = 0; k < kVPT; ++k)
                            x[k][t] = (act[k] && j + t < d1) ? __ldg(fb + (size_t)(j + t) * np + v0 + k * T) : 0.0f;
#pragma unroll
                    for (int t = 0; t < DB; ++t) {
                        if (j + t < d1) {
                            const float qv = sh.qf[j + t];
#pragma unroll
                            for (int k = 0; k < kVPT; ++k) {
                                const float dd = __fsub_rn(qv, x[k][t]);
                                acc[k] = __fmaf_rn(dd, dd, acc[k]);
                            }
                        }
                    }
                }
                const float tf = __uint_as_float(thr);
#pragma unroll
                for (int k = 0; k < kVPT; ++k) {
                    keep[k] = act[k] && acc[k] < tf;
                    if (act[k]) {
                        sh.dist[v0 + k * T] = __float_as_uint(acc[k]);
                        pruned += (count && acc[k] >= tf) ? 1u : 0u;
                    }
                }
            }
            if (count) {
#pragma unroll
                for (int k = 0; k < kVPT; ++k) {
                    const unsigned m = __ballot_sync(0xffffffffu, keep[k]);
                    if (lane == 0 && wb + k * T < n) sh.bits[(wb + k * T) >> 5] = m;
                }
            }
        }
        return count ? block_sum<T>(pruned, s) : 0u;
    }

    // Positions of the set bits of sh.bits over [0, n), ascending, into sh.pos; returns their
    // number. sh.bits must be complete (a barrier after it was written).
    __device__ uint32_t compact_bits(uint32_t n) {
        const uint32_t words = (n + 31) >> 5;
        uint32_t* pref = sh.bits + p.bits_cap;
        if (threadIdx.x < 32) {
            const uint32_t lane = lane_id();
            uint32_t carry = 0;
            for (uint32_t w0 = 0; w0 < words; w0 += 32) {
                const uint32_t w = w0 + lane;
                const uint32_t cnt = w < words ? __popc(sh.bits[w]) : 0u;
                uint32_t incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= (uint32_t)o) incl += t;
                }
                if (w < words) pref[w] = carry + incl - cnt;
                carry += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) s.sc[2] = carry;
        }
        __syncthreads();
        for (uint32_t w = threadIdx.x; w < words; w += T) {
            uint32_t b = sh.bits[w], at = pref[w];
            while (b) {
                const uint32_t i = __ffs(b) - 1;
                b &= b - 1;
                sh.pos[at++] = w * 32 + i;
            }
        }
        const uint32_t total = s.sc[2];
        __syncthreads();
        return total;
    }

    // Vertical dims [d0, d1) for the first npos listed positions (gathered access).
    __device__ void vertical_pos(const DevCluster& c, uint32_t d0, uint32_t d1, uint32_t npos) {
        const uint32_t* base = vert(c);
        const uint32_t np = c.n_pad;
        if constexpr (U8) {
            const uint32_t g0 = d0 >> 2, g1 = (d1 + 3) >> 2;
            for (uint32_t i = threadIdx.x; i < npos; i += T) {
                const uint32_t v = sh.pos[i];
                uint32_t acc = sh.dist[v];
                for (uint32_t g = g0; g < g1; ++g)
                    acc = sqdiff4(sh.qw[g], __ldg(base + (size_t)g * np + v), acc);
                sh.dist[v] = acc;
            }
        } else {
            const float* fb = reinterpret_cast<const float*>(base);
            for (uint32_t i = threadIdx.x; i < npos; i += T) {
                const uint32_t v = sh.pos[i];
                float acc = __uint_as_float(sh.dist[v]);
                for (uint32_t j = d0; j < d1; ++j) {
                    const float t = __fsub_rn(sh.qf[j], __ldg(fb + (size_t)j * np + v));
                    acc = __fmaf_rn(t, t, acc);
                }
                sh.dist[v] = __float_as_uint(acc);
            }
        }
        __syncthreads();
    }

    // Adds horizontal block b to the distances of positions[0, npos) (all vectors when
    // all_vectors is set, npos = n). Several rows per thread group are in flight at once.
    __device__ void horizontal(const DevCluster& c, uint32_t b, uint32_t npos, bool all_vectors) {
        const uint32_t np = c.n_pad;
        const uint32_t lane = lane_id();
        if constexpr (U8) {
            constexpr int RPG = 4;  // rows per 4-thread group per pass
            const uint8_t* hb = p.arena + c.hor_off + (size_t)b * np * kHDim;
            const uint32_t* qh = sh.qw + lv.qw_hoff + b * 16;
            const uint32_t sub = lane & 3;
            const uint32_t groups = T / 4;
            const uint4 q4 = *reinterpret_cast<const uint4*>(qh + sub * 4);
            for (uint32_t base = 0; base < npos; base += groups * RPG) {
                uint32_t v[RPG];
                bool active[RPG];
                uint4 x[RPG];
#pragma unroll
                for (int r = 0; r < RPG; ++r) {
                    const uint32_t i = base + r * groups + (threadIdx.x >> 2);
                    active[r] = i < npos;
                    v[r] = active[r] ? (all_vectors ? i : sh.pos[i]) : 0u;
                }
#pragma unroll
                for (int r = 0; r < RPG; ++r)
                    x[r] = active[r] ? __ldg(reinterpret_cast<const uint4*>(hb + (size_t)v[r] * kHDim) + sub)
                                     : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
                for (int r = 0; r < RPG; ++r) {
                    uint32_t acc = 0;
                    acc = sqdiff4(q4.x, x[r].x, acc);
                    acc = sqdiff4(q4.y, x[r].y, acc);
                    acc = sqdiff4(q4.z, x[r].z, acc);
                    acc = sqdiff4(q4.w, x[r].w, acc);
                    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
                    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
                    if (active[r] && sub == 0) sh.dist[v[r]] += acc;
                }
            }
        } else {
            constexpr int RPG = 2;  // rows per 8-thread group per pass
            const float* hb = reinterpret_cast<const float*>(p.arena + c.hor_off) + (size_t)b * np * kHDim;
            const float* qh = sh.qf + lv.dv + b * kHDim;
            const uint32_t sub = lane & 7;
            const uint32_t groups = T / 8;
            for (uint32_t base = 0; base < npos; base += groups * RPG) {
                uint32_t v[RPG];
                bool active[RPG];
                float x[RPG][8];
#pragma unroll
                for (int r = 0; r < RPG; ++r) {
                    const uint32_t i = base + r * groups + (threadIdx.x >> 3);
                    active[r] = i < npos;
                    v[r] = active[r] ? (all_vectors ? i : sh.pos[i]) : 0u;
                }
#pragma unroll
                for (int r = 0; r < RPG; ++r)
#pragma unroll
                    for (int t = 0; t < 8; ++t)
                        x[r][t] = active[r] ? __ldg(hb + (size_t)v[r] * kHDim + sub + 8 * t) : 0.0f;
#pragma unroll
                for (int r = 0; r < RPG; ++r) {
                    // avx2_computers.hpp:47-98: lane sub accumulates dims sub, sub+8, ... with FMA
                    float acc = 0.0f;
#pragma unroll
                    for (int t = 0; t < 8; ++t) {
                        const float dd = __fsub_rn(qh[sub + 8 * t], x[r][t]);
                        acc = __fmaf_rn(dd, dd, acc);
                    }
                    double sm = (double)acc + (double)__shfl_down_sync(0xffffffffu, acc, 4, 8);
                    sm = sm + __shfl_down_sync(0xffffffffu, sm, 2, 8);
                    sm = sm + __shfl_down_sync(0xffffffffu, sm, 1, 8);
                    if (active[r] && sub == 0)
                        sh.dist[v[r]] = __float_as_uint(__fadd_rn(__uint_as_float(sh.dist[v[r]]), (float)sm));
                }
            }
        }
        __syncthreads();
    }

    __device__ void zero_dist(uint32_t n) {
        for (uint32_t v = threadIdx.x; v < n; v += T) sh.dist[v] = 0u;
        __syncthreads();
    }

    // Largest heap distance and its lowest slot, on every lane of the calling warp. Heap
    // distances are non-negative floats, ordered as their bit patterns.
    __device__ __forceinline__ void warp_heap_top(uint32_t hsize, float& top, uint32_t& slot) const {
        const uint32_t lane = lane_id();
        uint32_t best = 0, bs = 0xFFFFFFFFu;
        for (uint32_t i = lane; i < hsize; i += 32) {
            const uint32_t x = __float_as_uint(sh.hd[i]);
            if (bs == 0xFFFFFFFFu || x > best) {
                best = x;
                bs = i;
            }
        }
        const uint32_t gmax = __reduce_max_sync(0xffffffffu, best);
        slot = __reduce_min_sync(0xffffffffu, best == gmax ? bs : 0xFFFFFFFFu);
        top = __uint_as_float(gmax);
    }

    __device__ void recompute_top() {
        if (threadIdx.x < 32) {
            float top;
            uint32_t slot;
            warp_heap_top(s.hsize, top, slot);
            if (threadIdx.x == 0) {
                s.top = top;
                s.top_slot = slot;
            }
        }
        __syncthreads();
    }

    // Pushes the m smallest raw distances of the cluster (searcher.hpp:256-280).
    __device__ void push_smallest(const DevCluster& c, uint32_t m) {
        if (m == 0) return;
        uint32_t kth, less;
        block_radix_select<T>(sh.dist, c.n, m, s, kth, less);
        const uint32_t* idp = ids(c);
        uint32_t* dist = sh.dist;
        const uint32_t nl = block_compact<T>(
            c.n, [&](uint32_t, uint32_t v) { return dist[v] < kth; }, [](uint32_t i) { return i; },
            sh.pos, s);
        const uint32_t ties_needed = m - nl;
        // ties at the m-th key: lowest positions first
        const uint32_t nt = block_compact<T>(
            c.n, [&](uint32_t, uint32_t v) { return dist[v] == kth; }, [](uint32_t i) { return i; },
            sh.pos + nl, s);
        (void)nt;
        const uint32_t hs = s.hsize;
        for (uint32_t j = threadIdx.x; j < m; j += T) {
            const uint32_t v = sh.pos[j];
            sh.hd[hs + j] = reported(dist[v]);
            sh.hid[hs + j] = __ldg(idp + v);
        }
        (void)ties_needed;
        __syncthreads();
        if (threadIdx.x == 0) s.hsize = hs + m;
        __syncthreads();
        recompute_top();
    }

    // searcher.hpp:217-281
    __device__ void start(const DevCluster& c, uint32_t k) {
        count_bytes((unsigned long long)c.n * lv.d * kElem, kStart);
        zero_dist(c.n);
        vertical_all(c, 0, lv.dv, false, 0);
        __syncthreads();
        for (uint32_t b = 0; b < lv.n_hblocks; ++b) horizontal(c, b, c.n, true);
        if (has_tombstones(c)) mask_tombstones(c, false);
        uint32_t m = k - s.hsize;
        if (m > c.n) m = c.n;
        push_smallest(c, m);
    }

    // searcher.hpp:217-281 on distances computed ahead by the batched Start (pdxg_start.cu):
    // the same exact U8 sums, read instead of recomputed.
    __device__ void start_pre(const DevCluster& c, uint32_t k) {
        count_bytes((unsigned long long)c.n * lv.d * kElem, kStart);
        const uint32_t* src = p.start_dist + (size_t)pre_row * p.start_stride;
        for (uint32_t v = threadIdx.x; v < c.n; v += T) sh.dist[v] = __ldg(src + v);
        __syncthreads();
        if (has_tombstones(c)) mask_tombstones(c, false);
        uint32_t m = k - s.hsize;
        if (m > c.n) m = c.n;
        push_smallest(c, m);
    }

    // searcher.hpp:283-372
    __device__ void filtered_start(const DevCluster& c, uint32_t k, uint32_t passing) {
        zero_dist(c.n);
        const uint32_t nsel = block_compact<T>(
            c.n, [&](uint32_t i, uint32_t) { return selected(c, i); }, [](uint32_t i) { return i; },
            sh.pos, s);
        count_bytes((unsigned long long)nsel * lv.dh * kElem +
                    (unsigned long long)((__fdiv_rn((float)passing, (float)c.n) > (1.0f - kSelectivity)) ? c.n : nsel) *
                        lv.dv * kElem, kStart);
        for (uint32_t b = 0; b < lv.n_hblocks; ++b) horizontal(c, b, nsel, false);
        const float pct = __fdiv_rn((float)passing, (float)c.n);
        if (pct > (1.0f - kSelectivity)) {
            vertical_all(c, 0, lv.dv, false, 0);
            __syncthreads();
        } else {
            vertical_pos(c, 0, lv.dv, nsel);
        }
        uint32_t m = k - s.hsize;
        if (m > passing) m = passing;
        const uint32_t mask = mask_raw();
        for (uint32_t v = threadIdx.x; v < c.n; v += T)
            if (!selected(c, v)) sh.dist[v] = mask;
        __syncthreads();
        push_smallest(c, m);
    }

    // Warmup + Prune + MergeIntoHeap for one cluster with a full heap.
    __device__ void prune_cluster(const DevCluster& c, uint32_t k, uint32_t passing) {
        const uint32_t n = c.n;
        uint32_t cur = 0;
        bool skip_warmup = false;
        if (fsel) {
            zero_dist(n);
            const uint32_t mask = mask_raw();
            for (uint32_t v = threadIdx.x; v < n; v += T)
                if (!selected(c, v)) sh.dist[v] = mask;
            __syncthreads();
            const float pct = __fdiv_rn((float)passing, (float)n);
            skip_warmup = pct < (1.0f - kSelectivity);
        }
        bool bits_ready = false;  // sh.bits holds the vectors below the bound at `cur`
        // tombstoned slots (unfiltered; a filter never selects them) start the warmup at the
        // mask value and are reset to it before the survivors are taken (searcher.hpp:393, 453)
        if (!fsel && has_tombstones(c)) mask_tombstones(c, true);
        if (!skip_warmup) {
            // Warmup (searcher.hpp:374-435); the first step starts the distances from 0
            const uint32_t needed = (uint32_t)ceilf(__fmul_rn(kSelectivity, (float)n));
            uint32_t n_pruned = 0, step = 0;
            while (n_pruned < needed && cur < lv.dv) {
                uint32_t last = cur + c_fetch_sizes[step < kNumFetchSizes ? step : kNumFetchSizes - 1];
                if (last > lv.dv) last = lv.dv;
                const uint32_t thr = thr_raw(last);
                count_bytes((unsigned long long)n * (last - cur) * kElem, kWarmup);
                n_pruned = vertical_all(c, cur, last, true, thr, cur == 0 && !fsel && !has_tombstones(c));  // ends with a barrier
                cur = last;
                ++step;
                bits_ready = !fsel;
            }
        }
        if (!fsel && has_tombstones(c)) {
            mask_tombstones(c, false);
            bits_ready = false;
        }
        // Prune (searcher.hpp:437-540): the vectors below the bound at the warmup's last
        // checkpoint, in position order
        const uint32_t thr = thr_raw(cur);
        uint32_t* dist = sh.dist;
        const LevelOps* self = this;  // captured by the predicate
        const uint32_t nsurv =
            bits_ready ? compact_bits(n)
                       : block_compact<T>(
                             n,
                             [&](uint32_t i, uint32_t) { return self->below(dist[i], thr) && self->selected(c, i); },
                             [](uint32_t i) { return i; }, sh.pos, s);
        // The bound's heap top is fixed until the merge, so a survivor's way through the
        // horizontal blocks and the remaining vertical dims depends on that vector alone: each
        // thread follows whole survivors, and the vectors reaching the merge, and their order,
        // are those of the reference's block-by-block compaction.
        uint32_t hbytes = 0, vbytes = 0;
        for (uint32_t i = threadIdx.x; i < nsurv; i += T) {
            const uint32_t v = sh.pos[i];
            uint32_t raw = sh.dist[v];
            if (follow_survivor(c, v, cur, raw, hbytes, vbytes)) sh.dist[v] = raw;
            else sh.pos[i] = 0xFFFFFFFFu;
        }
        if (p.stats) {  // block-uniform
            const uint32_t hb = block_sum<T>(hbytes, s), vb = block_sum<T>(vbytes, s);
            count_bytes(hb, kSurvivorH);
            count_bytes(vb, kSurvivorV);
        }
        __syncthreads();
        // MergeIntoHeap (searcher.hpp:542-566): sequential, strict-<, in position order.
        if (threadIdx.x < 32 && nsurv) {
            const uint32_t lane = lane_id();
            const uint32_t* idp = ids(c);
            float top = s.top;
            uint32_t slot = s.top_slot;
            uint32_t hsize = s.hsize;
            uint32_t merged = 0;
            for (uint32_t i0 = 0; i0 < nsurv; i0 += 32) {
                const uint32_t i = i0 + lane;
                const uint32_t v = i < nsurv ? sh.pos[i] : 0xFFFFFFFFu;
                const bool alive = v != 0xFFFFFFFFu;
                const float dd = alive ? reported(sh.dist[v]) : 0.0f;
                const uint32_t idv = alive ? __ldg(idp + v) : 0u;
                unsigned bal = __ballot_sync(0xffffffffu, alive);
                merged += __popc(bal);
                while (bal) {
                    const int j = __ffs(bal) - 1;
                    bal &= bal - 1;
                    const float ddj = __shfl_sync(0xffffffffu, dd, j);
                    const uint32_t idj = __shfl_sync(0xffffffffu, idv, j);
                    if (hsize < k || ddj < top) {
                        if (lane == 0) {
                            const uint32_t at = (hsize >= k) ? slot : hsize;
                            sh.hd[at] = ddj;
                            sh.hid[at] = idj;
                        }
                        if (hsize < k) ++hsize;
                        __syncwarp();
                        warp_heap_top(hsize, top, slot);
                    }
                }
            }
            if (lane == 0) {
                s.top = top;
                s.top_slot = slot;
                s.hsize = hsize;
                if (p.stats) s.merged += merged;
            }
        }
        __syncthreads();
    }

    // Raw distance of vector v plus horizontal block b (searcher.hpp:437-540 per vector).
    __device__ __forceinline__ uint32_t add_hblock(const DevCluster& c, uint32_t b, uint32_t v, uint32_t raw) const {
        const uint32_t np = c.n_pad;
        if constexpr (U8) {
            const uint4* row = reinterpret_cast<const uint4*>(p.arena + c.hor_off + ((size_t)b * np + v) * kHDim);
            const uint4* qh = reinterpret_cast<const uint4*>(sh.qw + lv.qw_hoff + b * 16);
            uint4 x[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) x[t] = __ldg(row + t);
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const uint4 q4 = qh[t];
                raw = sqdiff4(q4.x, x[t].x, raw);
                raw = sqdiff4(q4.y, x[t].y, raw);
                raw = sqdiff4(q4.z, x[t].z, raw);
                raw = sqdiff4(q4.w, x[t].w, raw);
            }
            return raw;
        } else {
            // avx2_computers.hpp:47-98: lane j of 8 accumulates dims j, j + 8, ... with FMA;
            // lanes j and j + 4 are added in double, then (0 + 2) + (1 + 3)
            const float* row = reinterpret_cast<const float*>(p.arena + c.hor_off) + ((size_t)b * np + v) * kHDim;
            const float* qh = sh.qf + lv.dv + b * kHDim;
            double sj[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const float d0 = __fsub_rn(qh[j + 8 * t], __ldg(row + j + 8 * t));
                    a0 = __fmaf_rn(d0, d0, a0);
                    const float d1 = __fsub_rn(qh[j + 4 + 8 * t], __ldg(row + j + 4 + 8 * t));
                    a1 = __fmaf_rn(d1, d1, a1);
                }
                sj[j] = (double)a0 + (double)a1;
            }
            const float h = (float)((sj[0] + sj[2]) + (sj[1] + sj[3]));
            return __float_as_uint(__fadd_rn(__uint_as_float(raw), h));
        }
    }

    // Raw distance of vector v plus vertical dims [d0, d1) in dimension order.
    __device__ __forceinline__ uint32_t add_vertical(const DevCluster& c, uint32_t v, uint32_t d0, uint32_t d1,
                                                     uint32_t raw) const {
        const uint32_t* base = vert(c);
        const uint32_t np = c.n_pad;
        if constexpr (U8) {
            const uint32_t g0 = d0 >> 2, g1 = (d1 + 3) >> 2;
            for (uint32_t g = g0; g < g1; ++g) raw = sqdiff4(sh.qw[g], __ldg(base + (size_t)g * np + v), raw);
            return raw;
        } else {
            const float* fb = reinterpret_cast<const float*>(base);
            float acc = __uint_as_float(raw);
            for (uint32_t j = d0; j < d1; ++j) {
                const float t = __fsub_rn(sh.qf[j], __ldg(fb + (size_t)j * np + v));
                acc = __fmaf_rn(t, t, acc);
            }
            return __float_as_uint(acc);
        }
    }

    // One survivor of the warmup bound from checkpoint cur0 on: the horizontal blocks, then the
    // remaining vertical dims in 64-dim steps, re-tested after each (searcher.hpp:437-540).
    // Returns whether it is still below the bound at the end; raw is its running distance.
    __device__ __forceinline__ bool follow_survivor(const DevCluster& c, uint32_t v, uint32_t cur0, uint32_t& raw,
                                                    uint32_t& hbytes, uint32_t& vbytes) const {
        uint32_t cur = cur0;
        for (uint32_t b = 0; b < lv.n_hblocks; ++b) {
            hbytes += kHDim * kElem;
            raw = add_hblock(c, b, v, raw);
            cur += kHDim;
            if (!below(raw, thr_raw(cur))) return false;
        }
        uint32_t cur_v = cur0;
        while (cur_v < lv.dv) {
            const uint32_t last = (cur_v + kHDim < lv.dv) ? cur_v + kHDim : lv.dv;
            vbytes += (last - cur_v) * kElem;
            raw = add_vertical(c, v, cur_v, last, raw);
            cur = (cur + kHDim < lv.d) ? cur + kHDim : lv.d;
            cur_v = last;
            if (!below(raw, thr_raw(cur))) return false;
            if (cur == lv.d) break;
        }
        return true;
    }

    // Visits clusters order[0, nvisit) (searcher.hpp:655-721 / 776-853).
    // `order` is sh.order or, for visit orders computed ahead of the scan, the query's row of
    // them in global memory.
    __device__ void run(uint32_t k, uint32_t nvisit, const uint32_t* order) {
        if (threadIdx.x == 0) {
            s.hsize = 0;
            s.top = 0.0f;
            s.top_slot = 0;
        }
        __syncthreads();
        for (uint32_t ci = 0; ci < nvisit; ++ci) {
            const uint32_t cidx = order[ci];
            const DevCluster c = lv.clusters[cidx];
            uint32_t passing = 0;
            if (fsel) {
                passing = __ldg(fpass + cidx);
                if (passing == 0) continue;
            }
            if ((TOMB ? c.live : c.n) == 0) continue;  // num_embeddings == 0 (searcher.hpp:662)
            if (p.stats && threadIdx.x == 0) s.visits += 1;
            if (s.hsize < k) {
                long long t0 = 0;
                if (p.stats && threadIdx.x == 0) t0 = clock64();
                if (fsel)
                    filtered_start(c, k, passing);
                else if (pre_row >= 0 && s.hsize == 0 && cidx == pre_cluster)
                    start_pre(c, k);
                else
                    start(c, k);
                if (p.stats && threadIdx.x == 0 && !top_level)
                    s.cycles[1] += (unsigned long long)(clock64() - t0);
                continue;
            }
            prune_cluster(c, k, passing);
        }
    }

    // Sorts the heap ascending into sh.sortw; returns the result count (searcher.hpp:568-585).
    __device__ uint32_t sort_heap(uint32_t k) {
        uint32_t hs = s.hsize;
        const uint32_t N = next_pow2(hs ? hs : 1);
        for (uint32_t i = threadIdx.x; i < N; i += T)
            sh.sortw[i] = (i < hs) ? ((uint64_t)__float_as_uint(sh.hd[i]) << 32) | sh.hid[i]
                                   : ~0ull;
        __syncthreads();
        block_bitonic_sort<T>(sh.sortw, N);
        // drop one FLT_MAX initialisation element when it is the maximum
        if (hs && __uint_as_float((uint32_t)(sh.sortw[hs - 1] >> 32)) == FLT_MAX) --hs;
        return hs < k ? hs : k;
    }

    // Probe order over the level's centroids: nearest `nprobe` sorted ascending into sh.order.
    __device__ uint32_t probe(uint32_t nprobe) {
        const uint32_t nc = lv.nclusters;
        count_bytes((unsigned long long)nc * lv.d * 4u, kProbe);
        const uint32_t lane = lane_id(), sub = lane & 7;
        for (uint32_t base = 0; base < nc; base += T / 8) {
            const uint32_t cidx = base + (threadIdx.x >> 3);
            const bool active = cidx < nc;
            const float d = horiz_f32_group8(sh.qf, lv.centroids + (size_t)(active ? cidx : 0) * lv.d,
                                             lv.d, sub, active);
            if (active && sub == 0) sh.dist[cidx] = __float_as_uint(d);
        }
        __syncthreads();
        const uint32_t m = nprobe < nc ? nprobe : nc;
        uint32_t kth, less;
        block_radix_select<T>(sh.dist, nc, m, s, kth, less);
        uint32_t* dist = sh.dist;
        const uint32_t nl = block_compact<T>(
            nc, [&](uint32_t, uint32_t v) { return dist[v] < kth; }, [](uint32_t i) { return i; },
            sh.pos, s);
        block_compact<T>(nc, [&](uint32_t, uint32_t v) { return dist[v] == kth; },
                         [](uint32_t i) { return i; }, sh.pos + nl, s);
        const uint32_t N = next_pow2(m);
        for (uint32_t i = threadIdx.x; i < N; i += T) {
            if (i < m) {
                const uint32_t ci = sh.pos[i];
                sh.sorth[i] = ((uint64_t)dist[ci] << 32) | ci;
            } else {
                sh.sorth[i] = ~0ull;
            }
        }
        __syncthreads();
        block_bitonic_sort<T>(sh.sorth, N);
        for (uint32_t i = threadIdx.x; i < m; i += T) sh.order[i] = (uint32_t)sh.sorth[i];
        __syncthreads();
        return m;
    }
};

// ------------------------------------------------------------------------------------------
template <int T>
__device__ void prepare_query(const SearchParams& p, Shared& sh, uint32_t q) {
    const DevLevel& lv = p.l1;
    const float* src = p.queries + (size_t)q * lv.d;
    for (uint32_t i = threadIdx.x; i < lv.d; i += T) sh.qf[i] = __ldg(src + i);
    __syncthreads();
    if (lv.is_u8) {
        // QuantizeEmbedding (scalar.hpp:76-94), packed into the device word layout
        const uint32_t nw = lv.qw_hoff + lv.n_hblocks * 16;
        for (uint32_t w = threadIdx.x; w < nw; w += T) sh.qw[w] = quantize_word(sh.qf, lv, w);
        __syncthreads();
    }
}

template <bool U8, int T, bool TOMB>
__global__ void __launch_bounds__(T) search_kernel(const __grid_constant__ SearchParams p) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ Scalars s;
    Shared sh;
    sh.qf = reinterpret_cast<float*>(smem + p.smem_qf);
    sh.qw = reinterpret_cast<uint32_t*>(smem + p.smem_qw);
    sh.dist = reinterpret_cast<uint32_t*>(smem + p.smem_work);
    sh.pos = sh.dist + p.work_cap;
    sh.sortw = reinterpret_cast<uint64_t*>(smem + p.smem_work);
    sh.hd = reinterpret_cast<float*>(smem + p.smem_heap);
    sh.hid = reinterpret_cast<uint32_t*>(smem + p.smem_heap) + p.heap_cap;
    sh.sorth = reinterpret_cast<uint64_t*>(smem + p.smem_heap);
    sh.order = reinterpret_cast<uint32_t*>(smem + p.smem_order);
    sh.bits = reinterpret_cast<uint32_t*>(smem + p.smem_bits);

    const uint32_t n_list = p.q_list ? __ldg(p.q_list_n) : p.nq;
    for (;;) {
        if (threadIdx.x == 0) s.query = atomicAdd(p.queue, 1u);
        __syncthreads();
        const uint32_t slot = s.query;
        __syncthreads();
        if (slot >= n_list) break;
        const uint32_t q = p.q_list ? __ldg(p.q_list + slot) : slot;
        if (threadIdx.x == 0) {
            for (int i = 0; i < 6; ++i) s.bytes[i] = 0;
            for (int i = 0; i < 3; ++i) s.cycles[i] = 0;
            s.visits = 0;
            s.merged = 0;
        }
        const int filter = p.filter_of ? p.filter_of[q] : -1;
        prepare_query<T>(p, sh, q);

        long long t_q0 = 0;
        if (p.stats && threadIdx.x == 0) t_q0 = clock64();
        // per-query parameters (serving batches mix them); p.k is the output row stride
        const uint32_t kq = p.q_k ? __ldg(p.q_k + q) : p.k;
        const uint32_t npq = p.q_nprobe ? __ldg(p.q_nprobe + q) : p.nprobe;
        const uint32_t topq = p.q_top ? __ldg(p.q_top + q) : p.top_nprobe;
        uint32_t nvisit;
        const uint32_t* visit = sh.order;  // the query's L1 visit order
        if (p.order) {
            // caller-provided access order (PDXearch::SetClusterAccessOrder, searcher.hpp:48-54)
            nvisit = npq < p.n_order ? npq : p.n_order;
            for (uint32_t i = threadIdx.x; i < nvisit; i += T) sh.order[i] = __ldg(p.order + i);
            __syncthreads();
        } else if (filter == -1 && p.q_order) {
            // the tree top level (pdxg_toplevel.cu) or a probe ahead of the scan (pdxg_probe.cu)
            // already produced this query's L1 order: read in place
            nvisit = __ldg(p.q_order_count + q);
            visit = p.q_order + (size_t)q * p.q_order_stride;
        } else if (p.is_tree && filter == -1) {
            // PDXTreeIndex::Search (index.hpp:545-566): pruned F32 search over the meso
            // clusters with k = nprobe returns the L1 clusters to visit, nearest first.
            LevelOps<T, false> top(p, p.l0, sh, s, -1, true);
            const uint32_t nv0 = topq < p.l0.nclusters ? topq : p.l0.nclusters;
            top.probe(topq);
            top.run(npq, nv0, sh.order);
            const uint32_t cnt = top.sort_heap(npq);
            for (uint32_t i = threadIdx.x; i < cnt; i += T) sh.order[i] = (uint32_t)sh.sortw[i];
            __syncthreads();
            nvisit = cnt;
        } else {
            LevelOps<T, false> probe_ops(p, p.l1, sh, s, -1);
            nvisit = probe_ops.probe(npq);
        }

        if (p.stats && threadIdx.x == 0) {
            const long long now = clock64();
            s.cycles[0] += (unsigned long long)(now - t_q0);
            t_q0 = now;
        }
        LevelOps<T, U8, TOMB> ops(p, p.l1, sh, s, filter);
        if (U8 && p.start_row && filter == -1) {
            ops.pre_row = __ldg(p.start_row + q);
            ops.pre_cluster = __ldg(p.start_first + q);
        }
        ops.run(kq, nvisit, visit);
        const uint32_t cnt = ops.sort_heap(kq);
        uint32_t* oi = p.out_ids + (size_t)q * p.k;
        float* od = p.out_dists + (size_t)q * p.k;
        for (uint32_t i = threadIdx.x; i < p.k; i += T) {
            if (i < cnt) {
                const uint64_t e = sh.sortw[i];
                oi[i] = (uint32_t)e;
                od[i] = __uint_as_float((uint32_t)(e >> 32));
            } else {
                oi[i] = 0xFFFFFFFFu;
                od[i] = __int_as_float(0x7f800000);
            }
        }
        if (threadIdx.x == 0) {
            p.out_counts[q] = cnt;
            if (p.stats) {
                s.cycles[2] += (unsigned long long)(clock64() - t_q0) - s.cycles[1];
                for (int i = 0; i < 3; ++i) atomicAdd(p.stats + 9 + i, s.cycles[i]);
                unsigned long long tot = 0;
                for (int i = 0; i < 6; ++i) {
                    tot += s.bytes[i];
                    atomicAdd(p.stats + 3 + i, s.bytes[i]);
                }
                atomicAdd(p.stats, tot);
                atomicAdd(p.stats + 1, s.visits);
                atomicAdd(p.stats + 2, s.merged);
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------
// Tree top level as its own launch (PDXTreeIndex::Search, index.hpp:545-566): small CTAs, one
// per query, run the same per-query top-level search as search_kernel's tree branch -- meso
// probe, pruned F32 search over the meso clusters with k = L1 nprobe -- and write the sorted
// L1 order. Meso clusters are small, so 64 threads keep busy and many more queries are in
// flight than with the L1 search's 256-thread CTAs. search_kernel then reads p.q_order.
template <int T>
__global__ void __launch_bounds__(T) top_level_kernel(const __grid_constant__ SearchParams p) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ Scalars s;
    Shared sh;
    sh.qf = reinterpret_cast<float*>(smem + p.smem_qf);
    sh.qw = nullptr;
    sh.dist = reinterpret_cast<uint32_t*>(smem + p.smem_work);
    sh.pos = sh.dist + p.work_cap;
    sh.sortw = reinterpret_cast<uint64_t*>(smem + p.smem_work);
    sh.hd = reinterpret_cast<float*>(smem + p.smem_heap);
    sh.hid = reinterpret_cast<uint32_t*>(smem + p.smem_heap) + p.heap_cap;
    sh.sorth = reinterpret_cast<uint64_t*>(smem + p.smem_heap);
    sh.order = reinterpret_cast<uint32_t*>(smem + p.smem_order);
    sh.bits = reinterpret_cast<uint32_t*>(smem + p.smem_bits);
    uint32_t* out_order = const_cast<uint32_t*>(p.q_order);
    uint32_t* out_count = const_cast<uint32_t*>(p.q_order_count);
    for (;;) {
        if (threadIdx.x == 0) s.query = atomicAdd(p.queue, 1u);
        __syncthreads();
        const uint32_t q = s.query;
        __syncthreads();
        if (q >= p.nq) break;
        if (p.filter_of && __ldg(p.filter_of + q) != -1) {
            // filtered queries probe the L1 centroids directly (no top-level search)
            if (threadIdx.x == 0) out_count[q] = 0;
            continue;
        }
        if (threadIdx.x == 0) {
            for (int i = 0; i < 6; ++i) s.bytes[i] = 0;
            s.visits = 0;
            s.merged = 0;
        }
        const float* src = p.queries + (size_t)q * p.l0.d;
        for (uint32_t i = threadIdx.x; i < p.l0.d; i += T) sh.qf[i] = __ldg(src + i);
        __syncthreads();
        LevelOps<T, false> top(p, p.l0, sh, s, -1, true);
        const uint32_t npq = p.q_nprobe ? __ldg(p.q_nprobe + q) : p.nprobe;
        const uint32_t topq = p.q_top ? __ldg(p.q_top + q) : p.top_nprobe;
        const uint32_t nv0 = topq < p.l0.nclusters ? topq : p.l0.nclusters;
        top.probe(topq);
        top.run(npq, nv0, sh.order);
        const uint32_t cnt = top.sort_heap(npq);
        for (uint32_t i = threadIdx.x; i < cnt; i += T)
            out_order[(size_t)q * p.q_order_stride + i] = (uint32_t)sh.sortw[i];
        if (threadIdx.x == 0) {
            out_count[q] = cnt;
            if (p.stats) {
                atomicAdd(p.stats + 3, s.bytes[kTopLevel]);
                atomicAdd(p.stats, s.bytes[kTopLevel]);
                atomicAdd(p.stats + 1, s.visits);
            }
        }
        __syncthreads();
    }
}

// 64 threads per query for batches (many CTAs per SM), 256 when a few queries have the GPU to
// themselves (an Append, a single query): the same decisions, less latency.
cudaError_t launch_top_level(const SearchParams& p, int grid, cudaStream_t st, int threads) {
    auto kern = threads == 256 ? top_level_kernel<256> : top_level_kernel<64>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem_total);
    if (e != cudaSuccess) return e;
    kern<<<grid, threads == 256 ? 256 : 64, p.smem_total, st>>>(p);
    return cudaGetLastError();
}

// Resident CTAs per SM, remembered per (device, kernel form, threads, shared memory): the planner
// asks for every search, and a single-row Append pays the driver query otherwise.
template <class F>
static int cached_occupancy(int kind, int threads, size_t smem, F query) {
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, size_t>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(dev, kind, threads, smem);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    const int blocks = query();
    if (blocks > 0) {
        std::lock_guard<std::mutex> lock(mu);
        cache[key] = blocks;
    }
    return blocks;
}

int top_level_occupancy(size_t smem, int threads) {
    return cached_occupancy(-1, threads, smem, [&] {
        int blocks = 0;
        auto kern = threads == 256 ? top_level_kernel<256> : top_level_kernel<64>;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, threads == 256 ? 256 : 64, smem);
        return blocks;
    });
}

// ------------------------------------------------------------------------------------------
template <bool U8, int T>
static cudaError_t launch_t(const SearchParams& p, int grid, cudaStream_t st) {
    auto kern = p.l1.tomb ? search_kernel<U8, T, true> : search_kernel<U8, T, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)p.smem_total);
    if (e != cudaSuccess) return e;
    kern<<<grid, T, p.smem_total, st>>>(p);
    return cudaGetLastError();
}

template <bool U8, int T>
static int occupancy_u(size_t smem) {
    int blocks = 0;
    cudaFuncSetAttribute(search_kernel<U8, T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, search_kernel<U8, T, false>, T, smem);
    return blocks;
}
template <int T>
static int occupancy_t(bool u8, size_t smem) {
    return u8 ? occupancy_u<true, T>(smem) : occupancy_u<false, T>(smem);
}

int search_occupancy(bool u8, int threads, size_t smem) {
    return cached_occupancy(u8 ? 1 : 0, threads, smem, [&] {
        switch (threads) {
        case 64: return occupancy_t<64>(u8, smem);
        case 128: return occupancy_t<128>(u8, smem);
        case 256: return occupancy_t<256>(u8, smem);
        case 512: return occupancy_t<512>(u8, smem);
        default: return 0;
        }
    });
}

cudaError_t launch_search(const SearchParams& p, bool u8, int threads, int grid, cudaStream_t st) {
    switch (threads) {
    case 64: return u8 ? launch_t<true, 64>(p, grid, st) : launch_t<false, 64>(p, grid, st);
    case 128: return u8 ? launch_t<true, 128>(p, grid, st) : launch_t<false, 128>(p, grid, st);
    case 256: return u8 ? launch_t<true, 256>(p, grid, st) : launch_t<false, 256>(p, grid, st);
    case 512: return u8 ? launch_t<true, 512>(p, grid, st) : launch_t<false, 512>(p, grid, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace pdxg
