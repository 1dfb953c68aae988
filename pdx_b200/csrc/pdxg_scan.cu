// Cluster-major scan of U8 levels: PDXearch (searcher.hpp:217-566) for a whole batch, with the
// first warmup step computed once per cluster for all the queries that visit it.
//
// Per query, PDXearch visits its clusters in order. The first non-empty one is a Start (full
// distances, the best k pushed); every later one runs Warmup: partial distances over the
// vertical dims in steps of 16, 16, 32, ... (DIMENSIONS_FETCHING_SIZES), testing after each step
// how many vectors reach the ADSampling bound thr(top) = top * ratio[dims] (as U8 raw distances)
// and stopping once ceil(0.8 n) do. On the IVF2 SQ8 workloads that exit comes after the first
// step almost always, so most of the scan is the first 16 dims of every vector of every visited
// cluster, one query at a time, each query re-reading the same clusters.
//
// The heap top only falls once the heap is full (MergeIntoHeap replaces the top with a smaller
// distance), and the bound is monotone in it. So the bound a query applies at any later cluster
// is at most tau0, its heap top right after the Start, and a vector below that later bound at
// the first checkpoint is below the bound at tau0. That set -- the candidates -- is computed
// cluster-major: every cluster's first-checkpoint rows are read once per group of 64 queries and
// each (query, cluster) pair gets a bitmap of its candidates. Then one warp per query replays
// PDXearch in visit order with its true heap top: the vectors below the bound are the
// candidates whose exact first-checkpoint distance is below it, so the warmup's count and its
// survivors are exact; where the warmup would not stop after the first step the warp runs the
// whole warmup itself. Survivors then follow Prune (searcher.hpp:437-540) one per lane and are
// merged in position order (searcher.hpp:542-566), as in the per-query kernel.
//
//   scan_prep_kernel   : warp per query -- quantized query words, the Start's pushes (the m
//                        smallest batched-Start distances, ties by position) and tau0's bound;
//                        every later visit appended to its cluster's list, with a work item per
//                        64 list entries; queries this path does not take go to a list for the
//                        per-query kernel
//   scan_bitmap_kernel : persistent CTAs over the items: candidate bitmaps with dp4a, exact
//                        |q - x|^2 = |q|^2 + |x|^2 - 2 q.x over the first checkpoint's dims
//   scan_replay_kernel : warp per query -- Warmup / Prune / MergeIntoHeap / result
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "pdxg_block.cuh"
#include "pdxg_common.cuh"

namespace pdxg {

constexpr uint32_t kScanCQ = 64;         // visits per bitmap work item
constexpr int kBitmapThreads = 256;
constexpr int kBitmapBPW = 4;            // 32-vector blocks a bitmap warp holds at once
constexpr int kScanWarps = 8;            // queries per prep / replay CTA
constexpr uint32_t kOffPath = 0xFFFFFFFFu;

// DIMENSIONS_FETCHING_SIZES (common.hpp:47-49)
__constant__ uint32_t c_scan_fetch[kNumFetchSizes] = {16, 16, 32, 32, 32, 32, 64, 64, 64, 64,
                                                     128, 128, 128, 128, 256, 256, 512, 1024, 2048, 16384};

__device__ __forceinline__ uint32_t sq4(uint32_t a, uint32_t b, uint32_t acc) {
    const uint32_t d = __vabsdiffu4(a, b);
    return __dp4a(d, d, acc);
}

// GetPruningThreshold (searcher.hpp:75-91) for U8: top * ratio[cur] scaled to the raw domain,
// saturating (the same float steps as LevelOps::thr_raw).
__device__ __forceinline__ uint32_t thr_u8(float top, uint32_t cur, const DevLevel& lv, const float* ratios) {
    const float r = (cur == lv.d) ? 1.0f : __ldg(ratios + cur);
    const float scaled = __fmul_rn(__fmul_rn(top, r), lv.scale_sq);
    return scaled >= 4294967296.0f ? 0xFFFFFFFFu : __float2uint_rz(scaled);
}

__device__ __forceinline__ float reported_u8(uint32_t raw, const DevLevel& lv) {
    return __fmul_rn(__uint2float_rn(raw), lv.inv_scale_sq);
}

__device__ __forceinline__ void add_stat(const ScanParams& sp, int idx, unsigned long long v) {
    if (v) atomicAdd(sp.stats + idx, v);
}

// ------------------------------------------------------------------------------------ prep
constexpr int kRegKeys = 32;  // Start distances a prep lane keeps in registers (clusters <= 1024)

// The m-th smallest of the n keys key(v) (exact radix select, 8 bits a pass; hist: 256 words of
// this warp's shared memory).
template <class Key>
__device__ __forceinline__ uint32_t warp_radix_select(uint32_t n, uint32_t m, uint32_t* hist, Key key) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t prefix = 0, mask = 0, rem = m;
    for (int shift = 24; shift >= 0; shift -= 8) {
#pragma unroll
        for (int j = 0; j < 8; ++j) hist[lane * 8 + j] = 0;
        __syncwarp();
        key.for_each(n, [&](uint32_t, uint32_t k) {
            if ((k & mask) == prefix) atomicAdd(&hist[(k >> shift) & 255u], 1u);
        });
        __syncwarp();
        uint32_t loc[8], sum = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            loc[j] = hist[lane * 8 + j];
            sum += loc[j];
        }
        uint32_t tot;
        const uint32_t excl = warp_exclusive_scan(sum, tot);
        const unsigned own = __ballot_sync(0xffffffffu, excl < rem && rem <= excl + sum);
        const uint32_t owner = __ffs(own) - 1;
        uint32_t bin = 0, cum = excl;
        if (lane == owner) {
            int b = 0;
            for (; b < 7; ++b) {
                if (cum + loc[b] >= rem) break;
                cum += loc[b];
            }
            bin = lane * 8 + b;
        }
        bin = __shfl_sync(0xffffffffu, bin, owner);
        cum = __shfl_sync(0xffffffffu, cum, owner);
        prefix |= bin << shift;
        mask |= 0xFFu << shift;
        rem -= cum;
        __syncwarp();
    }
    return prefix;
}

// Start distances held by the lanes: key j of a lane is vector 32 j + lane (all loads issued
// together).
struct RegKeys {
    uint32_t k[kRegKeys];
    __device__ __forceinline__ void load(const uint32_t* src, uint32_t n) {
        const uint32_t lane = threadIdx.x & 31;
#pragma unroll
        for (int j = 0; j < kRegKeys; ++j) {
            const uint32_t v = 32u * j + lane;
            k[j] = v < n ? __ldg(src + v) : 0xFFFFFFFFu;
        }
    }
    template <class F>
    __device__ __forceinline__ void for_each(uint32_t n, F f) const {
        const uint32_t lane = threadIdx.x & 31;
#pragma unroll
        for (int j = 0; j < kRegKeys; ++j)
            if (32u * j + lane < n) f(32u * j + lane, k[j]);
    }
    // f(v0, key of v0 + lane) for the 32-vector chunks v0 = 0, 32, ... below n, in order
    template <class F>
    __device__ __forceinline__ void for_chunks(uint32_t n, F f) const {
#pragma unroll
        for (int j = 0; j < kRegKeys; ++j)
            if (32u * j < n) f(32u * j, k[j]);
    }
};

// Start distances read from global memory (clusters larger than the register form).
struct MemKeys {
    const uint32_t* src;
    template <class F>
    __device__ __forceinline__ void for_each(uint32_t n, F f) const {
        for (uint32_t v = threadIdx.x & 31; v < n; v += 32) f(v, src[v]);
    }
    template <class F>
    __device__ __forceinline__ void for_chunks(uint32_t n, F f) const {
        for (uint32_t v0 = 0; v0 < n; v0 += 32) {
            const uint32_t v = v0 + (threadIdx.x & 31);
            f(v0, v < n ? src[v] : 0xFFFFFFFFu);
        }
    }
};

// Start (searcher.hpp:256-280): the m smallest keys pushed in the order of
// LevelOps::push_smallest -- the keys below the m-th in position order, then the ties at it.
// Returns the m-th key.
template <class Key>
__device__ __forceinline__ uint32_t start_push(const Key& key, uint32_t n, uint32_t m, uint32_t* hist,
                                               const uint32_t* ids, const DevLevel& lv, float* hd, uint32_t* hid) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t kth = warp_radix_select(n, m, hist, key);
    uint32_t pushed = 0;
    for (int pass = 0; pass < 2 && pushed < m; ++pass) {
        key.for_chunks(n, [&](uint32_t v0, uint32_t kv) {
            const uint32_t v = v0 + lane;
            const bool sel = pushed < m && v < n && (pass == 0 ? kv < kth : kv == kth);
            const unsigned b = __ballot_sync(0xffffffffu, sel);
            const uint32_t at = pushed + __popc(b & ((1u << lane) - 1u));
            if (sel && at < m) {
                hd[at] = reported_u8(kv, lv);
                hid[at] = __ldg(ids + v);
            }
            pushed += __popc(b);
        });
    }
    return kth;
}

// Dynamic shared memory: the warps' query rows (prep_qs set: kScanWarps x d floats), staged
// with one coalesced pass; without it the query is read from global memory.
__global__ void __launch_bounds__(kScanWarps * 32) scan_prep_kernel(const __grid_constant__ ScanParams sp) {
    __shared__ uint32_t hist_all[kScanWarps][256];
    extern __shared__ __align__(16) float qs_all[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t q = blockIdx.x * kScanWarps + warp;
    if (q >= sp.nq) return;  // whole warp
    uint32_t* hist = hist_all[warp];
    const DevLevel& lv = sp.l1;
    const bool plain = !sp.filter_of || __ldg(sp.filter_of + q) == -1;
    const int32_t row = plain ? __ldg(sp.start_row + q) : -1;
    const uint32_t kq = sp.q_k ? __ldg(sp.q_k + q) : sp.k;
    auto leave = [&]() {
        if (lane == 0) {
            sp.first_i[q] = kOffPath;
            sp.left[atomicAdd(sp.left_n, 1u)] = q;
        }
    };
    if (row < 0) {
        leave();
        return;
    }
    const uint32_t first = __ldg(sp.start_first + q);
    const DevCluster cl = lv.clusters[first];
    const uint32_t n = cl.n;
    const uint32_t m = kq < n ? kq : n;
    if (m < kq) {  // the heap is not full after the Start: the next cluster is a Start too
        leave();
        return;
    }
    // position of the Start cluster in the visit order
    const uint32_t* ord = sp.q_order + (size_t)q * sp.q_order_stride;
    const uint32_t cnt = __ldg(sp.q_order_count + q);
    uint32_t fi = kOffPath;
    for (uint32_t i0 = 0; i0 < cnt && fi == kOffPath; i0 += 32) {
        const uint32_t i = i0 + lane;
        const unsigned b = __ballot_sync(0xffffffffu, i < cnt && __ldg(ord + i) == first);
        if (b) fi = i0 + __ffs(b) - 1;
    }
    if (fi == kOffPath) {
        leave();
        return;
    }
    const uint32_t* src = sp.start_dist + (size_t)row * sp.start_stride;
    RegKeys rk;
    if (n <= 32u * kRegKeys) rk.load(src, n);  // in flight while the query is quantized
    // QuantizeEmbedding (scalar.hpp:76-94) in the scan's packed word layout; |q|^2 over the
    // first checkpoint's words
    const float* qf = sp.queries + (size_t)q * lv.d;
    if (sp.prep_qs) {
        float* qs = qs_all + (size_t)warp * sp.prep_qs_stride;
        for (uint32_t i0 = 0; i0 < lv.d; i0 += 128) {
            float t[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t i = i0 + 32 * u + lane;
                t[u] = i < lv.d ? __ldg(qf + i) : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t i = i0 + 32 * u + lane;
                if (i < lv.d) qs[i] = t[u];
            }
        }
        __syncwarp();
        qf = qs;
    }
    uint32_t* qw = sp.qwords + (size_t)q * sp.nwords;
    uint32_t qn = 0;
    for (uint32_t w = lane; w < sp.nwords; w += 32) {
        const uint32_t word = quantize_word(qf, lv, w);
        qw[w] = word;
        if (w < sp.g1) qn = __dp4a(word, word, qn);
    }
    qn = __reduce_add_sync(0xffffffffu, qn);
    // every later non-empty visit into its cluster's list; the visit that opens a chunk of
    // kScanCQ list entries also opens the bitmap work item of that chunk
    for (uint32_t i = fi + 1 + lane; i < cnt; i += 32) {
        const uint32_t c = __ldg(ord + i);
        if (lv.clusters[c].n == 0) continue;  // num_embeddings == 0 (searcher.hpp:662)
        const uint32_t slot = atomicAdd(sp.vl_count + c, 1u);
        sp.vl[(size_t)c * sp.nq + slot] = q * sp.q_order_stride + i;
        if (slot % kScanCQ == 0) {
            const uint32_t it = atomicAdd(sp.n_items, 1u);
            sp.items[2 * it] = c;
            sp.items[2 * it + 1] = slot / kScanCQ;
        }
    }
    const uint32_t* ids = reinterpret_cast<const uint32_t*>(sp.arena + cl.ids_off);
    float* hd = sp.heap_d + (size_t)q * sp.k;
    uint32_t* hid = sp.heap_id + (size_t)q * sp.k;
    const uint32_t kth = n <= 32u * kRegKeys ? start_push(rk, n, m, hist, ids, lv, hd, hid)
                                             : start_push(MemKeys{src}, n, m, hist, ids, lv, hd, hid);
    if (lane == 0) {
        // heap top after the pushes: the m-th key; the first checkpoint's bound at it
        const float tau0 = reported_u8(kth, lv);
        const long long lim = (long long)thr_u8(tau0, sp.cp1, lv, sp.ratios) - (long long)qn;
        sp.lim[q] = lim > 0x7FFFFFFFll ? 0x7FFFFFFF : (int32_t)lim;
        sp.first_i[q] = fi;
        if (sp.stats) {
            add_stat(sp, 0, (unsigned long long)n * lv.d);
            add_stat(sp, 3 + kStart, (unsigned long long)n * lv.d);
            add_stat(sp, 1, 1ull);
        }
    }
}

// ------------------------------------------------------------------------------------ bitmaps
// CTA = one work item: up to 64 visits of one cluster. Warp w holds the first-checkpoint words
// of vector blocks w, w + 8, ... (lane = vector) in registers with |x|^2, and loops over the
// item's queries: 4 dp4a give q.x, and the ballot of |x|^2 - 2 q.x < lim is the 32-bit word of
// that block in the query's bitmap. Lane j keeps the word of query j mod 32 and the 32 words are
// stored together.
__global__ void __launch_bounds__(kBitmapThreads) scan_bitmap_kernel(const __grid_constant__ ScanParams sp) {
    __shared__ uint4 qv[kScanCQ];
    __shared__ int32_t ql[kScanCQ];
    __shared__ uint32_t qe[kScanCQ];
    __shared__ uint32_t item;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr uint32_t kWarps = kBitmapThreads / 32;
    const DevLevel& lv = sp.l1;
    const uint32_t g1 = sp.g1;
    for (;;) {
        if (threadIdx.x == 0) item = atomicAdd(sp.queue, 1u);
        __syncthreads();
        const uint32_t it = item;
        __syncthreads();
        if (it >= sp.n_items[0]) break;
        const uint32_t c = sp.items[2 * it], a = sp.items[2 * it + 1];
        const uint32_t L = sp.vl_count[c];
        const uint32_t nqc = (L - a * kScanCQ) < kScanCQ ? (L - a * kScanCQ) : kScanCQ;
        if (threadIdx.x < nqc) {
            const uint32_t e = sp.vl[(size_t)c * sp.nq + a * kScanCQ + threadIdx.x];
            const uint32_t q = e / sp.q_order_stride;
            const uint32_t* w = sp.qwords + (size_t)q * sp.nwords;
            qv[threadIdx.x] = make_uint4(__ldg(w), g1 > 1 ? __ldg(w + 1) : 0u, g1 > 2 ? __ldg(w + 2) : 0u,
                                         g1 > 3 ? __ldg(w + 3) : 0u);
            ql[threadIdx.x] = sp.lim[q];
            qe[threadIdx.x] = e;
        }
        __syncthreads();
        const DevCluster cl = lv.clusters[c];
        const uint32_t n = cl.n;
        const uint32_t nb = (n + 31) >> 5;
        const uint32_t* vert = reinterpret_cast<const uint32_t*>(sp.arena + cl.vert_off);
        for (uint32_t b0 = warp; b0 < nb; b0 += kWarps * kBitmapBPW) {
            uint32_t x[kBitmapBPW][4], xn[kBitmapBPW], word[kBitmapBPW];
            bool valid[kBitmapBPW];
#pragma unroll
            for (int b = 0; b < kBitmapBPW; ++b) {
                const uint32_t blk = b0 + b * kWarps;
                const uint32_t v = blk * 32 + lane;
                valid[b] = blk < nb && v < n;
                xn[b] = 0;
                word[b] = 0;
#pragma unroll
                for (int g = 0; g < 4; ++g) {
                    // rows past the cluster's vectors but inside n_pad hold padding: never read
                    x[b][g] = (valid[b] && (uint32_t)g < g1) ? __ldg(vert + (size_t)g * cl.n_pad + v) : 0u;
                    xn[b] = __dp4a(x[b][g], x[b][g], xn[b]);
                }
            }
            for (uint32_t j = 0; j < nqc; ++j) {
                const uint4 qq = qv[j];
                const int32_t lj = ql[j];
#pragma unroll
                for (int b = 0; b < kBitmapBPW; ++b) {
                    uint32_t dot = __dp4a(qq.x, x[b][0], 0u);
                    dot = __dp4a(qq.y, x[b][1], dot);
                    dot = __dp4a(qq.z, x[b][2], dot);
                    dot = __dp4a(qq.w, x[b][3], dot);
                    const int32_t val = (int32_t)xn[b] - 2 * (int32_t)dot;  // |q - x|^2 - |q|^2
                    const unsigned bal = __ballot_sync(0xffffffffu, valid[b] && val < lj);
                    if (lane == (j & 31)) word[b] = bal;
                }
                if ((j & 31) == 31 || j + 1 == nqc) {
                    const uint32_t jj = (j & ~31u) + lane;
                    if (jj <= j) {
                        const size_t base = (size_t)qe[jj] * sp.bm_words;
#pragma unroll
                        for (int b = 0; b < kBitmapBPW; ++b) {
                            const uint32_t blk = b0 + b * kWarps;
                            if (blk < nb) sp.bm[base + blk] = word[b];
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------ replay
// Per-warp shared memory: qw [nwords] | hd, hid [r_heap_cap] | area [r_area_bytes] (candidate
// offsets as u16, or the final sort) | sbits [bm_words] survivor bitmap of one cluster |
// sv_pos, sv_d [r_surv_cap] the survivors of a first warmup step and their distances.
struct ReplayWarp {
    uint32_t* qw;
    float* hd;
    uint32_t* hid;
    uint16_t* cand;
    uint64_t* sortbuf;
    uint32_t* sbits;
    uint32_t* sv_pos;
    uint32_t* sv_d;
};

constexpr int kCandPerLane = 4;  // candidates a replay lane tests per memory round trip
constexpr int kFallPerLane = 4;  // vectors a replay lane carries through a full warmup step

__device__ __forceinline__ uint32_t sq16(const uint4& q, const uint4& x, uint32_t acc) {
    acc = sq4(q.x, x.x, acc);
    acc = sq4(q.y, x.y, acc);
    acc = sq4(q.z, x.z, acc);
    return sq4(q.w, x.w, acc);
}

// One survivor of the warmup bound at checkpoint cur0: the horizontal blocks, then the
// remaining vertical dims in 64-dim steps, tested after each against the bound of the heap top
// `top` fixed for the whole cluster (searcher.hpp:437-540). Returns whether it is still below
// the bound at the end; raw is its running distance.
__device__ __forceinline__ bool scan_follow(const ScanParams& sp, const DevCluster& c, const uint32_t* qw,
                                            uint32_t v, uint32_t cur0, float top, uint32_t& raw,
                                            unsigned long long& hbytes, unsigned long long& vbytes) {
    const DevLevel& lv = sp.l1;
    const uint32_t nhb = lv.n_hblocks;
    uint32_t cur = cur0;
    if (nhb) {
        const uint4* row = reinterpret_cast<const uint4*>(sp.arena + c.hor_off) + (size_t)v * 4;
        const size_t bstride = (size_t)c.n_pad * 4;  // uint4 per block
        for (uint32_t b = 0; b < nhb; ++b) {
            uint4 x[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) x[t] = __ldg(row + b * bstride + t);
            const uint4* qh = reinterpret_cast<const uint4*>(qw + lv.qw_hoff + b * 16);
#pragma unroll
            for (int t = 0; t < 4; ++t) raw = sq16(qh[t], x[t], raw);
            hbytes += kHDim;
            cur += kHDim;
            if (!(raw < thr_u8(top, cur, lv, sp.ratios))) return false;
        }
    }
    const uint32_t* vert = reinterpret_cast<const uint32_t*>(sp.arena + c.vert_off);
    uint32_t cur_v = cur0;
    while (cur_v < lv.dv) {
        const uint32_t last = (cur_v + kHDim < lv.dv) ? cur_v + kHDim : lv.dv;
        vbytes += last - cur_v;
        for (uint32_t g = cur_v >> 2; g < ((last + 3) >> 2); ++g)
            raw = sq4(qw[g], __ldg(vert + (size_t)g * c.n_pad + v), raw);
        cur = (cur + kHDim < lv.d) ? cur + kHDim : lv.d;
        cur_v = last;
        if (!(raw < thr_u8(top, cur, lv, sp.ratios))) return false;
        if (cur == lv.d) break;
    }
    return true;
}

// Positions of the set bits of one word per lane (word index w_rel of a group of 32 words),
// ascending, as offsets from the group's first vector into cand; returns their number.
__device__ __forceinline__ uint32_t scan_bits_to_offsets(uint32_t word, uint32_t w_rel, uint16_t* cand) {
    uint32_t total;
    uint32_t at = warp_exclusive_scan(__popc(word), total);
    while (word) {
        const uint32_t bit = __ffs(word) - 1;
        word &= word - 1;
        cand[at++] = (uint16_t)(w_rel * 32 + bit);
    }
    __syncwarp();
    return total;
}

__global__ void __launch_bounds__(kScanWarps * 32, 3) scan_replay_kernel(const __grid_constant__ ScanParams sp) {
    extern __shared__ __align__(16) uint8_t smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t q = blockIdx.x * kScanWarps + warp;
    if (q >= sp.nq) return;  // whole warp
    const uint32_t fi = sp.first_i[q];
    if (fi == kOffPath) return;
    const DevLevel& lv = sp.l1;
    uint8_t* base = smem + (size_t)warp * sp.r_warp_bytes;
    ReplayWarp R;
    R.qw = reinterpret_cast<uint32_t*>(base);
    R.hd = reinterpret_cast<float*>(base + ((size_t)sp.nwords * 4 + 15) / 16 * 16);
    R.hid = reinterpret_cast<uint32_t*>(R.hd + sp.r_heap_cap);
    R.cand = reinterpret_cast<uint16_t*>(R.hid + sp.r_heap_cap);
    R.sortbuf = reinterpret_cast<uint64_t*>(R.cand);
    R.sbits = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(R.cand) + sp.r_area_bytes);
    R.sv_pos = R.sbits + (sp.bm_words + 3) / 4 * 4;
    R.sv_d = R.sv_pos + sp.r_surv_cap;
    const uint32_t kq = sp.q_k ? __ldg(sp.q_k + q) : sp.k;
    const uint32_t stride = sp.q_order_stride;
    for (uint32_t w = lane; w < sp.nwords; w += 32) R.qw[w] = __ldg(sp.qwords + (size_t)q * sp.nwords + w);
    for (uint32_t j = lane; j < kq; j += 32) {
        R.hd[j] = __ldg(sp.heap_d + (size_t)q * sp.k + j);
        R.hid[j] = __ldg(sp.heap_id + (size_t)q * sp.k + j);
    }
    __syncwarp();
    uint4 q1 = make_uint4(0u, 0u, 0u, 0u);  // first checkpoint's query words (zero past g1)
    q1.x = R.qw[0];
    if (sp.g1 > 1) q1.y = R.qw[1];
    if (sp.g1 > 2) q1.z = R.qw[2];
    if (sp.g1 > 3) q1.w = R.qw[3];
    float top;
    uint32_t slot;
    warp_heap_top(R.hd, kq, top, slot);
    uint32_t* scratch = sp.start_dist + (size_t)__ldg(sp.start_row + q) * sp.start_stride;
    const uint32_t* ord = sp.q_order + (size_t)q * stride;
    const uint32_t cnt = __ldg(sp.q_order_count + q);
    const uint32_t S = sp.r_surv_cap;
    unsigned long long b_warm = 0, b_h = 0, b_v = 0, visits = 0, merged = 0;
    unsigned long long n_cand = 0, n_surv = 0, n_fast = 0, n_full = 0;

    // Follows the lane's survivor (alive, v, raw) through Prune with the bound at `tp`, then
    // merges the warp's survivors in lane order (MergeIntoHeap, searcher.hpp:542-566).
    auto prune_merge = [&](const DevCluster& c, bool alive, uint32_t v, uint32_t raw, uint32_t cur, float tp) {
        uint32_t idv = 0;
        if (alive) {
            alive = scan_follow(sp, c, R.qw, v, cur, tp, raw, b_h, b_v);
            if (alive) idv = __ldg(reinterpret_cast<const uint32_t*>(sp.arena + c.ids_off) + v);
        }
        const float dd = reported_u8(raw, lv);
        unsigned bal = __ballot_sync(0xffffffffu, alive);
        merged += __popc(bal);
        while (bal) {
            const int l = __ffs(bal) - 1;
            bal &= bal - 1;
            const float ddl = __shfl_sync(0xffffffffu, dd, l);
            const uint32_t idl = __shfl_sync(0xffffffffu, idv, l);
            if (ddl < top) {
                if (lane == 0) {
                    R.hd[slot] = ddl;
                    R.hid[slot] = idl;
                }
                __syncwarp();
                warp_heap_top(R.hd, kq, top, slot);
            }
        }
    };

    // the next visit's cluster record and first bitmap words, loaded one visit ahead
    DevCluster c_nx{};
    uint32_t bw_nx = 0;
    auto prefetch = [&](uint32_t ii) {
        if (ii < cnt) {
            c_nx = lv.clusters[__ldg(ord + ii)];
            bw_nx = lane < sp.bm_words ? __ldg(sp.bm + ((size_t)q * stride + ii) * sp.bm_words + lane) : 0u;
        }
    };
    prefetch(fi + 1);
    for (uint32_t i = fi + 1; i < cnt; ++i) {
        const DevCluster c = c_nx;
        const uint32_t bw0 = bw_nx;
        prefetch(i + 1);
        const uint32_t n = c.n;
        if (n == 0) continue;  // num_embeddings == 0 (searcher.hpp:662)
        ++visits;
        const uint32_t* vert = reinterpret_cast<const uint32_t*>(sp.arena + c.vert_off);
        const uint32_t W = (n + 31) >> 5;
        const uint32_t needed = (uint32_t)ceilf(__fmul_rn(kSelectivity, (float)n));
        const uint32_t* bmp = sp.bm + ((size_t)q * stride + i) * sp.bm_words;
        // Warmup step 1 from the candidates: the exact first-checkpoint distance of each, and the
        // survivors under the current bound, in position order
        const uint32_t thr1 = thr_u8(top, sp.cp1, lv, sp.ratios);
        uint32_t ns = 0;
        for (uint32_t w0 = 0; w0 < W; w0 += 32) {
            const uint32_t w = w0 + lane;
            uint32_t word = w0 == 0 ? bw0 : (w < W ? __ldg(bmp + w) : 0u);
            if (w >= W) word = 0u;
            const uint32_t total = scan_bits_to_offsets(word, lane, R.cand);
            n_cand += total;
            for (uint32_t j0 = 0; j0 < total; j0 += 32 * kCandPerLane) {
                uint32_t v[kCandPerLane];
                uint4 x[kCandPerLane];
#pragma unroll
                for (int u = 0; u < kCandPerLane; ++u) {
                    const uint32_t j = j0 + 32 * u + lane;
                    v[u] = j < total ? w0 * 32 + R.cand[j] : 0xFFFFFFFFu;
                    const bool in = v[u] != 0xFFFFFFFFu;
                    const uint32_t* col = vert + (in ? v[u] : 0u);
                    x[u].x = in ? __ldg(col) : 0u;
                    x[u].y = (in && sp.g1 > 1) ? __ldg(col + (size_t)c.n_pad) : 0u;
                    x[u].z = (in && sp.g1 > 2) ? __ldg(col + 2 * (size_t)c.n_pad) : 0u;
                    x[u].w = (in && sp.g1 > 3) ? __ldg(col + 3 * (size_t)c.n_pad) : 0u;
                }
#pragma unroll
                for (int u = 0; u < kCandPerLane; ++u) {
                    const uint32_t d1 = sq16(q1, x[u], 0u);
                    const bool s = v[u] != 0xFFFFFFFFu && d1 < thr1;
                    const unsigned bal = __ballot_sync(0xffffffffu, s);
                    const uint32_t r = ns + __popc(bal & ((1u << lane) - 1u));
                    if (s && r < S) {
                        R.sv_pos[r] = v[u];
                        R.sv_d[r] = d1;
                    }
                    ns += __popc(bal);
                }
            }
            __syncwarp();
        }
        b_warm += (unsigned long long)n * sp.cp1;
        const bool exits = sp.cp1 >= lv.dv || n - ns >= needed;  // the warmup stops after step 1
        const float tp = top;  // the bound's heap top, fixed for the whole cluster
        n_surv += ns;
        if (exits && ns <= S) {
            ++n_fast;
            // Prune and MergeIntoHeap of the survivors, 32 at a time in position order
            for (uint32_t g0 = 0; g0 < ns; g0 += 32) {
                const uint32_t j = g0 + lane;
                const bool alive = j < ns;
                prune_merge(c, alive, alive ? R.sv_pos[j] : 0u, alive ? R.sv_d[j] : 0u, sp.cp1, tp);
            }
            continue;
        }
        // the warmup continues past its first step (or keeps more survivors than the list
        // holds): the whole Warmup (searcher.hpp:374-435) over every vector, the running
        // distances in the query's scratch row
        ++n_full;
        uint32_t cur = 0, step = 0, n_pruned = 0;
        while (n_pruned < needed && cur < lv.dv) {
            uint32_t last = cur + c_scan_fetch[step < kNumFetchSizes ? step : kNumFetchSizes - 1];
            if (last > lv.dv) last = lv.dv;
            const uint32_t thr = thr_u8(top, last, lv, sp.ratios);
            const uint32_t g0 = cur >> 2, g_end = (last + 3) >> 2;
            uint32_t cntp = 0;
            for (uint32_t v0 = 0; v0 < n; v0 += 32 * kFallPerLane) {
                uint32_t acc[kFallPerLane];
#pragma unroll
                for (int u = 0; u < kFallPerLane; ++u) {
                    const uint32_t v = v0 + 32 * u + lane;
                    acc[u] = (v < n && cur > 0) ? scratch[v] : 0u;
                }
                for (uint32_t g = g0; g < g_end; g += 4) {
                    uint32_t xs[4][kFallPerLane];
#pragma unroll
                    for (int gg = 0; gg < 4; ++gg)
#pragma unroll
                        for (int u = 0; u < kFallPerLane; ++u) {
                            const uint32_t v = v0 + 32 * u + lane;
                            xs[gg][u] = (v < n && g + gg < g_end) ? __ldg(vert + (size_t)(g + gg) * c.n_pad + v) : 0u;
                        }
#pragma unroll
                    for (int gg = 0; gg < 4; ++gg) {
                        const uint32_t qv = g + gg < g_end ? R.qw[g + gg] : 0u;
#pragma unroll
                        for (int u = 0; u < kFallPerLane; ++u) acc[u] = sq4(qv, xs[gg][u], acc[u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < kFallPerLane; ++u) {
                    const uint32_t v = v0 + 32 * u + lane;
                    if (v < n) {
                        scratch[v] = acc[u];
                        cntp += acc[u] >= thr ? 1u : 0u;
                    }
                }
            }
            n_pruned = __reduce_add_sync(0xffffffffu, cntp);
            if (cur > 0) b_warm += (unsigned long long)n * (last - cur);
            cur = last;
            ++step;
        }
        // Prune: the vectors below the bound at the warmup's last checkpoint, in position order
        const uint32_t thr = thr_u8(top, cur, lv, sp.ratios);
        for (uint32_t v0 = 0; v0 < n; v0 += 32) {
            const uint32_t v = v0 + lane;
            const unsigned bal = __ballot_sync(0xffffffffu, v < n && scratch[v] < thr);
            if (lane == 0) R.sbits[v0 >> 5] = bal;
        }
        __syncwarp();
        for (uint32_t w0 = 0; w0 < W; w0 += 32) {
            const uint32_t w = w0 + lane;
            const uint32_t total = scan_bits_to_offsets(w < W ? R.sbits[w] : 0u, lane, R.cand);
            for (uint32_t j0 = 0; j0 < total; j0 += 32) {
                const uint32_t j = j0 + lane;
                const bool alive = j < total;
                const uint32_t v = alive ? w0 * 32 + R.cand[j] : 0u;
                prune_merge(c, alive, v, alive ? scratch[v] : 0u, cur, tp);
            }
            __syncwarp();  // cand is rewritten by the next word group
        }
    }
    // BuildResultSetFromHeap (searcher.hpp:568-585)
    const uint32_t N = next_pow2(kq);
    for (uint32_t j = lane; j < N; j += 32)
        R.sortbuf[j] = j < kq ? (((uint64_t)__float_as_uint(R.hd[j]) << 32) | R.hid[j]) : ~0ull;
    __syncwarp();
    warp_sort_u64(R.sortbuf, N);
    uint32_t hs = kq;
    if (__uint_as_float((uint32_t)(R.sortbuf[hs - 1] >> 32)) == FLT_MAX) --hs;
    uint32_t* oi = sp.out_ids + (size_t)q * sp.k;
    float* od = sp.out_dists + (size_t)q * sp.k;
    for (uint32_t j = lane; j < sp.k; j += 32) {
        if (j < hs) {
            const uint64_t e = R.sortbuf[j];
            oi[j] = (uint32_t)e;
            od[j] = __uint_as_float((uint32_t)(e >> 32));
        } else {
            oi[j] = 0xFFFFFFFFu;
            od[j] = __int_as_float(0x7f800000);
        }
    }
    if (lane == 0) sp.out_counts[q] = hs;
    if (sp.stats) {
        const unsigned long long h = __reduce_add_sync(0xffffffffu, (uint32_t)b_h);
        const unsigned long long vv = __reduce_add_sync(0xffffffffu, (uint32_t)b_v);
        if (lane == 0) {
            add_stat(sp, 0, b_warm + h + vv);
            add_stat(sp, 3 + kWarmup, b_warm);
            add_stat(sp, 3 + kSurvivorH, h);
            add_stat(sp, 3 + kSurvivorV, vv);
            add_stat(sp, 1, visits);
            add_stat(sp, 2, merged);
            add_stat(sp, 12, n_cand);
            add_stat(sp, 13, n_surv);
            add_stat(sp, 14, n_fast);
            add_stat(sp, 15, n_full);
        }
    }
}

// ------------------------------------------------------------------------------------ launch
uint64_t scan_item_bound(uint32_t nq, uint32_t stride, uint32_t n1) {
    return (uint64_t)nq * stride / kScanCQ + n1 + 1;
}

int scan_bitmap_occupancy() {
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, scan_bitmap_kernel, kBitmapThreads, 0);
    return blocks;
}

uint32_t scan_queries_per_cta() { return kScanWarps; }

// ev (optional, 3 events): recorded after the prep kernel, the bitmaps and the replay.
cudaError_t launch_scan(const ScanParams& sp, int bitmap_grid, cudaStream_t st, const cudaEvent_t* ev) {
    cudaError_t e = cudaMemsetAsync(sp.vl_count, 0, sizeof(uint32_t) * sp.l1.nclusters, st);
    if (e != cudaSuccess) return e;
    // left_n, n_items and queue are consecutive
    if ((e = cudaMemsetAsync(sp.left_n, 0, 3 * sizeof(uint32_t), st)) != cudaSuccess) return e;
    const uint32_t ctas = (sp.nq + kScanWarps - 1) / kScanWarps;
    const size_t prep_smem = sp.prep_qs ? (size_t)kScanWarps * sp.prep_qs_stride * 4 : 0;
    if (prep_smem) {
        e = cudaFuncSetAttribute(scan_prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)prep_smem);
        if (e != cudaSuccess) return e;
    }
    scan_prep_kernel<<<ctas, kScanWarps * 32, prep_smem, st>>>(sp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (ev && (e = cudaEventRecord(ev[0], st)) != cudaSuccess) return e;
    scan_bitmap_kernel<<<bitmap_grid, kBitmapThreads, 0, st>>>(sp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (ev && (e = cudaEventRecord(ev[1], st)) != cudaSuccess) return e;
    const size_t smem = (size_t)kScanWarps * sp.r_warp_bytes;
    e = cudaFuncSetAttribute(scan_replay_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    scan_replay_kernel<<<ctas, kScanWarps * 32, smem, st>>>(sp);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (ev && (e = cudaEventRecord(ev[2], st)) != cudaSuccess) return e;
    return cudaSuccess;
}

}  // namespace pdxg
