// Shared definitions of the B200 PDX search engine: the device-resident index layout and the
// kernel parameter blocks. Host and device code both include this header.
//
// Device layout of one cluster (all offsets in bytes from the arena base, 256-byte aligned):
//   vertical block   : n_vwords rows x n_pad 32-bit words. F32: one row per vertical dimension
//                      (dim-major, consecutive vectors in consecutive words). U8: one row per
//                      group of 4 vertical dimensions, each word holding the 4 interleaved bytes
//                      of one vector (the reference's U8_INTERLEAVE_SIZE packing); a trailing
//                      group of d_v % 4 dims is zero-padded to a full word.
//   horizontal blocks: n_hblocks x n_pad rows of 64 elements (F32: 256 B rows, U8: 64 B rows),
//                      the reference's 64-dim row-major sub-blocks.
//   row ids          : n u32.
// n_pad rounds the cluster size up to 32 so every dimension row starts on a 128-byte line.
#pragma once
#include <cstdint>

namespace pdxg {

constexpr int kHDim = 64;               // H_DIM_SIZE (common.hpp:45)
constexpr int kMaxDims = 16384;         // PDX_MAX_DIMS (common.hpp:44)
constexpr int kNumFetchSizes = 20;      // DIMENSIONS_FETCHING_SIZES (common.hpp:47-49)
constexpr float kSelectivity = 0.80f;   // selectivity_threshold (searcher.hpp:57)
// Counters of a search with PDXG_COLLECT_STATS: [0..11] as SearchParams::stats describes,
// [12..15] the cluster-major scan's (candidates tested, first-step survivors, visits whose warmup
// stops after its first step, visits that ran the whole warmup).
constexpr int kStatsWords = 16;

struct DevCluster {
    uint64_t vert_off;  // vertical block
    uint64_t hor_off;   // horizontal blocks
    uint64_t ids_off;   // row ids
    uint32_t n;         // vectors in the cluster (used capacity, tombstoned slots included)
    uint32_t n_pad;     // row stride in vectors (multiple of 32)
    uint32_t sel_word;  // first 32-bit word of this cluster in a filter selection bitmap
    uint32_t live;      // vectors not tombstoned (num_embeddings); n when there are none
};

struct DevLevel {
    const DevCluster* clusters;  // [nclusters]
    const float* centroids;      // [nclusters x d] f32 (rotated space)
    uint32_t nclusters;
    uint32_t d, dv, dh;
    uint32_t n_vwords;           // vertical words per vector: F32 dv, U8 ceil(dv / 4)
    uint32_t qw_hoff;            // U8: first horizontal word of the packed query (16B aligned)
    uint32_t n_hblocks;          // dh / 64
    uint32_t max_n;              // largest cluster
    uint32_t is_u8;
    uint32_t sel_words;          // words of one selection bitmap over this level
    float scale_sq;              // U8: quantization_scale^2
    float inv_scale_sq;          // U8: 1 / quantization_scale^2
    float base, scale;           // U8 quantization parameters
    const uint32_t* tomb;        // tombstoned slots, one bit per slot in the selection-bitmap
                                 // layout (sel_word); null when the level has none
};

// One batched search launch.
struct SearchParams {
    const uint8_t* arena;
    DevLevel l1;                 // data clusters
    DevLevel l0;                 // meso clusters (tree indexes only)
    int is_tree;
    const float* ratios;         // ADSampling ratio table [d] (adsampling.hpp:147-157)
    const float* queries;        // prepared (normalized + rotated) queries [nq x d]
    uint32_t nq;
    uint32_t k;
    uint32_t nprobe;             // L1 clusters to visit (already resolved: 1..nclusters)
    uint32_t top_nprobe;         // tree: meso clusters probed by the top-level search
    const uint32_t* order;       // optional caller cluster order [n_order] shared by all queries
    uint32_t n_order;
    const uint32_t* sel_bits;    // optional: [n_filters x l1.sel_words] selection bitmaps
    const uint32_t* passing;     // optional: [n_filters x l1.nclusters] passing counts
    const int32_t* filter_of;    // optional: [nq] filter per query: -1 unfiltered, f >= 0 the
                                 // batch's filter f, -2 - r the registered filter r
    const uint32_t* reg_sel;     // registered filters: [slots x l1.sel_words] selection bitmaps
    const uint32_t* reg_pass;    // registered filters: [slots x l1.nclusters] passing counts
    const uint32_t* q_k;         // optional per-query k (<= k, the output row stride)
    const uint32_t* q_nprobe;    // optional per-query resolved nprobe (<= nprobe)
    const uint32_t* q_top;       // optional per-query tree top-level probe (<= top_nprobe)
    uint32_t* out_ids;           // [nq x k]
    float* out_dists;            // [nq x k]
    uint32_t* out_counts;        // [nq]
    uint32_t* queue;             // work counter (zeroed before launch)
    unsigned long long* stats;   // optional [12]: [0] index bytes the algorithm reads, [1] clusters
                                 // visited, [2] vectors reaching the merge, [3..8] bytes by phase:
                                 // top-level search, Start, warmup, survivor horizontal blocks,
                                 // survivor vertical dims, centroid probe; [9..11] SM cycles
                                 // in the top-level search, in L1 Start, in the rest
    // tree top level, batched form (pdxg_toplevel.cu): each query's L1 visit order
    const uint32_t* q_order;        // [nq x q_order_stride]
    const uint32_t* q_order_count;  // [nq]
    uint32_t q_order_stride;
    // batched Start (pdxg_start.cu): exact U8 distances to every vector of each query's first
    // visited cluster, computed ahead with reuse across queries
    const int32_t* start_row;       // optional [nq]: row in start_dist, -1 = none
    const uint32_t* start_first;    // [nq] the cluster of that row
    const uint32_t* start_dist;     // [rows x start_stride]
    uint32_t start_stride;
    // optional: only the queries q_list[0 .. *q_list_n) are searched (the rest of a batch went
    // through the cluster-major scan, pdxg_scan.cu)
    const uint32_t* q_list;
    const uint32_t* q_list_n;
    // shared-memory carve-up (bytes), computed by the host
    uint32_t smem_qf, smem_qw, smem_work, smem_heap, smem_order, smem_bits, smem_total;
    uint32_t bits_cap;           // words of the survivor bitmap (work_cap / 32); the prefix follows
    uint32_t work_cap;           // entries of the dist / pos work arrays (multiple of 32, >= heap_cap)
    uint32_t heap_cap;           // entries of the heap arrays (power of two)
    uint32_t order_cap;          // entries of the cluster order list
};

// Tiled tree top level (pdxg_toplevel.cu): meso probe, per-(meso cluster, query tile) exact
// partial distances, warp-per-query replay of the top-level PDXearch.
constexpr int kMaxCheckpoints = 32;

struct TopLevelParams {
    const uint8_t* arena;
    DevLevel l0;                 // meso level (F32): its "vectors" are the L1 centroids
    const float* ratios;         // ADSampling ratio table [d]
    const float* queries;        // prepared queries [nq x d]
    uint32_t nq;
    uint32_t top;                // meso clusters probed per query (row stride of order / off)
    uint32_t k1;                 // L1 nprobe (row stride of l1_order)
    const uint32_t* q_nprobe;    // optional per-query L1 nprobe (<= k1)
    const uint32_t* q_top;       // optional per-query meso probe count (<= top)
    const int32_t* filter_of;    // optional: queries with filter_of != -1 get no L1 order
    uint32_t* order;             // [nq x top] probed meso clusters, nearest first
    uint32_t* off;               // [nq x top] float offset of each probed cluster's partials
    uint32_t* ntop;              // [nq] meso clusters probed
    uint32_t* list_count;        // [nL0] queries probing each meso cluster (zeroed before)
    uint32_t* lists;             // [nL0 x nq] entries q * top + r
    float* vals;                 // [nq x per_query] partials: ncp checkpoint rows, nb block rows
    unsigned long long per_query;
    uint32_t ncp;                // vertical checkpoints (cp[ncp - 1] == dv)
    uint32_t nvals;              // ncp + n_hblocks rows per probed cluster
    uint32_t cp[kMaxCheckpoints];
    uint32_t* l1_order;          // [nq x k1] L1 clusters to visit, nearest first
    uint32_t* l1_count;          // [nq]
    unsigned long long* stats;   // optional, SearchParams::stats layout
    // replay shared memory (bytes per warp and carve-up)
    uint32_t r_heap_cap, r_work_cap, r_sort_cap, r_pre_floats, r_warp_bytes, r_smem;
    uint32_t probe_smem;         // meso probe CTA: queries + sort keys
    uint32_t probe_q;            // queries per meso probe CTA (1..8)
};

// Reduced-precision centroid probe (pdxg_probe.cu).
struct ProbeParams {
    const float* queries;        // prepared queries [nq x d] (FP32)
    const float* centroids;      // [nclusters x d] FP32
    const float* scores;         // [nq x ld_scores] approximate |c|^2 - 2 q.c
    uint32_t ld_scores;
    uint32_t nq, d, nclusters;
    uint32_t nprobe;             // resolved nprobe (row stride of order)
    const uint32_t* q_nprobe;    // optional per-query resolved nprobe (<= nprobe)
    uint32_t* order;             // [nq x stride] clusters to visit, nearest first
    uint32_t stride;
    uint32_t* count;             // [nq]
    uint32_t cand_cap, sort_cap; // shared-memory capacities (candidates, sort keys)
    uint32_t score_bytes;        // bytes per centroid element read by the approximate scores
    unsigned long long* stats;   // optional, SearchParams::stats layout
};

// Batched Start (pdxg_start.cu).
struct StartParams {
    const uint8_t* arena;
    DevLevel l1;
    const float* queries;         // prepared queries [nq x d]
    uint32_t nq;
    const uint32_t* q_order;      // [nq x q_order_stride] each query's L1 visit order
    const uint32_t* q_order_count;
    uint32_t q_order_stride;
    const int32_t* filter_of;     // optional: queries with filter_of != -1 are left out
    uint32_t* cl_count;           // [n1] queries per first cluster (zeroed before)
    uint32_t* cl_off;             // [n1] first row of each cluster
    uint32_t* cl_items;           // [n1] first work item of each cluster
    uint32_t* first_cl;           // [nq] first non-empty visited cluster (~0u: none)
    uint32_t* slot_of;            // [nq] position among that cluster's queries
    int32_t* row_of;              // [nq] row in dist (-1: none)
    uint32_t* sorted_q;           // [nq] queries grouped by first cluster (row order)
    uint32_t* items;              // [2 x item bound] (cluster, query chunk << 16 | vector chunk)
    uint32_t* n_items;            // [1]
    uint32_t* queue;              // [1] work counter
    uint32_t* dist;               // [nq x stride] exact U8 distances
    uint32_t stride;              // >= largest L1 cluster
};

// Cluster-major scan of U8 levels (pdxg_scan.cu): the first warmup step of every (query,
// visited cluster) pair computed per cluster for all its queries, then one warp per query
// replaying PDXearch on those results.
struct ScanParams {
    const uint8_t* arena;
    DevLevel l1;
    const float* ratios;          // ADSampling ratio table [d]
    const float* queries;         // prepared queries [nq x d]
    uint32_t nq;
    uint32_t k;                   // output row stride (the largest per-query k)
    const uint32_t* q_k;          // optional per-query k (<= k)
    const int32_t* filter_of;     // optional: only queries with -1 take this path
    const uint32_t* q_order;      // [nq x q_order_stride] L1 visit orders
    const uint32_t* q_order_count;
    uint32_t q_order_stride;
    const int32_t* start_row;     // batched Start (pdxg_start.cu): row of each query, -1 none
    const uint32_t* start_first;  // [nq] the cluster of that row
    uint32_t* start_dist;         // [rows x start_stride]; a query's row is its scratch afterwards
    uint32_t start_stride;
    uint32_t cp1;                 // first warmup checkpoint: min(16, d_v)
    uint32_t g1;                  // vertical words it covers: ceil(cp1 / 4) (<= 4)
    uint32_t nwords;              // packed query words: qw_hoff + 16 n_hblocks
    uint32_t* qwords;             // [nq x nwords] quantized queries, packed as the scan packs them
    uint32_t* first_i;            // [nq] position of the Start cluster in the order; ~0u: not here
    int32_t* lim;                 // [nq] a vector is a candidate when |x|^2 - 2 q.x < lim
    float* heap_d;                // [nq x k] the Start's pushes, in push order
    uint32_t* heap_id;
    uint32_t* left;               // [nq] queries left to the per-query scan kernel
    uint32_t* left_n;             // [1] (zeroed before; n_items and queue follow it)
    uint32_t* vl_count;           // [n1] visits per cluster (zeroed before)
    uint32_t* vl;                 // [n1 x nq] visits of each cluster: q * q_order_stride + i
    uint32_t* items;              // [2 x item bound] (cluster, chunk of 64 list entries)
    uint32_t* n_items;            // [1] (zeroed before)
    uint32_t* queue;              // [1] work counter (zeroed before)
    uint32_t* bm;                 // [nq x q_order_stride x bm_words] candidate bitmaps
    uint32_t bm_words;            // ceil(largest cluster / 32)
    uint32_t* out_ids;            // [nq x k]
    float* out_dists;             // [nq x k]
    uint32_t* out_counts;         // [nq]
    unsigned long long* stats;    // optional, SearchParams::stats layout
    uint32_t prep_qs;             // 1: the prep kernel stages each query row in shared memory
    uint32_t prep_qs_stride;      // floats per staged row
    uint32_t r_surv_cap;          // replay: survivors of one cluster's first warmup step it keeps
    uint32_t r_heap_cap;          // replay shared memory per warp: heap entries,
    uint32_t r_area_bytes;        // candidate offsets / final sort area,
    uint32_t r_warp_bytes;        // and the whole per-warp region
};

}  // namespace pdxg
