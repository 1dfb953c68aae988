// Host-side engine state shared by pdxg_index.cu (loading, search, C ABI) and pdxg_maint.cu
// (Append / Delete): the index object, its levels, workspace and maintenance state, and the few
// internal helpers both use. Not part of the C ABI (include/pdx_b200.h).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_set>
#include <vector>

#include "../../include/pdx_b200.h"
#include "pdxg_common.cuh"
#include "pdxg_gemm.cuh"

namespace pdxg {
namespace host {

// Last error message of the calling thread (pdxg_last_error) and the status-code helper.
extern thread_local std::string g_err;
int fail(int code, const std::string& msg);

#define PDXG_CUDA(x)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (x);                                                             \
        if (e_ != cudaSuccess)                                                            \
            return fail(PDXG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

inline uint32_t next_pow2(uint32_t x) {
    uint32_t p = 1;
    while (p < x) p <<= 1;
    return p;
}
inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

struct FileCluster {
    uint32_t n = 0, max_cap = 0;
    const uint8_t* data = nullptr;  // compact PDX block inside the file buffer
    const uint8_t* ids = nullptr;   // u32[n]
};

struct HostLevel {
    bool u8 = false;
    uint32_t d = 0, dv = 0, dh = 0;
    std::vector<FileCluster> fc;
    std::vector<DevCluster> meta;
    std::vector<uint32_t> n, max_cap;
    std::vector<uint64_t> ids_start;
    std::vector<uint32_t> ids;  // host copy of all row ids, cluster after cluster
    std::vector<float> centroids;
    uint32_t max_n = 0, sel_words = 0, n_vwords = 0, qw_hoff = 0, n_hblocks = 0;
    uint64_t total_vectors = 0;
};

struct Workspace {
    uint32_t q_cap = 0, k_cap = 0;
    float* d_q = nullptr;
    float* d_rq = nullptr;
    float* d_norms = nullptr;
    uint32_t* d_ids = nullptr;
    float* d_dists = nullptr;
    uint32_t* d_counts = nullptr;
    uint32_t* d_queue = nullptr;
    uint32_t* d_order = nullptr;
    uint32_t order_cap = 0;
    uint32_t* d_sel = nullptr;
    uint64_t sel_cap = 0;
    uint32_t* d_pass = nullptr;
    uint64_t pass_cap = 0;
    int32_t* d_filter_of = nullptr;
    uint32_t fo_cap = 0;
    unsigned long long* d_stats = nullptr;
    // batched tree top level
    uint32_t* d_top_order = nullptr;
    uint64_t top_order_cap = 0;
    uint32_t* d_top_off = nullptr;
    uint64_t top_off_cap = 0;
    uint32_t* d_top_lists = nullptr;
    uint64_t top_lists_cap = 0;
    uint32_t* d_top_count = nullptr;
    uint64_t top_count_cap = 0;
    float* d_top_vals = nullptr;
    uint64_t top_vals_cap = 0;
    uint32_t* d_l1_order = nullptr;
    uint64_t l1_order_cap = 0;
    uint32_t* d_l1_count = nullptr;
    uint64_t l1_count_cap = 0;
    // batched Start: per-cluster counters ([3 x n1]), per-query arrays ([4 x nq]), work items,
    // counters, distances
    uint32_t* d_st_cl = nullptr;
    uint64_t st_cl_cap = 0;
    uint32_t* d_st_q = nullptr;
    uint64_t st_q_cap = 0;
    uint32_t* d_st_items = nullptr;
    uint64_t st_items_cap = 0;
    uint32_t* d_st_dist = nullptr;
    uint64_t st_dist_cap = 0;
    // reduced-precision probe: BF16 queries, BF16 / E4M3 rotated queries (+ row scales), scores
    uint16_t* d_pq_b16 = nullptr;
    uint64_t pq_b16_cap = 0;
    uint16_t* d_pq_r16 = nullptr;
    uint64_t pq_r16_cap = 0;
    uint8_t* d_pq_r8 = nullptr;
    uint64_t pq_r8_cap = 0;
    float* d_pq_r8s = nullptr;
    uint64_t pq_r8s_cap = 0;
    float* d_pq_scores = nullptr;
    uint64_t pq_scores_cap = 0;
    // per-query request parameters (pdxg_search_requests)
    uint32_t* d_req = nullptr;  // q_k | q_nprobe | q_top | filter_of, nq each
    uint64_t req_cap = 0;
    unsigned long long* d_foff = nullptr;
    uint64_t foff_cap = 0;
    uint32_t* d_rows = nullptr;
    uint64_t rows_cap = 0;
    // tensor-core rotation: TF32 hi / lo planes of the (normalized) queries, GEMM error flag
    float* d_qhi = nullptr;
    float* d_qlo = nullptr;
    uint64_t qhi_cap = 0, qlo_cap = 0;
    int* d_gemm_err = nullptr;
    // cluster-major scan (pdxg_scan.cu): packed query words, per-query state ([3 x nq + 4]:
    // first_i | lim | left | left_n, n_items, queue), Start heaps, per-cluster visit lists and
    // counters, work items, candidate bitmaps
    uint32_t* d_sc_qw = nullptr;
    uint64_t sc_qw_cap = 0;
    uint32_t* d_sc_q = nullptr;
    uint64_t sc_q_cap = 0;
    uint32_t* d_sc_heap = nullptr;
    uint64_t sc_heap_cap = 0;
    uint32_t* d_sc_cl = nullptr;
    uint64_t sc_cl_cap = 0;
    uint32_t* d_sc_vl = nullptr;
    uint64_t sc_vl_cap = 0;
    uint32_t* d_sc_items = nullptr;
    uint64_t sc_items_cap = 0;
    uint32_t* d_sc_bm = nullptr;
    uint64_t sc_bm_cap = 0;
};

// Mutable state of a tree index once Append / Delete have been used (PDXTreeIndex,
// index.hpp:580-638, and Cluster, cluster.hpp:86-154, 260-294).
struct MaintCluster {
    uint32_t num_embeddings = 0, used = 0, max_cap = 0, min_cap = 0;
    // the reference's container (cluster.hpp:20): PopTombstone takes begin(), so the same
    // sequence of inserts and erases reuses and compacts the same slots
    std::unordered_set<uint32_t> tombstones;
    std::vector<uint32_t> indices;  // row id of every used slot
};

struct Maint {
    std::vector<MaintCluster> cl;
    uint64_t arena_cap = 0;       // bytes allocated for the arena (arena_bytes are in use)
    uint32_t* d_tomb = nullptr;   // tombstone bitmap in the selection-bitmap layout
    uint64_t tomb_cap = 0;        // words allocated
    std::vector<uint32_t> tomb;   // host copy (l1.sel_words words)
    uint64_t n_tomb = 0;          // tombstoned slots over all clusters
    uint64_t live = 0;            // total_num_embeddings
    uint64_t rid_cap = 0;         // entries allocated for the device row maps
    uint64_t appends = 0, deletes = 0, compactions = 0, grown = 0, merges_deferred = 0;
    // device state waiting for the next search (flush_maintenance)
    bool dirty = false;           // any of the below pending
    bool records_dirty = false;   // cluster records
    bool tomb_dirty = false;      // tombstone bitmap
    std::vector<uint32_t> dirty_rows;  // row ids whose map entries changed
    bool quiet = false;           // no search launched since the last device synchronization
    cudaEvent_t ev_flush = nullptr;  // after the last upload of changes: later searches wait on it
    cudaEvent_t ev_stage = nullptr;  // after the last copy out of h_stage (before it is rewritten)
    bool in_op = false;           // inside Append: its own top-level search skips the flush
    uint32_t* d_stage = nullptr;  // row-map entries (row, cluster, position) being uploaded
    uint32_t* h_stage = nullptr;  // pinned
    // appends: pinned staging of one chunk of rows, the chosen clusters, the slot writes
    float* h_rows = nullptr;
    uint32_t* h_res = nullptr;    // nearest cluster and count per row, then the GEMM status
    void* h_writes = nullptr;     // RowWrite records (pinned)
    void* d_writes = nullptr;
    uint32_t stage_rows = 0;      // rows the append staging holds
};

struct Launch {
    SearchParams p{};
    bool u8 = false;
    int threads = 256;
    int grid = 1;
    uint32_t top_launches = 0;  // kernels of a separate tree top level
    uint32_t scan_launches = 0;  // kernels of the cluster-major scan ahead of the per-query kernel
    uint32_t start_launches = 0;  // kernels of the batched Start
    uint32_t probe_launches = 0;  // kernels of the reduced-precision probe (rotation included)
};

// Incremented whenever a device buffer is replaced: a captured search graph holds raw buffer
// pointers and refuses to launch once any of them may have moved.
extern std::atomic<uint64_t> g_alloc_gen;

template <class T>
int dev_grow(T*& ptr, uint64_t& cap, uint64_t need) {
    if (need <= cap && ptr) return PDXG_OK;
    g_alloc_gen.fetch_add(1);
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    const uint64_t n = std::max<uint64_t>(need, 1);
    PDXG_CUDA(cudaMalloc(&ptr, n * sizeof(T)));
    cap = n;
    return PDXG_OK;
}

// Search plumbing (pdxg_index.cu).
int ensure_ws(pdxg_index* ix, Workspace& w, uint32_t nq, uint32_t k);
// normalize: -1 follows the index's is_normalized flag (queries), 0 / 1 force it (appended rows
// follow PDXIndexConfig::normalize); allow_tc: the tensor-core rotation may be used.
int prepare_dev(pdxg_index* ix, Workspace& w, const float* q, uint32_t nq, float* out, cudaStream_t st,
                int normalize = -1, bool allow_tc = true);
// st: the stream the search runs on (nullptr = the index's own); pending Append / Delete changes
// are uploaded on it first (flush_maintenance).
int plan_search(pdxg_index* ix, uint32_t nq, uint32_t k, uint32_t n_order, bool any_filter, Launch& L,
                uint32_t np_flat_max = 0xFFFFFFFFu, uint32_t top_max = 0xFFFFFFFFu, bool probe_ahead = false,
                cudaStream_t st = nullptr);
// The tensor-core (TF32x3) rotation of nq queries; hi / lo are nq x d planes, err its wait status.
bool rotation_on_tensor_cores(const pdxg_index* ix, uint32_t nq);
int rotate_tf32x3(pdxg_index* ix, const float* q, uint32_t nq, bool norm, float* hi, float* lo, int* err,
                  float* out, cudaStream_t st);
int run_top_level(pdxg_index* ix, Workspace& w, const float* qp, uint32_t nq, Launch& L, cudaStream_t st,
                  uint32_t q_offset = 0, bool timed = false);
// The cluster-major scan for the queries it can take (U8 level after a batched Start, visit
// orders ahead, no tombstones); sets L.p.q_list to the rest, for the per-query kernel.
int run_scan_cluster_major(pdxg_index* ix, Workspace& w, uint32_t nq, Launch& L, cudaStream_t st,
                           bool timed = false);
int check_index(const pdxg_index* ix);
// Selection bitmap + passing counts of one row-id list in the device bitmap layout.
void build_filter(const pdxg_index* ix, const uint64_t* rows, uint64_t n, uint32_t* sel, uint32_t* pass);

// Append / Delete support (pdxg_maint.cu).
int maint_prepare_save(pdxg_index* ix);
int refresh_registered_filters(pdxg_index* ix);
// Enqueues the upload of what Append / Delete changed on `st` (nullptr = the index's own stream)
// and makes `st` wait for the last such upload; fails while `st` is being captured with changes
// pending (the upload cannot be part of a graph).
int flush_maintenance(pdxg_index* ix, cudaStream_t st = nullptr);
void free_maintenance(Maint& M);

}  // namespace host
}  // namespace pdxg

struct pdxg_index {
    int device = 0;
    int type = 0;
    uint32_t d = 0, dv = 0, dh = 0;
    bool tree = false, u8 = false, normalized = false;
    float base = 0.0f, scale = 1.0f;
    uint32_t rot_rows = 0, rot_cols = 0;
    std::vector<float> rotation;       // d x d matrix of y = x M used by the engine
    std::vector<float> file_rotation;  // as stored in the file (d x d, or 1 x d DCT signs)
    pdxg::host::HostLevel l1, l0;
    uint8_t* arena = nullptr;
    uint64_t arena_bytes = 0;
    pdxg::DevCluster* d_cl1 = nullptr;
    pdxg::DevCluster* d_cl0 = nullptr;
    float* d_cent1 = nullptr;
    float* d_cent0 = nullptr;
    float* d_rot = nullptr;
    float* d_rot_hi = nullptr;  // M^T split into TF32 hi / lo planes (tensor-core rotation)
    float* d_rot_lo = nullptr;
    pdxg::GemmOperand rot_op{};
    bool rot_tc = false;        // tensor-core rotation available for this index
    uint32_t rot_mode = 0;      // 0: tensor cores when available, 1: FP32 SIMT GEMM
    float* d_ratios = nullptr;
    uint32_t* d_rid_cluster = nullptr;  // row id -> cluster (device copy, filters)
    uint32_t* d_rid_pos = nullptr;      // row id -> position in its cluster
    float eps0 = 1.5f;
    uint32_t nprobe = 0;
    uint32_t threads = 0;
    uint32_t top_mode = 0;  // tree top level: 0 auto, 1 inside the search CTA, 2 own launch of
                            // per-query CTAs, 3 tiled (probe, partials, replay)
    uint32_t start_mode = 0;  // U8 first-cluster Start: 0 batched when it fits, 1 in the scan
    uint32_t scan_mode = 0;   // U8 scan after a batched Start: 0 cluster-major when it fits,
                              // 1 the per-query kernel only
    // centroid probe: 0 the reference's (exact FP32 probe / tree top-level search), 1 BF16
    // tensor-core rotation and centroid scores + widened list + FP32 rescore, 2 the same with
    // FP8-E4M3 centroid scores. Operands are built on first use.
    uint32_t probe_mode = 0;
    bool pp_ready = false;
    void* d_rot_b16 = nullptr;   // M^T, BF16 (K-major B operand of the rotation)
    void* d_c1_b16 = nullptr;    // L1 centroids, BF16
    uint8_t* d_c1_e4 = nullptr;  // L1 centroids, E4M3 with one scale per row
    float* d_c1_e4s = nullptr;
    float* d_c1_sq = nullptr;    // |c|^2 of the FP32 L1 centroids
    pdxg::GemmOperand rot_op16{}, c1_op16{}, c1_op8{};
    int num_sms = 0;
    size_t max_smem = 0;
    std::vector<uint32_t> rid_cluster, rid_pos;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // host-buffer search: query upload of later chunks
    cudaEvent_t chunk_ev[8] = {};
    cudaStream_t stats_stream = nullptr;
    // PDXG_TIME_KERNELS marks: start, after preparation, after top level / probe, after the
    // batched Start, end
    // PDXG_TIME_KERNELS: [0..4] stage boundaries (start, after query preparation, after the top
    // level, after the batched Start, after the scan); [5..7] inside the cluster-major scan (after
    // its planning kernels, after the bitmaps, after the replay); [8..9] inside the tiled top level
    // (after the meso probe, after the partials)
    cudaEvent_t tev[10] = {};
    bool tev_ready = false, tev_top = false, tev_prep = false, tev_scan = false, tev_tiled = false;
    uint32_t last_launches = 0;  // engine kernels launched by the last search_device_impl
    uint32_t last_order_stride = 0;  // row stride of the visit orders of the last search (0: none)
    pdxg::host::Workspace ws;
    std::mutex mu;
    // registered filters (pdxg_filter_register): resident selection bitmaps + passing counts,
    // one slot each; reg_mu is held from a batch's validation through its launch
    uint32_t* d_reg_sel = nullptr;   // [reg_cap x l1.sel_words]
    uint32_t* d_reg_pass = nullptr;  // [reg_cap x l1 clusters]
    uint32_t reg_cap = 0;
    std::vector<uint8_t> reg_used;
    std::vector<std::vector<uint64_t>> reg_rows;  // row ids of each registered filter
    bool reg_dirty = false;  // slots moved since the bitmaps were built (Append / Delete)
    std::mutex reg_mu;
    // Append / Delete (tree indexes): created on first use
    std::unique_ptr<pdxg::host::Maint> maint;
    uint64_t l0_start = 0;          // first arena byte of the meso level
    bool append_normalize = false;  // PDXIndexConfig::normalize: set by a build, false after a
                                    // load (LoadPDXIndex uses the default config)
};
