/*
 * pdx_b200.h -- C ABI of the B200 PDX search engine (libpdx_b200.so).
 *
 * Drop-in boundary for the reference's search path: every entry point below replaces one
 * member of the reference's C++ index interface (include/pdx/index.hpp) or of its pybind
 * surface (include/pdx/lib/lib.hpp, python/lib.cpp), with plain pointers and sizes instead of
 * C++ / numpy types. Status codes are returned, never thrown; pdxg_last_error() describes the
 * last failure on the calling thread.
 *
 * Index files are the reference's own serialized format (PDXIndex/PDXTreeIndex::Save,
 * index.hpp:213-239 and 483-514); an index is loaded once into GPU memory and searched there.
 * The search path has no CPU fallback: without a usable CUDA device every call fails with
 * PDXG_ERR_CUDA.
 */
#ifndef PDX_B200_H
#define PDX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pdxg_index pdxg_index;

/* Status codes. */
#define PDXG_OK 0
#define PDXG_ERR_INVALID_ARGUMENT 1 /* std::invalid_argument in the reference */
#define PDXG_ERR_IO 2               /* file missing / unreadable / truncated */
#define PDXG_ERR_FORMAT 3           /* unknown index type or inconsistent header */
#define PDXG_ERR_CUDA 4             /* CUDA runtime failure (no device, launch error, OOM) */
#define PDXG_ERR_UNSUPPORTED 5      /* operation not available for this index type */
#define PDXG_ERR_CAPACITY 6         /* request exceeds a stated engine limit */

/* Index types: the type byte of the file (common.hpp:78, PDXIndexType). */
#define PDXG_TYPE_F32 0
#define PDXG_TYPE_U8 1
#define PDXG_TYPE_TREE_F32 2
#define PDXG_TYPE_TREE_U8 3

/* Search flags. */
#define PDXG_QUERY_TRANSFORMED 1u /* queries are already normalized + rotated: the reference's
                                     Search(query, k, is_query_transformed = true),
                                     searcher.hpp:596-613 */
#define PDXG_COLLECT_STATS 2u     /* count the index bytes the search algorithm reads (centroid
                                     probes, Start scans, warmup steps, survivor gathers);
                                     read them back with pdxg_get_stats */
#define PDXG_TIME_KERNELS 4u      /* record CUDA events around the query preparation, the tree
                                     top level and the scan kernel on the search's stream;
                                     read the durations with pdxg_kernel_times */

/* Last error message of the calling thread (never NULL). */
const char* pdxg_last_error(void);

/* Replaces LoadPDXIndex(path) (index.hpp:1736-1760) + Restore (index.hpp:242-267, 516-543) and
 * the pybind module function load_index (python/lib.cpp:52-57). Loads the file into GPU memory
 * on `device`. */
int pdxg_load(const char* path, int device, pdxg_index** out);

/* Same as pdxg_load, from an in-memory copy of the file bytes. */
int pdxg_load_buffer(const void* data, uint64_t size, int device, pdxg_index** out);

/* Replaces IPDXIndex::BuildIndex (index.hpp:174, 329-403 for PDXIndex, 640-758 for PDXTreeIndex;
 * PDXIndexConfig index.hpp:27-40) and the pybind PDXIndex.build_index (python/lib.cpp:35): builds
 * the index on `device` from `n` row-major float rows of `d` dims and loads it. `rotation` is the
 * d x d row-major matrix applied to every (normalized, if `normalize`) row; index_type is one of
 * PDXG_TYPE_*. num_clusters = 0 takes ComputeNumberOfClusters (common.hpp:191-199);
 * num_meso_clusters = 0 takes sqrt(num_clusters) (trees only). k-means runs `kmeans_iters` Lloyd
 * updates with BF16 tensor-core assignment (spherical for normalized data); the clustering is this
 * engine's own, so cluster contents differ from the reference's (its SuperKMeans), while the file
 * layout, the SQ8 parameters, the rotation and everything a search reads follow the reference.
 * The same inputs and seed give the same index bytes. PDXG_ERR_UNSUPPORTED when d is not a
 * multiple of 8 or the tensor-core GEMM is not available. */
int pdxg_build(const float* data, uint64_t n, uint32_t d, uint32_t index_type, uint32_t num_clusters,
               uint32_t num_meso_clusters, int normalize, const float* rotation, uint64_t seed,
               uint32_t kmeans_iters, int device, pdxg_index** out);

/* Releases the index and its GPU memory. NULL is ignored. */
void pdxg_free(pdxg_index* index);

/* Replaces IPDXIndex::SetNProbe (index.hpp:171, 282) / PDXIndex.set_nprobe (lib.cpp:41).
 * 0 means "all clusters", as in PDXearch::Search (searcher.hpp:614-616). */
int pdxg_set_nprobe(pdxg_index* index, uint32_t nprobe);

/* Replaces ADSamplingPruner::SetPruningAggresiveness (adsampling.hpp:80-85): epsilon0 of the
 * ADSampling bound (default 1.5, common.hpp:67). Very large values disable pruning. */
int pdxg_set_pruning_aggressiveness(pdxg_index* index, float epsilon0);

/* Replaces IPDXIndex::Search (index.hpp:167, 269-271, 545-566) and PDXIndex.search
 * (lib.hpp:92-112), batched: `queries` is nq x d row-major float32 in HOST memory; results go
 * to host arrays ids[nq*k], distances[nq*k] (ascending per query; unused slots hold
 * UINT32_MAX / +inf) and counts[nq]. Synchronous. */
int pdxg_search(pdxg_index* index, const float* queries, uint32_t nq, uint32_t k, uint32_t flags,
                uint32_t* ids, float* distances, uint32_t* counts);

/* Device-resident variant of pdxg_search: every pointer is GPU memory on the index's device;
 * the work is enqueued on `stream` (a cudaStream_t, NULL = the index's own stream) and the call
 * returns without waiting. Workspace is allocated on first use and reused (growing it may
 * synchronize the device). After Append / Delete the first search enqueues the upload of the
 * changes on its stream ahead of its kernels, without a device synchronisation; a search issued
 * inside a stream capture while changes are pending fails with PDXG_ERR_INVALID_ARGUMENT. */
int pdxg_search_device(pdxg_index* index, const float* queries, uint32_t nq, uint32_t k,
                       uint32_t flags, uint32_t* ids, float* distances, uint32_t* counts,
                       void* stream);

/* Replaces PDXearch::SetClusterAccessOrder (searcher.hpp:48-54) followed by Search: visits the
 * given clusters (at most nprobe of them) in the given order instead of probing centroids.
 * Host pointers, synchronous. */
int pdxg_search_with_order(pdxg_index* index, const float* queries, uint32_t nq, uint32_t k,
                           const uint32_t* order, uint32_t n_order, uint32_t flags, uint32_t* ids,
                           float* distances, uint32_t* counts);

/* Replaces IPDXIndex::FilteredSearch (index.hpp:168-172, 273-280, 568-578) and
 * PDXIndex.filtered_search (lib.hpp:114-142): one query, only rows whose id is listed in
 * row_ids[n_row_ids] can be returned. Host pointers, synchronous; *count receives the number
 * of results written to ids[k] / distances[k]. Unknown row ids are ignored. */
int pdxg_filtered_search(pdxg_index* index, const float* query, uint32_t k,
                         const uint64_t* row_ids, uint64_t n_row_ids, uint32_t flags,
                         uint32_t* ids, float* distances, uint32_t* count);

/* Batched filtered search: nq queries, each with its own row-id list. Query q uses
 * row_ids[offsets[q] .. offsets[q+1]) (offsets has nq+1 entries); offsets[q] == UINT64_MAX
 * marks query q as unfiltered. Host pointers, synchronous. */
int pdxg_filtered_search_batch(pdxg_index* index, const float* queries, uint32_t nq, uint32_t k,
                               const uint64_t* row_ids, const uint64_t* offsets, uint32_t flags,
                               uint32_t* ids, float* distances, uint32_t* counts);

/* Replaces IPDXIndex::Save (index.hpp:173, 213-239, 483-514): writes the reference's format.
 * After Append / Delete it first compacts every cluster, as the reference's tree Save does,
 * which moves slots for later searches too. */
int pdxg_save(pdxg_index* index, const char* path);

/* Replaces PDXTreeIndex::Append (index.hpp:580-616) and PDXIndex.append (python/lib.cpp:51,
 * lib.hpp:166-172): row_id must be the next row id (the row count so far); the embedding (d
 * floats, host memory) is normalized when the index was built with normalize (an index loaded
 * from a file keeps LoadPDXIndex's default config, which does not normalize: see
 * pdxg_set_append_normalization) and rotated, then placed in the L1 cluster the top-level search
 * finds (k = 1 over max(1, n_L0 / 8) meso clusters), in a tombstoned slot if the cluster has one
 * (quantized with the index's SQ8 parameters for U8). PDXG_QUERY_TRANSFORMED in flags: the
 * embedding is already normalized and rotated. Flat indexes answer PDXG_ERR_UNSUPPORTED
 * ("Append is not implemented in PDXIndex", index.hpp:405-407). Not concurrent with searches. */
int pdxg_append(pdxg_index* index, uint64_t row_id, const float* embedding, uint32_t flags);

/* n appends of rows first_row_id, first_row_id + 1, ... (n x d floats, host memory, row-major),
 * with the results of n pdxg_append calls in that order: a row's cluster comes from the top-level
 * search over the meso level, which appends never change, so one batched rotation and top-level
 * search serve the batch, and the slots and health checks follow row by row. */
int pdxg_append_batch(pdxg_index* index, uint64_t first_row_id, uint32_t n, const float* embeddings,
                      uint32_t flags);

/* Replaces PDXTreeIndex::Delete (index.hpp:619-638) and PDXIndex.delete (python/lib.cpp:52):
 * tombstones the row's slot. PDXG_ERR_INVALID_ARGUMENT for a row never appended or already
 * deleted. After Append and Delete the cluster health check of index.hpp:1241-1255 runs: a full
 * cluster with tombstones is compacted exactly as the reference does; where the reference would
 * split a full cluster or merge a small one (SuperKMeans, not in the reference tree) this engine
 * grows the cluster's capacity to max(1.3 x used, 256) slots, or keeps the cluster. */
int pdxg_delete(pdxg_index* index, uint64_t row_id);

/* PDXIndexConfig::normalize for Append (index.hpp:590-591): 1 for an index the caller built with
 * normalize (pdxg_build sets it), 0 after pdxg_load (the reference's LoadPDXIndex default). */
int pdxg_set_append_normalization(pdxg_index* index, int normalize);

/* Maintenance counters: appends, deletes, compactions, capacity growths in place of splits,
 * merges not performed, tombstoned slots now. */
int pdxg_maintenance_stats(const pdxg_index* index, uint64_t out[6]);

/* Getters: IPDXIndex::GetNumDimensions / GetNumClusters / GetClusterSize / GetClusterRowIds /
 * GetInMemorySizeInBytes (index.hpp:175-179) and the pybind getters (lib.hpp:148-164). */
int pdxg_index_type(const pdxg_index* index);
uint32_t pdxg_num_dimensions(const pdxg_index* index);
uint32_t pdxg_num_clusters(const pdxg_index* index);
uint32_t pdxg_nprobe(const pdxg_index* index);
uint32_t pdxg_cluster_size(const pdxg_index* index, uint32_t cluster_id);
int pdxg_cluster_row_ids(const pdxg_index* index, uint32_t cluster_id, uint32_t* out,
                         uint32_t capacity);
uint64_t pdxg_in_memory_size_in_bytes(const pdxg_index* index);
uint64_t pdxg_num_embeddings(const pdxg_index* index);

/* Rotated (normalized when the index is) queries, as the search sees them: the reference's
 * ADSamplingPruner::PreprocessQuery (adsampling.hpp:100-113) on nq host queries. */
int pdxg_prepare_queries(pdxg_index* index, const float* queries, uint32_t nq, float* out);

/* Counters of the last search launched with PDXG_COLLECT_STATS (synchronizes the index's
 * stream): out[0] index bytes read by the algorithm, out[1] clusters visited, out[2] vectors
 * that reached the heap merge, out[3..8] the bytes of out[0] by phase (tree top-level search,
 * Start scans, warmup steps, survivor horizontal blocks, survivor vertical dims, centroid
 * probe), out[9..11] SM cycles spent per query in the top-level search, in Start, and in
 * the rest of the scan. No counterpart in the reference (its profiler times phases, profiler.hpp:36-320);
 * used for the roofline accounting. */
int pdxg_get_stats(pdxg_index* index, uint64_t out[12]);

/* Counters of the cluster-major scan in the last search launched with PDXG_COLLECT_STATS
 * (synchronizes the index's stream): out[0] candidates tested (vectors below the first warmup
 * checkpoint's bound at the heap top after the Start), out[1] of those below the bound at the
 * heap top of their visit, out[2] visits whose warmup stopped after its first step, out[3]
 * visits that ran the whole warmup. No counterpart in the reference; diagnostics of
 * pdxg_set_scan_mode 0. */
int pdxg_get_scan_stats(pdxg_index* index, uint64_t out[4]);

/* Engine kernels launched by the last pdxg_search_device call on this index (query
 * preparation, tree top level and scan; memsets not counted). No counterpart in the reference. */
uint32_t pdxg_last_launch_count(const pdxg_index* index);

/* Durations (ms) of the last search launched with PDXG_TIME_KERNELS through pdxg_search_device:
 * out[0] query preparation (normalization + rotation), out[1] tree top level, out[2] the scan
 * kernel (0 for a stage that did not run). Waits for that search to finish. No counterpart in
 * the reference; used for the roofline accounting. */
int pdxg_kernel_times(pdxg_index* index, float out[3]);
/* As pdxg_kernel_times, split finer: out[0] query preparation, out[1] tree top level or the
 * reduced-precision probe, out[2] the batched Start, out[3] the scan (n >= 4); with n >= 11 also
 * out[4] the cluster-major scan's prep kernel (Start pushes, visit lists), out[5] its bitmaps, out[6] its replay, out[7]
 * the per-query scan kernel, out[8] the tiled top level's meso probe, out[9] its partials, out[10]
 * its replay (0 for what did not run). */
int pdxg_kernel_times_ex(pdxg_index* index, float* out, uint32_t n);

/* Size of the fixed scratch array behind pdxg_search_device_noalloc, per GPU. */
#define PDXG_NOALLOC_SCRATCH_BYTES (8u << 20)

/* Allocation-free variant of pdxg_search_device, for callers that must not have the library
 * call cudaMalloc: hosts whose framework already owns the GPU's memory through its own pool,
 * serving loops that cannot afford the device-wide synchronisation cudaMalloc/cudaFree may
 * cause, plugins running under an allocation policy they do not control. It has no
 * counterpart in the reference (whose CPU search allocates per call, searcher.hpp:601-653).
 *
 * Same arguments and results as pdxg_search_device (all pointers GPU memory; NULL stream = the
 * index's own stream): raw queries are rotated by the same kernels pdxg_search_device picks for
 * the batch (the TF32x3 tensor-core GEMM for more than 8 queries at d >= 512 with rotation mode
 * 0, else the FP32 SIMT kernels), and the search runs the same per-query decisions, so ids and
 * distances are identical. The scratch -- work counter, GEMM wait status, query norms or the
 * TF32 hi / lo planes, rotated queries -- comes from one fixed array of
 * PDXG_NOALLOC_SCRATCH_BYTES compiled into the library; every GPU that loads the library holds it
 * until the process exits. Limit for raw queries: 12*nq*d + 512 bytes with the tensor-core
 * rotation (682 queries at d = 1024), else 4*nq*d + 4*nq + 512 (about 2,040 at d = 1024); larger
 * batches fail with PDXG_ERR_CAPACITY. With PDXG_QUERY_TRANSFORMED only the work counter is used,
 * so any nq fits. PDXG_COLLECT_STATS is rejected and PDXG_TIME_KERNELS ignored; an index set to
 * the reduced-precision probe (pdxg_set_probe_mode 1 or 2) is refused with PDXG_ERR_UNSUPPORTED.
 * The first call on a device looks up the array's device address (with that device current);
 * make that first call before any stream capture. After Append / Delete the first search uploads
 * the changes on its stream (no allocation, no device synchronisation); it fails with
 * PDXG_ERR_INVALID_ARGUMENT if that stream is being captured. All calls share the one array and
 * it keeps the previous call's contents: calls whose work overlaps on the GPU (different
 * streams, or different indexes on the same GPU) race on it and must be serialised by the
 * caller. */
int pdxg_search_device_noalloc(pdxg_index* index, const float* queries, uint32_t nq, uint32_t k,
                               uint32_t flags, uint32_t* ids, float* distances, uint32_t* counts,
                               void* stream);

/* PDXG_NOALLOC_SCRATCH_BYTES as built into the library. */
uint64_t pdxg_noalloc_scratch_bytes(void);

/* Engine tuning, tree indexes: how the top-level (meso-cluster) search of
 * PDXTreeIndex::Search (index.hpp:545-566) runs. 0 = automatic (the tiled form when the index
 * and batch fit it, else per-query CTAs), 1 = inside each query's search CTA, 2 = its own
 * launch of small per-query CTAs, 3 = tiled: a meso probe, exact partial distances per
 * (meso cluster, query tile) computed once with reuse across queries, and a warp per query
 * replaying the reference's decisions on them (needs d and the vertical dims to be multiples
 * of 4 and 16-byte aligned queries). Modes 2 and 3 write the L1 visit orders the search kernel
 * then reads and fail with PDXG_ERR_CAPACITY if they cannot run. Results are identical in
 * every mode. */
int pdxg_set_top_level_mode(pdxg_index* index, uint32_t mode);

/* Engine tuning, U8 tree indexes: the Start of PDXearch (searcher.hpp:217-281) on each query's
 * first visited cluster. 0 = batched when the batch has at least 32 queries and the L1 visit
 * orders come from a separate top level: queries are grouped by first cluster and the exact
 * distances computed once per cluster and group, ahead of the scan; 1 = inside each query's
 * scan CTA. Results are identical in both modes. No counterpart in the reference. */
int pdxg_set_start_mode(pdxg_index* index, uint32_t mode);

/* The centroid probe (GetClustersAccessOrderIVF, searcher.hpp:181-215; for tree indexes the
 * top-level search of PDXTreeIndex::Search, index.hpp:545-566). 0 = the reference's (default);
 * 1 = reduced precision: the rotation and the scores against every L1 centroid run as BF16
 * tensor-core GEMMs with FP32 accumulation, the nprobe list is widened by 10 %, and those
 * candidates are rescored in FP32 with the reference's arithmetic to keep the nprobe nearest;
 * 2 = the same with FP8-E4M3 centroid scores. Modes 1 and 2 need tensor cores and d a multiple
 * of 16 (PDXG_ERR_UNSUPPORTED otherwise); their results differ from the reference's where the
 * reduced precision changes a probe set or a quantized query. No counterpart in the reference
 * (a precision form of its probe). */
int pdxg_set_probe_mode(pdxg_index* index, uint32_t mode);

/* The L1 visit orders of the last pdxg_search_device call, when it computed them ahead of the
 * scan (tree top level in its own launch, or probe modes 1 and 2): orders[i * stride + j] for
 * j < counts[i]. Waits for the device. No counterpart in the reference. */
int pdxg_last_visit_orders(pdxg_index* index, uint32_t nq, uint32_t stride, uint32_t* orders, uint32_t* counts);

/* ---------------------------------------------------------------------------------------
 * Serving-style batches. A context owns a workspace and a CUDA stream; work issued on
 * different contexts of one index runs concurrently. No counterpart in the reference (one
 * query per call there); the per-query semantics are those of Search / FilteredSearch. */
typedef struct pdxg_context pdxg_context;

/* One request of a batch: k results (1 <= k <= k_max), nprobe as SetNProbe (0 = all
 * clusters), and an optional filter: a registered filter (filter_id >= 0, see
 * pdxg_filter_register) or else the row ids rows[filter_begin, filter_end) (filter_id = -1 and
 * filter_begin = UINT64_MAX: no filter). */
typedef struct {
    uint32_t k;
    uint32_t nprobe;
    uint64_t filter_begin;
    uint64_t filter_end;
    int32_t filter_id;
    uint32_t reserved;  /* 0 */
} pdxg_request;

int pdxg_context_create(pdxg_index* index, pdxg_context** out);
void pdxg_context_free(pdxg_context* context);
/* The context's cudaStream_t. */
void* pdxg_context_stream(pdxg_context* context);

/* Enqueues one batch on the context's stream and returns without waiting. `queries` (nq x d)
 * and the outputs ids / distances (nq x k_max, row stride k_max) and counts (nq) are GPU
 * memory; `requests` (nq) and `rows` (the filters' row ids) are host memory, staged before the
 * call returns. Filters are built on the GPU as one bit per cluster slot. A second call on the
 * same context waits for the first call's host-to-device copies only. */
int pdxg_search_requests(pdxg_context* context, const float* queries, uint32_t nq,
                         const pdxg_request* requests, const uint32_t* rows, uint32_t k_max,
                         uint32_t flags, uint32_t* ids, float* distances, uint32_t* counts);

/* Registered filters: the selection bitmap and per-cluster passing counts of a row-id list
 * (CreatePredicateEvaluator, index.hpp:436-446), built once and kept in GPU memory, so that
 * requests naming it stage no row ids. Unknown row ids are ignored, repeated ones count once.
 * Registering may synchronize the device when the filter pool grows. A filter may be released
 * only once the batches that name it have completed. */
int pdxg_filter_register(pdxg_index* index, const uint64_t* row_ids, uint64_t n, int32_t* filter_id);
int pdxg_filter_release(pdxg_index* index, int32_t filter_id);

/* Engine tuning: how queries are rotated (ADSamplingPruner::Rotate, adsampling.hpp:192-246,
 * an FP32 BLAS sgemm in the reference). 0 = tcgen05 tensor cores with FP32 operands split
 * into TF32 hi / lo planes (three products, FP32 rounding level) when the device and the
 * dimension allow it (d >= 512 and a multiple of 4), else the FP32 SIMT GEMM; 1 = always the
 * FP32 SIMT GEMM. pdxg_rotation_uses_tensor_cores tells which one runs. */
int pdxg_set_rotation_mode(pdxg_index* index, uint32_t mode);
int pdxg_rotation_uses_tensor_cores(const pdxg_index* index);

/* Engine tuning, U8 indexes: how the scan (Warmup / Prune / MergeIntoHeap of PDXearch,
 * searcher.hpp:374-566) runs after a batched Start. 0 = cluster-major when it fits (default):
 * each cluster's first warmup step is computed once for all the queries that visit it, bounded
 * by each query's heap top after its Start, and a warp per query replays PDXearch on those
 * results (queries with a filter, or a Start that leaves the heap short of k, take the per-query
 * kernel); 1 = the per-query kernel for every query. Results are identical in both modes. No
 * counterpart in the reference. */
int pdxg_set_scan_mode(pdxg_index* index, uint32_t mode);

/* Engine tuning: threads per query CTA (64, 128, 256 or 512; 0 = automatic). */
int pdxg_set_threads_per_query(pdxg_index* index, uint32_t threads);

#ifdef __cplusplus
}
#endif

#endif /* PDX_B200_H */
