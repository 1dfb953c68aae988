// C-ABI wrapper around the reference PDX search code, compiled from the reference's own
// headers (include/pdx/{common,cluster,ivf_wrapper,searcher,...}.hpp) by oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY. Tests, the smoke check and bench.py's CPU-baseline / reference arm
// use this library as the checker or the timed CPU baseline. The product (libpdx_b200.so) never
// links or calls it.
//
// index.hpp cannot be included: it pulls clustering.hpp -> SuperKMeans, an empty submodule.
// This file therefore restates the few lines of index.hpp that sit on the load/search path:
//   - LoadPDXIndex type dispatch                      (index.hpp:1736-1760)
//   - PDXIndex / PDXTreeIndex ::Restore               (index.hpp:242-267, 516-543)
//   - PDXTreeIndex::Search (top-level search + order) (index.hpp:545-566)
//   - CreatePredicateEvaluator + BuildRowIdClusterMapping (index.hpp:421-446, 818-845)
//   - PDXTreeIndex::Append / Delete / CheckClusterHealth and Save's compaction
//     (index.hpp:580-638, 1241-1255, 484-494) on the reference's Cluster (cluster.hpp); the
//     split and merge branches run SuperKMeans, so they are replaced by the substitutes the
//     engine uses (capacity growth to max(uint32(1.3 used), 256); no merge)
// Everything below those calls (IVF::Load, ADSamplingPruner, PDXearch::Search/FilteredSearch,
// distance computers) is the reference's unmodified code.
#include <cstddef>
#include <cstdint>

extern "C" void sgemm_(const char* transa, const char* transb, const int* m, const int* n,
                       const int* k, const float* alpha, const float* a, const int* lda,
                       const float* b, const int* ldb, const float* beta, float* c,
                       const int* ldc);

#include "pdx/common.hpp"
#include "pdx/db_mock/predicate_evaluator.hpp"
#include "pdx/ivf_wrapper.hpp"
#include "pdx/pruners/adsampling.hpp"
#include "pdx/quantizers/scalar.hpp"
#include "pdx/searcher.hpp"
#include "pdx/utils.hpp"

#include <cstring>
#include <limits>
#include <memory>
#include <omp.h>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

struct RefIndexBase {
    virtual ~RefIndexBase() = default;
    uint8_t type = 0;
    std::unique_ptr<PDX::ADSamplingPruner> pruner;
    uint32_t nprobe = 0;
    virtual uint32_t Dims() const = 0;
    virtual uint32_t NumClusters() const = 0;
    virtual uint32_t ClusterSize(uint32_t c) const = 0;
    virtual const uint32_t* ClusterIds(uint32_t c) const = 0;
    virtual void Search(const float* q, uint32_t k, bool transformed,
                        std::vector<PDX::KNNCandidate>& out) = 0;
    virtual void FilteredSearch(const float* q, uint32_t k, const uint64_t* row_ids, size_t n,
                                bool transformed, std::vector<PDX::KNNCandidate>& out) = 0;
    virtual void SearchWithOrder(const float* q, uint32_t k, const uint32_t* order, size_t n_order,
                                 bool transformed, std::vector<PDX::KNNCandidate>& out) = 0;
    // GetClusterRowIds (index.hpp:772-782): the used slots that are not tombstoned
    virtual void LiveRowIds(uint32_t c, uint32_t* out) const {
        std::memcpy(out, ClusterIds(c), sizeof(uint32_t) * ClusterSize(c));
    }
    virtual void Append(uint64_t, const float*, bool) {
        throw std::runtime_error("Append is not implemented in PDXIndex. Use PDXTreeIndex instead.");
    }
    virtual void Delete(uint64_t) {
        throw std::runtime_error("Delete is not implemented in PDXIndex. Use PDXTreeIndex instead.");
    }
    virtual void CompactAll() {}
    bool append_normalize = false;  // PDXIndexConfig::normalize (false after LoadPDXIndex)
    uint64_t maint_stats[5] = {0, 0, 0, 0, 0};  // appends, deletes, compactions, growths, merges
};

template <class IndexT, PDX::Quantization Q>
PDX::PredicateEvaluator MakeEvaluator(const IndexT& index,
                                      const std::vector<std::pair<uint32_t, uint32_t>>& mapping,
                                      const uint64_t* row_ids, size_t n) {
    PDX::PredicateEvaluator ev(index.num_clusters, index.total_capacity);
    for (size_t i = 0; i < n; ++i) {
        if (row_ids[i] >= mapping.size()) continue;
        const auto& [cluster_id, pos] = mapping[row_ids[i]];
        if (cluster_id == std::numeric_limits<uint32_t>::max()) continue;  // DELETED_MARKER
        ev.n_passing_tuples[cluster_id]++;
        ev.selection_vector[index.cluster_offsets[cluster_id] + pos] = 1;
    }
    return ev;
}

template <class IndexT>
std::vector<std::pair<uint32_t, uint32_t>> RowIdMapping(const IndexT& index) {
    size_t total = 0;
    for (size_t c = 0; c < index.num_clusters; c++) total += index.clusters[c].num_embeddings;
    std::vector<std::pair<uint32_t, uint32_t>> m(total);
    for (uint32_t c = 0; c < index.num_clusters; c++)
        for (uint32_t p = 0; p < index.clusters[c].num_embeddings; p++) {
            uint32_t rid = index.clusters[c].indices[p];
            if (rid < total) m[rid] = {c, p};
        }
    return m;
}

template <PDX::Quantization Q>
struct RefFlat : RefIndexBase {
    PDX::IVF<Q> index;
    std::vector<std::pair<uint32_t, uint32_t>> mapping;
    uint32_t Dims() const override { return index.num_dimensions; }
    uint32_t NumClusters() const override { return index.num_clusters; }
    uint32_t ClusterSize(uint32_t c) const override { return index.clusters[c].num_embeddings; }
    const uint32_t* ClusterIds(uint32_t c) const override { return index.clusters[c].indices; }
    void Search(const float* q, uint32_t k, bool transformed,
                std::vector<PDX::KNNCandidate>& out) override {
        PDX::PDXearch<Q> s(index, *pruner);
        s.SetNProbe(nprobe);
        out = s.Search(q, k, transformed);
    }
    void FilteredSearch(const float* q, uint32_t k, const uint64_t* row_ids, size_t n,
                        bool transformed, std::vector<PDX::KNNCandidate>& out) override {
        PDX::PDXearch<Q> s(index, *pruner);
        s.SetNProbe(nprobe);
        auto ev = MakeEvaluator<PDX::IVF<Q>, Q>(index, mapping, row_ids, n);
        out = s.FilteredSearch(q, k, ev, transformed);
    }
    void SearchWithOrder(const float* q, uint32_t k, const uint32_t* order, size_t n_order,
                         bool transformed, std::vector<PDX::KNNCandidate>& out) override {
        PDX::PDXearch<Q> s(index, *pruner);
        s.SetNProbe(nprobe);
        s.SetClusterAccessOrder(std::vector<uint32_t>(order, order + n_order));
        out = s.Search(q, k, transformed);
    }
};

template <PDX::Quantization Q>
struct RefTree : RefIndexBase {
    PDX::IVFTree<Q> index;
    std::vector<std::pair<uint32_t, uint32_t>> mapping;
    uint32_t Dims() const override { return index.num_dimensions; }
    uint32_t NumClusters() const override { return index.num_clusters; }
    uint32_t ClusterSize(uint32_t c) const override { return index.clusters[c].num_embeddings; }
    const uint32_t* ClusterIds(uint32_t c) const override { return index.clusters[c].indices; }

    // Mirrors PDXTreeIndex::Search (index.hpp:545-566) with fresh per-call searchers so that
    // concurrent callers never share the mutable searcher state the reference keeps.
    std::vector<uint32_t> TopLevelOrder(const float* q, bool transformed, uint32_t& l1_nprobe) {
        PDX::PDXearch<Q> s(index, *pruner);
        PDX::PDXearch<PDX::F32> top(index.l0, *pruner);
        l1_nprobe = nprobe == 0 ? index.num_clusters : nprobe;
        uint32_t n_probe_top = index.l0.num_clusters;
        if (l1_nprobe < index.num_clusters / 2) n_probe_top /= 2;
        top.SetNProbe(n_probe_top);
        auto res = top.Search(q, l1_nprobe, transformed);
        std::vector<uint32_t> ids(res.size());
        for (size_t i = 0; i < res.size(); i++) ids[i] = res[i].index;
        return ids;
    }
    void Search(const float* q, uint32_t k, bool transformed,
                std::vector<PDX::KNNCandidate>& out) override {
        uint32_t l1_nprobe = 0;
        auto ids = TopLevelOrder(q, transformed, l1_nprobe);
        PDX::PDXearch<Q> s(index, *pruner);
        s.SetNProbe(l1_nprobe);
        s.SetClusterAccessOrder(ids);
        out = s.Search(q, k, transformed);
    }
    void FilteredSearch(const float* q, uint32_t k, const uint64_t* row_ids, size_t n,
                        bool transformed, std::vector<PDX::KNNCandidate>& out) override {
        // The reference's restored tree has no L1 centroid array (IVFTree::Save omits it), so
        // PDXearch::FilteredSearch would read an empty vector. The L1 centroids are the L0
        // clusters' vectors; rebuild them here exactly as the in-memory built tree holds them.
        if (index.centroids.size() != static_cast<size_t>(index.num_clusters) * index.num_dimensions)
            RebuildL1Centroids();
        PDX::PDXearch<Q> s(index, *pruner);
        s.SetNProbe(nprobe);
        auto ev = MakeEvaluator<PDX::IVFTree<Q>, Q>(index, mapping, row_ids, n);
        out = s.FilteredSearch(q, k, ev, transformed);
    }
    void SearchWithOrder(const float* q, uint32_t k, const uint32_t* order, size_t n_order,
                         bool transformed, std::vector<PDX::KNNCandidate>& out) override {
        PDX::PDXearch<Q> s(index, *pruner);
        s.SetNProbe(nprobe == 0 ? index.num_clusters : nprobe);
        s.SetClusterAccessOrder(std::vector<uint32_t>(order, order + n_order));
        out = s.Search(q, k, transformed);
    }
    void LiveRowIds(uint32_t c, uint32_t* out) const override {
        const auto& cl = index.clusters[c];
        uint32_t j = 0;
        for (uint32_t i = 0; i < cl.used_capacity; i++)
            if (!cl.HasTombstone(i)) out[j++] = cl.indices[i];
    }

    static constexpr uint32_t kDeleted = std::numeric_limits<uint32_t>::max();  // index.hpp:462

    // PDXTreeIndex::Append (index.hpp:580-616)
    void Append(uint64_t row_id, const float* embedding, bool transformed) override {
        if (row_id != mapping.size())
            throw std::invalid_argument("Append: row_id " + std::to_string(row_id) +
                                        " is not sequential (expected " + std::to_string(mapping.size()) + ")");
        const uint32_t d = index.num_dimensions;
        std::unique_ptr<float[]> pre(new float[d]);
        if (transformed) {
            std::memcpy(pre.get(), embedding, sizeof(float) * d);
        } else {  // NormalizeAndRotate (index.hpp:75-97)
            const float* in = embedding;
            std::unique_ptr<float[]> normalized;
            if (append_normalize) {
                normalized.reset(new float[d]);
                PDX::Quantizer qz(d);
                qz.NormalizeQuery(embedding, normalized.get());
                in = normalized.get();
            }
            pruner->PreprocessEmbeddings(in, pre.get(), 1);
        }
        PDX::PDXearch<PDX::F32> top(index.l0, *pruner);
        top.SetNProbe(std::max(1u, index.l0.num_clusters / 8));
        auto cand = top.Search(pre.get(), 1, true);
        const uint32_t c = cand[0].index;
        auto& cluster = index.clusters[c];
        uint32_t pos;
        if constexpr (Q == PDX::U8) {  // QuantizeAndAppend (index.hpp:885-896)
            std::unique_ptr<uint8_t[]> qv(new uint8_t[d]);
            PDX::ScalarQuantizer<Q> quantizer(d);
            quantizer.QuantizeEmbedding(pre.get(), index.quantization_base, index.quantization_scale, qv.get());
            pos = cluster.AppendEmbedding(static_cast<uint32_t>(row_id), qv.get());
        } else {
            pos = cluster.AppendEmbedding(static_cast<uint32_t>(row_id), pre.get());
        }
        mapping.emplace_back(c, pos);
        index.total_num_embeddings++;
        maint_stats[0]++;
        CheckHealth(c);
    }

    // PDXTreeIndex::Delete (index.hpp:619-638)
    void Delete(uint64_t row_id) override {
        if (row_id >= mapping.size())
            throw std::invalid_argument("Delete: row_id " + std::to_string(row_id) + " is not in the index");
        const auto [c, pos] = mapping[row_id];
        if (c == kDeleted)
            throw std::invalid_argument("Delete: row_id " + std::to_string(row_id) + " was already deleted");
        index.clusters[c].DeleteEmbedding(pos);
        mapping[row_id] = {kDeleted, kDeleted};
        index.total_num_embeddings--;
        maint_stats[1]++;
        CheckHealth(c);
    }

    // CheckClusterHealth (index.hpp:1241-1255) with the split / merge substitutes
    void CheckHealth(uint32_t c) {
        auto& cluster = index.clusters[c];
        if (cluster.used_capacity == cluster.max_capacity) {
            if (cluster.num_embeddings < cluster.used_capacity) {
                for (const auto& [rid, idx] : cluster.CompactCluster()) mapping[rid] = {c, idx};
                maint_stats[2]++;
            } else {
                Grow(c);
            }
        } else if (cluster.num_embeddings <= cluster.min_capacity) {
            maint_stats[4]++;
        }
    }

    // In place of SplitCluster: the same rows, in the same slots, in a buffer of
    // max(uint32(1.3 used), 256) slots.
    void Grow(uint32_t c) {
        auto& old = index.clusters[c];
        const uint32_t d = index.num_dimensions;
        uint32_t cap = std::max<uint32_t>(static_cast<uint32_t>(static_cast<float>(old.used_capacity) * 1.3f), 256u);
        if (cap <= old.used_capacity) cap = old.used_capacity + 1;
        auto rows = old.GetHorizontalEmbeddingsFromPDXBuffer();
        PDX::Cluster<Q> grown(0u, cap, d);
        for (uint32_t i = 0; i < old.num_embeddings; i++)
            grown.AppendEmbedding(old.indices[i], rows.get() + static_cast<size_t>(i) * d);
        grown.min_capacity = old.min_capacity;
        grown.id = old.id;
        grown.mesocluster_id = old.mesocluster_id;
        index.clusters[c] = std::move(grown);
        index.ComputeClusterOffsets();
        maint_stats[3]++;
    }

    // The compaction of PDXTreeIndex::Save (index.hpp:484-494)
    void CompactAll() override {
        for (uint32_t c = 0; c < index.num_clusters; c++)
            for (const auto& [rid, idx] : index.clusters[c].CompactCluster()) mapping[rid] = {c, idx};
        for (uint32_t c = 0; c < index.l0.num_clusters; c++) index.l0.clusters[c].CompactCluster();
    }

    void RebuildL1Centroids() {
        const uint32_t d = index.num_dimensions;
        std::vector<float> cents(static_cast<size_t>(index.num_clusters) * d, 0.0f);
        const uint32_t dv = index.l0.num_vertical_dimensions;
        const uint32_t dh = index.l0.num_horizontal_dimensions;
        for (auto& c : index.l0.clusters) {
            const size_t stride = c.max_capacity;
            for (uint32_t p = 0; p < c.num_embeddings; p++) {
                float* dst = cents.data() + static_cast<size_t>(c.indices[p]) * d;
                for (uint32_t j = 0; j < dv; j++) dst[j] = c.data[j * stride + p];
                for (uint32_t b = 0; b < dh; b += 64)
                    for (uint32_t j = 0; j < 64; j++)
                        dst[dv + b + j] = c.data[(dv + b) * stride + static_cast<size_t>(p) * 64 + j];
            }
        }
        index.centroids = std::move(cents);
    }
};

thread_local std::string g_last_error;

RefIndexBase* LoadRef(const char* path) {
    auto buffer = MmapFile(path);
    char* ptr = buffer.get();
    const uint8_t type = static_cast<uint8_t>(ptr[0]);
    ptr += 1;
    uint32_t rows, cols;
    std::memcpy(&rows, ptr, 4);
    ptr += 4;
    std::memcpy(&cols, ptr, 4);
    ptr += 4;
    std::unique_ptr<float[]> matrix(new float[static_cast<size_t>(rows) * cols]);
    std::memcpy(matrix.get(), ptr, sizeof(float) * rows * cols);
    ptr += sizeof(float) * rows * cols;
    std::unique_ptr<RefIndexBase> out;
    switch (type) {
    case 0: {
        auto r = std::make_unique<RefFlat<PDX::F32>>();
        r->index.Load(ptr);
        r->pruner = std::make_unique<PDX::ADSamplingPruner>(r->index.num_dimensions, matrix.get());
        r->mapping = RowIdMapping(r->index);
        out = std::move(r);
        break;
    }
    case 1: {
        auto r = std::make_unique<RefFlat<PDX::U8>>();
        r->index.Load(ptr);
        r->pruner = std::make_unique<PDX::ADSamplingPruner>(r->index.num_dimensions, matrix.get());
        r->mapping = RowIdMapping(r->index);
        out = std::move(r);
        break;
    }
    case 2: {
        auto r = std::make_unique<RefTree<PDX::F32>>();
        r->index.Load(ptr);
        r->pruner = std::make_unique<PDX::ADSamplingPruner>(r->index.num_dimensions, matrix.get());
        r->mapping = RowIdMapping(r->index);
        out = std::move(r);
        break;
    }
    case 3: {
        auto r = std::make_unique<RefTree<PDX::U8>>();
        r->index.Load(ptr);
        r->pruner = std::make_unique<PDX::ADSamplingPruner>(r->index.num_dimensions, matrix.get());
        r->mapping = RowIdMapping(r->index);
        out = std::move(r);
        break;
    }
    default:
        throw std::runtime_error("Unknown PDX index type: " + std::to_string(type));
    }
    out->type = type;
    return out.release();
}

int Emit(const std::vector<PDX::KNNCandidate>& res, uint32_t* ids, float* dists) {
    for (size_t i = 0; i < res.size(); i++) {
        ids[i] = res[i].index;
        dists[i] = res[i].distance;
    }
    return static_cast<int>(res.size());
}

} // namespace

extern "C" {

const char* pdxref_last_error() { return g_last_error.c_str(); }

void* pdxref_load(const char* path) {
    try {
        return LoadRef(path);
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return nullptr;
    }
}

void pdxref_free(void* h) { delete static_cast<RefIndexBase*>(h); }

int pdxref_type(void* h) { return static_cast<RefIndexBase*>(h)->type; }
uint32_t pdxref_num_dimensions(void* h) { return static_cast<RefIndexBase*>(h)->Dims(); }
uint32_t pdxref_num_clusters(void* h) { return static_cast<RefIndexBase*>(h)->NumClusters(); }
uint32_t pdxref_cluster_size(void* h, uint32_t c) {
    return static_cast<RefIndexBase*>(h)->ClusterSize(c);
}
void pdxref_cluster_row_ids(void* h, uint32_t c, uint32_t* out) {
    static_cast<RefIndexBase*>(h)->LiveRowIds(c, out);
}

// 0, 1 (std::invalid_argument) or 2 (other error); the message in pdxref_last_error.
int pdxref_append(void* h, uint64_t row_id, const float* embedding, int transformed) {
    try {
        static_cast<RefIndexBase*>(h)->Append(row_id, embedding, transformed != 0);
        return 0;
    } catch (const std::invalid_argument& e) {
        g_last_error = e.what();
        return 1;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return 2;
    }
}

int pdxref_delete(void* h, uint64_t row_id) {
    try {
        static_cast<RefIndexBase*>(h)->Delete(row_id);
        return 0;
    } catch (const std::invalid_argument& e) {
        g_last_error = e.what();
        return 1;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return 2;
    }
}

void pdxref_set_append_normalization(void* h, int on) {
    static_cast<RefIndexBase*>(h)->append_normalize = on != 0;
}

void pdxref_compact_all(void* h) { static_cast<RefIndexBase*>(h)->CompactAll(); }

void pdxref_maintenance_stats(void* h, uint64_t* out) {
    std::memcpy(out, static_cast<RefIndexBase*>(h)->maint_stats, sizeof(uint64_t) * 5);
}


void pdxref_set_nprobe(void* h, uint32_t nprobe) { static_cast<RefIndexBase*>(h)->nprobe = nprobe; }

void pdxref_set_pruning_aggressiveness(void* h, float eps0) {
    static_cast<RefIndexBase*>(h)->pruner->SetPruningAggresiveness(eps0);
}

// ADSamplingPruner::PreprocessEmbeddings (adsampling.hpp:107-113): out = rotate(in), n rows.
void pdxref_rotate(void* h, const float* in, float* out, uint32_t n) {
    static_cast<RefIndexBase*>(h)->pruner->PreprocessEmbeddings(in, out, n);
}

int pdxref_search(void* h, const float* q, uint32_t k, int transformed, uint32_t* ids,
                  float* dists) {
    try {
        std::vector<PDX::KNNCandidate> res;
        static_cast<RefIndexBase*>(h)->Search(q, k, transformed != 0, res);
        return Emit(res, ids, dists);
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

int pdxref_search_with_order(void* h, const float* q, uint32_t k, const uint32_t* order,
                             uint32_t n_order, int transformed, uint32_t* ids, float* dists) {
    try {
        std::vector<PDX::KNNCandidate> res;
        static_cast<RefIndexBase*>(h)->SearchWithOrder(q, k, order, n_order, transformed != 0, res);
        return Emit(res, ids, dists);
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

int pdxref_filtered_search(void* h, const float* q, uint32_t k, const uint64_t* row_ids,
                           uint64_t n_row_ids, int transformed, uint32_t* ids, float* dists) {
    try {
        std::vector<PDX::KNNCandidate> res;
        static_cast<RefIndexBase*>(h)->FilteredSearch(q, k, row_ids, n_row_ids, transformed != 0,
                                                      res);
        return Emit(res, ids, dists);
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return -1;
    }
}

// nq queries (row-major nq x d), results in [nq x k] slots with per-query counts. Each OpenMP
// thread runs its own searcher objects, as a multi-threaded caller of the reference must.
int pdxref_search_batch(void* h, const float* q, uint32_t nq, uint32_t k, int transformed,
                        int n_threads, uint32_t* ids, float* dists, uint32_t* counts) {
    auto* r = static_cast<RefIndexBase*>(h);
    const uint32_t d = r->Dims();
    int failed = 0;
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads)
    for (int64_t i = 0; i < static_cast<int64_t>(nq); i++) {
        try {
            std::vector<PDX::KNNCandidate> res;
            r->Search(q + static_cast<size_t>(i) * d, k, transformed != 0, res);
            counts[i] = static_cast<uint32_t>(res.size());
            Emit(res, ids + static_cast<size_t>(i) * k, dists + static_cast<size_t>(i) * k);
        } catch (...) {
#pragma omp atomic write
            failed = 1;
        }
    }
    return failed ? -1 : 0;
}

} // extern "C"
