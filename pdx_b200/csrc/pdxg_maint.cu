// Append / Delete on device-resident tree indexes (PDXTreeIndex::Append / Delete,
// index.hpp:580-638); the C ABI entry points pdxg_append, pdxg_append_batch, pdxg_delete,
// pdxg_set_append_normalization and pdxg_maintenance_stats.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "pdxg_engine.cuh"

using namespace pdxg;
using namespace pdxg::host;

// PDXTreeIndex::Append / Delete (index.hpp:580-638) on the device-resident index. The first call
// re-lays the L1 clusters at their max_capacity strides (the buffer of Cluster, cluster.hpp:26-38),
// so an append, a delete and a compaction touch single slots in place; the meso level is copied
// unchanged. The host keeps each cluster's counters, tombstone set and row ids and decides every
// slot; the device holds the slot data (written by a kernel, moved by copies on the index's
// stream), the cluster records, a tombstone bitmap that the scan masks exactly where the
// reference's searcher does (searcher.hpp:169-179 and its callers), and the row-id maps of the
// filters. Records, bitmap and maps are uploaded in one batch before the next search
// (flush_maintenance), so a delete is host bookkeeping and an append costs one device round trip
// (the rotation and the top-level search that choose its cluster).
// Split and merge maintenance (index.hpp:1000-1729) runs the reference's SuperKMeans, whose
// sources are not part of the reference tree: where the reference would split a full cluster
// (used == max_capacity, no tombstones) this engine grows the cluster's capacity to
// max(uint32(1.3 used), 256) slots, and where it would merge a cluster (num_embeddings <=
// min_capacity) it keeps the cluster. Both are counted (pdxg_maintenance_stats); results equal the
// reference's up to the first such event.
namespace {

constexpr uint32_t kNoCluster = 0xFFFFFFFFu;  // DELETED_MARKER (index.hpp:462)
constexpr uint32_t kStageRows = 65536;        // row-map entries per upload batch

uint32_t slot_stride(uint32_t cap) { return std::max<uint32_t>(32, (cap + 31) / 32 * 32); }

uint64_t cluster_block_bytes(const HostLevel& lv, uint32_t np) {
    const uint64_t esz = lv.u8 ? 1 : 4;
    return align_up((uint64_t)lv.n_vwords * np * 4, 256) + align_up((uint64_t)lv.n_hblocks * np * kHDim * esz, 256) +
           align_up((uint64_t)np * 4, 256);
}

// Cluster record m placed at arena offset off (256-byte aligned) with a stride of np slots.
void place_cluster(const HostLevel& lv, DevCluster& m, uint64_t off, uint32_t np) {
    const uint64_t esz = lv.u8 ? 1 : 4;
    m.n_pad = np;
    m.vert_off = off;
    off = align_up(off + (uint64_t)lv.n_vwords * np * 4, 256);
    m.hor_off = off;
    off = align_up(off + (uint64_t)lv.n_hblocks * np * kHDim * esz, 256);
    m.ids_off = off;
}

// The first n slots of cluster src (in src_arena) into cluster dst (in dst_arena).
cudaError_t copy_cluster_slots(const HostLevel& lv, uint8_t* dst_arena, const DevCluster& dst,
                               const uint8_t* src_arena, const DevCluster& src, uint32_t n, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const size_t esz = lv.u8 ? 1 : 4;
    cudaError_t e = cudaMemcpy2DAsync(dst_arena + dst.vert_off, (size_t)dst.n_pad * 4, src_arena + src.vert_off,
                                      (size_t)src.n_pad * 4, (size_t)n * 4, lv.n_vwords, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && lv.n_hblocks)
        e = cudaMemcpy2DAsync(dst_arena + dst.hor_off, (size_t)dst.n_pad * kHDim * esz, src_arena + src.hor_off,
                              (size_t)src.n_pad * kHDim * esz, (size_t)n * kHDim * esz, lv.n_hblocks,
                              cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dst_arena + dst.ids_off, src_arena + src.ids_off, (size_t)n * 4, cudaMemcpyDeviceToDevice,
                            st);
    return e;
}

// Slot `from` of a cluster copied over slot `to` (CopyEmbeddingInPDXLayout, cluster.hpp).
cudaError_t move_slot(const HostLevel& lv, uint8_t* arena, const DevCluster& m, uint32_t from, uint32_t to,
                      cudaStream_t st) {
    const size_t esz = lv.u8 ? 1 : 4;
    const size_t vp = (size_t)m.n_pad * 4, hr = (size_t)kHDim * esz, hp = (size_t)m.n_pad * hr;
    cudaError_t e = cudaMemcpy2DAsync(arena + m.vert_off + (size_t)to * 4, vp, arena + m.vert_off + (size_t)from * 4, vp,
                                      4, lv.n_vwords, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && lv.n_hblocks)
        e = cudaMemcpy2DAsync(arena + m.hor_off + (size_t)to * hr, hp, arena + m.hor_off + (size_t)from * hr, hp, hr,
                              lv.n_hblocks, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(arena + m.ids_off + (size_t)to * 4, arena + m.ids_off + (size_t)from * 4, 4,
                            cudaMemcpyDeviceToDevice, st);
    return e;
}

// One appended row: the cluster record at the time of the write, the slot, the row id and the
// row's index among the prepared rows of the batch.
struct RowWrite {
    DevCluster m;
    uint32_t slot, row_id, src, pad_;
};

// Prepared rows into their slots, one CTA per row: U8 rows quantized as QuantizeEmbedding
// (scalar.hpp:76-94: round half away from zero of (x - base) * scale, clamped to 0..255); vertical
// dims dimension-major (U8 in 4-byte interleaved groups, the tail group's padding stays zero),
// 64-dim horizontal blocks row-major, then the row id.
__global__ void write_rows_kernel(const float* __restrict__ rows, uint32_t d, uint32_t dv, int u8, float base,
                                  float scale, uint8_t* __restrict__ arena, const RowWrite* __restrict__ writes) {
    const RowWrite wr = writes[blockIdx.x];
    const DevCluster& m = wr.m;
    const uint64_t np = m.n_pad, slot = wr.slot;
    const float* row = rows + (uint64_t)wr.src * d;
    for (uint32_t j = threadIdx.x; j < d; j += blockDim.x) {
        const float x = row[j];
        if (u8) {
            const float r = roundf(__fmul_rn(__fsub_rn(x, base), scale));
            const uint8_t q = r > 255.0f ? (uint8_t)255 : (r < 0.0f ? (uint8_t)0 : (uint8_t)r);
            uint64_t off;
            if (j < dv) off = m.vert_off + ((uint64_t)(j >> 2) * np + slot) * 4 + (j & 3);
            else off = m.hor_off + ((uint64_t)((j - dv) / kHDim) * np + slot) * kHDim + (j - dv) % kHDim;
            arena[off] = q;
        } else {
            uint64_t off;
            if (j < dv) off = m.vert_off + ((uint64_t)j * np + slot) * 4;
            else off = m.hor_off + (((uint64_t)((j - dv) / kHDim) * np + slot) * kHDim + (j - dv) % kHDim) * 4;
            *reinterpret_cast<float*>(arena + off) = x;
        }
    }
    if (threadIdx.x == 0) *reinterpret_cast<uint32_t*>(arena + m.ids_off + slot * 4) = wr.row_id;
}

// Row-map entries (row, cluster, position) into the device maps of the filters.
__global__ void scatter_row_map_kernel(const uint32_t* __restrict__ tri, uint32_t n, uint32_t* __restrict__ rid_cluster,
                                       uint32_t* __restrict__ rid_pos) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t r = tri[3 * i];
        rid_cluster[r] = tri[3 * i + 1];
        rid_pos[r] = tri[3 * i + 2];
    }
}

void mark_cluster(pdxg_index* ix, uint32_t c) {
    Maint& M = *ix->maint;
    const MaintCluster& K = M.cl[c];
    DevCluster& m = ix->l1.meta[c];
    m.n = K.used;
    m.live = K.num_embeddings;
    ix->l1.n[c] = K.used;
    ix->l1.max_n = std::max(ix->l1.max_n, K.used);
    M.records_dirty = M.dirty = true;
}

void mark_tombstone(pdxg_index* ix, uint32_t c, uint32_t slot, bool on) {
    Maint& M = *ix->maint;
    const uint32_t w = ix->l1.meta[c].sel_word + (slot >> 5);
    const uint32_t bit = 1u << (slot & 31);
    M.tomb[w] = on ? (M.tomb[w] | bit) : (M.tomb[w] & ~bit);
    if (on) ++M.n_tomb;
    else --M.n_tomb;
    M.tomb_dirty = M.dirty = true;
}

void mark_row(pdxg_index* ix, uint32_t r) {
    ix->maint->dirty_rows.push_back(r);
    ix->maint->dirty = true;
    ix->reg_dirty = true;
}

// Device row maps large enough for `need` rows (moved when they grow).
int grow_row_maps(pdxg_index* ix, uint64_t need, cudaStream_t st) {
    Maint& M = *ix->maint;
    if (need <= M.rid_cap) return PDXG_OK;
    const uint64_t cap = std::max<uint64_t>({need, M.rid_cap * 2, 1024});
    uint32_t *c = nullptr, *p = nullptr;
    if (cudaMalloc(&c, cap * 4) != cudaSuccess || cudaMalloc(&p, cap * 4) != cudaSuccess) {
        cudaFree(c);
        return fail(PDXG_ERR_CUDA, "cannot grow the row id map");
    }
    const uint64_t have = M.rid_cap;
    if (have) {
        PDXG_CUDA(cudaMemcpyAsync(c, ix->d_rid_cluster, have * 4, cudaMemcpyDeviceToDevice, st));
        PDXG_CUDA(cudaMemcpyAsync(p, ix->d_rid_pos, have * 4, cudaMemcpyDeviceToDevice, st));
    }
    PDXG_CUDA(cudaStreamSynchronize(st));
    g_alloc_gen.fetch_add(1);
    cudaFree(ix->d_rid_cluster);
    cudaFree(ix->d_rid_pos);
    ix->d_rid_cluster = c;
    ix->d_rid_pos = p;
    M.rid_cap = cap;
    return PDXG_OK;
}

// Selection-bitmap words of every L1 cluster from its stride and the tombstone bitmap in that
// layout (after a cluster's stride changed); uploaded by the next flush.
int relayout_bitmaps(pdxg_index* ix) {
    Maint& M = *ix->maint;
    HostLevel& lv = ix->l1;
    uint32_t sel = 0;
    for (DevCluster& m : lv.meta) {
        m.sel_word = sel;
        sel += m.n_pad / 32;
    }
    lv.sel_words = sel;
    M.tomb.assign(sel, 0u);
    for (size_t c = 0; c < M.cl.size(); ++c)
        for (uint32_t t : M.cl[c].tombstones) M.tomb[lv.meta[c].sel_word + (t >> 5)] |= 1u << (t & 31);
    if (sel > M.tomb_cap) {
        uint32_t* t = nullptr;
        PDXG_CUDA(cudaMalloc(&t, (size_t)sel * 4));
        g_alloc_gen.fetch_add(1);
        cudaFree(M.d_tomb);
        M.d_tomb = t;
        M.tomb_cap = sel;
    }
    M.records_dirty = M.tomb_dirty = M.dirty = true;
    ix->reg_dirty = true;
    return PDXG_OK;
}

// Waits for the device once before the first change after a search: searches in flight read the
// slots, records and maps being changed.
int quiesce(pdxg_index* ix) {
    if (ix->maint && ix->maint->quiet) return PDXG_OK;
    PDXG_CUDA(cudaDeviceSynchronize());
    if (ix->maint) ix->maint->quiet = true;
    return PDXG_OK;
}

}  // namespace

// Uploads what Append / Delete changed (cluster records, tombstone bitmap, row maps) before a
// search launches; a no-op without pending changes. Stream-ordered: the copies and the row-map
// scatter run on the search's stream after the index stream's slot writes, and every later search
// on any stream waits for them through ev_flush. The host waits only before it rewrites the
// pinned row-map staging, for the previous copy out of it.
int pdxg::host::flush_maintenance(pdxg_index* ix, cudaStream_t st) {
    Maint* M = ix->maint.get();
    if (!M || M->in_op) return PDXG_OK;
    if (!st) st = ix->stream;
    M->quiet = false;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PDXG_CUDA(cudaStreamIsCapturing(st, &cs));
    const bool capturing = cs != cudaStreamCaptureStatusNone;
    if (M->dirty) {
        if (capturing)
            return fail(PDXG_ERR_INVALID_ARGUMENT,
                        "Append / Delete changes are pending: run one search outside stream capture first");
        if (!M->ev_flush) PDXG_CUDA(cudaEventCreateWithFlags(&M->ev_flush, cudaEventDisableTiming));
        if (!M->ev_stage) PDXG_CUDA(cudaEventCreateWithFlags(&M->ev_stage, cudaEventDisableTiming));
        if (st != ix->stream) {  // slot writes and moves on the index's stream
            PDXG_CUDA(cudaEventRecord(M->ev_flush, ix->stream));
            PDXG_CUDA(cudaStreamWaitEvent(st, M->ev_flush, 0));
        }
        HostLevel& lv = ix->l1;
        // pageable sources: staged by the driver before the call returns
        if (M->records_dirty)
            PDXG_CUDA(cudaMemcpyAsync(ix->d_cl1, lv.meta.data(), lv.meta.size() * sizeof(DevCluster),
                                      cudaMemcpyHostToDevice, st));
        if (M->tomb_dirty && lv.sel_words)
            PDXG_CUDA(cudaMemcpyAsync(M->d_tomb, M->tomb.data(), (size_t)lv.sel_words * 4,
                                      cudaMemcpyHostToDevice, st));
        std::vector<uint32_t>& rows = M->dirty_rows;
        for (size_t a = 0; a < rows.size(); a += kStageRows) {
            const uint32_t m = (uint32_t)std::min<size_t>(kStageRows, rows.size() - a);
            PDXG_CUDA(cudaEventSynchronize(M->ev_stage));  // the previous copy out of h_stage
            for (uint32_t i = 0; i < m; ++i) {
                const uint32_t r = rows[a + i];
                M->h_stage[3 * i] = r;
                M->h_stage[3 * i + 1] = ix->rid_cluster[r];
                M->h_stage[3 * i + 2] = ix->rid_pos[r];
            }
            PDXG_CUDA(cudaMemcpyAsync(M->d_stage, M->h_stage, (size_t)m * 12, cudaMemcpyHostToDevice, st));
            PDXG_CUDA(cudaEventRecord(M->ev_stage, st));
            scatter_row_map_kernel<<<(m + 255) / 256, 256, 0, st>>>(M->d_stage, m, ix->d_rid_cluster, ix->d_rid_pos);
            PDXG_CUDA(cudaGetLastError());
        }
        rows.clear();
        M->dirty = M->records_dirty = M->tomb_dirty = false;
        PDXG_CUDA(cudaEventRecord(M->ev_flush, st));
        return PDXG_OK;
    }
    // the last upload may still run on another stream; a capture relies on the host order of
    // pdxg_graph_launch instead (it waits on ev_flush outside the capture)
    if (M->ev_flush && !capturing) PDXG_CUDA(cudaStreamWaitEvent(st, M->ev_flush, 0));
    return PDXG_OK;
}

namespace {

int enable_maintenance(pdxg_index* ix, const char* op) {
    if (ix->maint) return PDXG_OK;
    if (!ix->tree)
        return fail(PDXG_ERR_UNSUPPORTED, std::string(op) + " is not implemented in PDXIndex. Use PDXTreeIndex instead.");
    HostLevel& lv = ix->l1;
    for (uint32_t c : ix->rid_cluster)
        if (c == kNoCluster) return fail(PDXG_ERR_UNSUPPORTED, "the index's row ids are not 0 .. n - 1");
    cudaStream_t st = ix->stream;
    auto M = std::make_unique<Maint>();
    const size_t n1 = lv.meta.size();
    M->cl.resize(n1);
    std::vector<DevCluster> meta(lv.meta);
    uint64_t off = 0;
    for (size_t c = 0; c < n1; ++c) {
        MaintCluster& K = M->cl[c];
        const uint32_t n = lv.n[c];
        K.num_embeddings = K.used = n;
        K.max_cap = std::max({lv.max_cap[c], n, 1u});
        K.min_cap = static_cast<uint32_t>(static_cast<float>(n) * 0.5f);  // MIN_CAPACITY_THRESHOLD
        K.indices.assign(lv.ids.begin() + lv.ids_start[c], lv.ids.begin() + lv.ids_start[c] + n);
        off = align_up(off, 256);
        place_cluster(lv, meta[c], off, slot_stride(K.max_cap));
        off += cluster_block_bytes(lv, meta[c].n_pad);
        M->live += n;
    }
    const uint64_t l1_bytes = align_up(off, 256);
    const uint64_t l0_bytes = ix->arena_bytes - ix->l0_start;
    const uint64_t used = l1_bytes + l0_bytes;
    const uint64_t cap = used + std::max<uint64_t>(used / 4, 64ull << 20);
    PDXG_CUDA(cudaDeviceSynchronize());  // searches in flight read the current arena
    if (cudaHostAlloc(&M->h_stage, (size_t)kStageRows * 12, cudaHostAllocDefault) != cudaSuccess ||
        cudaMalloc(&M->d_stage, (size_t)kStageRows * 12) != cudaSuccess) {
        free_maintenance(*M);
        return fail(PDXG_ERR_CUDA, "cannot allocate the maintenance staging buffers");
    }
    uint8_t* arena = nullptr;
    if (cudaMalloc(&arena, cap) != cudaSuccess) {
        free_maintenance(*M);
        return fail(PDXG_ERR_CUDA, "cannot allocate the arena at capacity strides");
    }
    auto undo = [&](cudaError_t e) {
        cudaFree(arena);
        free_maintenance(*M);
        return fail(PDXG_ERR_CUDA, std::string("maintenance layout: ") + cudaGetErrorString(e));
    };
    cudaError_t e = cudaMemsetAsync(arena, 0, cap, st);
    for (size_t c = 0; c < n1 && e == cudaSuccess; ++c)
        e = copy_cluster_slots(lv, arena, meta[c], ix->arena, lv.meta[c], lv.n[c], st);
    if (e == cudaSuccess && l0_bytes)
        e = cudaMemcpyAsync(arena + l1_bytes, ix->arena + ix->l0_start, l0_bytes, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return undo(e);
    std::vector<DevCluster> meta0(ix->l0.meta);
    for (DevCluster& m : meta0) {
        m.vert_off = m.vert_off - ix->l0_start + l1_bytes;
        m.hor_off = m.hor_off - ix->l0_start + l1_bytes;
        m.ids_off = m.ids_off - ix->l0_start + l1_bytes;
    }
    if (!meta0.empty())
        e = cudaMemcpy(ix->d_cl0, meta0.data(), meta0.size() * sizeof(DevCluster), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return undo(e);
    g_alloc_gen.fetch_add(1);
    cudaFree(ix->arena);
    ix->arena = arena;
    ix->arena_bytes = used;
    ix->l0_start = l1_bytes;
    ix->l0.meta = meta0;
    lv.meta = meta;
    for (size_t c = 0; c < n1; ++c) lv.max_cap[c] = M->cl[c].max_cap;
    M->arena_cap = cap;
    M->rid_cap = ix->rid_cluster.size();
    ix->maint = std::move(M);
    if (int rc = relayout_bitmaps(ix)) return rc;
    ix->maint->quiet = true;
    if (int rc = flush_maintenance(ix)) return rc;
    PDXG_CUDA(cudaStreamSynchronize(ix->stream));
    return PDXG_OK;
}

// The arena holds at least `need` bytes (the whole arena moves when it grows).
int reserve_arena(pdxg_index* ix, uint64_t need, cudaStream_t st) {
    Maint& M = *ix->maint;
    if (need <= M.arena_cap) return PDXG_OK;
    const uint64_t cap = std::max(need + (need >> 2), M.arena_cap * 2);
    uint8_t* arena = nullptr;
    PDXG_CUDA(cudaMalloc(&arena, cap));
    cudaError_t e = cudaMemsetAsync(arena, 0, cap, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(arena, ix->arena, ix->arena_bytes, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaFree(arena);
        return fail(PDXG_ERR_CUDA, std::string("cannot grow the arena: ") + cudaGetErrorString(e));
    }
    g_alloc_gen.fetch_add(1);
    cudaFree(ix->arena);
    ix->arena = arena;
    M.arena_cap = cap;
    return PDXG_OK;
}

// In place of SplitCluster (index.hpp:1314-1610): the cluster's capacity grows to
// max(uint32(1.3 used), 256) slots and its block moves to a fresh region of that stride.
int grow_cluster(pdxg_index* ix, uint32_t c, cudaStream_t st) {
    Maint& M = *ix->maint;
    MaintCluster& K = M.cl[c];
    HostLevel& lv = ix->l1;
    uint32_t cap = std::max<uint32_t>(static_cast<uint32_t>(static_cast<float>(K.used) * 1.3f), 256u);
    if (cap <= K.used) cap = K.used + 1;
    const uint32_t np = slot_stride(cap);
    K.max_cap = cap;
    lv.max_cap[c] = cap;
    ++M.grown;
    if (np == lv.meta[c].n_pad) return PDXG_OK;
    const uint64_t off = align_up(ix->arena_bytes, 256);
    const uint64_t bytes = cluster_block_bytes(lv, np);
    if (int rc = reserve_arena(ix, off + bytes, st)) return rc;
    DevCluster nm = lv.meta[c];
    place_cluster(lv, nm, off, np);
    PDXG_CUDA(copy_cluster_slots(lv, ix->arena, nm, ix->arena, lv.meta[c], K.used, st));
    lv.meta[c] = nm;
    ix->arena_bytes = off + bytes;
    return relayout_bitmaps(ix);
}

// Cluster::CompactCluster (cluster.hpp:260-294) with the row-id map updates of
// CheckClusterHealth / Save (index.hpp:1245-1248, 484-490).
int compact_cluster(pdxg_index* ix, uint32_t c, cudaStream_t st) {
    Maint& M = *ix->maint;
    MaintCluster& K = M.cl[c];
    if (K.tombstones.empty()) return PDXG_OK;
    const DevCluster m = ix->l1.meta[c];
    auto drain_tail = [&]() {
        while (K.used > 0 && K.tombstones.count(K.used - 1)) {
            K.tombstones.erase(K.used - 1);
            mark_tombstone(ix, c, K.used - 1, false);
            K.indices[K.used - 1] = 0;
            --K.used;
        }
    };
    drain_tail();
    while (!K.tombstones.empty()) {
        auto it = K.tombstones.begin();  // PopTombstone
        const uint32_t t = *it;
        K.tombstones.erase(it);
        mark_tombstone(ix, c, t, false);
        const uint32_t last = K.used - 1;
        PDXG_CUDA(move_slot(ix->l1, ix->arena, m, last, t, st));
        K.indices[t] = K.indices[last];
        ix->rid_pos[K.indices[t]] = t;
        mark_row(ix, K.indices[t]);
        K.indices[last] = 0;
        --K.used;
        drain_tail();
    }
    K.indices.resize(K.used);
    mark_cluster(ix, c);
    return PDXG_OK;
}

// CheckClusterHealth (index.hpp:1241-1255) with the split / merge substitutes above.
int check_cluster_health(pdxg_index* ix, uint32_t c, cudaStream_t st) {
    Maint& M = *ix->maint;
    MaintCluster& K = M.cl[c];
    if (K.used == K.max_cap) {
        if (K.num_embeddings < K.used) {
            ++M.compactions;
            return compact_cluster(ix, c, st);
        }
        return grow_cluster(ix, c, st);
    }
    if (K.num_embeddings <= K.min_cap) ++M.merges_deferred;
    return PDXG_OK;
}

constexpr uint32_t kAppendChunk = 4096;  // rows per rotation + top-level search launch

// Pinned / device staging for appends of up to `rows` rows at a time.
int ensure_append_staging(pdxg_index* ix, uint32_t rows) {
    Maint& M = *ix->maint;
    if (rows <= M.stage_rows) return PDXG_OK;
    if (M.h_rows) cudaFreeHost(M.h_rows);
    if (M.h_res) cudaFreeHost(M.h_res);
    if (M.h_writes) cudaFreeHost(M.h_writes);
    cudaFree(M.d_writes);
    M.h_rows = nullptr;
    M.h_res = nullptr;
    M.h_writes = nullptr;
    M.d_writes = nullptr;
    M.stage_rows = 0;
    void* hw = nullptr;
    if (cudaHostAlloc(&M.h_rows, (size_t)rows * ix->d * 4, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc(&M.h_res, ((size_t)rows * 2 + 1) * 4, cudaHostAllocDefault) != cudaSuccess ||
        cudaHostAlloc(&hw, (size_t)rows * sizeof(RowWrite), cudaHostAllocDefault) != cudaSuccess ||
        cudaMalloc(&M.d_writes, (size_t)rows * sizeof(RowWrite)) != cudaSuccess) {
        if (hw) cudaFreeHost(hw);
        return fail(PDXG_ERR_CUDA, "cannot allocate the append staging buffers");
    }
    M.h_writes = hw;
    M.stage_rows = rows;
    return PDXG_OK;
}

// Slot writes [from, to) of the current chunk, in order, on the index's stream.
int launch_row_writes(pdxg_index* ix, const float* d_rows, uint32_t from, uint32_t to) {
    if (to <= from) return PDXG_OK;
    Maint& M = *ix->maint;
    cudaStream_t st = ix->stream;
    RowWrite* hw = reinterpret_cast<RowWrite*>(M.h_writes);
    RowWrite* dw = reinterpret_cast<RowWrite*>(M.d_writes);
    PDXG_CUDA(cudaMemcpyAsync(dw + from, hw + from, (size_t)(to - from) * sizeof(RowWrite), cudaMemcpyHostToDevice, st));
    const HostLevel& lv = ix->l1;
    write_rows_kernel<<<to - from, 256, 0, st>>>(d_rows, ix->d, lv.dv, lv.u8 ? 1 : 0, ix->base, ix->scale, ix->arena,
                                                 dw + from);
    PDXG_CUDA(cudaGetLastError());
    return PDXG_OK;
}

// Device work that picks the clusters of m staged rows (M.h_rows): upload, NormalizeAndRotate
// (index.hpp:75-97, 592-594) unless the rows are prepared, and the nearest L1 cluster of every
// row (index.hpp:597-607): the top-level search with k = 1 over max(1, n_L0 / 8) meso clusters in
// the per-query top-level kernel; the clusters, their counts and the GEMM status land in M.h_res.
int enqueue_probe(pdxg_index* ix, uint32_t m, bool transformed, const float*& d_rows) {
    Maint& M = *ix->maint;
    Workspace& w = ix->ws;
    cudaStream_t st = ix->stream;
    const uint32_t d = ix->d;
    int rc;
    PDXG_CUDA(cudaMemcpyAsync(w.d_q, M.h_rows, (size_t)m * d * 4, cudaMemcpyHostToDevice, st));
    d_rows = w.d_q;
    if (!transformed) {
        if ((rc = prepare_dev(ix, w, w.d_q, m, w.d_rq, st, ix->append_normalize ? 1 : 0))) return rc;
        d_rows = w.d_rq;
    }
    const uint32_t top = std::max<uint32_t>(1u, (uint32_t)ix->l0.meta.size() / 8);
    Launch L;
    M.in_op = true;
    rc = plan_search(ix, m, 1, 0, false, L, 1, top);
    M.in_op = false;
    if (rc) return rc;
    L.p.queries = d_rows;
    const uint32_t mode = ix->top_mode;
    ix->top_mode = 2;
    rc = run_top_level(ix, w, d_rows, m, L, st);
    ix->top_mode = mode;
    if (rc) return rc;
    if (!L.p.q_order || L.p.q_order_stride != 1) return fail(PDXG_ERR_CAPACITY, "top-level kernel does not fit this index");
    PDXG_CUDA(cudaMemcpyAsync(M.h_res, L.p.q_order, (size_t)m * 4, cudaMemcpyDeviceToHost, st));
    PDXG_CUDA(cudaMemcpyAsync(M.h_res + m, L.p.q_order_count, (size_t)m * 4, cudaMemcpyDeviceToHost, st));
    if (w.d_gemm_err) PDXG_CUDA(cudaMemcpyAsync(M.h_res + 2 * m, w.d_gemm_err, 4, cudaMemcpyDeviceToHost, st));
    return PDXG_OK;
}

// enqueue_probe, then a synchronization and the GEMM status.
int probe_rows(pdxg_index* ix, uint32_t m, bool transformed, const float*& d_rows) {
    Maint& M = *ix->maint;
    Workspace& w = ix->ws;
    int rc;
    if ((rc = ensure_ws(ix, w, m, 1))) return rc;
    M.h_res[2 * m] = 0;
    if ((rc = enqueue_probe(ix, m, transformed, d_rows))) return rc;
    PDXG_CUDA(cudaStreamSynchronize(ix->stream));
    if (M.h_res[2 * m]) {
        cudaMemset(w.d_gemm_err, 0, sizeof(int));
        return fail(PDXG_ERR_CUDA, "tensor-core GEMM gave up waiting (code " + std::to_string(M.h_res[2 * m]) + ")");
    }
    return PDXG_OK;
}

// PDXTreeIndex::Append (index.hpp:580-616) for rows row0, row0 + 1, ... in order. A row's cluster
// comes from the top-level search over the meso level, which Append never changes, so one batched
// rotation and top-level search choose the same clusters as one call per row; slots, counters and
// health checks then run row by row on the host, and the slot writes are issued in that order
// (before any compaction or growth copies that follow them).
int append_rows(pdxg_index* ix, uint64_t row0, uint32_t n, const float* rows, bool transformed) {
    Maint& M = *ix->maint;
    if (row0 != ix->rid_cluster.size())
        return fail(PDXG_ERR_INVALID_ARGUMENT, "Append: row_id " + std::to_string(row0) +
                                                   " is not sequential (expected " +
                                                   std::to_string(ix->rid_cluster.size()) + ")");
    if (row0 + n >= 0xFFFFFFFFull) return fail(PDXG_ERR_CAPACITY, "Append: row ids are 32-bit");
    cudaStream_t st = ix->stream;
    const uint32_t d = ix->d;
    int rc;
    if ((rc = grow_row_maps(ix, row0 + n, st))) return rc;
    if ((rc = ensure_append_staging(ix, std::min(n, kAppendChunk)))) return rc;
    RowWrite* hw = reinterpret_cast<RowWrite*>(M.h_writes);
    for (uint32_t a = 0; a < n; a += kAppendChunk) {
        const uint32_t m = std::min(kAppendChunk, n - a);
        std::memcpy(M.h_rows, rows + (size_t)a * d, (size_t)m * d * 4);
        const float* d_rows = nullptr;
        if ((rc = probe_rows(ix, m, transformed, d_rows))) return rc;
        uint32_t* res = M.h_res;
        uint32_t issued = 0;
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t c = res[i];
            const uint64_t row_id = row0 + a + i;
            if (res[m + i] == 0 || c >= ix->l1.meta.size()) {
                launch_row_writes(ix, d_rows, issued, i);
                return fail(PDXG_ERR_FORMAT, "Append: no L1 cluster found");
            }
            // QuantizeAndAppend + Cluster::AppendEmbedding (index.hpp:885-896, cluster.hpp:121-146)
            MaintCluster& K = M.cl[c];
            uint32_t slot = K.used;
            bool reused = false;
            if (!K.tombstones.empty()) {
                auto it = K.tombstones.begin();  // PopTombstone
                slot = *it;
                K.tombstones.erase(it);
                reused = true;
            }
            if (slot >= K.max_cap) {
                if (reused) K.tombstones.insert(slot);
                launch_row_writes(ix, d_rows, issued, i);
                return fail(PDXG_ERR_CAPACITY, "AppendEmbedding: cluster buffer overflow (used_capacity=" +
                                                    std::to_string(K.used) + ", max_capacity=" +
                                                    std::to_string(K.max_cap) + ")");
            }
            hw[i] = RowWrite{ix->l1.meta[c], slot, (uint32_t)row_id, i, 0};
            if (reused) {
                mark_tombstone(ix, c, slot, false);
                K.indices[slot] = (uint32_t)row_id;
            } else {
                K.indices.push_back((uint32_t)row_id);
                ++K.used;
            }
            ++K.num_embeddings;
            ix->rid_cluster.push_back(c);
            ix->rid_pos.push_back(slot);
            mark_row(ix, (uint32_t)row_id);
            ++M.live;
            ++M.appends;
            mark_cluster(ix, c);
            if (K.used == K.max_cap) {  // compaction or growth moves slots: the writes go first
                if ((rc = launch_row_writes(ix, d_rows, issued, i + 1))) return rc;
                issued = i + 1;
            }
            if ((rc = check_cluster_health(ix, c, st))) return rc;
        }
        if ((rc = launch_row_writes(ix, d_rows, issued, m))) return rc;
    }
    return PDXG_OK;
}

// PDXTreeIndex::Delete (index.hpp:619-638).
int delete_impl(pdxg_index* ix, uint64_t row_id) {
    Maint& M = *ix->maint;
    if (row_id >= ix->rid_cluster.size())
        return fail(PDXG_ERR_INVALID_ARGUMENT, "Delete: row_id " + std::to_string(row_id) + " is not in the index");
    const uint32_t c = ix->rid_cluster[row_id];
    if (c == kNoCluster)
        return fail(PDXG_ERR_INVALID_ARGUMENT, "Delete: row_id " + std::to_string(row_id) + " was already deleted");
    const uint32_t slot = ix->rid_pos[row_id];
    MaintCluster& K = M.cl[c];
    // Cluster::DeleteEmbedding (cluster.hpp:148-154): the slot keeps its data and row id
    K.tombstones.insert(slot);
    --K.num_embeddings;
    mark_tombstone(ix, c, slot, true);
    ix->rid_cluster[row_id] = kNoCluster;
    ix->rid_pos[row_id] = kNoCluster;
    mark_row(ix, (uint32_t)row_id);
    --M.live;
    ++M.deletes;
    mark_cluster(ix, c);
    return check_cluster_health(ix, c, ix->stream);
}

}  // namespace

// Save compacts every cluster first (index.hpp:484-494) and writes the ids of the used slots.
int pdxg::host::maint_prepare_save(pdxg_index* ix) {
    if (!ix->maint) return PDXG_OK;
    if (int rc = quiesce(ix)) return rc;
    for (uint32_t c = 0; c < ix->maint->cl.size(); ++c)
        if (int rc = compact_cluster(ix, c, ix->stream)) return rc;
    if (int rc = flush_maintenance(ix)) return rc;
    PDXG_CUDA(cudaStreamSynchronize(ix->stream));  // Save reads the device state next
    HostLevel& lv = ix->l1;
    lv.total_vectors = 0;
    for (size_t c = 0; c < lv.meta.size(); ++c) {
        lv.ids_start[c] = lv.total_vectors;
        lv.total_vectors += ix->maint->cl[c].used;
    }
    lv.ids_start[lv.meta.size()] = lv.total_vectors;
    lv.ids.resize(lv.total_vectors);
    for (size_t c = 0; c < lv.meta.size(); ++c) {
        const auto& ind = ix->maint->cl[c].indices;
        std::copy(ind.begin(), ind.end(), lv.ids.begin() + lv.ids_start[c]);
    }
    g_alloc_gen.fetch_add(1);
    return PDXG_OK;
}

void pdxg::host::free_maintenance(Maint& M) {
    if (M.ev_flush) cudaEventDestroy(M.ev_flush);
    if (M.ev_stage) cudaEventDestroy(M.ev_stage);
    cudaFree(M.d_tomb);
    cudaFree(M.d_stage);
    cudaFree(M.d_writes);
    if (M.h_rows) cudaFreeHost(M.h_rows);
    if (M.h_res) cudaFreeHost(M.h_res);
    if (M.h_writes) cudaFreeHost(M.h_writes);
    if (M.h_stage) cudaFreeHost(M.h_stage);
    M = Maint{};
}

// Registered filters after Append / Delete moved slots: every bitmap rebuilt from its row ids in
// the current layout. Called with reg_mu held.
int pdxg::host::refresh_registered_filters(pdxg_index* ix) {
    if (!ix->reg_dirty) return PDXG_OK;
    const uint32_t words = ix->l1.sel_words;
    const uint32_t n1 = (uint32_t)ix->l1.meta.size();
    if (ix->reg_cap) {
        PDXG_CUDA(cudaDeviceSynchronize());  // batches in flight read the pool
        uint32_t* sel = nullptr;
        PDXG_CUDA(cudaMalloc(&sel, (size_t)ix->reg_cap * std::max(words, 1u) * 4));
        g_alloc_gen.fetch_add(1);
        cudaFree(ix->d_reg_sel);
        ix->d_reg_sel = sel;
        std::vector<uint32_t> bits(words), pass(n1);
        for (uint32_t slot = 0; slot < ix->reg_cap; ++slot) {
            if (!ix->reg_used[slot]) continue;
            std::fill(bits.begin(), bits.end(), 0u);
            std::fill(pass.begin(), pass.end(), 0u);
            const auto& rows = ix->reg_rows[slot];
            build_filter(ix, rows.data(), rows.size(), bits.data(), pass.data());
            PDXG_CUDA(cudaMemcpy(ix->d_reg_sel + (size_t)slot * words, bits.data(), (size_t)words * 4,
                                 cudaMemcpyHostToDevice));
            PDXG_CUDA(cudaMemcpy(ix->d_reg_pass + (size_t)slot * n1, pass.data(), (size_t)n1 * 4,
                                 cudaMemcpyHostToDevice));
        }
    }
    ix->reg_dirty = false;
    return PDXG_OK;
}

extern "C" {

int pdxg_append(pdxg_index* ix, uint64_t row_id, const float* embedding, uint32_t flags) {
    if (int rc = check_index(ix)) return rc;
    if (!embedding) return fail(PDXG_ERR_INVALID_ARGUMENT, "embedding is NULL");
    std::lock_guard<std::mutex> lock(ix->mu);
    std::lock_guard<std::mutex> reg_lock(ix->reg_mu);
    PDXG_CUDA(cudaSetDevice(ix->device));
    if (int rc = enable_maintenance(ix, "Append")) return rc;
    if (int rc = quiesce(ix)) return rc;
    g_alloc_gen.fetch_add(1);  // captured searches hold the old cluster records
    return append_rows(ix, row_id, 1, embedding, (flags & PDXG_QUERY_TRANSFORMED) != 0);
}

int pdxg_append_batch(pdxg_index* ix, uint64_t first_row_id, uint32_t n, const float* embeddings, uint32_t flags) {
    if (int rc = check_index(ix)) return rc;
    if (n && !embeddings) return fail(PDXG_ERR_INVALID_ARGUMENT, "embeddings is NULL");
    std::lock_guard<std::mutex> lock(ix->mu);
    std::lock_guard<std::mutex> reg_lock(ix->reg_mu);
    PDXG_CUDA(cudaSetDevice(ix->device));
    if (int rc = enable_maintenance(ix, "Append")) return rc;
    if (n == 0) return PDXG_OK;
    if (int rc = quiesce(ix)) return rc;
    g_alloc_gen.fetch_add(1);
    return append_rows(ix, first_row_id, n, embeddings, (flags & PDXG_QUERY_TRANSFORMED) != 0);
}

int pdxg_delete(pdxg_index* ix, uint64_t row_id) {
    if (int rc = check_index(ix)) return rc;
    std::lock_guard<std::mutex> lock(ix->mu);
    std::lock_guard<std::mutex> reg_lock(ix->reg_mu);
    PDXG_CUDA(cudaSetDevice(ix->device));
    if (int rc = enable_maintenance(ix, "Delete")) return rc;
    if (int rc = quiesce(ix)) return rc;
    g_alloc_gen.fetch_add(1);
    return delete_impl(ix, row_id);
}

int pdxg_set_append_normalization(pdxg_index* ix, int normalize) {
    if (int rc = check_index(ix)) return rc;
    ix->append_normalize = normalize != 0;
    return PDXG_OK;
}

int pdxg_maintenance_stats(const pdxg_index* ix, uint64_t out[6]) {
    if (int rc = check_index(ix)) return rc;
    if (!out) return fail(PDXG_ERR_INVALID_ARGUMENT, "out is NULL");
    const Maint* M = ix->maint.get();
    out[0] = M ? M->appends : 0;
    out[1] = M ? M->deletes : 0;
    out[2] = M ? M->compactions : 0;
    out[3] = M ? M->grown : 0;
    out[4] = M ? M->merges_deferred : 0;
    out[5] = M ? M->n_tomb : 0;
    return PDXG_OK;
}

}  // extern "C"
