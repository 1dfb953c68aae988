// Host side of the B200 PDX engine: index-file parsing, the device arena, workspaces and the
// C ABI declared in include/pdx_b200.h.
//
// Loading follows LoadPDXIndex / Restore (index.hpp:1736-1760, 242-267, 516-543) and
// IVF::Load / IVFTree::Load (ivf_wrapper.hpp:89-131, 218-312) for the byte layout, then
// re-lays every cluster into the device format described in pdxg_common.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <atomic>
#include <functional>
#include <mutex>
#include <string>
#include <unordered_set>
#include <vector>

#include "../../include/pdx_b200.h"
#include "pdxg_common.cuh"
#include "pdxg_gemm.cuh"
#include "pdxg_engine.cuh"

namespace pdxg {
cudaError_t launch_search(const SearchParams& p, bool u8, int threads, int grid, cudaStream_t st);
int search_occupancy(bool u8, int threads, size_t smem);
cudaError_t launch_prepare_queries(const float* q, uint32_t nq, uint32_t d, const float* rotation,
                                   bool normalize, float* norms_ws, float* out, cudaStream_t st);
cudaError_t launch_top_level(const SearchParams& p, int grid, cudaStream_t st, int threads);
int top_level_occupancy(size_t smem, int threads);
cudaError_t launch_top_level_tiled(const TopLevelParams& tp, uint32_t vtiles, int replay_warps,
                                   cudaStream_t st, const cudaEvent_t* ev);
cudaError_t launch_start_batched(const StartParams& sp, int grid, cudaStream_t st);
cudaError_t launch_scan(const ScanParams& sp, int bitmap_grid, cudaStream_t st, const cudaEvent_t* ev);
uint64_t scan_item_bound(uint32_t nq, uint32_t stride, uint32_t n1);
int scan_bitmap_occupancy();
uint32_t scan_queries_per_cta();
cudaError_t launch_row_sq(const float* x, uint32_t n, uint32_t d, float* out, cudaStream_t st);
size_t probe_select_smem(uint32_t d, uint32_t n1, uint32_t cand_cap, uint32_t sort_cap);
cudaError_t launch_probe_select(const ProbeParams& pp, cudaStream_t st);
cudaError_t launch_probe_exact(const ProbeParams& pp, cudaStream_t st);
int start_dist_occupancy(size_t smem);
size_t start_dist_smem(const DevLevel& lv);
uint64_t start_item_bound(uint32_t nq, uint32_t n1, uint32_t max_n);
}  // namespace pdxg

using namespace pdxg;
using namespace pdxg::host;

namespace pdxg {
namespace host {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

// Incremented whenever a device buffer is replaced: a captured search graph holds raw buffer
// pointers and refuses to launch once any of them may have moved.
std::atomic<uint64_t> g_alloc_gen{0};

}  // namespace host
}  // namespace pdxg

namespace {

// ADSamplingPruner::GetRatio (adsampling.hpp:147-157), same types and operation order.
float adsampling_ratio(const size_t& visited, uint32_t d, float eps0) {
    if (visited == 0) return 1;
    if (visited == d) return 1.0;
    return static_cast<float>(visited) / d * (1.0 + eps0 / std::sqrt(visited)) *
           (1.0 + eps0 / std::sqrt(visited));
}

void dimension_split(uint32_t d, uint32_t& h, uint32_t& v) {  // common.hpp:133-159
    float prop = 0.75f;
    if (d <= 128) prop = 0.25f;
    h = static_cast<uint32_t>(static_cast<float>(d) * prop);
    v = d - h;
    if (h % kHDim > 0) {
        h = ((h + kHDim / 2) / kHDim) * kHDim;
        v = d - h;
    }
    if (!v) {
        h = kHDim;
        v = d - h;
    }
    if (d <= kHDim) {
        h = 0;
        v = d;
    }
}

struct Cursor {
    const uint8_t* p;
    const uint8_t* end;
    bool ok = true;
    bool need(uint64_t n) {
        if (!ok || (uint64_t)(end - p) < n) ok = false;
        return ok;
    }
    uint32_t u32() {
        uint32_t v = 0;
        if (need(4)) {
            std::memcpy(&v, p, 4);
            p += 4;
        }
        return v;
    }
    uint8_t u8() {
        uint8_t v = 0;
        if (need(1)) v = *p++;
        return v;
    }
    float f32() {
        float v = 0;
        if (need(4)) {
            std::memcpy(&v, p, 4);
            p += 4;
        }
        return v;
    }
    const uint8_t* take(uint64_t n) {
        if (!need(n)) return nullptr;
        const uint8_t* r = p;
        p += n;
        return r;
    }
};

bool read_level(Cursor& c, HostLevel& lv, uint32_t ncl) {
    lv.fc.resize(ncl);
    for (uint32_t i = 0; i < ncl; ++i) {
        lv.fc[i].n = c.u32();
        lv.fc[i].max_cap = c.u32();
    }
    if (!c.ok) return false;
    const uint64_t esz = lv.u8 ? 1 : 4;
    for (uint32_t i = 0; i < ncl; ++i) {
        lv.fc[i].data = c.take((uint64_t)lv.fc[i].n * lv.d * esz);
        if (!c.ok) return false;
    }
    for (uint32_t i = 0; i < ncl; ++i) {
        lv.fc[i].ids = c.take((uint64_t)lv.fc[i].n * 4);
        if (!c.ok) return false;
    }
    return true;
}

// Byte layout of the level's clusters inside the arena, starting at `off`.
uint64_t plan_level(HostLevel& lv, uint64_t off) {
    lv.n_vwords = lv.u8 ? (lv.dv + 3) / 4 : lv.dv;
    lv.qw_hoff = (lv.n_vwords + 3) / 4 * 4;
    lv.n_hblocks = lv.dh / kHDim;
    const uint64_t esz = lv.u8 ? 1 : 4;
    const size_t ncl = lv.fc.size();
    lv.meta.resize(ncl);
    lv.n.resize(ncl);
    lv.max_cap.resize(ncl);
    lv.ids_start.resize(ncl + 1);
    lv.max_n = 0;
    lv.total_vectors = 0;
    uint32_t sel = 0;
    for (size_t i = 0; i < ncl; ++i) {
        const uint32_t n = lv.fc[i].n;
        const uint32_t n_pad = std::max<uint32_t>(32, (n + 31) / 32 * 32);
        DevCluster& m = lv.meta[i];
        m.n = n;
        m.n_pad = n_pad;
        m.sel_word = sel;
        m.live = n;
        sel += n_pad / 32;
        off = align_up(off, 256);
        m.vert_off = off;
        off += (uint64_t)lv.n_vwords * n_pad * 4;
        off = align_up(off, 256);
        m.hor_off = off;
        off += (uint64_t)lv.n_hblocks * n_pad * kHDim * esz;
        off = align_up(off, 256);
        m.ids_off = off;
        off += (uint64_t)n_pad * 4;
        lv.n[i] = n;
        lv.max_cap[i] = lv.fc[i].max_cap;
        lv.ids_start[i] = lv.total_vectors;
        lv.total_vectors += n;
        lv.max_n = std::max(lv.max_n, n);
    }
    lv.ids_start[ncl] = lv.total_vectors;
    lv.sel_words = sel;
    return align_up(off, 256);
}

// Fills the staging image of the arena for one level (compact file block -> device layout).
void fill_level(HostLevel& lv, uint8_t* img) {
    const uint32_t dv = lv.dv;
    lv.ids.resize(lv.total_vectors);
    for (size_t i = 0; i < lv.fc.size(); ++i) {
        const FileCluster& f = lv.fc[i];
        const DevCluster& m = lv.meta[i];
        const uint64_t n = f.n, np = m.n_pad;
        if (!lv.u8) {
            for (uint32_t j = 0; j < dv; ++j)
                std::memcpy(img + m.vert_off + (uint64_t)j * np * 4, f.data + (uint64_t)j * n * 4, n * 4);
            const uint8_t* hsrc = f.data + (uint64_t)dv * n * 4;
            for (uint32_t b = 0; b < lv.n_hblocks; ++b)
                std::memcpy(img + m.hor_off + (uint64_t)b * np * kHDim * 4,
                            hsrc + (uint64_t)b * n * kHDim * 4, n * kHDim * 4);
        } else {
            const uint32_t full = dv / 4, rem = dv % 4;
            for (uint32_t g = 0; g < full; ++g)
                std::memcpy(img + m.vert_off + (uint64_t)g * np * 4, f.data + (uint64_t)g * n * 4, n * 4);
            if (rem) {
                const uint8_t* src = f.data + (uint64_t)full * n * 4;
                uint8_t* dst = img + m.vert_off + (uint64_t)full * np * 4;
                for (uint64_t v = 0; v < n; ++v)
                    for (uint32_t t = 0; t < rem; ++t) dst[v * 4 + t] = src[v * rem + t];
            }
            const uint8_t* hsrc = f.data + (uint64_t)dv * n;
            for (uint32_t b = 0; b < lv.n_hblocks; ++b)
                std::memcpy(img + m.hor_off + (uint64_t)b * np * kHDim, hsrc + (uint64_t)b * n * kHDim,
                            n * kHDim);
        }
        std::memcpy(img + m.ids_off, f.ids, n * 4);
        std::memcpy(lv.ids.data() + lv.ids_start[i], f.ids, n * 4);
    }
}

void free_workspace(Workspace& w) {
    void* ptrs[] = {w.d_q, w.d_rq, w.d_norms, w.d_ids, w.d_dists, w.d_counts, w.d_queue, w.d_order,
                    w.d_sel, w.d_pass, w.d_filter_of, w.d_stats, w.d_top_order, w.d_top_off,
                    w.d_top_lists, w.d_top_count, w.d_top_vals, w.d_l1_order, w.d_l1_count,
                    w.d_st_cl, w.d_st_q, w.d_st_items, w.d_st_dist, w.d_pq_b16, w.d_pq_r16, w.d_pq_r8,
                    w.d_pq_r8s, w.d_pq_scores,
                    w.d_req, w.d_foff, w.d_rows, w.d_qhi, w.d_qlo, w.d_gemm_err, w.d_sc_qw, w.d_sc_q,
                    w.d_sc_heap, w.d_sc_cl, w.d_sc_vl, w.d_sc_items, w.d_sc_bm};
    for (void* q : ptrs) cudaFree(q);
    w = Workspace();
}



int upload_ratios(pdxg_index* ix) {
    std::vector<float> r(ix->d);
    for (size_t i = 0; i < ix->d; ++i) r[i] = adsampling_ratio(i, ix->d, ix->eps0);
    PDXG_CUDA(cudaMemcpy(ix->d_ratios, r.data(), sizeof(float) * ix->d, cudaMemcpyHostToDevice));
    return PDXG_OK;
}

DevLevel make_level(const HostLevel& lv, const DevCluster* dcl, const float* cent, float base,
                    float scale, const uint32_t* tomb = nullptr) {
    DevLevel L{};
    L.tomb = tomb;
    L.clusters = dcl;
    L.centroids = cent;
    L.nclusters = (uint32_t)lv.fc.size();
    L.d = lv.d;
    L.dv = lv.dv;
    L.dh = lv.dh;
    L.n_vwords = lv.n_vwords;
    L.qw_hoff = lv.qw_hoff;
    L.n_hblocks = lv.n_hblocks;
    L.max_n = lv.max_n;
    L.is_u8 = lv.u8 ? 1 : 0;
    L.sel_words = lv.sel_words;
    L.base = base;
    L.scale = scale;
    L.scale_sq = scale * scale;
    L.inv_scale_sq = 1.0f / L.scale_sq;
    return L;
}

void free_index(pdxg_index* ix) {
    if (!ix) return;
    cudaSetDevice(ix->device);
    cudaFree(ix->arena);
    cudaFree(ix->d_cl1);
    cudaFree(ix->d_cl0);
    cudaFree(ix->d_cent1);
    cudaFree(ix->d_cent0);
    cudaFree(ix->d_rot);
    cudaFree(ix->d_rot_hi);
    cudaFree(ix->d_rot_b16);
    cudaFree(ix->d_c1_b16);
    cudaFree(ix->d_c1_e4);
    cudaFree(ix->d_c1_e4s);
    cudaFree(ix->d_c1_sq);
    cudaFree(ix->d_rot_lo);
    cudaFree(ix->d_ratios);
    cudaFree(ix->d_rid_cluster);
    cudaFree(ix->d_rid_pos);
    cudaFree(ix->d_reg_sel);
    cudaFree(ix->d_reg_pass);
    if (ix->maint) free_maintenance(*ix->maint);
    for (cudaEvent_t e : ix->tev)
        if (e) cudaEventDestroy(e);
    free_workspace(ix->ws);
    if (ix->stream) cudaStreamDestroy(ix->stream);
    if (ix->copy_stream) cudaStreamDestroy(ix->copy_stream);
    for (cudaEvent_t e : ix->chunk_ev)
        if (e) cudaEventDestroy(e);
    delete ix;
}

int load_from_bytes(const uint8_t* buf, uint64_t size, int device, pdxg_index** out) {
    if (!out) return fail(PDXG_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    Cursor c{buf, buf + size};
    const uint8_t type = c.u8();
    if (!c.ok) return fail(PDXG_ERR_FORMAT, "index file is empty");
    if (type > 3) return fail(PDXG_ERR_FORMAT, "Unknown PDX index type: " + std::to_string(type));
    auto* ix = new pdxg_index();
    ix->device = device;
    ix->type = type;
    ix->tree = type >= 2;
    ix->u8 = (type == 1 || type == 3);
    ix->rot_rows = c.u32();
    ix->rot_cols = c.u32();
    const uint8_t* rot = c.take((uint64_t)ix->rot_rows * ix->rot_cols * 4);
    uint32_t d = c.u32(), dv = c.u32(), dh = c.u32();
    if (!c.ok) {
        free_index(ix);
        return fail(PDXG_ERR_FORMAT, "truncated index header");
    }
    uint32_t eh = 0, ev = 0;
    if (d == 0 || d > (uint32_t)kMaxDims) {
        free_index(ix);
        return fail(PDXG_ERR_FORMAT, "num_dimensions out of range: " + std::to_string(d));
    }
    dimension_split(d, eh, ev);
    if (dv != ev || dh != eh) {
        free_index(ix);
        return fail(PDXG_ERR_FORMAT, "dimension split in file does not match GetPDXDimensionSplit");
    }
    const bool dct = ix->rot_rows == 1 && ix->rot_cols == d;
    if (!dct && (ix->rot_rows != d || ix->rot_cols != d)) {
        free_index(ix);
        return fail(PDXG_ERR_FORMAT, "rotation matrix shape does not match num_dimensions");
    }
    ix->d = d;
    ix->dv = dv;
    ix->dh = dh;
    ix->file_rotation.resize((size_t)ix->rot_rows * ix->rot_cols);
    std::memcpy(ix->file_rotation.data(), rot, ix->file_rotation.size() * 4);
    ix->rotation.resize((size_t)d * d);
    if (dct) {
        // Files built with the FFTW rotation store a 1 x d sign vector (adsampling.hpp:192-246):
        // flip dimension j where it is negative, then the orthonormal DCT-II (FFTW_REDFT10 with
        // output 0 scaled by sqrt(1/(4d)), the others by sqrt(2/(4d))). The engine applies it as
        // the d x d matrix of y = x M: M[j][k] = s_j c_k cos(pi (2j + 1) k / (2d)), c_0 = sqrt(1/d),
        // c_k = sqrt(2/d), through the same rotation GEMMs.
        for (uint32_t j = 0; j < d; ++j) {
            const double sj = ix->file_rotation[j] < 0.0f ? -1.0 : 1.0;
            for (uint32_t k = 0; k < d; ++k) {
                const double ck = k == 0 ? std::sqrt(1.0 / d) : std::sqrt(2.0 / d);
                ix->rotation[(size_t)j * d + k] =
                    (float)(sj * ck * std::cos(M_PI * (2.0 * j + 1.0) * k / (2.0 * d)));
            }
        }
    } else {
        std::memcpy(ix->rotation.data(), rot, (size_t)d * d * 4);
    }
    for (HostLevel* lv : {&ix->l1, &ix->l0}) {
        lv->d = d;
        lv->dv = dv;
        lv->dh = dh;
    }
    ix->l1.u8 = ix->u8;
    ix->l0.u8 = false;
    bool ok;
    uint32_t n1, n0 = 0;
    if (!ix->tree) {
        n1 = c.u32();
        ok = c.ok && read_level(c, ix->l1, n1);
    } else {
        n1 = c.u32();
        n0 = c.u32();
        ok = c.ok && read_level(c, ix->l0, n0) && read_level(c, ix->l1, n1);
    }
    if (!ok) {
        free_index(ix);
        return fail(PDXG_ERR_FORMAT, "truncated index payload");
    }
    ix->normalized = c.u8() != 0;
    const uint32_t ncent = ix->tree ? n0 : n1;
    const uint8_t* cent = c.take((uint64_t)ncent * d * 4);
    if (ix->u8) {
        ix->base = c.f32();
        ix->scale = c.f32();
    }
    if (!c.ok) {
        free_index(ix);
        return fail(PDXG_ERR_FORMAT, "truncated index trailer");
    }
    if (ix->tree) {
        ix->l0.centroids.assign(reinterpret_cast<const float*>(cent),
                                reinterpret_cast<const float*>(cent) + (size_t)n0 * d);
        // L1 centroids are the vectors of the L0 clusters (IVFTree::Save does not store them).
        ix->l1.centroids.assign((size_t)n1 * d, 0.0f);
        for (const FileCluster& f : ix->l0.fc) {
            const float* data = reinterpret_cast<const float*>(f.data);
            for (uint32_t p = 0; p < f.n; ++p) {
                uint32_t id;
                std::memcpy(&id, f.ids + (size_t)p * 4, 4);
                if (id >= n1) {
                    free_index(ix);
                    return fail(PDXG_ERR_FORMAT, "meso cluster references an unknown cluster");
                }
                float* dst = ix->l1.centroids.data() + (size_t)id * d;
                for (uint32_t j = 0; j < dv; ++j) dst[j] = data[(size_t)j * f.n + p];
                for (uint32_t b = 0; b < dh; b += kHDim)
                    std::memcpy(dst + dv + b, data + (size_t)dv * f.n + (size_t)b * f.n + (size_t)p * kHDim,
                                kHDim * 4);
            }
        }
    } else {
        ix->l1.centroids.assign(reinterpret_cast<const float*>(cent),
                                reinterpret_cast<const float*>(cent) + (size_t)n1 * d);
    }

    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        free_index(ix);
        return fail(PDXG_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
    cudaDeviceGetAttribute(&ix->num_sms, cudaDevAttrMultiProcessorCount, device);
    int smem_optin = 0;
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    ix->max_smem = (size_t)smem_optin;

    uint64_t off = plan_level(ix->l1, 0);
    if (ix->tree) {
        for (DevCluster& m : ix->l0.meta) (void)m;
        const uint64_t start0 = off;
        ix->l0_start = start0;
        off = plan_level(ix->l0, start0);
    }
    ix->arena_bytes = off;
    std::vector<uint8_t> img(off, 0);
    fill_level(ix->l1, img.data());
    if (ix->tree) fill_level(ix->l0, img.data());

    int rc = PDXG_OK;
    auto step = [&](cudaError_t err, const char* what) {
        if (rc == PDXG_OK && err != cudaSuccess)
            rc = fail(PDXG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(err));
    };
    step(cudaStreamCreateWithFlags(&ix->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    step(cudaMalloc(&ix->arena, std::max<uint64_t>(off, 256)), "cudaMalloc(arena)");
    if (rc == PDXG_OK)
        step(cudaMemcpy(ix->arena, img.data(), off, cudaMemcpyHostToDevice), "cudaMemcpy(arena)");
    img.clear();
    img.shrink_to_fit();
    auto upload = [&](auto*& dptr, const auto& vec, const char* what) {
        using T = typename std::decay<decltype(vec)>::type::value_type;
        if (rc != PDXG_OK) return;
        step(cudaMalloc(&dptr, std::max<size_t>(vec.size(), 1) * sizeof(T)), what);
        if (rc == PDXG_OK && !vec.empty())
            step(cudaMemcpy(dptr, vec.data(), vec.size() * sizeof(T), cudaMemcpyHostToDevice), what);
    };
    upload(ix->d_cl1, ix->l1.meta, "clusters");
    upload(ix->d_cent1, ix->l1.centroids, "centroids");
    if (ix->tree) {
        upload(ix->d_cl0, ix->l0.meta, "meso clusters");
        upload(ix->d_cent0, ix->l0.centroids, "meso centroids");
    }
    upload(ix->d_rot, ix->rotation, "rotation");
    // Tensor-core rotation for d >= 512: its error (a fixed number of truncations per K = 32
    // stage) is below the FP32 SIMT GEMM's (which grows with sqrt(d)) from about that size on;
    // smaller dimensions keep the SIMT GEMM, the closer match to the reference's sgemm there.
    if (rc == PDXG_OK && d >= 512 && gemm_available() && gemm_shape_ok(kGemmTF32x3, d)) {
        // B operand of the tensor-core rotation: M^T (K-major) as TF32 hi / lo planes
        std::vector<float> th((size_t)d * d), tl((size_t)d * d);
        for (uint32_t i = 0; i < d; ++i)
            for (uint32_t j = 0; j < d; ++j) {
                const float x = ix->rotation[(size_t)i * d + j];
                uint32_t bits;
                std::memcpy(&bits, &x, 4);
                bits &= 0xFFFFE000u;
                float h;
                std::memcpy(&h, &bits, 4);
                th[(size_t)j * d + i] = h;
                tl[(size_t)j * d + i] = x - h;
            }
        upload(ix->d_rot_hi, th, "rotation planes");
        upload(ix->d_rot_lo, tl, "rotation planes");
        if (rc == PDXG_OK)
            ix->rot_tc = make_gemm_operand(ix->rot_op, kGemmTF32x3, ix->d_rot_hi, ix->d_rot_lo, d, d) == 0;
    }
    if (rc == PDXG_OK) step(cudaMalloc(&ix->d_ratios, sizeof(float) * d), "ratios");
    if (rc == PDXG_OK) rc = upload_ratios(ix);
    if (rc != PDXG_OK) {
        free_index(ix);
        return rc;
    }
    // row id -> (cluster, position), as BuildRowIdClusterMapping (index.hpp:421-433)
    const uint64_t total = ix->l1.total_vectors;
    ix->rid_cluster.assign(total, 0xFFFFFFFFu);
    ix->rid_pos.assign(total, 0);
    for (size_t ci = 0; ci < ix->l1.fc.size(); ++ci)
        for (uint32_t p = 0; p < ix->l1.n[ci]; ++p) {
            const uint32_t rid = ix->l1.ids[ix->l1.ids_start[ci] + p];
            if (rid < total) {
                ix->rid_cluster[rid] = (uint32_t)ci;
                ix->rid_pos[rid] = p;
            }
        }
    if (cudaMalloc(&ix->d_rid_cluster, std::max<size_t>(total, 1) * 4) != cudaSuccess ||
        cudaMalloc(&ix->d_rid_pos, std::max<size_t>(total, 1) * 4) != cudaSuccess ||
        (total && cudaMemcpy(ix->d_rid_cluster, ix->rid_cluster.data(), total * 4, cudaMemcpyHostToDevice) != cudaSuccess) ||
        (total && cudaMemcpy(ix->d_rid_pos, ix->rid_pos.data(), total * 4, cudaMemcpyHostToDevice) != cudaSuccess)) {
        free_index(ix);
        return fail(PDXG_ERR_CUDA, "cannot upload the row id map");
    }
    // file buffer pointers are not kept
    for (HostLevel* lv : {&ix->l1, &ix->l0})
        for (FileCluster& f : lv->fc) {
            f.data = nullptr;
            f.ids = nullptr;
        }
    *out = ix;
    return PDXG_OK;
}

}  // namespace

namespace pdxg {
namespace host {

int plan_search(pdxg_index* ix, uint32_t nq, uint32_t k, uint32_t n_order, bool any_filter,
                Launch& L, uint32_t np_flat_max, uint32_t top_max, bool probe_ahead, cudaStream_t st) {
    if (int rc = flush_maintenance(ix, st)) return rc;
    SearchParams& p = L.p;
    p.arena = ix->arena;
    p.l1 = make_level(ix->l1, ix->d_cl1, ix->d_cent1, ix->base, ix->scale,
                      (ix->maint && ix->maint->n_tomb) ? ix->maint->d_tomb : nullptr);
    p.is_tree = ix->tree ? 1 : 0;
    if (ix->tree) p.l0 = make_level(ix->l0, ix->d_cl0, ix->d_cent0, 0.0f, 1.0f);
    p.ratios = ix->d_ratios;
    p.nq = nq;
    p.k = k;
    const uint32_t n1 = p.l1.nclusters;
    // flat: searcher.hpp:614-616; tree: index.hpp:546-556
    uint32_t np_flat = (ix->nprobe == 0 || ix->nprobe > n1) ? n1 : ix->nprobe;
    uint32_t top = 0;
    if (ix->tree) {
        top = p.l0.nclusters;
        const uint32_t l1np = ix->nprobe == 0 ? n1 : ix->nprobe;
        if (l1np < n1 / 2) top /= 2;
    }
    // per-query batches (pdxg_search_requests) size everything for their largest values
    if (np_flat_max != 0xFFFFFFFFu) np_flat = np_flat_max;
    if (top_max != 0xFFFFFFFFu) top = top_max;
    p.nprobe = np_flat;
    p.top_nprobe = top;
    p.n_order = n_order;
    const uint32_t d = ix->d;
    // the heap region also holds the sorted probe list of an in-kernel probe (flat: nprobe,
    // tree L0: top entries); orders computed ahead are read in place
    const uint32_t heap_cap = probe_ahead ? next_pow2(std::max(k, 1u)) : next_pow2(std::max({k, np_flat, top, 1u}));
    uint32_t work = std::max({p.l1.max_n, heap_cap, 32u});
    // an in-kernel probe keeps one entry per centroid (not needed when the visit orders are
    // computed ahead of the scan)
    if ((!ix->tree && !probe_ahead) || any_filter) work = std::max(work, n1);
    if (ix->tree) work = std::max({work, p.l0.max_n, p.l0.nclusters});
    // dist/pos need max cluster size (or centroid count for a probe); sorts viewing the region as
    // u64 need at most heap_cap (a power of two) entries, so no power-of-two padding here
    const uint32_t work_cap = (work + 31) / 32 * 32;
    const uint32_t order_cap = probe_ahead ? std::max(n_order, 1u) : std::max({np_flat, top, n_order, 1u});
    uint32_t off = 0;
    p.smem_qf = off;
    off += (uint32_t)align_up((uint64_t)d * 4, 16);
    p.smem_qw = off;
    if (ix->u8) off += (uint32_t)align_up((uint64_t)(p.l1.qw_hoff + p.l1.n_hblocks * 16) * 4, 16);
    p.smem_work = off;
    off += work_cap * 8;
    p.smem_heap = off;
    off += heap_cap * 8;
    p.smem_order = off;
    off += (uint32_t)align_up((uint64_t)order_cap * 4, 16);
    p.smem_bits = off;
    p.bits_cap = work_cap / 32;
    off += (uint32_t)align_up((uint64_t)p.bits_cap * 8, 16);
    p.smem_total = off;
    p.work_cap = work_cap;
    p.heap_cap = heap_cap;
    p.order_cap = order_cap;
    if ((size_t)off + 2048 > ix->max_smem)
        return fail(PDXG_ERR_CAPACITY, "per-query shared memory (" + std::to_string(off) +
                                           " B) exceeds the device limit; cluster, k or nprobe too large");
    L.u8 = ix->u8;
    int threads = (int)ix->threads;
    if (threads == 0) threads = 128;  // measured fastest on B200 (IVF2 SQ8 1M x 1024)
    L.threads = threads;
    const int occ = search_occupancy(L.u8, threads, off);
    if (occ <= 0) return fail(PDXG_ERR_CAPACITY, "search kernel cannot be resident with this configuration");
    L.grid = (int)std::min<uint64_t>(nq, (uint64_t)occ * ix->num_sms);
    return PDXG_OK;
}


int ensure_ws(pdxg_index* ix, Workspace& w, uint32_t nq, uint32_t k) {
    uint64_t cap;
    if (nq > w.q_cap || !w.d_rq) {
        cap = 0;
        int rc = dev_grow(w.d_rq, cap, (uint64_t)nq * ix->d);
        if (rc) return rc;
        cap = 0;
        if ((rc = dev_grow(w.d_norms, cap, nq))) return rc;
        cap = 0;
        if ((rc = dev_grow(w.d_counts, cap, nq))) return rc;
        cap = 0;
        if ((rc = dev_grow(w.d_q, cap, (uint64_t)nq * ix->d))) return rc;
        w.q_cap = nq;
        w.k_cap = 0;
    }
    if ((uint64_t)nq * k > (uint64_t)w.q_cap * w.k_cap || !w.d_ids) {
        cap = 0;
        int rc = dev_grow(w.d_ids, cap, (uint64_t)w.q_cap * k);
        if (rc) return rc;
        cap = 0;
        if ((rc = dev_grow(w.d_dists, cap, (uint64_t)w.q_cap * k))) return rc;
        w.k_cap = k;
    }
    if (!w.d_queue) PDXG_CUDA(cudaMalloc(&w.d_queue, 4 * sizeof(uint32_t)));  // search, -, top
    return PDXG_OK;
}

}  // namespace host
}  // namespace pdxg

namespace {

// NormalizeQuery + rotation of nq device queries into `out` (ADSamplingPruner::PreprocessQuery,
// adsampling.hpp:100-113): TF32x3 tensor-core GEMM when available, else the FP32 SIMT GEMM.
}  // namespace

namespace pdxg {
namespace host {

bool rotation_on_tensor_cores(const pdxg_index* ix, uint32_t nq) {
    // up to 8 rows (a single query, an appended row): the FP32 GEMV has the shorter latency
    return ix->rot_tc && ix->rot_mode == 0 && nq > 8;
}

int rotate_tf32x3(pdxg_index* ix, const float* q, uint32_t nq, bool norm, float* hi, float* lo, int* err,
                  float* out, cudaStream_t st) {
    const uint32_t d = ix->d;
    PDXG_CUDA(launch_split_rows(q, nq, d, norm, hi, lo, st));
    GemmOperand a;
    if (make_gemm_operand(a, kGemmTF32x3, hi, lo, nq, d) != 0)
        return fail(PDXG_ERR_CUDA, "cannot encode the query tensor maps");
    GemmArgs g{};
    g.M = nq;
    g.N = d;
    g.K = d;
    g.out = out;
    g.ldo = d;
    g.error = err;
    PDXG_CUDA(launch_gemm(a, ix->rot_op, kEpiStore, g, st));
    return PDXG_OK;
}

// normalize: -1 follows the index's is_normalized flag (queries), 0 / 1 force it (appended rows
// follow PDXIndexConfig::normalize).
int prepare_dev(pdxg_index* ix, Workspace& w, const float* q, uint32_t nq, float* out, cudaStream_t st,
                int normalize, bool allow_tc) {
    if (nq == 0) return PDXG_OK;
    const uint32_t d = ix->d;
    const bool norm = normalize < 0 ? ix->normalized : normalize != 0;
    if (allow_tc && rotation_on_tensor_cores(ix, nq)) {
        int rc;
        if ((rc = dev_grow(w.d_qhi, w.qhi_cap, (uint64_t)nq * d))) return rc;
        if ((rc = dev_grow(w.d_qlo, w.qlo_cap, (uint64_t)nq * d))) return rc;
        if (!w.d_gemm_err) {
            PDXG_CUDA(cudaMalloc(&w.d_gemm_err, sizeof(int)));
            PDXG_CUDA(cudaMemsetAsync(w.d_gemm_err, 0, sizeof(int), st));
        }
        return rotate_tf32x3(ix, q, nq, norm, w.d_qhi, w.d_qlo, w.d_gemm_err, out, st);
    }
    PDXG_CUDA(launch_prepare_queries(q, nq, d, ix->d_rot, norm, w.d_norms, out, st));
    return PDXG_OK;
}

}  // namespace host
}  // namespace pdxg

namespace {

// After a synchronization: fails if a tensor-core GEMM of this workspace gave up a wait.
int check_gemm_error(Workspace& w) {
    if (!w.d_gemm_err) return PDXG_OK;
    int h = 0;
    PDXG_CUDA(cudaMemcpy(&h, w.d_gemm_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h == 0) return PDXG_OK;
    cudaMemset(w.d_gemm_err, 0, sizeof(int));
    return fail(PDXG_ERR_CUDA, "tensor-core GEMM gave up waiting (code " + std::to_string(h) + ")");
}

// Warmup checkpoints of the top-level search: the cumulative DIMENSIONS_FETCHING_SIZES steps
// from 0, capped at dv (searcher.hpp:374-435, common.hpp:47-49).
uint32_t warmup_checkpoints(uint32_t dv, uint32_t* cp, uint32_t cap) {
    static const uint32_t fetch[kNumFetchSizes] = {16, 16, 32, 32, 32, 32, 64, 64, 64, 64,
                                                   128, 128, 128, 128, 256, 256, 512, 1024, 2048, 16384};
    uint32_t cur = 0, n = 0;
    while (cur < dv) {
        uint32_t last = cur + fetch[n < kNumFetchSizes ? n : kNumFetchSizes - 1];
        if (last > dv) last = dv;
        if (n >= cap) return cap + 1;
        cp[n++] = last;
        cur = last;
    }
    return n;
}

// Tiled top level (pdxg_toplevel.cu). Returns PDXG_OK with L.p.q_order set when it ran,
// PDXG_OK with L.p.q_order unset when this index or batch does not fit its limits (the caller
// then uses the per-query form), or an error.
int run_top_level_tiled(pdxg_index* ix, Workspace& w, const float* qp, uint32_t nq, Launch& L, cudaStream_t st,
                        uint32_t q_offset = 0, bool timed = false) {
    const DevLevel& l0 = L.p.l0;
    const HostLevel& h0 = ix->l0;
    if (l0.d % 4 || l0.dv % 4 || l0.dv == 0 || ((uintptr_t)qp & 15) || h0.fc.empty()) return PDXG_OK;
    TopLevelParams tp{};
    tp.ncp = warmup_checkpoints(l0.dv, tp.cp, kMaxCheckpoints);
    if (tp.ncp > (uint32_t)kMaxCheckpoints) return PDXG_OK;
    const uint32_t k1 = L.p.nprobe, top = L.p.top_nprobe, nL0 = l0.nclusters;
    if (top == 0 || k1 == 0 || nL0 > 65535 || (uint64_t)nq * top >= (1ull << 32)) return PDXG_OK;
    tp.nvals = tp.ncp + l0.n_hblocks;
    // partials of one query: its `top` largest meso clusters at most
    std::vector<uint32_t> strides(nL0);
    for (uint32_t i = 0; i < nL0; ++i) strides[i] = (h0.n[i] + 3u) & ~3u;
    std::sort(strides.begin(), strides.end(), std::greater<uint32_t>());
    uint64_t per_query = 0;
    for (uint32_t i = 0; i < std::min(top, nL0); ++i) per_query += (uint64_t)strides[i] * tp.nvals;
    if (per_query >= (1ull << 31)) return PDXG_OK;
    const uint64_t vals_bytes = (uint64_t)nq * per_query * 4;
    if (vals_bytes + (uint64_t)nL0 * nq * 4 > (8ull << 30)) return PDXG_OK;
    const uint32_t max_n0 = std::max(l0.max_n, 1u);
    if (max_n0 > (1u << 20)) return PDXG_OK;
    tp.probe_q = 8;
    auto probe_bytes = [&](uint32_t qn) {
        return align_up((uint64_t)qn * l0.d * 4, 16) + (uint64_t)qn * next_pow2(nL0) * 8;
    };
    while (tp.probe_q > 1 && probe_bytes(tp.probe_q) + 1024 > ix->max_smem) tp.probe_q >>= 1;
    if (probe_bytes(tp.probe_q) + 1024 > ix->max_smem) return PDXG_OK;
    tp.probe_smem = (uint32_t)probe_bytes(tp.probe_q);
    tp.r_heap_cap = next_pow2(std::max(k1, 2u));
    tp.r_work_cap = (max_n0 + 31) / 32 * 32;
    tp.r_sort_cap = std::max({next_pow2(max_n0), tp.r_heap_cap, 2u});
    tp.r_pre_floats = (uint32_t)((uint64_t)tp.nvals * ((max_n0 + 3) & ~3u));
    const uint64_t wb = align_up((uint64_t)tp.r_sort_cap * 8 + (uint64_t)tp.r_pre_floats * 8 +
                                 (uint64_t)tp.r_heap_cap * 8 + (uint64_t)tp.r_work_cap * 8 +
                                 (uint64_t)top * 8, 16);
    const uint64_t ratio_bytes = align_up((uint64_t)l0.d * 4, 16);
    int warps = 4;
    while (warps > 1 && ratio_bytes + (uint64_t)warps * wb + 1024 > ix->max_smem) warps >>= 1;
    if (ratio_bytes + (uint64_t)warps * wb + 1024 > ix->max_smem) return PDXG_OK;
    tp.r_warp_bytes = (uint32_t)wb;

    int rc;
    if ((rc = dev_grow(w.d_top_order, w.top_order_cap, (uint64_t)nq * top))) return rc;
    if ((rc = dev_grow(w.d_top_off, w.top_off_cap, (uint64_t)nq * top))) return rc;
    if ((rc = dev_grow(w.d_top_lists, w.top_lists_cap, (uint64_t)nL0 * nq))) return rc;
    if ((rc = dev_grow(w.d_top_count, w.top_count_cap, (uint64_t)nL0 + nq))) return rc;
    if ((rc = dev_grow(w.d_top_vals, w.top_vals_cap, std::max<uint64_t>((uint64_t)nq * per_query, 4)))) return rc;
    if ((rc = dev_grow(w.d_l1_order, w.l1_order_cap, (uint64_t)(q_offset + nq) * k1))) return rc;
    if ((rc = dev_grow(w.d_l1_count, w.l1_count_cap, q_offset + nq))) return rc;
    tp.arena = ix->arena;
    tp.l0 = l0;
    tp.ratios = L.p.ratios;
    tp.queries = qp;
    tp.nq = nq;
    tp.top = top;
    tp.k1 = k1;
    tp.q_nprobe = L.p.q_nprobe;
    tp.q_top = L.p.q_top;
    tp.filter_of = L.p.filter_of;
    tp.order = w.d_top_order;
    tp.off = w.d_top_off;
    tp.list_count = w.d_top_count;
    tp.ntop = w.d_top_count + nL0;
    tp.lists = w.d_top_lists;
    tp.vals = w.d_top_vals;
    tp.per_query = per_query;
    tp.l1_order = w.d_l1_order + (uint64_t)q_offset * k1;
    tp.l1_count = w.d_l1_count + q_offset;
    tp.stats = L.p.stats;
    const uint32_t vtiles = (max_n0 + 31) / 32;
    tp.r_smem = (uint32_t)(ratio_bytes + (uint64_t)warps * wb);
    PDXG_CUDA(launch_top_level_tiled(tp, vtiles, warps, st, timed ? ix->tev + 8 : nullptr));
    ix->tev_tiled = timed;
    L.top_launches = 3;
    L.p.q_order = w.d_l1_order;
    L.p.q_order_count = w.d_l1_count;
    L.p.q_order_stride = k1;
    return PDXG_OK;
}

// Tree top level as its own launch: the tiled form (mode 3, and mode 0 when it fits), else
// small per-query CTAs (top_level_kernel; mode 2, and mode 0 otherwise). On success the search
// kernel reads each query's L1 order from L.p.q_order; in mode 1 the search kernel runs the
// top level itself.
}  // namespace

namespace pdxg {
namespace host {

int run_top_level(pdxg_index* ix, Workspace& w, const float* qp, uint32_t nq, Launch& L, cudaStream_t st,
                  uint32_t q_offset, bool timed) {
    L.p.q_order = nullptr;
    L.p.q_order_count = nullptr;
    ix->tev_tiled = false;
    if (ix->top_mode == 1) return PDXG_OK;
    // auto mode: a few queries (a single search, an Append) take the one-launch per-query
    // kernel, batches the tiled form
    const bool small = ix->top_mode == 0 && nq <= 32;
    if ((ix->top_mode == 0 && !small) || ix->top_mode == 3) {
        int rc = run_top_level_tiled(ix, w, qp, nq, L, st, q_offset, timed);
        if (rc || L.p.q_order) return rc;
        if (ix->top_mode == 3)
            return fail(PDXG_ERR_CAPACITY, "tiled top level cannot run on this index or batch "
                                           "(needs d and d_v multiples of 4, 16-byte aligned queries)");
    }
    SearchParams tp = L.p;
    tp.queries = qp;
    const uint32_t k1 = L.p.nprobe;
    const uint32_t top = L.p.top_nprobe;
    // shared memory of one top-level CTA: query, work (meso clusters / probe), heap, order
    const uint32_t heap_cap = next_pow2(std::max({k1, top, 1u}));
    uint32_t work = std::max({tp.l0.max_n, tp.l0.nclusters, heap_cap, 32u});
    const uint32_t work_cap = (work + 31) / 32 * 32;
    uint32_t off = 0;
    tp.smem_qf = 0;
    off += (uint32_t)align_up((uint64_t)ix->d * 4, 16);
    tp.smem_qw = off;
    tp.smem_work = off;
    off += work_cap * 8;
    tp.smem_heap = off;
    off += heap_cap * 8;
    tp.smem_order = off;
    off += (uint32_t)align_up((uint64_t)std::max(top, 1u) * 4, 16);
    tp.smem_bits = off;
    tp.bits_cap = work_cap / 32;
    off += (uint32_t)align_up((uint64_t)tp.bits_cap * 8, 16);
    tp.smem_total = off;
    tp.work_cap = work_cap;
    tp.heap_cap = heap_cap;
    tp.order_cap = top;
    if ((size_t)off + 2048 > ix->max_smem) {
        if (ix->top_mode == 2) return fail(PDXG_ERR_CAPACITY, "top-level kernel does not fit in shared memory");
        return PDXG_OK;
    }
    int rc;
    if ((rc = dev_grow(w.d_l1_order, w.l1_order_cap, (uint64_t)(q_offset + nq) * k1))) return rc;
    if ((rc = dev_grow(w.d_l1_count, w.l1_count_cap, q_offset + nq))) return rc;
    tp.q_order = w.d_l1_order + (uint64_t)q_offset * k1;
    tp.q_order_count = w.d_l1_count + q_offset;
    tp.q_order_stride = k1;
    tp.queue = w.d_queue + 2;
    PDXG_CUDA(cudaMemsetAsync(tp.queue, 0, sizeof(uint32_t), st));
    const int threads = nq <= (uint32_t)ix->num_sms ? 256 : 64;
    const int occ = top_level_occupancy(off, threads);
    if (occ <= 0) return fail(PDXG_ERR_CAPACITY, "top-level kernel cannot be resident");
    const int grid = (int)std::min<uint64_t>(nq, (uint64_t)occ * ix->num_sms);
    PDXG_CUDA(launch_top_level(tp, grid, st, threads));
    L.top_launches = 1;
    L.p.q_order = w.d_l1_order;
    L.p.q_order_count = w.d_l1_count;
    L.p.q_order_stride = k1;
    return PDXG_OK;
}

}  // namespace host
}  // namespace pdxg

namespace {

uint16_t bf16_rne(float x) {
    uint32_t b;
    std::memcpy(&b, &x, 4);
    return (uint16_t)((b + 0x7FFFu + ((b >> 16) & 1u)) >> 16);
}

// Whether the reduced-precision probe can run on this index (tensor cores, d a multiple of
// 16, candidate arrays within shared memory).
bool probe_gemm_ok(const pdxg_index* ix) {
    const uint32_t n1 = (uint32_t)ix->l1.fc.size();
    return gemm_available() && ix->d % 16 == 0 && gemm_shape_ok(kGemmBF16, ix->d) && gemm_shape_ok(kGemmE4M3, ix->d) &&
           probe_select_smem(ix->d, n1, (n1 + 3) & ~3u, next_pow2(n1)) + 2048 <= ix->max_smem;
}

int prepare_probe_gemm(pdxg_index* ix, cudaStream_t st) {
    if (ix->pp_ready) return PDXG_OK;
    const uint32_t d = ix->d, n1 = (uint32_t)ix->l1.fc.size();
    std::vector<uint16_t> rt((size_t)d * d);
    for (uint32_t i = 0; i < d; ++i)
        for (uint32_t j = 0; j < d; ++j) rt[(size_t)j * d + i] = bf16_rne(ix->rotation[(size_t)i * d + j]);
    PDXG_CUDA(cudaMalloc(&ix->d_rot_b16, rt.size() * 2));
    PDXG_CUDA(cudaMemcpy(ix->d_rot_b16, rt.data(), rt.size() * 2, cudaMemcpyHostToDevice));
    PDXG_CUDA(cudaMalloc(&ix->d_c1_b16, (size_t)n1 * d * 2));
    PDXG_CUDA(cudaMalloc(&ix->d_c1_e4, (size_t)n1 * d));
    PDXG_CUDA(cudaMalloc(&ix->d_c1_e4s, (size_t)n1 * 4));
    PDXG_CUDA(cudaMalloc(&ix->d_c1_sq, (size_t)n1 * 4));
    PDXG_CUDA(launch_bf16_rows(ix->d_cent1, n1, d, false, ix->d_c1_b16, st));
    PDXG_CUDA(launch_e4m3_rows(ix->d_cent1, n1, d, ix->d_c1_e4, ix->d_c1_e4s, st));
    PDXG_CUDA(launch_row_sq(ix->d_cent1, n1, d, ix->d_c1_sq, st));
    if (make_gemm_operand(ix->rot_op16, kGemmBF16, ix->d_rot_b16, nullptr, d, d) != 0 ||
        make_gemm_operand(ix->c1_op16, kGemmBF16, ix->d_c1_b16, nullptr, n1, d) != 0 ||
        make_gemm_operand(ix->c1_op8, kGemmE4M3, ix->d_c1_e4, nullptr, n1, d) != 0)
        return fail(PDXG_ERR_CUDA, "cannot encode the probe tensor maps");
    ix->pp_ready = true;
    return PDXG_OK;
}

// Reduced-precision probe (probe modes 1 and 2): BF16 rotation of the raw queries into w.d_rq
// (skipped for transformed queries), tensor-core centroid scores, widened list, FP32 rescore.
// Sets L.p.queries to the rotated queries and L.p.q_order to the visit orders.
int run_probe_gemm(pdxg_index* ix, Workspace& w, const float* q, uint32_t nq, bool transformed, Launch& L,
                   cudaStream_t st) {
    const uint32_t d = ix->d, n1 = L.p.l1.nclusters;
    int rc;
    if ((rc = prepare_probe_gemm(ix, st))) return rc;
    if (!w.d_gemm_err) {
        PDXG_CUDA(cudaMalloc(&w.d_gemm_err, sizeof(int)));
        PDXG_CUDA(cudaMemsetAsync(w.d_gemm_err, 0, sizeof(int), st));
    }
    if ((rc = dev_grow(w.d_pq_r16, w.pq_r16_cap, (uint64_t)nq * d))) return rc;
    if ((rc = dev_grow(w.d_pq_scores, w.pq_scores_cap, (uint64_t)nq * n1))) return rc;
    const float* rq = q;
    if (!transformed) {
        // NormalizeQuery + Rotate as one BF16 GEMM, FP32 accumulation; BF16 copy for the scores
        if ((rc = dev_grow(w.d_pq_b16, w.pq_b16_cap, (uint64_t)nq * d))) return rc;
        PDXG_CUDA(launch_bf16_rows(q, nq, d, ix->normalized, w.d_pq_b16, st));
        GemmOperand a;
        if (make_gemm_operand(a, kGemmBF16, w.d_pq_b16, nullptr, nq, d) != 0)
            return fail(PDXG_ERR_CUDA, "cannot encode the query tensor map");
        GemmArgs g{};
        g.M = nq;
        g.N = d;
        g.K = d;
        g.out = w.d_rq;
        g.ldo = d;
        g.out_b16 = w.d_pq_r16;
        g.ldo16 = d;
        g.error = w.d_gemm_err;
        PDXG_CUDA(launch_gemm(a, ix->rot_op16, kEpiStore, g, st));
        rq = w.d_rq;
        L.probe_launches += 2;
    } else {
        PDXG_CUDA(launch_bf16_rows(q, nq, d, false, w.d_pq_r16, st));
        L.probe_launches += 1;
    }
    GemmArgs g{};
    g.M = nq;
    g.N = n1;
    g.K = d;
    g.out = w.d_pq_scores;
    g.ldo = n1;
    g.col_add = ix->d_c1_sq;
    g.error = w.d_gemm_err;
    if (ix->probe_mode == 2) {
        if ((rc = dev_grow(w.d_pq_r8, w.pq_r8_cap, (uint64_t)nq * d))) return rc;
        if ((rc = dev_grow(w.d_pq_r8s, w.pq_r8s_cap, nq))) return rc;
        PDXG_CUDA(launch_e4m3_rows(rq, nq, d, w.d_pq_r8, w.d_pq_r8s, st));
        GemmOperand a;
        if (make_gemm_operand(a, kGemmE4M3, w.d_pq_r8, nullptr, nq, d) != 0)
            return fail(PDXG_ERR_CUDA, "cannot encode the query tensor map");
        g.row_scale = w.d_pq_r8s;
        g.col_scale = ix->d_c1_e4s;
        PDXG_CUDA(launch_gemm(a, ix->c1_op8, kEpiDist, g, st));
        L.probe_launches += 2;
    } else {
        GemmOperand a;
        if (make_gemm_operand(a, kGemmBF16, w.d_pq_r16, nullptr, nq, d) != 0)
            return fail(PDXG_ERR_CUDA, "cannot encode the query tensor map");
        PDXG_CUDA(launch_gemm(a, ix->c1_op16, kEpiDist, g, st));
        L.probe_launches += 1;
    }
    const uint32_t k1 = L.p.nprobe;
    if ((rc = dev_grow(w.d_l1_order, w.l1_order_cap, (uint64_t)nq * k1))) return rc;
    if ((rc = dev_grow(w.d_l1_count, w.l1_count_cap, nq))) return rc;
    ProbeParams pp{};
    pp.queries = rq;
    pp.centroids = ix->d_cent1;
    pp.scores = w.d_pq_scores;
    pp.ld_scores = n1;
    pp.nq = nq;
    pp.d = d;
    pp.nclusters = n1;
    pp.nprobe = k1;
    pp.q_nprobe = L.p.q_nprobe;
    pp.order = w.d_l1_order;
    pp.stride = k1;
    pp.count = w.d_l1_count;
    pp.cand_cap = (n1 + 3) & ~3u;
    pp.sort_cap = next_pow2(n1);
    pp.score_bytes = ix->probe_mode == 2 ? 1u : 2u;
    pp.stats = L.p.stats;
    PDXG_CUDA(launch_probe_select(pp, st));
    L.probe_launches += 1;
    L.p.queries = rq;
    L.p.q_order = w.d_l1_order;
    L.p.q_order_count = w.d_l1_count;
    L.p.q_order_stride = k1;
    return PDXG_OK;
}

// Exact probe of a flat index ahead of the scan (probe_exact_kernel): same order as the scan
// kernel's own probe; lets the scan keep per-vector arrays only.
constexpr uint32_t kProbeAheadMinQueries = 32;

bool probe_exact_ok(const pdxg_index* ix) {
    const uint32_t n1 = (uint32_t)ix->l1.fc.size();
    return !ix->tree && probe_select_smem(ix->d, n1, (n1 + 3) & ~3u, next_pow2(n1)) + 2048 <= ix->max_smem;
}

int run_probe_exact(pdxg_index* ix, Workspace& w, const float* qp, uint32_t nq, Launch& L, cudaStream_t st) {
    const uint32_t n1 = L.p.l1.nclusters, k1 = L.p.nprobe;
    int rc;
    if ((rc = dev_grow(w.d_l1_order, w.l1_order_cap, (uint64_t)nq * k1))) return rc;
    if ((rc = dev_grow(w.d_l1_count, w.l1_count_cap, nq))) return rc;
    ProbeParams pp{};
    pp.queries = qp;
    pp.centroids = ix->d_cent1;
    pp.nq = nq;
    pp.d = ix->d;
    pp.nclusters = n1;
    pp.nprobe = k1;
    pp.q_nprobe = L.p.q_nprobe;
    pp.order = w.d_l1_order;
    pp.stride = k1;
    pp.count = w.d_l1_count;
    pp.cand_cap = (n1 + 3) & ~3u;
    pp.sort_cap = next_pow2(n1);
    pp.stats = L.p.stats;
    PDXG_CUDA(launch_probe_exact(pp, st));
    L.probe_launches += 1;
    L.p.q_order = w.d_l1_order;
    L.p.q_order_count = w.d_l1_count;
    L.p.q_order_stride = k1;
    return PDXG_OK;
}

// Batched Start (pdxg_start.cu) for U8 levels whose visit orders are known before the scan
// (tree indexes with a separate top level). Sets L.p.start_* when it ran; a batch outside its
// limits leaves them unset and the scan runs Start itself.
constexpr uint32_t kStartMinQueries = 32;

int run_start_batched(pdxg_index* ix, Workspace& w, const float* qp, uint32_t nq, Launch& L, cudaStream_t st) {
    L.p.start_row = nullptr;
    if (!ix->u8 || !L.p.q_order || ix->start_mode == 1 || nq < kStartMinQueries) return PDXG_OK;
    const uint32_t n1 = L.p.l1.nclusters;
    const uint32_t stride = (std::max(L.p.l1.max_n, 1u) + 3) & ~3u;
    const uint64_t items = start_item_bound(nq, n1, std::max(L.p.l1.max_n, 1u));
    if ((uint64_t)nq * stride * 4 > (4ull << 30) || items > 0xFFFFFFFFull || nq > (1u << 20)) return PDXG_OK;
    const size_t smem = start_dist_smem(L.p.l1);
    if (smem + 1024 > ix->max_smem) return PDXG_OK;
    const int occ = start_dist_occupancy(smem);
    if (occ <= 0) return PDXG_OK;
    int rc;
    if ((rc = dev_grow(w.d_st_cl, w.st_cl_cap, (uint64_t)3 * n1))) return rc;
    if ((rc = dev_grow(w.d_st_q, w.st_q_cap, (uint64_t)4 * nq + 2))) return rc;
    if ((rc = dev_grow(w.d_st_items, w.st_items_cap, 2 * items))) return rc;
    if ((rc = dev_grow(w.d_st_dist, w.st_dist_cap, (uint64_t)nq * stride))) return rc;
    StartParams sp{};
    sp.arena = ix->arena;
    sp.l1 = L.p.l1;
    sp.queries = qp;
    sp.nq = nq;
    sp.q_order = L.p.q_order;
    sp.q_order_count = L.p.q_order_count;
    sp.q_order_stride = L.p.q_order_stride;
    sp.filter_of = L.p.filter_of;
    sp.cl_count = w.d_st_cl;
    sp.cl_off = w.d_st_cl + n1;
    sp.cl_items = w.d_st_cl + 2 * (uint64_t)n1;
    sp.first_cl = w.d_st_q;
    sp.slot_of = w.d_st_q + nq;
    sp.row_of = reinterpret_cast<int32_t*>(w.d_st_q + 2 * (uint64_t)nq);
    sp.sorted_q = w.d_st_q + 3 * (uint64_t)nq;
    sp.n_items = w.d_st_q + 4 * (uint64_t)nq;
    sp.queue = w.d_st_q + 4 * (uint64_t)nq + 1;
    sp.items = w.d_st_items;
    sp.dist = w.d_st_dist;
    sp.stride = stride;
    PDXG_CUDA(launch_start_batched(sp, occ * ix->num_sms, st));
    L.p.start_row = sp.row_of;
    L.p.start_first = sp.first_cl;
    L.p.start_dist = sp.dist;
    L.p.start_stride = stride;
    L.start_launches = 3;
    return PDXG_OK;
}

}  // namespace

int pdxg::host::run_scan_cluster_major(pdxg_index* ix, Workspace& w, uint32_t nq, Launch& L, cudaStream_t st,
                                       bool timed) {
    L.p.q_list = nullptr;
    L.p.q_list_n = nullptr;
    L.scan_launches = 0;
    ix->tev_scan = false;
    if (ix->scan_mode != 0 || !L.u8 || !L.p.start_row || !L.p.q_order || L.p.order || L.p.l1.tomb) return PDXG_OK;
    const DevLevel& lv = L.p.l1;
    const uint32_t n1 = lv.nclusters, stride = L.p.q_order_stride, k = L.p.k;
    const uint32_t nwords = lv.qw_hoff + lv.n_hblocks * 16;
    const uint32_t bm_words = (std::max(lv.max_n, 1u) + 31) / 32;
    if ((uint64_t)nq * stride >= 0xFFFFFFFFull || (uint64_t)n1 * nq > (256ull << 20) || stride == 0) return PDXG_OK;
    ScanParams sp{};
    sp.r_heap_cap = (k + 3) & ~3u;
    sp.r_area_bytes = (uint32_t)align_up(std::max<uint64_t>(2048, 8ull * next_pow2(k)), 16);
    // a first warmup step that ends the warmup keeps at most n - ceil(0.8 n) survivors
    sp.r_surv_cap = (std::max(lv.max_n, 1u) / 5 + 33 + 31) / 32 * 32;
    sp.r_warp_bytes = (uint32_t)(align_up((uint64_t)nwords * 4, 16) + 8ull * sp.r_heap_cap + sp.r_area_bytes +
                                 align_up((uint64_t)bm_words * 4, 16) + 8ull * sp.r_surv_cap);
    sp.prep_qs_stride = (lv.d + 3) & ~3u;
    sp.prep_qs = (uint64_t)scan_queries_per_cta() * sp.prep_qs_stride * 4 + 9 * 1024 <= ix->max_smem ? 1u : 0u;
    if ((uint64_t)sp.r_warp_bytes * scan_queries_per_cta() + 1024 > ix->max_smem) return PDXG_OK;
    const int occ = scan_bitmap_occupancy();
    if (occ <= 0) return PDXG_OK;
    const uint64_t items = scan_item_bound(nq, stride, n1);
    int rc;
    if ((rc = dev_grow(w.d_sc_qw, w.sc_qw_cap, (uint64_t)nq * nwords))) return rc;
    if ((rc = dev_grow(w.d_sc_q, w.sc_q_cap, 3ull * nq + 4))) return rc;
    if ((rc = dev_grow(w.d_sc_heap, w.sc_heap_cap, 2ull * nq * k))) return rc;
    if ((rc = dev_grow(w.d_sc_cl, w.sc_cl_cap, (uint64_t)n1))) return rc;
    if ((rc = dev_grow(w.d_sc_vl, w.sc_vl_cap, (uint64_t)n1 * nq))) return rc;
    if ((rc = dev_grow(w.d_sc_items, w.sc_items_cap, 2 * items))) return rc;
    if ((rc = dev_grow(w.d_sc_bm, w.sc_bm_cap, (uint64_t)nq * stride * bm_words))) return rc;
    sp.arena = L.p.arena;
    sp.l1 = lv;
    sp.ratios = L.p.ratios;
    sp.queries = L.p.queries;
    sp.nq = nq;
    sp.k = k;
    sp.q_k = L.p.q_k;
    sp.filter_of = L.p.filter_of;
    sp.q_order = L.p.q_order;
    sp.q_order_count = L.p.q_order_count;
    sp.q_order_stride = stride;
    sp.start_row = L.p.start_row;
    sp.start_first = L.p.start_first;
    sp.start_dist = const_cast<uint32_t*>(L.p.start_dist);
    sp.start_stride = L.p.start_stride;
    sp.cp1 = std::min(16u, lv.dv);
    sp.g1 = (sp.cp1 + 3) / 4;
    sp.nwords = nwords;
    sp.qwords = w.d_sc_qw;
    sp.first_i = w.d_sc_q;
    sp.lim = reinterpret_cast<int32_t*>(w.d_sc_q + nq);
    sp.left = w.d_sc_q + 2ull * nq;
    sp.left_n = w.d_sc_q + 3ull * nq;
    sp.n_items = w.d_sc_q + 3ull * nq + 1;
    sp.queue = w.d_sc_q + 3ull * nq + 2;
    sp.heap_d = reinterpret_cast<float*>(w.d_sc_heap);
    sp.heap_id = w.d_sc_heap + (uint64_t)nq * k;
    sp.vl_count = w.d_sc_cl;
    sp.vl = w.d_sc_vl;
    sp.items = w.d_sc_items;
    sp.bm = w.d_sc_bm;
    sp.bm_words = bm_words;
    sp.out_ids = L.p.out_ids;
    sp.out_dists = L.p.out_dists;
    sp.out_counts = L.p.out_counts;
    sp.stats = L.p.stats;
    PDXG_CUDA(launch_scan(sp, occ * ix->num_sms, st, timed ? ix->tev + 5 : nullptr));
    ix->tev_scan = timed;
    L.p.q_list = sp.left;
    L.p.q_list_n = sp.left_n;
    L.scan_launches = 3;
    return PDXG_OK;
}

namespace {

// Core device-side search: queries/ids/dists/counts are device pointers.
int search_device_impl(pdxg_index* ix, Workspace& w, const float* q, uint32_t nq, uint32_t k, uint32_t flags,
                       const uint32_t* d_order, uint32_t n_order, const uint32_t* d_sel,
                       const uint32_t* d_pass, const int32_t* d_filter_of, bool any_filter,
                       uint32_t* ids, float* dists, uint32_t* counts, cudaStream_t st) {
    if (nq == 0) return PDXG_OK;
    if (k == 0) {
        PDXG_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * nq, st));
        return PDXG_OK;
    }
    int rc = ensure_ws(ix, w, nq, k);
    if (rc) return rc;
    const bool timed = (flags & PDXG_TIME_KERNELS) != 0;
    if (timed) {
        for (cudaEvent_t& e : ix->tev)
            if (!e) PDXG_CUDA(cudaEventCreate(&e));
        ix->tev_ready = false;
        PDXG_CUDA(cudaEventRecord(ix->tev[0], st));
    }
    const float* qp = q;
    // the reduced-precision probe rotates the queries itself (BF16 GEMM)
    const bool gemm_probe = ix->probe_mode != 0 && !d_order && probe_gemm_ok(ix);
    ix->tev_prep = !(flags & PDXG_QUERY_TRANSFORMED) && !gemm_probe;
    uint32_t launches = 1;  // the scan
    if (!(flags & PDXG_QUERY_TRANSFORMED) && !gemm_probe) {
        if ((rc = prepare_dev(ix, w, q, nq, w.d_rq, st))) return rc;
        qp = w.d_rq;
        // TF32 split + tensor-core GEMM, or [norms +] SIMT GEMM
        launches += (ix->rot_tc && ix->rot_mode == 0 && nq > 8) ? 2 : (ix->normalized ? 2 : 1);
    }
    if (timed) PDXG_CUDA(cudaEventRecord(ix->tev[1], st));
    Launch L;
    const bool probe_ahead = !gemm_probe && !ix->tree && !any_filter && !d_order && nq >= kProbeAheadMinQueries &&
                             probe_exact_ok(ix);
    rc = plan_search(ix, nq, k, n_order, any_filter, L, 0xFFFFFFFFu, 0xFFFFFFFFu, probe_ahead, st);
    if (rc) return rc;
    L.p.queries = qp;
    L.p.order = d_order;
    L.p.sel_bits = d_sel;
    L.p.passing = d_pass;
    L.p.filter_of = d_filter_of;
    L.p.out_ids = ids;
    L.p.out_dists = dists;
    L.p.out_counts = counts;
    L.p.queue = w.d_queue;
    L.p.stats = nullptr;
    if (flags & PDXG_COLLECT_STATS) {
        if (!w.d_stats) PDXG_CUDA(cudaMalloc(&w.d_stats, kStatsWords * sizeof(unsigned long long)));
        PDXG_CUDA(cudaMemsetAsync(w.d_stats, 0, kStatsWords * sizeof(unsigned long long), st));
        L.p.stats = w.d_stats;
        ix->stats_stream = st;
    }
    if (gemm_probe) {
        rc = run_probe_gemm(ix, w, q, nq, (flags & PDXG_QUERY_TRANSFORMED) != 0, L, st);
        if (rc) return rc;
        qp = L.p.queries;
        launches += L.probe_launches;
    } else if (ix->tree && !any_filter && !d_order) {
        rc = run_top_level(ix, w, qp, nq, L, st, 0, timed);
        if (rc) return rc;
        launches += L.top_launches;
    } else if (probe_ahead) {
        rc = run_probe_exact(ix, w, qp, nq, L, st);
        if (rc) return rc;
        launches += L.probe_launches;
    }
    ix->tev_top = L.p.q_order != nullptr;
    ix->last_order_stride = L.p.q_order ? L.p.q_order_stride : 0;
    // the batched Start belongs to the scan's time
    if (timed) PDXG_CUDA(cudaEventRecord(ix->tev[2], st));
    if ((rc = run_start_batched(ix, w, qp, nq, L, st))) return rc;
    launches += L.start_launches;
    if (timed) PDXG_CUDA(cudaEventRecord(ix->tev[3], st));
    if ((rc = run_scan_cluster_major(ix, w, nq, L, st, timed))) return rc;
    launches += L.scan_launches;
    ix->last_launches = launches;
    PDXG_CUDA(cudaMemsetAsync(w.d_queue, 0, sizeof(uint32_t), st));
    PDXG_CUDA(launch_search(L.p, L.u8, L.threads, L.grid, st));
    if (timed) {
        PDXG_CUDA(cudaEventRecord(ix->tev[4], st));
        ix->tev_ready = true;
    }
    return PDXG_OK;
}

}  // namespace

// Whether pdxg_search_device rotates a batch of nq raw queries on the tensor cores (TF32x3), and
// whether its probe is the reduced-precision one: the allocation-free search sizes its scratch by
// the first and refuses the second.
bool pdxg_rotation_on_tensor_cores(const pdxg_index* ix, uint32_t nq) { return rotation_on_tensor_cores(ix, nq); }
bool pdxg_reduced_precision_probe(const pdxg_index* ix) { return ix->probe_mode != 0 && probe_gemm_ok(ix); }

// Search on caller-provided workspace: never allocates. Raw queries are rotated as
// pdxg_search_device rotates them: on the tensor cores (hi / lo need nq * d floats each, 16-byte
// aligned; gemm_err one int) when pdxg_rotation_on_tensor_cores, else by the FP32 SIMT kernels
// (norms: nq floats). `rotated` needs nq * d floats; all of these are unused with
// PDXG_QUERY_TRANSFORMED. `queue` is one u32.
int pdxg_search_on_workspace(pdxg_index* ix, const float* q, uint32_t nq, uint32_t k,
                             uint32_t flags, float* norms, float* rotated, float* hi, float* lo,
                             int* gemm_err, uint32_t* queue, uint32_t* ids, float* dists,
                             uint32_t* counts, cudaStream_t st) {
    if (nq == 0) return PDXG_OK;
    if (k == 0) {
        PDXG_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * nq, st));
        return PDXG_OK;
    }
    const float* qp = q;
    int rc;
    if (!(flags & PDXG_QUERY_TRANSFORMED)) {
        if (rotation_on_tensor_cores(ix, nq)) {
            PDXG_CUDA(cudaMemsetAsync(gemm_err, 0, sizeof(int), st));
            if ((rc = rotate_tf32x3(ix, q, nq, ix->normalized, hi, lo, gemm_err, rotated, st))) return rc;
        } else {
            PDXG_CUDA(launch_prepare_queries(q, nq, ix->d, ix->d_rot, ix->normalized, norms, rotated, st));
        }
        qp = rotated;
    }
    Launch L;
    rc = plan_search(ix, nq, k, 0, false, L, 0xFFFFFFFFu, 0xFFFFFFFFu, false, st);
    if (rc) return rc;
    L.p.queries = qp;
    L.p.out_ids = ids;
    L.p.out_dists = dists;
    L.p.out_counts = counts;
    L.p.queue = queue;
    PDXG_CUDA(cudaMemsetAsync(queue, 0, sizeof(uint32_t), st));
    PDXG_CUDA(launch_search(L.p, L.u8, L.threads, L.grid, st));
    return PDXG_OK;
}

int pdxg_index_device(const pdxg_index* ix) { return ix->device; }
uint32_t pdxg_index_dims(const pdxg_index* ix) { return ix->d; }
std::mutex& pdxg_index_mutex(pdxg_index* ix) { return ix->mu; }
cudaStream_t pdxg_index_stream(pdxg_index* ix) { return ix->stream; }
int pdxg_set_error(int code, const char* msg) { return fail(code, msg); }
void pdxg_split_dims(uint32_t d, uint32_t& h, uint32_t& v) { dimension_split(d, h, v); }

namespace pdxg {
namespace host {

int check_index(const pdxg_index* ix) {
    if (!ix) return fail(PDXG_ERR_INVALID_ARGUMENT, "index is NULL");
    return PDXG_OK;
}

}  // namespace host
}  // namespace pdxg

namespace {

// Host-buffer search shared by pdxg_search / _with_order / filtered variants.
// Host-buffer search of a plain batch (no order, no filter) with the query upload pipelined:
// the batch goes up in chunks on a copy stream, each chunk is rotated and runs its tree top
// level on the compute stream while the next chunk uploads; the batched Start and the scan then
// run once over the whole batch (their cross-query reuse grows with the batch).
constexpr uint32_t kPipelineMinQueries = 4096;

int search_host_pipelined(pdxg_index* ix, const float* queries, uint32_t nq, uint32_t k, uint32_t flags,
                          uint32_t* ids, float* dists, uint32_t* counts) {
    Workspace& w = ix->ws;
    cudaStream_t st = ix->stream;
    const uint32_t d = ix->d;
    const bool transformed = (flags & PDXG_QUERY_TRANSFORMED) != 0;
    int rc;
    if (!ix->copy_stream) PDXG_CUDA(cudaStreamCreateWithFlags(&ix->copy_stream, cudaStreamNonBlocking));
    for (cudaEvent_t& e : ix->chunk_ev)
        if (!e) PDXG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    // two chunks (measured on B200: more chunks cost the top level its tile fill); the first is a
    // quarter of the batch, so that only its upload is exposed and the larger second upload
    // overlaps the first chunk's rotation and top level (10,000 x 1024 queries: first chunk
    // 1/8, 1/4, 1/3, 1/2 gave 2.68, 2.87, 2.80, 2.71 M queries/s end to end)
    const uint32_t nch = 2;
    const uint32_t first = nq >= 1024 ? (nq / 4 + 31) / 32 * 32 : nq;
    auto chunk_off = [&](uint32_t c) { return c == 0 ? 0u : std::min(first, nq); };
    auto chunk_len = [&](uint32_t c) { return c == 0 ? std::min(first, nq) : nq - std::min(first, nq); };
    Launch L;
    if ((rc = plan_search(ix, nq, k, 0, false, L))) return rc;
    L.p.out_ids = w.d_ids;
    L.p.out_dists = w.d_dists;
    L.p.out_counts = w.d_counts;
    L.p.queue = w.d_queue;
    const uint32_t k1 = L.p.nprobe;
    const bool top = ix->tree && ix->top_mode != 1;
    if (top) {
        if ((rc = dev_grow(w.d_l1_order, w.l1_order_cap, (uint64_t)nq * k1))) return rc;
        if ((rc = dev_grow(w.d_l1_count, w.l1_count_cap, nq))) return rc;
    }
    uint32_t launches = 1;
    bool orders = top;
    for (uint32_t c = 0; c < nch; ++c) {
        const uint32_t off = chunk_off(c), n = chunk_len(c);
        if (n == 0) break;
        PDXG_CUDA(cudaMemcpyAsync(w.d_q + (uint64_t)off * d, queries + (uint64_t)off * d, sizeof(float) * n * d,
                                  cudaMemcpyHostToDevice, ix->copy_stream));
        PDXG_CUDA(cudaEventRecord(ix->chunk_ev[c], ix->copy_stream));
        PDXG_CUDA(cudaStreamWaitEvent(st, ix->chunk_ev[c], 0));
        const float* qc = w.d_q + (uint64_t)off * d;
        if (!transformed) {
            if ((rc = prepare_dev(ix, w, qc, n, w.d_rq + (uint64_t)off * d, st))) return rc;
            qc = w.d_rq + (uint64_t)off * d;
            launches += (ix->rot_tc && ix->rot_mode == 0 && n > 8) ? 2 : (ix->normalized ? 2 : 1);
        }
        if (top) {
            Launch Lc = L;
            if ((rc = run_top_level(ix, w, qc, n, Lc, st, off))) return rc;
            orders = orders && Lc.p.q_order != nullptr;
            launches += Lc.top_launches;
        }
    }
    L.p.queries = transformed ? w.d_q : w.d_rq;
    if (orders) {
        L.p.q_order = w.d_l1_order;
        L.p.q_order_count = w.d_l1_count;
        L.p.q_order_stride = k1;
    }
    if ((rc = run_start_batched(ix, w, L.p.queries, nq, L, st))) return rc;
    launches += L.start_launches;
    if ((rc = run_scan_cluster_major(ix, w, nq, L, st))) return rc;
    launches += L.scan_launches;
    ix->last_launches = launches;
    ix->last_order_stride = L.p.q_order ? k1 : 0;
    PDXG_CUDA(cudaMemsetAsync(w.d_queue, 0, sizeof(uint32_t), st));
    PDXG_CUDA(launch_search(L.p, L.u8, L.threads, L.grid, st));
    PDXG_CUDA(cudaMemcpyAsync(ids, w.d_ids, sizeof(uint32_t) * nq * k, cudaMemcpyDeviceToHost, st));
    PDXG_CUDA(cudaMemcpyAsync(dists, w.d_dists, sizeof(float) * nq * k, cudaMemcpyDeviceToHost, st));
    PDXG_CUDA(cudaMemcpyAsync(counts, w.d_counts, sizeof(uint32_t) * nq, cudaMemcpyDeviceToHost, st));
    PDXG_CUDA(cudaStreamSynchronize(st));
    return check_gemm_error(w);
}

int search_host_impl(pdxg_index* ix, const float* queries, uint32_t nq, uint32_t k, uint32_t flags,
                     const uint32_t* order, uint32_t n_order,
                     const std::vector<uint32_t>* sel, const std::vector<uint32_t>* pass,
                     const std::vector<int32_t>* filter_of, uint32_t* ids, float* dists,
                     uint32_t* counts) {
    if (!queries || !ids || !dists || !counts)
        return fail(PDXG_ERR_INVALID_ARGUMENT, "NULL buffer");
    PDXG_CUDA(cudaSetDevice(ix->device));
    int rc = ensure_ws(ix, ix->ws, nq, k);
    if (rc) return rc;
    Workspace& w = ix->ws;
    cudaStream_t st = ix->stream;
    if (nq >= kPipelineMinQueries && k > 0 && !(order && n_order) && !(sel && !sel->empty()) &&
        ix->probe_mode == 0 && !(flags & PDXG_COLLECT_STATS) && !(flags & PDXG_TIME_KERNELS))
        return search_host_pipelined(ix, queries, nq, k, flags, ids, dists, counts);
    PDXG_CUDA(cudaMemcpyAsync(w.d_q, queries, sizeof(float) * nq * ix->d, cudaMemcpyHostToDevice, st));
    const uint32_t* d_order = nullptr;
    if (order && n_order) {
        uint64_t cap = w.order_cap;
        if ((rc = dev_grow(w.d_order, cap, n_order))) return rc;
        w.order_cap = (uint32_t)cap;
        PDXG_CUDA(cudaMemcpyAsync(w.d_order, order, sizeof(uint32_t) * n_order, cudaMemcpyHostToDevice, st));
        d_order = w.d_order;
    }
    const uint32_t* d_sel = nullptr;
    const uint32_t* d_pass = nullptr;
    const int32_t* d_fo = nullptr;
    bool any_filter = false;
    if (sel && !sel->empty()) {
        any_filter = true;
        if ((rc = dev_grow(w.d_sel, w.sel_cap, sel->size()))) return rc;
        if ((rc = dev_grow(w.d_pass, w.pass_cap, pass->size()))) return rc;
        uint64_t cap = w.fo_cap;
        if ((rc = dev_grow(w.d_filter_of, cap, filter_of->size()))) return rc;
        w.fo_cap = (uint32_t)cap;
        PDXG_CUDA(cudaMemcpyAsync(w.d_sel, sel->data(), sel->size() * 4, cudaMemcpyHostToDevice, st));
        PDXG_CUDA(cudaMemcpyAsync(w.d_pass, pass->data(), pass->size() * 4, cudaMemcpyHostToDevice, st));
        PDXG_CUDA(cudaMemcpyAsync(w.d_filter_of, filter_of->data(), filter_of->size() * 4,
                                  cudaMemcpyHostToDevice, st));
        d_sel = w.d_sel;
        d_pass = w.d_pass;
        d_fo = w.d_filter_of;
    }
    rc = search_device_impl(ix, w, w.d_q, nq, k, flags, d_order, n_order, d_sel, d_pass, d_fo,
                            any_filter, w.d_ids, w.d_dists, w.d_counts, st);
    if (rc) return rc;
    PDXG_CUDA(cudaMemcpyAsync(ids, w.d_ids, sizeof(uint32_t) * nq * k, cudaMemcpyDeviceToHost, st));
    PDXG_CUDA(cudaMemcpyAsync(dists, w.d_dists, sizeof(float) * nq * k, cudaMemcpyDeviceToHost, st));
    PDXG_CUDA(cudaMemcpyAsync(counts, w.d_counts, sizeof(uint32_t) * nq, cudaMemcpyDeviceToHost, st));
    PDXG_CUDA(cudaStreamSynchronize(st));
    return check_gemm_error(w);
}

}  // namespace

namespace pdxg {
namespace host {

// Selection bitmap + passing counts of one row-id list (CreatePredicateEvaluator,
// index.hpp:436-446), in the device bitmap layout (one bit per cluster slot).
void build_filter(const pdxg_index* ix, const uint64_t* rows, uint64_t n, uint32_t* sel,
                  uint32_t* pass) {
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t r = rows[i];
        if (r >= ix->rid_cluster.size()) continue;
        const uint32_t c = ix->rid_cluster[r];
        if (c == 0xFFFFFFFFu) continue;
        const uint32_t pos = ix->rid_pos[r];
        const uint32_t word = ix->l1.meta[c].sel_word + (pos >> 5);
        const uint32_t bit = 1u << (pos & 31);
        if (!(sel[word] & bit)) {
            sel[word] |= bit;
            pass[c]++;
        }
    }
}

}  // namespace host
}  // namespace pdxg

// =============================================================================== C ABI
extern "C" {

const char* pdxg_last_error(void) { return g_err.c_str(); }

int pdxg_load_buffer(const void* data, uint64_t size, int device, pdxg_index** out) {
    if (!data) return fail(PDXG_ERR_INVALID_ARGUMENT, "data is NULL");
    try {
        return load_from_bytes(static_cast<const uint8_t*>(data), size, device, out);
    } catch (const std::exception& e) {
        return fail(PDXG_ERR_IO, e.what());
    }
}

int pdxg_load(const char* path, int device, pdxg_index** out) {
    if (!path) return fail(PDXG_ERR_INVALID_ARGUMENT, "path is NULL");
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) return fail(PDXG_ERR_IO, std::string("Failed to open file: ") + path);
    const std::streamsize size = f.tellg();
    f.seekg(0);
    std::vector<uint8_t> buf((size_t)std::max<std::streamsize>(size, 0));
    if (size > 0 && !f.read(reinterpret_cast<char*>(buf.data()), size))
        return fail(PDXG_ERR_IO, std::string("Failed to read file: ") + path);
    return pdxg_load_buffer(buf.data(), buf.size(), device, out);
}

void pdxg_free(pdxg_index* index) { free_index(index); }

int pdxg_set_nprobe(pdxg_index* ix, uint32_t nprobe) {
    if (int rc = check_index(ix)) return rc;
    ix->nprobe = nprobe;
    return PDXG_OK;
}

int pdxg_set_pruning_aggressiveness(pdxg_index* ix, float eps0) {
    if (int rc = check_index(ix)) return rc;
    std::lock_guard<std::mutex> lock(ix->mu);
    PDXG_CUDA(cudaSetDevice(ix->device));
    ix->eps0 = eps0;
    return upload_ratios(ix);
}

int pdxg_set_top_level_mode(pdxg_index* ix, uint32_t mode) {
    if (int rc = check_index(ix)) return rc;
    if (mode > 3) return fail(PDXG_ERR_INVALID_ARGUMENT, "top-level mode must be 0, 1, 2 or 3");
    ix->top_mode = mode;
    return PDXG_OK;
}

int pdxg_set_probe_mode(pdxg_index* ix, uint32_t mode) {
    if (int rc = check_index(ix)) return rc;
    if (mode > 2) return fail(PDXG_ERR_INVALID_ARGUMENT, "probe mode must be 0, 1 or 2");
    if (mode != 0 && !probe_gemm_ok(ix))
        return fail(PDXG_ERR_UNSUPPORTED, "the reduced-precision probe needs tensor cores and d a multiple of 16");
    ix->probe_mode = mode;
    return PDXG_OK;
}

int pdxg_last_visit_orders(pdxg_index* ix, uint32_t nq, uint32_t stride, uint32_t* orders, uint32_t* counts) {
    if (int rc = check_index(ix)) return rc;
    std::lock_guard<std::mutex> lock(ix->mu);
    if (!ix->ws.d_l1_order || !ix->ws.d_l1_count || (uint64_t)nq * ix->last_order_stride > ix->ws.l1_order_cap ||
        nq > ix->ws.l1_count_cap || ix->last_order_stride == 0)
        return fail(PDXG_ERR_INVALID_ARGUMENT, "no visit orders of that size were computed by the last search");
    if (stride < ix->last_order_stride) return fail(PDXG_ERR_INVALID_ARGUMENT, "stride below the last nprobe");
    PDXG_CUDA(cudaSetDevice(ix->device));
    PDXG_CUDA(cudaDeviceSynchronize());
    std::vector<uint32_t> h((size_t)nq * ix->last_order_stride);
    PDXG_CUDA(cudaMemcpy(h.data(), ix->ws.d_l1_order, h.size() * 4, cudaMemcpyDeviceToHost));
    PDXG_CUDA(cudaMemcpy(counts, ix->ws.d_l1_count, (size_t)nq * 4, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < nq; ++i)
        std::memcpy(orders + (size_t)i * stride, h.data() + (size_t)i * ix->last_order_stride, ix->last_order_stride * 4);
    return PDXG_OK;
}

int pdxg_set_start_mode(pdxg_index* ix, uint32_t mode) {
    if (int rc = check_index(ix)) return rc;
    if (mode > 1) return fail(PDXG_ERR_INVALID_ARGUMENT, "start mode must be 0 or 1");
    ix->start_mode = mode;
    return PDXG_OK;
}

int pdxg_set_scan_mode(pdxg_index* ix, uint32_t mode) {
    if (int rc = check_index(ix)) return rc;
    if (mode > 1) return fail(PDXG_ERR_INVALID_ARGUMENT, "scan mode must be 0 or 1");
    std::lock_guard<std::mutex> lock(ix->mu);
    ix->scan_mode = mode;
    return PDXG_OK;
}

int pdxg_set_threads_per_query(pdxg_index* ix, uint32_t threads) {
    if (int rc = check_index(ix)) return rc;
    if (threads != 0 && threads != 64 && threads != 128 && threads != 256 && threads != 512)
        return fail(PDXG_ERR_INVALID_ARGUMENT, "threads per query must be 0, 64, 128, 256 or 512");
    ix->threads = threads;
    return PDXG_OK;
}

int pdxg_search(pdxg_index* ix, const float* queries, uint32_t nq, uint32_t k, uint32_t flags,
                uint32_t* ids, float* distances, uint32_t* counts) {
    if (int rc = check_index(ix)) return rc;
    std::lock_guard<std::mutex> lock(ix->mu);
    return search_host_impl(ix, queries, nq, k, flags, nullptr, 0, nullptr, nullptr, nullptr, ids,
                            distances, counts);
}

int pdxg_search_device(pdxg_index* ix, const float* queries, uint32_t nq, uint32_t k,
                       uint32_t flags, uint32_t* ids, float* distances, uint32_t* counts,
                       void* stream) {
    if (int rc = check_index(ix)) return rc;
    if (!queries || !ids || !distances || !counts)
        return fail(PDXG_ERR_INVALID_ARGUMENT, "NULL buffer");
    std::lock_guard<std::mutex> lock(ix->mu);
    PDXG_CUDA(cudaSetDevice(ix->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ix->stream;
    return search_device_impl(ix, ix->ws, queries, nq, k, flags, nullptr, 0, nullptr, nullptr, nullptr,
                              false, ids, distances, counts, st);
}

}  // extern "C"

struct pdxg_graph {
    pdxg_index* ix = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t gen = 0;  // g_alloc_gen at capture
};

extern "C" {

int pdxg_graph_create(pdxg_index* ix, const float* queries, uint32_t nq, uint32_t k, uint32_t flags,
                      uint32_t* ids, float* distances, uint32_t* counts, pdxg_graph** out) {
    if (int rc = check_index(ix)) return rc;
    if (!queries || !ids || !distances || !counts || !out) return fail(PDXG_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (flags & (PDXG_COLLECT_STATS | PDXG_TIME_KERNELS))
        return fail(PDXG_ERR_INVALID_ARGUMENT, "statistics and kernel timing are not captured in a graph");
    if (nq == 0 || k == 0) return fail(PDXG_ERR_INVALID_ARGUMENT, "empty batch");
    std::lock_guard<std::mutex> lock(ix->mu);
    PDXG_CUDA(cudaSetDevice(ix->device));
    // a direct run sizes every workspace buffer for this batch, so the capture allocates nothing
    int rc = search_device_impl(ix, ix->ws, queries, nq, k, flags, nullptr, 0, nullptr, nullptr, nullptr, false,
                                ids, distances, counts, ix->stream);
    if (rc) return rc;
    PDXG_CUDA(cudaStreamSynchronize(ix->stream));
    if ((rc = check_gemm_error(ix->ws))) return rc;
    const uint64_t gen = g_alloc_gen.load();
    cudaStream_t cs = nullptr;
    PDXG_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        rc = search_device_impl(ix, ix->ws, queries, nq, k, flags, nullptr, 0, nullptr, nullptr, nullptr, false,
                                ids, distances, counts, cs);
        e = cudaStreamEndCapture(cs, &graph);
    }
    cudaStreamDestroy(cs);
    if (rc == PDXG_OK && (e != cudaSuccess || g_alloc_gen.load() != gen))
        rc = fail(PDXG_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    if (rc == PDXG_OK && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
        rc = fail(PDXG_ERR_CUDA, "graph instantiation failed");
    if (rc != PDXG_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    pdxg_graph* g = new pdxg_graph();
    g->ix = ix;
    g->graph = graph;
    g->exec = exec;
    g->gen = gen;
    *out = g;
    return PDXG_OK;
}

int pdxg_graph_launch(pdxg_graph* g, void* stream) {
    if (!g) return fail(PDXG_ERR_INVALID_ARGUMENT, "graph is NULL");
    if (g_alloc_gen.load() != g->gen)
        return fail(PDXG_ERR_INVALID_ARGUMENT, "the engine's buffers changed since the capture; create the graph again");
    PDXG_CUDA(cudaSetDevice(g->ix->device));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : g->ix->stream;
    // the upload of the last Append / Delete changes may still run on another stream
    if (g->ix->maint && g->ix->maint->ev_flush) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        PDXG_CUDA(cudaStreamIsCapturing(st, &cs));
        if (cs == cudaStreamCaptureStatusNone) PDXG_CUDA(cudaStreamWaitEvent(st, g->ix->maint->ev_flush, 0));
    }
    PDXG_CUDA(cudaGraphLaunch(g->exec, st));
    return PDXG_OK;
}

void pdxg_graph_free(pdxg_graph* g) {
    if (!g) return;
    cudaSetDevice(g->ix->device);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
}

int pdxg_autotune(pdxg_index* ix, const float* queries, uint32_t nq, uint32_t k, uint32_t flags, uint32_t choice[3]) {
    if (int rc = check_index(ix)) return rc;
    if (!queries || !choice || nq == 0 || k == 0) return fail(PDXG_ERR_INVALID_ARGUMENT, "bad arguments");
    std::lock_guard<std::mutex> lock(ix->mu);
    PDXG_CUDA(cudaSetDevice(ix->device));
    flags &= ~(uint32_t)(PDXG_COLLECT_STATS | PDXG_TIME_KERNELS);
    uint32_t *ids = nullptr, *counts = nullptr;
    float* dists = nullptr;
    int rc = PDXG_OK;
    if (cudaMalloc(&ids, (size_t)nq * k * 4) != cudaSuccess || cudaMalloc(&dists, (size_t)nq * k * 4) != cudaSuccess ||
        cudaMalloc(&counts, (size_t)nq * 4) != cudaSuccess)
        rc = fail(PDXG_ERR_CUDA, "cannot allocate the tuning outputs");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (rc == PDXG_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        rc = fail(PDXG_ERR_CUDA, "cannot create events");
    const uint32_t old_threads = ix->threads, old_top = ix->top_mode, old_start = ix->start_mode;
    const uint32_t threads_c[3] = {64, 128, 256};
    const uint32_t tops_c[2] = {3, 2};
    const uint32_t starts_c[2] = {0, 1};
    const uint32_t ntop = ix->tree ? 2 : 1, nstart = (ix->tree && ix->u8) ? 2 : 1;
    float best = 1e30f;
    uint32_t bt = old_threads, btop = old_top, bstart = old_start;
    for (uint32_t a = 0; a < 3 && rc == PDXG_OK; ++a)
        for (uint32_t b = 0; b < ntop && rc == PDXG_OK; ++b)
            for (uint32_t c = 0; c < nstart && rc == PDXG_OK; ++c) {
                ix->threads = threads_c[a];
                ix->top_mode = ix->tree ? tops_c[b] : old_top;
                ix->start_mode = starts_c[c];
                float t_min = 1e30f;
                for (int rep = 0; rep < 4 && rc == PDXG_OK; ++rep) {
                    if (cudaEventRecord(e0, ix->stream) != cudaSuccess) rc = fail(PDXG_ERR_CUDA, "event");
                    if (rc == PDXG_OK)
                        rc = search_device_impl(ix, ix->ws, queries, nq, k, flags, nullptr, 0, nullptr, nullptr,
                                                nullptr, false, ids, dists, counts, ix->stream);
                    if (rc == PDXG_OK && (cudaEventRecord(e1, ix->stream) != cudaSuccess ||
                                          cudaEventSynchronize(e1) != cudaSuccess))
                        rc = fail(PDXG_ERR_CUDA, "event");
                    float ms = 0.0f;
                    if (rc == PDXG_OK && rep > 0 && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess)
                        t_min = std::min(t_min, ms);  // the first run of a form warms it up
                }
                if (rc == PDXG_OK && t_min < best) {
                    best = t_min;
                    bt = ix->threads;
                    btop = ix->top_mode;
                    bstart = ix->start_mode;
                }
            }
    if (rc == PDXG_OK) rc = check_gemm_error(ix->ws);
    ix->threads = rc == PDXG_OK ? bt : old_threads;
    ix->top_mode = rc == PDXG_OK ? btop : old_top;
    ix->start_mode = rc == PDXG_OK ? bstart : old_start;
    choice[0] = ix->threads;
    choice[1] = ix->top_mode;
    choice[2] = ix->start_mode;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(ids);
    cudaFree(dists);
    cudaFree(counts);
    return rc;
}

int pdxg_search_with_order(pdxg_index* ix, const float* queries, uint32_t nq, uint32_t k,
                           const uint32_t* order, uint32_t n_order, uint32_t flags, uint32_t* ids,
                           float* distances, uint32_t* counts) {
    if (int rc = check_index(ix)) return rc;
    if (!order && n_order) return fail(PDXG_ERR_INVALID_ARGUMENT, "order is NULL");
    const uint32_t n1 = (uint32_t)ix->l1.fc.size();
    for (uint32_t i = 0; i < n_order; ++i)
        if (order[i] >= n1) return fail(PDXG_ERR_INVALID_ARGUMENT, "cluster id out of range in order");
    std::lock_guard<std::mutex> lock(ix->mu);
    const uint32_t saved = ix->nprobe;
    if (ix->tree && ix->nprobe == 0) ix->nprobe = n1;
    int rc = search_host_impl(ix, queries, nq, k, flags, order, n_order ? n_order : 0, nullptr,
                              nullptr, nullptr, ids, distances, counts);
    ix->nprobe = saved;
    return rc;
}

int pdxg_filtered_search_batch(pdxg_index* ix, const float* queries, uint32_t nq, uint32_t k,
                               const uint64_t* row_ids, const uint64_t* offsets, uint32_t flags,
                               uint32_t* ids, float* distances, uint32_t* counts) {
    if (int rc = check_index(ix)) return rc;
    if (!offsets) return fail(PDXG_ERR_INVALID_ARGUMENT, "offsets is NULL");
    std::lock_guard<std::mutex> lock(ix->mu);
    const uint32_t words = ix->l1.sel_words;
    const uint32_t ncl = (uint32_t)ix->l1.fc.size();
    std::vector<int32_t> filter_of(nq, -1);
    uint32_t nf = 0;
    for (uint32_t q = 0; q < nq; ++q)
        if (offsets[q] != UINT64_MAX) filter_of[q] = (int32_t)nf++;
    std::vector<uint32_t> sel((uint64_t)nf * words, 0), pass((uint64_t)nf * ncl, 0);
    for (uint32_t q = 0; q < nq; ++q) {
        if (filter_of[q] < 0) continue;
        uint64_t a = offsets[q], b = offsets[q + 1];
        if (b == UINT64_MAX) {
            // next query unfiltered: find the next valid end offset
            uint32_t j = q + 1;
            while (j < nq && offsets[j] == UINT64_MAX) ++j;
            b = offsets[j];
        }
        if (b < a) return fail(PDXG_ERR_INVALID_ARGUMENT, "offsets must be non-decreasing");
        if (!row_ids && b > a) return fail(PDXG_ERR_INVALID_ARGUMENT, "row_ids is NULL");
        const uint32_t f = (uint32_t)filter_of[q];
        build_filter(ix, row_ids + a, b - a, sel.data() + (uint64_t)f * words,
                     pass.data() + (uint64_t)f * ncl);
    }
    if (nf == 0)
        return search_host_impl(ix, queries, nq, k, flags, nullptr, 0, nullptr, nullptr, nullptr,
                                ids, distances, counts);
    return search_host_impl(ix, queries, nq, k, flags, nullptr, 0, &sel, &pass, &filter_of, ids,
                            distances, counts);
}

int pdxg_filtered_search(pdxg_index* ix, const float* query, uint32_t k, const uint64_t* row_ids,
                         uint64_t n_row_ids, uint32_t flags, uint32_t* ids, float* distances,
                         uint32_t* count) {
    const uint64_t offsets[2] = {0, n_row_ids};
    return pdxg_filtered_search_batch(ix, query, 1, k, row_ids, offsets, flags, ids, distances,
                                      count);
}

int pdxg_prepare_queries(pdxg_index* ix, const float* queries, uint32_t nq, float* out) {
    if (int rc = check_index(ix)) return rc;
    if (!queries || !out) return fail(PDXG_ERR_INVALID_ARGUMENT, "NULL buffer");
    std::lock_guard<std::mutex> lock(ix->mu);
    PDXG_CUDA(cudaSetDevice(ix->device));
    int rc = ensure_ws(ix, ix->ws, nq, 1);
    if (rc) return rc;
    cudaStream_t st = ix->stream;
    PDXG_CUDA(cudaMemcpyAsync(ix->ws.d_q, queries, sizeof(float) * nq * ix->d, cudaMemcpyHostToDevice, st));
    if ((rc = prepare_dev(ix, ix->ws, ix->ws.d_q, nq, ix->ws.d_rq, st))) return rc;
    PDXG_CUDA(cudaMemcpyAsync(out, ix->ws.d_rq, sizeof(float) * nq * ix->d, cudaMemcpyDeviceToHost, st));
    PDXG_CUDA(cudaStreamSynchronize(st));
    return check_gemm_error(ix->ws);
}

int pdxg_get_scan_stats(pdxg_index* ix, uint64_t out[4]) {
    if (int rc = check_index(ix)) return rc;
    if (!out) return fail(PDXG_ERR_INVALID_ARGUMENT, "out is NULL");
    std::lock_guard<std::mutex> lock(ix->mu);
    if (!ix->ws.d_stats) return fail(PDXG_ERR_INVALID_ARGUMENT, "no search ran with PDXG_COLLECT_STATS");
    PDXG_CUDA(cudaSetDevice(ix->device));
    PDXG_CUDA(cudaStreamSynchronize(ix->stats_stream ? ix->stats_stream : ix->stream));
    unsigned long long h[4];
    PDXG_CUDA(cudaMemcpy(h, ix->ws.d_stats + 12, sizeof(h), cudaMemcpyDeviceToHost));
    for (int i = 0; i < 4; ++i) out[i] = h[i];
    return PDXG_OK;
}

int pdxg_get_stats(pdxg_index* ix, uint64_t out[12]) {
    if (int rc = check_index(ix)) return rc;
    if (!out) return fail(PDXG_ERR_INVALID_ARGUMENT, "out is NULL");
    std::lock_guard<std::mutex> lock(ix->mu);
    if (!ix->ws.d_stats) return fail(PDXG_ERR_INVALID_ARGUMENT, "no search ran with PDXG_COLLECT_STATS");
    PDXG_CUDA(cudaSetDevice(ix->device));
    PDXG_CUDA(cudaStreamSynchronize(ix->stats_stream ? ix->stats_stream : ix->stream));
    unsigned long long h[12];
    PDXG_CUDA(cudaMemcpy(h, ix->ws.d_stats, sizeof(h), cudaMemcpyDeviceToHost));
    for (int i = 0; i < 12; ++i) out[i] = h[i];
    return PDXG_OK;
}

int pdxg_set_rotation_mode(pdxg_index* ix, uint32_t mode) {
    if (int rc = check_index(ix)) return rc;
    if (mode > 1) return fail(PDXG_ERR_INVALID_ARGUMENT, "rotation mode must be 0 or 1");
    std::lock_guard<std::mutex> lock(ix->mu);
    ix->rot_mode = mode;
    return PDXG_OK;
}

int pdxg_rotation_uses_tensor_cores(const pdxg_index* ix) { return ix && ix->rot_tc && ix->rot_mode == 0; }

uint32_t pdxg_last_launch_count(const pdxg_index* ix) { return ix ? ix->last_launches : 0; }

int pdxg_kernel_times(pdxg_index* ix, float out[3]) {
    float t[4];
    if (int rc = pdxg_kernel_times_ex(ix, t, 4)) return rc;
    out[0] = t[0];
    out[1] = t[1];
    out[2] = t[2] + t[3];
    return PDXG_OK;
}

int pdxg_kernel_times_ex(pdxg_index* ix, float* out, uint32_t n) {
    if (int rc = check_index(ix)) return rc;
    if (!out || n < 4) return fail(PDXG_ERR_INVALID_ARGUMENT, "out must hold 4 values");
    std::lock_guard<std::mutex> lock(ix->mu);
    if (!ix->tev_ready) return fail(PDXG_ERR_INVALID_ARGUMENT, "no search ran with PDXG_TIME_KERNELS");
    PDXG_CUDA(cudaSetDevice(ix->device));
    PDXG_CUDA(cudaEventSynchronize(ix->tev[4]));
    float t[4];
    for (int i = 0; i < 4; ++i) PDXG_CUDA(cudaEventElapsedTime(&t[i], ix->tev[i], ix->tev[i + 1]));
    out[0] = ix->tev_prep ? t[0] : 0.0f;
    out[1] = ix->tev_top ? t[1] : 0.0f;
    out[2] = t[2];
    out[3] = t[3];
    // finer: [4] scan prep (Start pushes, visit lists, items), [5] bitmaps, [6] replay, [7] per-query scan
    // kernel (all of the scan without the cluster-major form); [8] meso probe, [9] partials,
    // [10] top-level replay (tiled top level only)
    float f[7] = {0, 0, 0, 0, 0, 0, 0};
    if (ix->tev_scan) {
        PDXG_CUDA(cudaEventElapsedTime(&f[0], ix->tev[3], ix->tev[5]));
        PDXG_CUDA(cudaEventElapsedTime(&f[1], ix->tev[5], ix->tev[6]));
        PDXG_CUDA(cudaEventElapsedTime(&f[2], ix->tev[6], ix->tev[7]));
        PDXG_CUDA(cudaEventElapsedTime(&f[3], ix->tev[7], ix->tev[4]));
    } else {
        f[3] = t[3];
    }
    if (ix->tev_tiled && ix->tev_top) {
        PDXG_CUDA(cudaEventElapsedTime(&f[4], ix->tev[1], ix->tev[8]));
        PDXG_CUDA(cudaEventElapsedTime(&f[5], ix->tev[8], ix->tev[9]));
        PDXG_CUDA(cudaEventElapsedTime(&f[6], ix->tev[9], ix->tev[2]));
    }
    for (uint32_t i = 4; i < n && i < 11; ++i) out[i] = f[i - 4];
    return PDXG_OK;
}

int pdxg_index_type(const pdxg_index* ix) { return ix ? ix->type : -1; }
uint32_t pdxg_num_dimensions(const pdxg_index* ix) { return ix ? ix->d : 0; }
uint32_t pdxg_num_clusters(const pdxg_index* ix) { return ix ? (uint32_t)ix->l1.fc.size() : 0; }
uint32_t pdxg_nprobe(const pdxg_index* ix) { return ix ? ix->nprobe : 0; }
uint64_t pdxg_num_embeddings(const pdxg_index* ix) {
    if (!ix) return 0;
    return ix->maint ? ix->maint->live : ix->l1.total_vectors;
}

// GetClusterSize / GetClusterRowIds (index.hpp:768-782): tombstoned slots are left out.
uint32_t pdxg_cluster_size(const pdxg_index* ix, uint32_t cluster_id) {
    if (!ix || cluster_id >= ix->l1.n.size()) return 0;
    return ix->maint ? ix->maint->cl[cluster_id].num_embeddings : ix->l1.n[cluster_id];
}

int pdxg_cluster_row_ids(const pdxg_index* ix, uint32_t cluster_id, uint32_t* out,
                         uint32_t capacity) {
    if (int rc = check_index(ix)) return rc;
    if (cluster_id >= ix->l1.n.size()) return fail(PDXG_ERR_INVALID_ARGUMENT, "cluster_id out of range");
    const uint32_t n = pdxg_cluster_size(ix, cluster_id);
    if (capacity < n || (!out && n)) return fail(PDXG_ERR_INVALID_ARGUMENT, "output buffer too small");
    if (ix->maint) {
        const MaintCluster& K = ix->maint->cl[cluster_id];
        uint32_t j = 0;
        for (uint32_t i = 0; i < K.used; ++i)
            if (!K.tombstones.count(i)) out[j++] = K.indices[i];
        return PDXG_OK;
    }
    std::memcpy(out, ix->l1.ids.data() + ix->l1.ids_start[cluster_id], (size_t)n * 4);
    return PDXG_OK;
}

uint64_t pdxg_in_memory_size_in_bytes(const pdxg_index* ix) {
    if (!ix) return 0;
    uint64_t s = ix->arena_bytes;
    s += (ix->l1.meta.size() + ix->l0.meta.size()) * sizeof(DevCluster);
    s += (ix->l1.centroids.size() + ix->l0.centroids.size() + ix->rotation.size() + ix->d) * 4;
    return s;
}

int pdxg_save(pdxg_index* ix, const char* path) {
    if (int rc = check_index(ix)) return rc;
    if (!path) return fail(PDXG_ERR_INVALID_ARGUMENT, "path is NULL");
    std::lock_guard<std::mutex> lock(ix->mu);
    PDXG_CUDA(cudaSetDevice(ix->device));
    if (ix->maint) {
        std::lock_guard<std::mutex> reg_lock(ix->reg_mu);
        if (int rc = maint_prepare_save(ix)) return rc;
    }
    std::vector<uint8_t> img(ix->arena_bytes);
    PDXG_CUDA(cudaMemcpy(img.data(), ix->arena, ix->arena_bytes, cudaMemcpyDeviceToHost));
    std::ofstream out(path, std::ios::binary);
    if (!out) return fail(PDXG_ERR_IO, std::string("Failed to open file for writing: ") + path);
    auto w32 = [&](uint32_t v) { out.write(reinterpret_cast<const char*>(&v), 4); };
    const uint8_t type = (uint8_t)ix->type;
    out.write(reinterpret_cast<const char*>(&type), 1);
    w32(ix->rot_rows);
    w32(ix->rot_cols);
    out.write(reinterpret_cast<const char*>(ix->file_rotation.data()), ix->file_rotation.size() * 4);
    auto write_level = [&](const HostLevel& lv) {
        for (size_t i = 0; i < lv.meta.size(); ++i) {
            w32(lv.n[i]);
            w32(lv.max_cap[i]);
        }
        std::vector<uint8_t> tmp;
        for (size_t i = 0; i < lv.meta.size(); ++i) {
            const DevCluster& m = lv.meta[i];
            const uint64_t n = m.n, np = m.n_pad;
            if (!lv.u8) {
                for (uint32_t j = 0; j < lv.dv; ++j)
                    out.write(reinterpret_cast<const char*>(img.data() + m.vert_off + (uint64_t)j * np * 4), n * 4);
                for (uint32_t b = 0; b < lv.n_hblocks; ++b)
                    out.write(reinterpret_cast<const char*>(img.data() + m.hor_off + (uint64_t)b * np * kHDim * 4),
                              n * kHDim * 4);
            } else {
                const uint32_t full = lv.dv / 4, rem = lv.dv % 4;
                for (uint32_t g = 0; g < full; ++g)
                    out.write(reinterpret_cast<const char*>(img.data() + m.vert_off + (uint64_t)g * np * 4), n * 4);
                if (rem) {
                    tmp.assign(n * rem, 0);
                    const uint8_t* src = img.data() + m.vert_off + (uint64_t)full * np * 4;
                    for (uint64_t v = 0; v < n; ++v)
                        for (uint32_t t = 0; t < rem; ++t) tmp[v * rem + t] = src[v * 4 + t];
                    out.write(reinterpret_cast<const char*>(tmp.data()), tmp.size());
                }
                for (uint32_t b = 0; b < lv.n_hblocks; ++b)
                    out.write(reinterpret_cast<const char*>(img.data() + m.hor_off + (uint64_t)b * np * kHDim),
                              n * kHDim);
            }
        }
        for (size_t i = 0; i < lv.meta.size(); ++i)
            out.write(reinterpret_cast<const char*>(lv.ids.data() + lv.ids_start[i]), (size_t)lv.n[i] * 4);
    };
    w32(ix->d);
    w32(ix->dv);
    w32(ix->dh);
    w32((uint32_t)ix->l1.meta.size());
    if (ix->tree) {
        w32((uint32_t)ix->l0.meta.size());
        write_level(ix->l0);
    }
    write_level(ix->l1);
    const uint8_t norm = ix->normalized ? 1 : 0;
    out.write(reinterpret_cast<const char*>(&norm), 1);
    const std::vector<float>& cent = ix->tree ? ix->l0.centroids : ix->l1.centroids;
    out.write(reinterpret_cast<const char*>(cent.data()), cent.size() * 4);
    if (ix->u8) {
        out.write(reinterpret_cast<const char*>(&ix->base), 4);
        out.write(reinterpret_cast<const char*>(&ix->scale), 4);
    }
    if (!out) return fail(PDXG_ERR_IO, std::string("Failed to write file: ") + path);
    return PDXG_OK;
}

}  // extern "C"

// =============================================================================== request batches
// Serving-style batches: every query carries its own k, nprobe and optional row-id filter.
// A context owns one workspace and one stream, so batches issued on different contexts run
// concurrently on the GPU without sharing scratch.

struct pdxg_context {
    pdxg_index* ix = nullptr;
    Workspace ws;
    cudaStream_t stream = nullptr;
    cudaEvent_t staged = nullptr;   // the previous call's host-to-device copies are done
    bool staged_pending = false;
    uint8_t* h_stage = nullptr;     // pinned staging of the per-query parameters and rows
    size_t h_cap = 0;
    std::mutex mu;
};

namespace {

// One bit per cluster slot: filter f selects row r when bit pos(r) of cluster(r) is set;
// passing[f][c] counts distinct selected rows (CreatePredicateEvaluator, index.hpp:436-446).
__global__ void build_filters_kernel(const uint32_t* __restrict__ rows,
                                     const unsigned long long* __restrict__ foff, uint32_t nf,
                                     const uint32_t* __restrict__ rid_cluster,
                                     const uint32_t* __restrict__ rid_pos, uint64_t n_rows,
                                     const DevCluster* __restrict__ clusters, uint32_t words,
                                     uint32_t ncl, uint32_t* sel, uint32_t* passing) {
    const uint32_t f = blockIdx.y;
    if (f >= nf) return;
    const unsigned long long a = foff[f], b = foff[f + 1];
    for (unsigned long long i = a + blockIdx.x * blockDim.x + threadIdx.x; i < b;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint32_t r = rows[i];
        if (r >= n_rows) continue;
        const uint32_t c = rid_cluster[r];
        if (c == 0xFFFFFFFFu) continue;
        const uint32_t pos = rid_pos[r];
        const uint32_t bit = 1u << (pos & 31);
        const uint32_t old = atomicOr(sel + (size_t)f * words + clusters[c].sel_word + (pos >> 5), bit);
        if (!(old & bit)) atomicAdd(passing + (size_t)f * ncl + c, 1u);
    }
}

int stage_grow(pdxg_context* ctx, size_t need) {
    if (need <= ctx->h_cap) return PDXG_OK;
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    ctx->h_stage = nullptr;
    ctx->h_cap = 0;
    PDXG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&ctx->h_stage), need, cudaHostAllocDefault));
    ctx->h_cap = need;
    return PDXG_OK;
}

}  // namespace

extern "C" {

int pdxg_context_create(pdxg_index* ix, pdxg_context** out) {
    if (int rc = check_index(ix)) return rc;
    if (!out) return fail(PDXG_ERR_INVALID_ARGUMENT, "out is NULL");
    PDXG_CUDA(cudaSetDevice(ix->device));
    auto* ctx = new pdxg_context();
    ctx->ix = ix;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->staged, cudaEventDisableTiming) != cudaSuccess) {
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return fail(PDXG_ERR_CUDA, "cannot create the context's stream");
    }
    *out = ctx;
    return PDXG_OK;
}

void pdxg_context_free(pdxg_context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->ix->device);
    cudaStreamSynchronize(ctx->stream);
    free_workspace(ctx->ws);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    cudaEventDestroy(ctx->staged);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

void* pdxg_context_stream(pdxg_context* ctx) { return ctx ? ctx->stream : nullptr; }

int pdxg_search_requests(pdxg_context* ctx, const float* queries, uint32_t nq,
                         const pdxg_request* requests, const uint32_t* rows, uint32_t k_max,
                         uint32_t flags, uint32_t* ids, float* distances, uint32_t* counts) {
    if (!ctx) return fail(PDXG_ERR_INVALID_ARGUMENT, "context is NULL");
    pdxg_index* ix = ctx->ix;
    if (!queries || !requests || !ids || !distances || !counts)
        return fail(PDXG_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (flags & PDXG_COLLECT_STATS) return fail(PDXG_ERR_INVALID_ARGUMENT, "stats are not collected here");
    std::lock_guard<std::mutex> lock(ctx->mu);
    PDXG_CUDA(cudaSetDevice(ix->device));
    cudaStream_t st = ctx->stream;
    if (nq == 0) return PDXG_OK;
    // the registry cannot grow (and move) between the checks below and the launch
    std::lock_guard<std::mutex> reg_lock(ix->reg_mu);
    if (int rc = refresh_registered_filters(ix)) return rc;
    if (int rc = flush_maintenance(ix, st)) return rc;  // the filters' device row maps
    // resolve every query's parameters as PDXearch / PDXTreeIndex::Search would
    const uint32_t n1 = (uint32_t)ix->l1.fc.size();
    const uint32_t n0 = (uint32_t)ix->l0.fc.size();
    uint32_t np_max = 1, top_max = 0, nf = 0;
    uint64_t nrows = 0;
    bool any_filter = false, any_plain = false;
    for (uint32_t q = 0; q < nq; ++q) {
        const pdxg_request& r = requests[q];
        if (r.k == 0 || r.k > k_max) return fail(PDXG_ERR_INVALID_ARGUMENT, "request k must be in [1, k_max]");
        if (r.filter_id >= 0) {
            if ((uint32_t)r.filter_id >= ix->reg_cap || !ix->reg_used[r.filter_id])
                return fail(PDXG_ERR_INVALID_ARGUMENT, "unknown filter id " + std::to_string(r.filter_id));
            any_filter = true;
        } else if (r.filter_id != -1) {
            return fail(PDXG_ERR_INVALID_ARGUMENT, "filter_id must be -1 or a registered filter");
        } else if (r.filter_begin != UINT64_MAX) {
            if (r.filter_end < r.filter_begin) return fail(PDXG_ERR_INVALID_ARGUMENT, "bad filter range");
            if (r.filter_end > r.filter_begin && !rows) return fail(PDXG_ERR_INVALID_ARGUMENT, "rows is NULL");
            ++nf;
            nrows += r.filter_end - r.filter_begin;
            any_filter = true;
        } else {
            any_plain = true;
        }
    }
    // pinned staging: q_k, q_np, q_top, filter_of (nq each), filter offsets (nf + 1), rows
    const size_t req_bytes = (size_t)nq * 16, foff_bytes = ((size_t)nf + 1) * 8, row_bytes = nrows * 4;
    if (ctx->staged_pending) PDXG_CUDA(cudaEventSynchronize(ctx->staged));
    int rc = stage_grow(ctx, req_bytes + foff_bytes + row_bytes + 64);
    if (rc) return rc;
    uint32_t* h_req = reinterpret_cast<uint32_t*>(ctx->h_stage);
    unsigned long long* h_foff = reinterpret_cast<unsigned long long*>(ctx->h_stage + req_bytes);
    uint32_t* h_rows = reinterpret_cast<uint32_t*>(ctx->h_stage + req_bytes + foff_bytes);
    uint32_t f = 0;
    unsigned long long pos = 0;
    for (uint32_t q = 0; q < nq; ++q) {
        const pdxg_request& r = requests[q];
        const uint32_t npf = (r.nprobe == 0 || r.nprobe > n1) ? n1 : r.nprobe;
        uint32_t top = 0;
        if (ix->tree) {
            top = n0;
            if ((r.nprobe == 0 ? n1 : r.nprobe) < n1 / 2) top /= 2;
        }
        h_req[q] = r.k;
        h_req[nq + q] = npf;
        h_req[2 * nq + q] = top;
        np_max = std::max(np_max, npf);
        top_max = std::max(top_max, top);
        if (r.filter_id >= 0) {
            h_req[3 * nq + q] = (uint32_t)(-2 - r.filter_id);
        } else if (r.filter_begin != UINT64_MAX) {
            h_req[3 * nq + q] = f;
            h_foff[f] = pos;
            const uint64_t len = r.filter_end - r.filter_begin;
            const uint32_t* src = rows + r.filter_begin;
            std::memcpy(h_rows + pos, src, len * 4);
            pos += len;
            ++f;
        } else {
            h_req[3 * nq + q] = 0xFFFFFFFFu;  // -1: unfiltered
        }
    }
    h_foff[nf] = pos;
    Workspace& w = ctx->ws;
    if ((rc = ensure_ws(ix, w, nq, k_max))) return rc;
    if ((rc = dev_grow(w.d_req, w.req_cap, (uint64_t)nq * 4))) return rc;
    if ((rc = dev_grow(w.d_foff, w.foff_cap, (uint64_t)nf + 1))) return rc;
    if ((rc = dev_grow(w.d_rows, w.rows_cap, std::max<uint64_t>(nrows, 1)))) return rc;
    PDXG_CUDA(cudaMemcpyAsync(w.d_req, h_req, req_bytes, cudaMemcpyHostToDevice, st));
    if (nf) {
        PDXG_CUDA(cudaMemcpyAsync(w.d_foff, h_foff, foff_bytes, cudaMemcpyHostToDevice, st));
        if (nrows) PDXG_CUDA(cudaMemcpyAsync(w.d_rows, h_rows, row_bytes, cudaMemcpyHostToDevice, st));
    }
    PDXG_CUDA(cudaEventRecord(ctx->staged, st));
    ctx->staged_pending = true;
    const uint32_t words = ix->l1.sel_words;
    if (nf) {
        if ((rc = dev_grow(w.d_sel, w.sel_cap, (uint64_t)nf * words))) return rc;
        if ((rc = dev_grow(w.d_pass, w.pass_cap, (uint64_t)nf * n1))) return rc;
        PDXG_CUDA(cudaMemsetAsync(w.d_sel, 0, (size_t)nf * words * 4, st));
        PDXG_CUDA(cudaMemsetAsync(w.d_pass, 0, (size_t)nf * n1 * 4, st));
        uint64_t max_len = 0;
        for (uint32_t i = 0; i < nf; ++i) max_len = std::max<uint64_t>(max_len, h_foff[i + 1] - h_foff[i]);
        dim3 grid((uint32_t)std::min<uint64_t>((max_len + 255) / 256 + 1, 64), nf);
        build_filters_kernel<<<grid, 256, 0, st>>>(w.d_rows, w.d_foff, nf, ix->d_rid_cluster, ix->d_rid_pos,
                                                   ix->rid_cluster.size(), ix->d_cl1, words, n1, w.d_sel,
                                                   w.d_pass);
        PDXG_CUDA(cudaGetLastError());
    }
    const float* qp = queries;
    const bool gemm_probe = ix->probe_mode != 0 && probe_gemm_ok(ix);
    if (!(flags & PDXG_QUERY_TRANSFORMED) && !gemm_probe) {
        if ((rc = prepare_dev(ix, w, queries, nq, w.d_rq, st))) return rc;
        qp = w.d_rq;
    }
    Launch L;
    if ((rc = plan_search(ix, nq, k_max, 0, any_filter, L, np_max, top_max, false, st))) return rc;
    L.p.queries = qp;
    L.p.q_k = w.d_req;
    L.p.q_nprobe = w.d_req + nq;
    L.p.q_top = w.d_req + 2 * nq;
    if (any_filter) {
        L.p.filter_of = reinterpret_cast<const int32_t*>(w.d_req + 3 * nq);
        L.p.sel_bits = nf ? w.d_sel : nullptr;
        L.p.passing = nf ? w.d_pass : nullptr;
        L.p.reg_sel = ix->d_reg_sel;
        L.p.reg_pass = ix->d_reg_pass;
    }
    L.p.out_ids = ids;
    L.p.out_dists = distances;
    L.p.out_counts = counts;
    L.p.queue = w.d_queue;
    if (gemm_probe) {
        if ((rc = run_probe_gemm(ix, w, queries, nq, (flags & PDXG_QUERY_TRANSFORMED) != 0, L, st))) return rc;
        qp = L.p.queries;
        if ((rc = run_start_batched(ix, w, qp, nq, L, st))) return rc;
    } else if (ix->tree && any_plain) {
        if ((rc = run_top_level(ix, w, qp, nq, L, st))) return rc;
        if ((rc = run_start_batched(ix, w, qp, nq, L, st))) return rc;
    }
    if ((rc = run_scan_cluster_major(ix, w, nq, L, st))) return rc;
    PDXG_CUDA(cudaMemsetAsync(w.d_queue, 0, sizeof(uint32_t), st));
    PDXG_CUDA(launch_search(L.p, L.u8, L.threads, L.grid, st));
    return PDXG_OK;
}

int pdxg_filter_register(pdxg_index* ix, const uint64_t* row_ids, uint64_t n, int32_t* filter_id) {
    if (int rc = check_index(ix)) return rc;
    if (!filter_id) return fail(PDXG_ERR_INVALID_ARGUMENT, "filter_id is NULL");
    if (n && !row_ids) return fail(PDXG_ERR_INVALID_ARGUMENT, "row_ids is NULL");
    std::lock_guard<std::mutex> lock(ix->reg_mu);
    PDXG_CUDA(cudaSetDevice(ix->device));
    if (int rc = refresh_registered_filters(ix)) return rc;
    const uint32_t words = ix->l1.sel_words;
    const uint32_t n1 = (uint32_t)ix->l1.fc.size();
    uint32_t slot = 0;
    while (slot < ix->reg_cap && ix->reg_used[slot]) ++slot;
    if (slot == ix->reg_cap) {
        if (ix->reg_cap >= (1u << 30)) return fail(PDXG_ERR_CAPACITY, "too many registered filters");
        const uint32_t cap = std::max(8u, ix->reg_cap * 2);
        uint32_t *sel = nullptr, *pass = nullptr;
        if (cudaMalloc(&sel, (size_t)cap * words * 4) != cudaSuccess ||
            cudaMalloc(&pass, (size_t)cap * n1 * 4) != cudaSuccess) {
            cudaFree(sel);
            return fail(PDXG_ERR_CUDA, "cannot grow the filter pool");
        }
        // batches already enqueued may still read the old pool: finish them before freeing it
        PDXG_CUDA(cudaDeviceSynchronize());
        if (ix->reg_cap) {
            PDXG_CUDA(cudaMemcpy(sel, ix->d_reg_sel, (size_t)ix->reg_cap * words * 4, cudaMemcpyDeviceToDevice));
            PDXG_CUDA(cudaMemcpy(pass, ix->d_reg_pass, (size_t)ix->reg_cap * n1 * 4, cudaMemcpyDeviceToDevice));
        }
        cudaFree(ix->d_reg_sel);
        cudaFree(ix->d_reg_pass);
        ix->d_reg_sel = sel;
        ix->d_reg_pass = pass;
        ix->reg_cap = cap;
        ix->reg_used.resize(cap, 0);
        ix->reg_rows.resize(cap);
    }
    std::vector<uint32_t> sel(words, 0), pass(n1, 0);
    build_filter(ix, row_ids, n, sel.data(), pass.data());
    PDXG_CUDA(cudaMemcpy(ix->d_reg_sel + (size_t)slot * words, sel.data(), (size_t)words * 4,
                         cudaMemcpyHostToDevice));
    PDXG_CUDA(cudaMemcpy(ix->d_reg_pass + (size_t)slot * n1, pass.data(), (size_t)n1 * 4,
                         cudaMemcpyHostToDevice));
    ix->reg_used[slot] = 1;
    if (ix->tree) ix->reg_rows[slot].assign(row_ids, row_ids + n);  // rebuilt after Append / Delete
    *filter_id = (int32_t)slot;
    return PDXG_OK;
}

int pdxg_filter_release(pdxg_index* ix, int32_t filter_id) {
    if (int rc = check_index(ix)) return rc;
    std::lock_guard<std::mutex> lock(ix->reg_mu);
    if (filter_id < 0 || (uint32_t)filter_id >= ix->reg_cap || !ix->reg_used[filter_id])
        return fail(PDXG_ERR_INVALID_ARGUMENT, "unknown filter id " + std::to_string(filter_id));
    ix->reg_used[filter_id] = 0;
    ix->reg_rows[filter_id].clear();
    ix->reg_rows[filter_id].shrink_to_fit();
    return PDXG_OK;
}

}  // extern "C"

