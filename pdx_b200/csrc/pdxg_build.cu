// Index build on the GPU (BuildIndex of the reference, index.hpp:329-403 / 640-758, with its own
// clustering in place of the SuperKMeans submodule).
//
//   1. NormalizeQuery + the rotation y = x M of every row (the FP32 SIMT GEMM of the query path).
//   2. SQ8 parameters from the global min / max of the rotated data (scalar.hpp:60-74).
//   3. Lloyd k-means on the rotated rows: assignment = argmin over |c|^2 - 2 x.c from a BF16
//      tensor-core GEMM (FP32 accumulation), update = one block per centroid summing its rows in
//      FP64 in row-id order (a build is reproducible); spherical (unit centroids) for normalized
//      data, empty clusters re-seeded from seeded random rows. Tree indexes cluster the L1
//      centroids again into meso clusters.
//   4. QuantizeEmbedding (U8) and the compact PDX block of every cluster (StoreClusterEmbeddings,
//      layout.hpp:12-87: vertical dims dimension-major, U8 in groups of 4 interleaved bytes,
//      64-dim horizontal blocks row-major), written by one kernel into the file's data region.
//   5. The reference's Save format assembled on the host, then loaded as any other file.
// Rows stay in row-id order inside each cluster.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/pdx_b200.h"
#include "pdxg_common.cuh"
#include "pdxg_gemm.cuh"

namespace pdxg {
cudaError_t launch_prepare_queries(const float* q, uint32_t nq, uint32_t d, const float* rotation,
                                   bool normalize, float* norms_ws, float* out, cudaStream_t st);
cudaError_t launch_row_sq(const float* x, uint32_t n, uint32_t d, float* out, cudaStream_t st);
}  // namespace pdxg

int pdxg_set_error(int code, const char* msg);
void pdxg_split_dims(uint32_t d, uint32_t& h, uint32_t& v);

namespace pdxg {
namespace {

__device__ __forceinline__ uint32_t ordered_key(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ inline float key_to_float(uint32_t k) {
    const uint32_t b = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

__global__ void minmax_kernel(const float* __restrict__ x, uint64_t n, uint32_t* __restrict__ mm) {
    uint32_t lo = 0xFFFFFFFFu, hi = 0u;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = ordered_key(x[i]);
        lo = min(lo, k);
        hi = max(hi, k);
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mm, lo);
        atomicMax(mm + 1, hi);
    }
}

// assign[row0 + r] = the column of the smallest score of row r (lowest column on ties); one
// warp per row.
__global__ void argmin_rows_kernel(const float* __restrict__ s, uint32_t rows, uint32_t k, uint32_t row0,
                                   uint32_t* __restrict__ assign) {
    const uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (r >= rows) return;
    const float* row = s + (size_t)r * k;
    float best = INFINITY;
    uint32_t bi = 0xFFFFFFFFu;
    for (uint32_t j = lane; j < k; j += 32) {
        const float v = row[j];
        if (v < best || (v == best && j < bi)) {
            best = v;
            bi = j;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, o);
        const uint32_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob < best || (ob == best && oi < bi)) {
            best = ob;
            bi = oi;
        }
    }
    if (lane == 0) assign[row0 + r] = bi == 0xFFFFFFFFu ? 0u : bi;
}

// One block per centroid: the mean of its rows (summed in FP64 in row-id order, so a build is
// reproducible) or, where src_rows names one, that row (initial centroids and re-seeded empty
// clusters); unit length for spherical k-means.
__global__ void centroid_update_kernel(const float* __restrict__ x, const uint32_t* __restrict__ order,
                                       const uint32_t* __restrict__ start, const uint32_t* __restrict__ src_rows,
                                       uint32_t d, int angular, float* __restrict__ c) {
    __shared__ float red[32];
    const uint32_t ci = blockIdx.x;
    float* row = c + (size_t)ci * d;
    const uint32_t src = src_rows[ci];
    const uint32_t r0 = src == 0xFFFFFFFFu ? start[ci] : 0, r1 = src == 0xFFFFFFFFu ? start[ci + 1] : 0;
    const double inv = r1 > r0 ? 1.0 / (double)(r1 - r0) : 0.0;
    float ss = 0.0f;
    for (uint32_t j = threadIdx.x; j < d; j += blockDim.x) {
        float v;
        if (src != 0xFFFFFFFFu) {
            v = x[(size_t)src * d + j];
        } else {
            double s = 0.0;
            for (uint32_t r = r0; r < r1; ++r) s += (double)x[(size_t)order[r] * d + j];
            v = (float)(s * inv);
        }
        row[j] = v;
        ss = __fmaf_rn(v, v, ss);
    }
    if (!angular) return;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
    __syncthreads();
    if (threadIdx.x < 32) {
        float t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (threadIdx.x == 0) red[0] = fmaxf(sqrtf(t), 1e-30f);
    }
    __syncthreads();
    const float nrm = red[0];
    for (uint32_t j = threadIdx.x; j < d; j += blockDim.x) row[j] = __fdiv_rn(row[j], nrm);
}

// QuantizeEmbedding (scalar.hpp:76-94): clamp(round((x - base) * scale), 0, 255).
__global__ void quantize_kernel(const float* __restrict__ x, uint64_t n, float base, float scale, uint8_t* __restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const int r = (int)roundf(__fmul_rn(__fsub_rn(x[i], base), scale));
        out[i] = (uint8_t)(r > 255 ? 255 : (r < 0 ? 0 : r));
    }
}

// Compact PDX blocks: element j of row perm[p] (cluster cl[p], position pos[p] of ncl[cl[p]])
// goes to its place in the cluster's block at blob + blob_off[cluster] (cluster.hpp:185-221).
__global__ void layout_kernel(const uint8_t* __restrict__ src, uint32_t esz, const uint32_t* __restrict__ perm,
                              const uint32_t* __restrict__ cl, const uint32_t* __restrict__ pos,
                              const uint32_t* __restrict__ ncl, const uint64_t* __restrict__ blob_off, uint64_t n,
                              uint32_t d, uint32_t dv, uint8_t* __restrict__ blob) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < n * d; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p = e / d;
        const uint32_t j = (uint32_t)(e - p * d);
        const uint32_t c = cl[p], i = pos[p];
        const uint64_t nc = ncl[c];
        uint64_t off;  // in elements
        if (j >= dv) {
            const uint32_t b = (j - dv) / kHDim, t = (j - dv) % kHDim;
            off = (uint64_t)dv * nc + (uint64_t)b * nc * kHDim + (uint64_t)i * kHDim + t;
        } else if (esz == 4) {
            off = (uint64_t)j * nc + i;
        } else {
            const uint32_t full = dv & ~3u;
            if (j < full) off = (uint64_t)(j & ~3u) * nc + (uint64_t)i * 4 + (j & 3u);
            else off = (uint64_t)full * nc + (uint64_t)i * (dv - full) + (j - full);
        }
        const uint8_t* s = src + ((uint64_t)perm[p] * d + j) * esz;
        uint8_t* t = blob + blob_off[c] + off * esz;
        for (uint32_t b = 0; b < esz; ++b) t[b] = s[b];
    }
}

int err(int code, const std::string& msg) { return pdxg_set_error(code, msg.c_str()); }

#define BCHK(x)                                                                          \
    do {                                                                                 \
        cudaError_t e_ = (x);                                                            \
        if (e_ != cudaSuccess) return err(PDXG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Device buffers of one build, freed on every exit path.
struct Bufs {
    std::vector<void*> ptrs;
    template <class T>
    cudaError_t alloc(T*& p, uint64_t count) {
        cudaError_t e = cudaMalloc(&p, std::max<uint64_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(p);
        return e;
    }
    ~Bufs() {
        for (void* p : ptrs) cudaFree(p);
    }
};

uint32_t grid_for(uint64_t work, uint32_t threads) {
    return (uint32_t)std::min<uint64_t>((work + threads - 1) / threads, 148ull * 32);
}

// Stable grouping of n items by their cluster: counts, and the items in (cluster, item) order.
void group_rows(const std::vector<uint32_t>& assign, uint32_t k, std::vector<uint32_t>& counts,
                std::vector<uint32_t>& order) {
    counts.assign(k, 0);
    for (uint32_t a : assign) counts[a]++;
    std::vector<uint64_t> start(k + 1, 0);
    for (uint32_t c = 0; c < k; ++c) start[c + 1] = start[c] + counts[c];
    order.resize(assign.size());
    std::vector<uint64_t> fill(start.begin(), start.end() - 1);
    for (uint64_t i = 0; i < assign.size(); ++i) order[fill[assign[i]]++] = (uint32_t)i;
}

// Lloyd k-means of x (n rows, device) into k centroids c (device, k x d) and assign (device, n):
// iters updates, iters + 1 assignments. Reproducible for a given seed.
int kmeans(const float* x, uint64_t n, uint32_t d, uint32_t k, uint32_t iters, uint64_t seed, bool angular,
           float* c, uint32_t* assign, cudaStream_t st) {
    Bufs b;
    uint16_t *xb = nullptr, *cb = nullptr;
    float *csq = nullptr, *scores = nullptr;
    uint32_t *order = nullptr, *start = nullptr, *src = nullptr;
    int* gerr = nullptr;
    const uint64_t chunk = std::max<uint64_t>(128, std::min<uint64_t>(n, (256ull << 20) / ((uint64_t)k * 4)));
    BCHK(b.alloc(xb, n * d));
    BCHK(b.alloc(cb, (uint64_t)k * d));
    BCHK(b.alloc(csq, k));
    BCHK(b.alloc(scores, chunk * k));
    BCHK(b.alloc(order, n));
    BCHK(b.alloc(start, (uint64_t)k + 1));
    BCHK(b.alloc(src, k));
    BCHK(b.alloc(gerr, 1));
    BCHK(cudaMemsetAsync(gerr, 0, sizeof(int), st));
    BCHK(cudaMemsetAsync(start, 0, ((size_t)k + 1) * 4, st));
    BCHK(launch_bf16_rows(x, (uint32_t)n, d, false, xb, st));
    std::mt19937_64 rng(seed * 0x9E3779B97F4A7C15ull + 104729u);
    // initial centroids: k distinct rows (partial Fisher-Yates over the row ids)
    std::vector<uint32_t> src_rows(k);
    {
        std::vector<uint32_t> idx(n);
        for (uint64_t i = 0; i < n; ++i) idx[i] = (uint32_t)i;
        for (uint32_t i = 0; i < k; ++i) {
            std::uniform_int_distribution<uint64_t> u(i, n - 1);
            std::swap(idx[i], idx[u(rng)]);
            src_rows[i] = idx[i];
        }
    }
    BCHK(cudaMemcpyAsync(src, src_rows.data(), (size_t)k * 4, cudaMemcpyHostToDevice, st));
    centroid_update_kernel<<<k, 256, 0, st>>>(x, order, start, src, d, angular ? 1 : 0, c);
    BCHK(cudaGetLastError());
    GemmOperand cop;
    if (make_gemm_operand(cop, kGemmBF16, cb, nullptr, k, d) != 0)
        return err(PDXG_ERR_CUDA, "cannot encode the centroid tensor map");
    std::vector<uint32_t> h_assign(n), counts, h_order, h_start(k + 1);
    for (uint32_t it = 0; it <= iters; ++it) {
        BCHK(launch_bf16_rows(c, k, d, false, cb, st));
        BCHK(launch_row_sq(c, k, d, csq, st));
        for (uint64_t r0 = 0; r0 < n; r0 += chunk) {
            const uint32_t rows = (uint32_t)std::min<uint64_t>(chunk, n - r0);
            GemmOperand aop;
            if (make_gemm_operand(aop, kGemmBF16, xb + r0 * d, nullptr, rows, d) != 0)
                return err(PDXG_ERR_CUDA, "cannot encode the data tensor map");
            GemmArgs g{};
            g.M = rows;
            g.N = k;
            g.K = d;
            g.out = scores;
            g.ldo = k;
            g.col_add = csq;
            g.error = gerr;
            BCHK(launch_gemm(aop, cop, kEpiDist, g, st));
            argmin_rows_kernel<<<(rows * 32 + 255) / 256, 256, 0, st>>>(scores, rows, k, (uint32_t)r0, assign);
            BCHK(cudaGetLastError());
        }
        if (it == iters) break;
        BCHK(cudaMemcpyAsync(h_assign.data(), assign, n * 4, cudaMemcpyDeviceToHost, st));
        BCHK(cudaStreamSynchronize(st));
        group_rows(h_assign, k, counts, h_order);
        std::uniform_int_distribution<uint64_t> u(0, n - 1);
        h_start[0] = 0;
        for (uint32_t i = 0; i < k; ++i) {
            h_start[i + 1] = h_start[i] + counts[i];
            src_rows[i] = counts[i] ? 0xFFFFFFFFu : (uint32_t)u(rng);
        }
        BCHK(cudaMemcpyAsync(order, h_order.data(), n * 4, cudaMemcpyHostToDevice, st));
        BCHK(cudaMemcpyAsync(start, h_start.data(), ((size_t)k + 1) * 4, cudaMemcpyHostToDevice, st));
        BCHK(cudaMemcpyAsync(src, src_rows.data(), (size_t)k * 4, cudaMemcpyHostToDevice, st));
        centroid_update_kernel<<<k, 256, 0, st>>>(x, order, start, src, d, angular ? 1 : 0, c);
        BCHK(cudaGetLastError());
    }
    int h = 0;
    BCHK(cudaMemcpyAsync(&h, gerr, sizeof(int), cudaMemcpyDeviceToHost, st));
    BCHK(cudaStreamSynchronize(st));
    if (h) return err(PDXG_ERR_CUDA, "tensor-core GEMM gave up waiting (code " + std::to_string(h) + ")");
    return PDXG_OK;
}

void put_u32(std::vector<uint8_t>& out, uint32_t v) {
    const uint8_t* p = reinterpret_cast<const uint8_t*>(&v);
    out.insert(out.end(), p, p + 4);
}
void put_bytes(std::vector<uint8_t>& out, const void* p, size_t n) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    out.insert(out.end(), b, b + n);
}
uint32_t max_capacity(uint32_t n) {  // cluster.hpp:22-33
    return std::max<uint32_t>((uint32_t)((float)n * 1.3f), 256u);
}

// One level in the file's layout from row-major host vectors (F32): headers, blocks, ids.
void write_level_host(std::vector<uint8_t>& out, const std::vector<float>& rows, uint32_t d, uint32_t dv,
                      const std::vector<uint32_t>& counts, const std::vector<uint32_t>& order) {
    for (uint32_t c : counts) {
        put_u32(out, c);
        put_u32(out, max_capacity(c));
    }
    uint64_t s = 0;
    for (uint32_t nc : counts) {
        const uint32_t* ids = order.data() + s;
        for (uint32_t j = 0; j < dv; ++j)
            for (uint32_t i = 0; i < nc; ++i) put_bytes(out, &rows[(size_t)ids[i] * d + j], 4);
        for (uint32_t b0 = dv; b0 < d; b0 += kHDim)
            for (uint32_t i = 0; i < nc; ++i) put_bytes(out, &rows[(size_t)ids[i] * d + b0], (size_t)kHDim * 4);
        s += nc;
    }
    put_bytes(out, order.data(), order.size() * 4);
}

}  // namespace
}  // namespace pdxg

using namespace pdxg;

extern "C" int pdxg_build(const float* data, uint64_t n, uint32_t d, uint32_t index_type, uint32_t num_clusters,
                          uint32_t num_meso_clusters, int normalize, const float* rotation, uint64_t seed,
                          uint32_t kmeans_iters, int device, pdxg_index** out) {
    if (!data || !rotation || !out) return err(PDXG_ERR_INVALID_ARGUMENT, "NULL argument");
    if (index_type > 3) return err(PDXG_ERR_INVALID_ARGUMENT, "index type must be 0..3");
    if (d == 0 || d > (uint32_t)kMaxDims) return err(PDXG_ERR_INVALID_ARGUMENT, "num_dimensions out of range");
    if (n == 0 || n > 0xFFFFFFFFull) return err(PDXG_ERR_INVALID_ARGUMENT, "number of embeddings out of range");
    const bool tree = index_type >= 2, u8 = index_type == 1 || index_type == 3;
    uint32_t k = num_clusters;
    if (k == 0) {  // ComputeNumberOfClusters (common.hpp:191-199)
        const double sq = std::sqrt((double)n);
        k = (uint32_t)std::ceil((n < 500000 ? 2.0 : (n < 2500000 ? 4.0 : 8.0)) * sq);
    }
    if (k > n) return err(PDXG_ERR_INVALID_ARGUMENT, "num_clusters exceeds the number of embeddings");
    uint32_t k0 = 0;
    if (tree) {
        k0 = num_meso_clusters ? num_meso_clusters : (uint32_t)std::sqrt((double)k);
        if (k0 == 0 || k0 >= k) return err(PDXG_ERR_INVALID_ARGUMENT, "num_meso_clusters must be in [1, num_clusters)");
    }
    if (!gemm_available() || !gemm_shape_ok(kGemmBF16, d) || d % 8)
        return err(PDXG_ERR_UNSUPPORTED, "the GPU build needs tensor cores and d a multiple of 8");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return err(PDXG_ERR_CUDA, "no usable CUDA device");
    BCHK(cudaSetDevice(device));
    uint32_t dh = 0, dv = 0;
    pdxg_split_dims(d, dh, dv);
    cudaStream_t st = nullptr;
    BCHK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{st};
    Bufs b;
    float *x = nullptr, *rot = nullptr, *norms = nullptr, *r = nullptr, *cent = nullptr;
    uint32_t *assign = nullptr, *mm = nullptr;
    BCHK(b.alloc(x, n * d));
    BCHK(b.alloc(rot, (uint64_t)d * d));
    BCHK(b.alloc(norms, n));
    BCHK(b.alloc(r, n * d));
    BCHK(b.alloc(cent, (uint64_t)k * d));
    BCHK(b.alloc(assign, n));
    BCHK(b.alloc(mm, 2));
    BCHK(cudaMemcpyAsync(x, data, n * d * 4, cudaMemcpyHostToDevice, st));
    BCHK(cudaMemcpyAsync(rot, rotation, (size_t)d * d * 4, cudaMemcpyHostToDevice, st));
    // 1. normalize + rotate (grid rows of 128: at most 65535 x 128 rows per launch)
    for (uint64_t r0 = 0; r0 < n; r0 += 4194304) {
        const uint32_t rows = (uint32_t)std::min<uint64_t>(4194304, n - r0);
        BCHK(launch_prepare_queries(x + r0 * d, rows, d, rot, normalize != 0, norms + r0, r + r0 * d, st));
    }
    // 2. SQ8 parameters (scalar.hpp:60-74)
    float base = 0.0f, scale = 1.0f;
    if (u8) {
        const uint32_t init_mm[2] = {0xFFFFFFFFu, 0u};
        BCHK(cudaMemcpyAsync(mm, init_mm, 8, cudaMemcpyHostToDevice, st));
        minmax_kernel<<<grid_for(n * d, 256), 256, 0, st>>>(r, n * d, mm);
        BCHK(cudaGetLastError());
        uint32_t hmm[2];
        BCHK(cudaMemcpyAsync(hmm, mm, 8, cudaMemcpyDeviceToHost, st));
        BCHK(cudaStreamSynchronize(st));
        const float lo = key_to_float(hmm[0]), hi = key_to_float(hmm[1]);
        const float rng = hi - lo;
        base = lo;
        scale = rng > 0.0f ? 255.0f / rng : 1.0f;
    }
    // 3. k-means of the rotated rows (spherical for normalized data)
    if (int rc = kmeans(r, n, d, k, kmeans_iters, seed, normalize != 0, cent, assign, st)) return rc;
    std::vector<uint32_t> h_assign(n);
    std::vector<float> h_cent((size_t)k * d);
    BCHK(cudaMemcpyAsync(h_assign.data(), assign, n * 4, cudaMemcpyDeviceToHost, st));
    BCHK(cudaMemcpyAsync(h_cent.data(), cent, (size_t)k * d * 4, cudaMemcpyDeviceToHost, st));
    BCHK(cudaStreamSynchronize(st));
    std::vector<uint32_t> counts, order;
    group_rows(h_assign, k, counts, order);
    // 4. stored values and the compact blocks of every cluster
    const uint32_t esz = u8 ? 1 : 4;
    const uint8_t* stored = reinterpret_cast<const uint8_t*>(r);
    if (u8) {
        uint8_t* q8 = nullptr;
        BCHK(b.alloc(q8, n * d));
        quantize_kernel<<<grid_for(n * d, 256), 256, 0, st>>>(r, n * d, base, scale, q8);
        BCHK(cudaGetLastError());
        stored = q8;
    }
    std::vector<uint32_t> cl(n), pos(n);
    std::vector<uint64_t> blob_off(k);
    {
        uint64_t s = 0, off = 0;
        for (uint32_t c = 0; c < k; ++c) {
            blob_off[c] = off;
            for (uint32_t i = 0; i < counts[c]; ++i) {
                cl[s + i] = c;
                pos[s + i] = i;
            }
            s += counts[c];
            off += (uint64_t)counts[c] * d * esz;
        }
    }
    uint32_t *d_perm = nullptr, *d_cl = nullptr, *d_pos = nullptr, *d_ncl = nullptr;
    uint64_t* d_off = nullptr;
    uint8_t* blob = nullptr;
    BCHK(b.alloc(d_perm, n));
    BCHK(b.alloc(d_cl, n));
    BCHK(b.alloc(d_pos, n));
    BCHK(b.alloc(d_ncl, k));
    BCHK(b.alloc(d_off, k));
    BCHK(b.alloc(blob, n * d * esz));
    BCHK(cudaMemcpyAsync(d_perm, order.data(), n * 4, cudaMemcpyHostToDevice, st));
    BCHK(cudaMemcpyAsync(d_cl, cl.data(), n * 4, cudaMemcpyHostToDevice, st));
    BCHK(cudaMemcpyAsync(d_pos, pos.data(), n * 4, cudaMemcpyHostToDevice, st));
    BCHK(cudaMemcpyAsync(d_ncl, counts.data(), (size_t)k * 4, cudaMemcpyHostToDevice, st));
    BCHK(cudaMemcpyAsync(d_off, blob_off.data(), (size_t)k * 8, cudaMemcpyHostToDevice, st));
    layout_kernel<<<grid_for(n * d, 256), 256, 0, st>>>(stored, esz, d_perm, d_cl, d_pos, d_ncl, d_off, n, d, dv, blob);
    BCHK(cudaGetLastError());
    std::vector<uint8_t> h_blob(n * d * esz);
    BCHK(cudaMemcpyAsync(h_blob.data(), blob, h_blob.size(), cudaMemcpyDeviceToHost, st));
    // tree: meso clusters of the L1 centroids (10 iterations, as the reference's second level)
    std::vector<uint32_t> m_counts, m_order;
    std::vector<float> h_mcent;
    if (tree) {
        float* mc = nullptr;
        uint32_t* ma = nullptr;
        BCHK(b.alloc(mc, (uint64_t)k0 * d));
        BCHK(b.alloc(ma, k));
        if (int rc = kmeans(cent, k, d, k0, 10, seed + 1, normalize != 0, mc, ma, st)) return rc;
        std::vector<uint32_t> h_ma(k);
        h_mcent.resize((size_t)k0 * d);
        BCHK(cudaMemcpyAsync(h_ma.data(), ma, (size_t)k * 4, cudaMemcpyDeviceToHost, st));
        BCHK(cudaMemcpyAsync(h_mcent.data(), mc, (size_t)k0 * d * 4, cudaMemcpyDeviceToHost, st));
        BCHK(cudaStreamSynchronize(st));
        group_rows(h_ma, k0, m_counts, m_order);
    }
    BCHK(cudaStreamSynchronize(st));
    // 5. the Save format (index.hpp:242-267, ivf_wrapper.hpp:133-165 / 314-380)
    std::vector<uint8_t> file;
    file.reserve(9 + (size_t)d * d * 4 + h_blob.size() + n * 4 + (size_t)k * (d * 4 + 8) + 64);
    file.push_back((uint8_t)index_type);
    put_u32(file, d);
    put_u32(file, d);
    put_bytes(file, rotation, (size_t)d * d * 4);
    put_u32(file, d);
    put_u32(file, dv);
    put_u32(file, dh);
    put_u32(file, k);
    if (tree) {
        put_u32(file, k0);
        write_level_host(file, h_cent, d, dv, m_counts, m_order);
    }
    for (uint32_t c : counts) {
        put_u32(file, c);
        put_u32(file, max_capacity(c));
    }
    put_bytes(file, h_blob.data(), h_blob.size());
    put_bytes(file, order.data(), order.size() * 4);
    file.push_back(normalize ? 1 : 0);
    if (tree) put_bytes(file, h_mcent.data(), h_mcent.size() * 4);
    else put_bytes(file, h_cent.data(), h_cent.size() * 4);
    if (u8) {
        put_bytes(file, &base, 4);
        put_bytes(file, &scale, 4);
    }
    int rc = pdxg_load_buffer(file.data(), file.size(), device, out);
    if (rc == PDXG_OK) pdxg_set_append_normalization(*out, normalize);
    return rc;
}
