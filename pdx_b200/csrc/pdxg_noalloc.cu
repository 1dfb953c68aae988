// Allocation-free search entry point (pdxg_search_device_noalloc in include/pdx_b200.h).
//
// Some callers cannot let a library call cudaMalloc: a host framework may already own the
// device's memory budget through its own pool, a latency-critical serving loop may forbid the
// device-wide synchronisation that cudaMalloc/cudaFree can cause, or a plugin may run inside a
// process whose allocation policy it does not control. This entry point therefore runs the
// same search kernels as pdxg_search_device, but takes its scratch space -- the queue counter,
// the query norms or the TF32 hi / lo planes of the tensor-core rotation, and the rotated queries
// -- from a fixed array compiled into the library instead of allocating a workspace.
//
// The array is a file-scope __device__ variable: every GPU that loads this library holds its
// own copy (kNoAllocScratchBytes) until the process exits. In host code the symbol is only a
// host-side stand-in, so its device address is looked up with cudaGetSymbolAddress, once per
// device, with that device current, the first time this entry point runs on it.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/pdx_b200.h"
#include "pdxg_common.cuh"

struct pdxg_index;
int pdxg_search_on_workspace(pdxg_index* ix, const float* q, uint32_t nq, uint32_t k,
                             uint32_t flags, float* norms, float* rotated, float* hi, float* lo,
                             int* gemm_err, uint32_t* queue, uint32_t* ids, float* dists,
                             uint32_t* counts, cudaStream_t st);
bool pdxg_rotation_on_tensor_cores(const pdxg_index* ix, uint32_t nq);
bool pdxg_reduced_precision_probe(const pdxg_index* ix);
int pdxg_index_device(const pdxg_index* ix);
uint32_t pdxg_index_dims(const pdxg_index* ix);
std::mutex& pdxg_index_mutex(pdxg_index* ix);
cudaStream_t pdxg_index_stream(pdxg_index* ix);
int pdxg_set_error(int code, const char* msg);

namespace {

constexpr uint64_t kNoAllocScratchBytes = PDXG_NOALLOC_SCRATCH_BYTES;
constexpr uint64_t kQueueBytes = 256;  // the work counter, padded to keep the rest aligned
constexpr uint64_t kErrBytes = 256;    // the rotation GEMM's wait status, padded likewise

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

uint64_t align256(uint64_t x) { return (x + 255) / 256 * 256; }

// Device address of this device's scratch array (set up on first use, device current).
int scratch_for_device(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices)
        return pdxg_set_error(PDXG_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_addr[device]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return pdxg_set_error(PDXG_ERR_CUDA, cudaGetErrorString(e));
        g_scratch_addr[device] = ptr;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[device]);
    return PDXG_OK;
}

}  // namespace

extern "C" uint64_t pdxg_noalloc_scratch_bytes(void) { return kNoAllocScratchBytes; }

extern "C" int pdxg_search_device_noalloc(pdxg_index* index, const float* queries, uint32_t nq,
                                          uint32_t k, uint32_t flags, uint32_t* ids,
                                          float* distances, uint32_t* counts, void* stream) {
    if (!index) return pdxg_set_error(PDXG_ERR_INVALID_ARGUMENT, "index is NULL");
    if (!queries || !ids || !distances || !counts)
        return pdxg_set_error(PDXG_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (flags & PDXG_COLLECT_STATS)
        return pdxg_set_error(PDXG_ERR_INVALID_ARGUMENT,
                              "PDXG_COLLECT_STATS needs a workspace; use pdxg_search_device");
    if (pdxg_reduced_precision_probe(index))
        return pdxg_set_error(PDXG_ERR_UNSUPPORTED,
                              "the reduced-precision probe (pdxg_set_probe_mode 1 or 2) needs a workspace; "
                              "use pdxg_search_device");
    const uint64_t d = pdxg_index_dims(index);
    const bool rotate = !(flags & PDXG_QUERY_TRANSFORMED);
    // raw queries are rotated exactly as pdxg_search_device rotates them: TF32x3 tensor-core
    // planes (hi, lo) when it would use them, else the FP32 SIMT kernels (norms)
    const bool tc = rotate && pdxg_rotation_on_tensor_cores(index, nq);
    const uint64_t plane = align256((uint64_t)nq * d * 4);
    const uint64_t norms_bytes = (rotate && !tc) ? align256((uint64_t)nq * 4) : 0;
    const uint64_t rot_bytes = rotate ? plane : 0;
    const uint64_t split_bytes = tc ? 2 * plane : 0;
    if (kQueueBytes + kErrBytes + norms_bytes + rot_bytes + split_bytes > kNoAllocScratchBytes)
        return pdxg_set_error(PDXG_ERR_CAPACITY,
                              "batch too large for the fixed scratch of pdxg_search_device_noalloc "
                              "(raw queries need 12 * nq * d + 512 bytes with the tensor-core rotation, "
                              "else 4 * nq * d + 4 * nq + 512, within PDXG_NOALLOC_SCRATCH_BYTES; "
                              "split the batch or pass PDXG_QUERY_TRANSFORMED queries)");
    std::lock_guard<std::mutex> lock(pdxg_index_mutex(index));
    const int device = pdxg_index_device(index);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return pdxg_set_error(PDXG_ERR_CUDA, cudaGetErrorString(e));
    unsigned char* scratch = nullptr;
    int rc = scratch_for_device(device, &scratch);
    if (rc) return rc;
    uint64_t at = 0;
    auto carve = [&](uint64_t bytes) {
        unsigned char* p = scratch + at;
        at += bytes;
        return p;
    };
    uint32_t* queue = reinterpret_cast<uint32_t*>(carve(kQueueBytes));
    int* gemm_err = reinterpret_cast<int*>(carve(kErrBytes));
    float* norms = reinterpret_cast<float*>(carve(norms_bytes));
    float* rotated = reinterpret_cast<float*>(carve(rot_bytes));
    float* hi = reinterpret_cast<float*>(carve(split_bytes / 2));
    float* lo = reinterpret_cast<float*>(carve(split_bytes / 2));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : pdxg_index_stream(index);
    return pdxg_search_on_workspace(index, queries, nq, k, flags, norms, rotated, hi, lo, gemm_err,
                                    queue, ids, distances, counts, st);
}
