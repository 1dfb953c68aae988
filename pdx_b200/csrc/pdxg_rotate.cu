// Query preparation: NormalizeQuery (scalar.hpp:23-40) and the ADSampling rotation
// y = M^T x of adsampling.hpp:225-245, batched as R[nq x d] = normalize(Q)[nq x d] @ M[d x d]
// (M row-major, as stored in the index file).
//
// The FP32 path is a register-tiled SIMT GEMM with FP32 accumulation (the reference's
// sgemm_ precision). Rotation parity against the reference is at FP32 rounding level, not
// bit-exact: the reference's own result depends on its BLAS build.
#include <cstdint>
#include <cuda_runtime.h>

namespace pdxg {

// One warp per query: norm = sqrt(sum x^2); inv stored as the divisor (0 -> row unchanged).
__global__ void query_norms_kernel(const float* __restrict__ q, uint32_t nq, uint32_t d,
                                   float* __restrict__ norms) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (warp >= nq) return;
    const float* row = q + (size_t)warp * d;
    float s = 0.0f;
    for (uint32_t i = lane; i < d; i += 32) s = __fmaf_rn(row[i], row[i], s);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) norms[warp] = (s == 0.0f) ? 1.0f : sqrtf(s);
}

// A few rows (nq <= kGemvRows, a single query or an appended row): C[nq x d] = (A / norm) @ B
// with 32 output columns per 1024-thread CTA, lane = column and warp = K slice (rows w, w + 32,
// ... of B, FMA in that order, eight rows of B loaded before their FMAs); the 32 warps' partial
// sums are then added in warp order, so the result does not depend on timing. B is read once,
// 128 contiguous bytes per warp and row.
constexpr uint32_t kGemvRows = 8;
constexpr uint32_t kGemvWarps = 32;

__global__ void __launch_bounds__(1024) rotate_gemv_kernel(const float* __restrict__ A,
                                                           const float* __restrict__ norms,
                                                           const float* __restrict__ B,
                                                           float* __restrict__ C, uint32_t M,
                                                           uint32_t N, uint32_t K) {
    __shared__ float part[kGemvWarps][kGemvRows][32];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t col = blockIdx.x * 32 + lane;
    float acc[kGemvRows];
#pragma unroll
    for (uint32_t r = 0; r < kGemvRows; ++r) acc[r] = 0.0f;
    for (uint32_t i0 = warp; i0 < K; i0 += kGemvWarps * 8) {
        float b[8];
#pragma unroll
        for (uint32_t t = 0; t < 8; ++t) {
            const uint32_t i = i0 + kGemvWarps * t;
            b[t] = (i < K && col < N) ? __ldg(B + (size_t)i * N + col) : 0.0f;
        }
#pragma unroll
        for (uint32_t t = 0; t < 8; ++t) {
            const uint32_t i = i0 + kGemvWarps * t;
            if (i >= K) break;
            for (uint32_t r = 0; r < M; ++r) {
                float a = __ldg(A + (size_t)r * K + i);
                if (norms) a = __fdiv_rn(a, __ldg(norms + r));
                acc[r] = __fmaf_rn(a, b[t], acc[r]);
            }
        }
    }
#pragma unroll
    for (uint32_t r = 0; r < kGemvRows; ++r)
        if (r < M) part[warp][r][lane] = acc[r];
    __syncthreads();
    if (warp == 0 && col < N) {
        for (uint32_t r = 0; r < M; ++r) {
            float s = part[0][r][lane];
            for (uint32_t w = 1; w < kGemvWarps; ++w) s = __fadd_rn(s, part[w][r][lane]);
            C[(size_t)r * N + col] = s;
        }
    }
}

// C[nq x d] = (A / norm)[nq x d] @ B[d x d]; 128x64 output tile per 256-thread CTA,
// 8x4 outputs per thread, K step 16, double-buffered through shared memory.
constexpr int RBM = 128, RBN = 64, RBK = 16;

__global__ void __launch_bounds__(256) rotate_sgemm_kernel(const float* __restrict__ A,
                                                           const float* __restrict__ norms,
                                                           const float* __restrict__ B,
                                                           float* __restrict__ C, uint32_t M,
                                                           uint32_t N, uint32_t K) {
    __shared__ float As[2][RBK][RBM + 4];
    __shared__ float Bs[2][RBK][RBN];
    const uint32_t tid = threadIdx.x;
    const uint32_t row0 = blockIdx.y * RBM, col0 = blockIdx.x * RBN;
    const uint32_t tr = tid / 16, tc = tid % 16;  // 16 x 16 thread grid: 8 rows x 4 cols each
    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0f;

    auto load_tile = [&](int buf, uint32_t k0) {
        // A tile: 128 rows x 16 k, 2048 elements, 8 per thread
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const uint32_t idx = tid + e * 256;
            const uint32_t r = idx / RBK, kk = idx % RBK;
            const uint32_t gr = row0 + r, gk = k0 + kk;
            float v = 0.0f;
            if (gr < M && gk < K) {
                v = A[(size_t)gr * K + gk];
                if (norms) v = __fdiv_rn(v, norms[gr]);
            }
            As[buf][kk][r] = v;
        }
        // B tile: 16 k x 64 cols, 1024 elements, 4 per thread
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const uint32_t idx = tid + e * 256;
            const uint32_t kk = idx / RBN, c = idx % RBN;
            const uint32_t gk = k0 + kk, gc = col0 + c;
            Bs[buf][kk][c] = (gk < K && gc < N) ? B[(size_t)gk * N + gc] : 0.0f;
        }
    };

    int buf = 0;
    load_tile(0, 0);
    __syncthreads();
    for (uint32_t k0 = 0; k0 < K; k0 += RBK) {
        if (k0 + RBK < K) load_tile(buf ^ 1, k0 + RBK);
#pragma unroll
        for (int kk = 0; kk < RBK; ++kk) {
            float a[8], b[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[buf][kk][tr * 8 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk][tc + 16 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = __fmaf_rn(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t gr = row0 + tr * 8 + i;
        if (gr >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t gc = col0 + tc + 16 * j;
            if (gc < N) C[(size_t)gr * N + gc] = acc[i][j];
        }
    }
}

cudaError_t launch_prepare_queries(const float* q, uint32_t nq, uint32_t d, const float* rotation,
                                   bool normalize, float* norms_ws, float* out, cudaStream_t st) {
    if (nq == 0) return cudaSuccess;
    if (normalize) {
        const uint32_t threads = 256;
        const uint32_t blocks = (nq * 32 + threads - 1) / threads;
        query_norms_kernel<<<blocks, threads, 0, st>>>(q, nq, d, norms_ws);
    }
    if (nq <= kGemvRows) {
        rotate_gemv_kernel<<<(d + 31) / 32, 1024, 0, st>>>(q, normalize ? norms_ws : nullptr, rotation, out, nq,
                                                           d, d);
        return cudaGetLastError();
    }
    dim3 grid((d + RBN - 1) / RBN, (nq + RBM - 1) / RBM);
    rotate_sgemm_kernel<<<grid, 256, 0, st>>>(q, normalize ? norms_ws : nullptr, rotation, out, nq,
                                              d, d);
    return cudaGetLastError();
}

}  // namespace pdxg
