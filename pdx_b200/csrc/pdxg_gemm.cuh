// Host interface of the tcgen05 tensor-core GEMMs (pdxg_gemm.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace pdxg {

enum GemmKind : int { kGemmTF32x3 = 0, kGemmBF16 = 1, kGemmE4M3 = 2 };
enum GemmEpi : int { kEpiStore = 0, kEpiDist = 1 };

// One K-major operand in global memory: `rows` x `k` elements, one tensor map per plane
// (TF32x3: hi and lo planes; BF16 / E4M3: one plane).
struct GemmOperand {
    CUtensorMap map[2];
    int kind;
    uint32_t rows, k;
};

// C = A . B^T epilogue arguments. Store: out[r][c] = acc * row_scale[r] * col_scale[c];
// Dist: out[r][c] = col_add[c] - 2 * acc * row_scale[r] * col_scale[c] (squared L2 up to the
// per-row constant |a_r|^2). Scales are optional (null = 1). out_b16 receives a BF16 copy.
struct GemmArgs {
    uint32_t M, N, K;
    float* out;
    uint32_t ldo;
    void* out_b16;
    uint32_t ldo16;
    const float* row_scale;
    const float* col_scale;
    const float* col_add;
    int* error;  // set (non-zero) when a bounded wait of the kernel gave up
};

bool gemm_available();
uint32_t gemm_elem_bytes(int kind);
// The tensor maps need the row pitch (k x element size) to be a multiple of 16 bytes.
bool gemm_shape_ok(int kind, uint32_t k);
// Encodes the tensor maps (planes are 16-byte aligned device pointers). 0 on success.
int make_gemm_operand(GemmOperand& op, int kind, const void* plane0, const void* plane1, uint32_t rows,
                      uint32_t k);
cudaError_t launch_gemm(const GemmOperand& a, const GemmOperand& b, int epi, const GemmArgs& g,
                        cudaStream_t st);
// TF32x3 planes of the rows of q (divided by their norm when normalize is set).
cudaError_t launch_split_rows(const float* q, uint32_t nq, uint32_t d, bool normalize, float* hi, float* lo,
                              cudaStream_t st);
cudaError_t launch_bf16_rows(const float* q, uint32_t nq, uint32_t d, bool normalize, void* out,
                             cudaStream_t st);
cudaError_t launch_e4m3_rows(const float* x, uint32_t n, uint32_t d, void* out, float* scale, cudaStream_t st);

}  // namespace pdxg
