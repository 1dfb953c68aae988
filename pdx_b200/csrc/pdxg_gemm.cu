// Tensor-core GEMMs (tcgen05, sm_100a) of the query preparation and of the centroid probe.
//
// C[M x N] = sum over products of A_p[M x K] . B_p[N x K]^T, both operands K-major in global
// memory, staged by TMA (cp.async.bulk.tensor, 128-byte swizzle, no multicast) into a
// multi-stage shared-memory ring, multiplied by one thread issuing tcgen05.mma into a
// 128 x 128 FP32 accumulator in tensor memory, and read back by all four warps with
// tcgen05.ld for the epilogue. One CTA per 128 x 128 output tile.
//
// Operand kinds:
//  * TF32x3: FP32 operands given as two planes each, hi = x with the low 13 mantissa bits
//    cleared (exactly representable in TF32) and lo = x - hi (exact in FP32); the three
//    products hi.hi + hi.lo + lo.hi carry about 21 bits per operand, so the result is at FP32
//    rounding level. Used for the ADSampling rotation of the exact search path
//    (adsampling.hpp:192-246 multiplies by the d x d matrix with BLAS sgemm in FP32).
//  * BF16 and FP8 (E4M3): one plane each; the reduced-precision centroid probe and rotation.
//
// Every wait on an mbarrier is bounded: a wait that gives up records an error code in
// GemmArgs::error and the CTA drains its own copies and tensor-core work (again with bounded
// waits), frees its tensor memory and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "pdxg_gemm.cuh"

namespace pdxg {

namespace {

constexpr uint32_t kTile = 128;                  // rows of an operand tile, rows/cols of C tile
constexpr uint32_t kRowBytes = 128;              // K bytes of one stage (one 128-byte swizzle row)
constexpr uint32_t kPlaneBytes = kTile * kRowBytes;  // 16 KB
constexpr uint32_t kTmemCols = 128;              // FP32 accumulator: 128 lanes x 128 columns
constexpr uint64_t kWaitNs = 500000000ull;       // 0.5 s: a wait that takes longer gives up

template <int KIND>
struct KindTraits;
template <>
struct KindTraits<kGemmTF32x3> {
    static constexpr int planes = 2, products = 3, stages = 3;
    static constexpr uint32_t elem = 4;
    static constexpr uint32_t fmt = 2;  // TF32 in the instruction descriptor
};
template <>
struct KindTraits<kGemmBF16> {
    static constexpr int planes = 1, products = 1, stages = 4;
    static constexpr uint32_t elem = 2;
    static constexpr uint32_t fmt = 1;  // BF16
};
template <>
struct KindTraits<kGemmE4M3> {
    static constexpr int planes = 1, products = 1, stages = 4;
    static constexpr uint32_t elem = 1;
    static constexpr uint32_t fmt = 0;  // E4M3
};

template <int KIND>
__host__ __device__ constexpr uint32_t stage_bytes() {
    return 2u * KindTraits<KIND>::planes * kPlaneBytes;
}
template <int KIND>
__host__ __device__ constexpr uint32_t gemm_smem_bytes() {
    return KindTraits<KIND>::stages * stage_bytes<KIND>() + 1024u;  // + alignment slack
}

// Instruction descriptor of a dense 128 x 128 MMA with FP32 accumulation, both operands
// K-major (PTX ISA, tcgen05 instruction descriptor: D format bits 4-5, A / B format bits
// 7-9 / 10-12, N >> 3 at bits 17-22, M >> 4 at bits 24-28).
template <int KIND>
__host__ __device__ constexpr uint32_t instr_desc() {
    return (1u << 4) | (KindTraits<KIND>::fmt << 7) | (KindTraits<KIND>::fmt << 10) |
           ((kTile >> 3) << 17) | ((kTile >> 4) << 24);
}

// Shared-memory matrix descriptor of a K-major operand tile written by TMA with the 128-byte
// swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart (stride byte offset), leading
// byte offset 16 (unused by the swizzled K-major form), descriptor version 1, layout 2
// (SWIZZLE_128B). The tile must start on a 1024-byte boundary.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | (1ull << 16) | (64ull << 32) | (1ull << 46) |
           (2ull << 61);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the phase of `parity` to complete: gives up after kWaitNs of wall time, or
// early once another thread of the CTA has given up (abort set; a null `abort` waits for
// in-flight work regardless).
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 1;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63u) == 0u && ((abort && *abort) || global_ns() - t0 > kWaitNs)) return false;
    }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int32_t x,
                                            int32_t y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

template <int KIND>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t acc) {
    constexpr uint32_t idesc = instr_desc<KIND>();
    if constexpr (KIND == kGemmTF32x3) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(acc));
    } else if constexpr (KIND == kGemmBF16) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(acc));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(a), "l"(b), "r"(idesc), "r"(acc));
    }
}

// Arrives on `bar` once every tcgen05.mma this thread issued before has completed.
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 32 lanes x 16 consecutive FP32 columns of the accumulator (one row per thread).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void set_error(const GemmArgs& g, int code, volatile int* abort) {
    *abort = 1;
    if (g.error) atomicExch(g.error, code);
}

template <int KIND, int EPI>
__global__ void __launch_bounds__(128, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap a0, const __grid_constant__ CUtensorMap a1,
                const __grid_constant__ CUtensorMap b0, const __grid_constant__ CUtensorMap b1,
                const GemmArgs g) {
    using TR = KindTraits<KIND>;
    constexpr int S = TR::stages;
    constexpr int NP = TR::planes;
    constexpr uint32_t SB = stage_bytes<KIND>();
    constexpr uint32_t KE = kRowBytes / TR::elem;  // K elements per stage
    extern __shared__ uint8_t dyn_smem[];
    __shared__ __align__(8) uint64_t full_bar[S];
    __shared__ __align__(8) uint64_t empty_bar[S];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int abort_sh;

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t m0 = blockIdx.x * kTile, n0 = blockIdx.y * kTile;
    const uint32_t nk = (g.K + KE - 1) / KE;
    const uint32_t ring = (smem_u32(dyn_smem) + 1023u) & ~1023u;
    volatile int* abort = &abort_sh;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(smem_u32(&full_bar[s]), 1);
            mbar_init(smem_u32(&empty_bar[s]), 1);
        }
        mbar_init(smem_u32(&done_bar), 1);
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_sh)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;

    if (warp == 0 && lane == 0) {
        // TMA producer
        uint32_t issued = 0;
        for (uint32_t kb = 0; kb < nk; ++kb) {
            const uint32_t s = kb % S, ph = (kb / S) & 1u;
            if (kb >= (uint32_t)S && !mbar_wait(smem_u32(&empty_bar[s]), ph ^ 1u, abort)) {
                set_error(g, 1, abort);
                break;
            }
            if (*abort) break;
            const uint32_t st = ring + s * SB;
            const uint32_t fb = smem_u32(&full_bar[s]);
            mbar_expect_tx(fb, SB);
            const int32_t x = (int32_t)(kb * KE);
            tma_load_2d(st, &a0, x, (int32_t)m0, fb);
            if constexpr (NP == 2) tma_load_2d(st + kPlaneBytes, &a1, x, (int32_t)m0, fb);
            tma_load_2d(st + NP * kPlaneBytes, &b0, x, (int32_t)n0, fb);
            if constexpr (NP == 2) tma_load_2d(st + (NP + 1) * kPlaneBytes, &b1, x, (int32_t)n0, fb);
            issued = kb + 1;
        }
        // every copy this thread started has landed before the CTA can exit
        const uint32_t first = issued > (uint32_t)S ? issued - S : 0u;
        for (uint32_t kb = first; kb < issued; ++kb)
            if (!mbar_wait(smem_u32(&full_bar[kb % S]), (kb / S) & 1u, nullptr)) set_error(g, 2, abort);
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        for (uint32_t kb = 0; kb < nk; ++kb) {
            const uint32_t s = kb % S, ph = (kb / S) & 1u;
            if (!mbar_wait(smem_u32(&full_bar[s]), ph, abort)) {
                set_error(g, 3, abort);
                break;
            }
            tc_fence_after();
            const uint32_t st = ring + s * SB;
#pragma unroll
            for (uint32_t kk = 0; kk < kRowBytes / 32; ++kk) {
                // each MMA consumes 32 bytes of K: advance the start address by 32 B (2 units)
#pragma unroll
                for (int pr = 0; pr < TR::products; ++pr) {
                    const uint32_t pa = (pr == 2) ? 1u : 0u;  // hi.hi, hi.lo, lo.hi
                    const uint32_t pb = (pr == 1) ? 1u : 0u;
                    const uint64_t da = sw128_desc(st + pa * kPlaneBytes) + 2u * kk;
                    const uint64_t db = sw128_desc(st + (NP + pb) * kPlaneBytes) + 2u * kk;
                    umma<KIND>(tmem, da, db, (kb | kk | (uint32_t)pr) != 0u ? 1u : 0u);
                }
            }
            umma_commit(smem_u32(&empty_bar[s]));
        }
        umma_commit(smem_u32(&done_bar));
    }
    __syncwarp();

    // epilogue: warp w owns accumulator lanes (rows) 32w .. 32w + 31
    const bool ok = mbar_wait(smem_u32(&done_bar), 0u, abort);
    if (!ok) set_error(g, 4, abort);
    tc_fence_after();
    if (ok && !*abort && nk > 0) {
        const uint32_t row = m0 + warp * 32 + lane;
        const float rs = (row < g.M && g.row_scale) ? g.row_scale[row] : 1.0f;
        for (uint32_t c0 = 0; c0 < kTile; c0 += 16) {
            if (n0 + c0 >= g.N) break;  // uniform across the CTA
            float v[16];
            __syncwarp();
            tmem_ld16(tmem + ((warp * 32u) << 16) + c0, v);
            if (row < g.M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const uint32_t col = n0 + c0 + j;
                    if (col < g.N) {
                        float r = v[j] * rs;
                        if (g.col_scale) r *= g.col_scale[col];
                        if constexpr (EPI == kEpiDist) r = fmaf(-2.0f, r, g.col_add[col]);
                        if (g.out) g.out[(size_t)row * g.ldo + col] = r;
                        if (g.out_b16)
                            static_cast<__nv_bfloat16*>(g.out_b16)[(size_t)row * g.ldo16 + col] =
                                __float2bfloat16_rn(r);
                    }
                }
            }
        }
    }
    // after an abort the tensor core may still be working: wait for its final commit
    if (*abort && threadIdx.x == 0) mbar_wait(smem_u32(&done_bar), 0u, nullptr);
    tc_fence_before();
    __syncthreads();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
    }
}

// TF32x3 with FP32 accumulation in registers. The tensor core's own FP32 accumulation
// truncates, so one accumulator over K = 1024 drifts to ~1e-5 relative (measured 1.2e-6 absolute
// on unit vectors); here each stage (K = 32) is accumulated in one of two tensor-memory
// buffers, and the drain warps add each stage's partial sums into FP32 registers (round to
// nearest) while the tensor core fills the other buffer. The remaining error is about a dozen
// truncations of a stage partial, independent of K (measured 1.5e-7 at d = 1024 with two-stage
// groups, against 2.1e-7 for the FP32 SIMT GEMM), while the SIMT GEMM's grows with sqrt(K).
// Six warps: warp 0 issues the TMA copies, warp 1 the MMAs, warps 2-5 drain the accumulator
// (warp w reads tensor-memory lanes 32 (w % 4) .. 32 (w % 4) + 31, the rows it owns).
constexpr uint32_t kDrainStages = 1;
constexpr uint32_t kTF32x3Threads = 192;

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__global__ void __launch_bounds__(kTF32x3Threads, 1)
    gemm_tf32x3_kernel(const __grid_constant__ CUtensorMap a0, const __grid_constant__ CUtensorMap a1,
                       const __grid_constant__ CUtensorMap b0, const __grid_constant__ CUtensorMap b1,
                       const GemmArgs g) {
    constexpr int KIND = kGemmTF32x3;
    using TR = KindTraits<KIND>;
    constexpr int S = TR::stages;
    constexpr uint32_t SB = stage_bytes<KIND>();
    constexpr uint32_t KE = kRowBytes / TR::elem;
    extern __shared__ uint8_t dyn_smem[];
    __shared__ __align__(8) uint64_t full_bar[S];
    __shared__ __align__(8) uint64_t empty_bar[S];
    __shared__ __align__(8) uint64_t acc_full[2];
    __shared__ __align__(8) uint64_t acc_empty[2];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int abort_sh;

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t m0 = blockIdx.x * kTile, n0 = blockIdx.y * kTile;
    const uint32_t nk = (g.K + KE - 1) / KE;
    const uint32_t ngroups = (nk + kDrainStages - 1) / kDrainStages;
    const uint32_t ring = (smem_u32(dyn_smem) + 1023u) & ~1023u;
    volatile int* abort = &abort_sh;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(smem_u32(&full_bar[s]), 1);
            mbar_init(smem_u32(&empty_bar[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&acc_full[b]), 1);
            mbar_init(smem_u32(&acc_empty[b]), 4);  // one arrival per epilogue warp
        }
        mbar_init(smem_u32(&done_bar), 1);
        abort_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_sh)),
                     "r"(2 * kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;

    if (warp == 0 && lane == 0) {
        uint32_t issued = 0;
        for (uint32_t kb = 0; kb < nk; ++kb) {
            const uint32_t s = kb % S, ph = (kb / S) & 1u;
            if (kb >= (uint32_t)S && !mbar_wait(smem_u32(&empty_bar[s]), ph ^ 1u, abort)) {
                set_error(g, 1, abort);
                break;
            }
            if (*abort) break;
            const uint32_t st = ring + s * SB;
            const uint32_t fb = smem_u32(&full_bar[s]);
            mbar_expect_tx(fb, SB);
            const int32_t x = (int32_t)(kb * KE);
            tma_load_2d(st, &a0, x, (int32_t)m0, fb);
            tma_load_2d(st + kPlaneBytes, &a1, x, (int32_t)m0, fb);
            tma_load_2d(st + 2 * kPlaneBytes, &b0, x, (int32_t)n0, fb);
            tma_load_2d(st + 3 * kPlaneBytes, &b1, x, (int32_t)n0, fb);
            issued = kb + 1;
        }
        const uint32_t first = issued > (uint32_t)S ? issued - S : 0u;
        for (uint32_t kb = first; kb < issued; ++kb)
            if (!mbar_wait(smem_u32(&full_bar[kb % S]), (kb / S) & 1u, nullptr)) set_error(g, 2, abort);
    } else if (warp == 1 && lane == 0) {
        uint32_t kb = 0;
        for (uint32_t gi = 0; gi < ngroups && !*abort; ++gi) {
            const uint32_t b = gi & 1u;
            if (gi >= 2 && !mbar_wait(smem_u32(&acc_empty[b]), ((gi >> 1) - 1u) & 1u, abort)) {
                set_error(g, 5, abort);
                break;
            }
            tc_fence_after();
            const uint32_t acc_tmem = tmem + b * kTmemCols;
            bool first_mma = true;
            for (uint32_t j = 0; j < kDrainStages && kb < nk; ++j, ++kb) {
                const uint32_t s = kb % S, ph = (kb / S) & 1u;
                if (!mbar_wait(smem_u32(&full_bar[s]), ph, abort)) {
                    set_error(g, 3, abort);
                    break;
                }
                tc_fence_after();
                const uint32_t st = ring + s * SB;
#pragma unroll
                for (uint32_t kk = 0; kk < kRowBytes / 32; ++kk) {
#pragma unroll
                    for (int pr = 0; pr < 3; ++pr) {
                        const uint32_t pa = (pr == 2) ? 1u : 0u;
                        const uint32_t pb = (pr == 1) ? 1u : 0u;
                        const uint64_t da = sw128_desc(st + pa * kPlaneBytes) + 2u * kk;
                        const uint64_t db = sw128_desc(st + (2u + pb) * kPlaneBytes) + 2u * kk;
                        umma<KIND>(acc_tmem, da, db, first_mma ? 0u : 1u);
                        first_mma = false;
                    }
                }
                umma_commit(smem_u32(&empty_bar[s]));
            }
            umma_commit(smem_u32(&acc_full[b]));
        }
        umma_commit(smem_u32(&done_bar));  // every MMA of this CTA has completed
    }
    __syncwarp();

    bool ok = true;
    if (warp >= 2) {
    // drain warps: rows 32 (warp % 4) .. + 31 of the tile, one row per thread
    const uint32_t quarter = warp & 3u;
    float sum[kTile];
#pragma unroll
    for (uint32_t c = 0; c < kTile; ++c) sum[c] = 0.0f;
    for (uint32_t gi = 0; gi < ngroups; ++gi) {
        const uint32_t b = gi & 1u;
        if (!mbar_wait(smem_u32(&acc_full[b]), (gi >> 1) & 1u, abort)) {
            set_error(g, 4, abort);
            ok = false;
            break;
        }
        tc_fence_after();
        __syncwarp();
#pragma unroll
        for (uint32_t c0 = 0; c0 < kTile; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + b * kTmemCols + ((quarter * 32u) << 16) + c0, v);
#pragma unroll
            for (int j = 0; j < 16; ++j) sum[c0 + j] = __fadd_rn(sum[c0 + j], v[j]);
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&acc_empty[b]));
    }
    if (ok && !*abort && nk > 0) {
        const uint32_t row = m0 + quarter * 32 + lane;
        if (row < g.M) {
            const float rs = g.row_scale ? g.row_scale[row] : 1.0f;
#pragma unroll
            for (uint32_t c = 0; c < kTile; ++c) {
                const uint32_t col = n0 + c;
                if (col < g.N) {
                    const float r = g.row_scale ? sum[c] * rs : sum[c];
                    if (g.out) g.out[(size_t)row * g.ldo + col] = r;
                    if (g.out_b16)
                        static_cast<__nv_bfloat16*>(g.out_b16)[(size_t)row * g.ldo16 + col] =
                            __float2bfloat16_rn(r);
                }
            }
        }
    }
    }
    // the tensor core may still be writing a buffer nobody waited for (after an abort)
    if (*abort && warp == 1 && lane == 0) mbar_wait(smem_u32(&done_bar), 0u, nullptr);
    tc_fence_before();
    __syncthreads();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kTmemCols)
                     : "memory");
    }
}

// TF32x3 planes of (optionally normalized) rows: x = q / norm (NormalizeQuery, scalar.hpp:23-40),
// hi = x with the low 13 mantissa bits cleared, lo = x - hi. One warp per row.
__global__ void split_rows_kernel(const float* __restrict__ q, uint32_t nq, uint32_t d, int normalize,
                                  float* __restrict__ hi, float* __restrict__ lo) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (row >= nq) return;
    const float* src = q + (size_t)row * d;
    float norm = 1.0f;
    if (normalize) {
        float s = 0.0f;
        for (uint32_t i = lane; i < d; i += 32) s = __fmaf_rn(src[i], src[i], s);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        norm = (s == 0.0f) ? 1.0f : sqrtf(s);
    }
    for (uint32_t i = lane; i < d; i += 32) {
        const float x = normalize ? __fdiv_rn(src[i], norm) : src[i];
        const float h = __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
        hi[(size_t)row * d + i] = h;
        lo[(size_t)row * d + i] = __fsub_rn(x, h);
    }
}

// BF16 copy of (optionally normalized) rows; one warp per row.
__global__ void bf16_rows_kernel(const float* __restrict__ q, uint32_t nq, uint32_t d, int normalize,
                                 __nv_bfloat16* __restrict__ out) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (row >= nq) return;
    const float* src = q + (size_t)row * d;
    float norm = 1.0f;
    if (normalize) {
        float s = 0.0f;
        for (uint32_t i = lane; i < d; i += 32) s = __fmaf_rn(src[i], src[i], s);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        norm = (s == 0.0f) ? 1.0f : sqrtf(s);
    }
    for (uint32_t i = lane; i < d; i += 32)
        out[(size_t)row * d + i] = __float2bfloat16_rn(normalize ? __fdiv_rn(src[i], norm) : src[i]);
}

// E4M3 copy of rows with one scale per row: x / s with s = max|x| / 448 (the largest finite
// E4M3 magnitude), saturating; scale[row] = s. One warp per row.
__global__ void e4m3_rows_kernel(const float* __restrict__ x, uint32_t n, uint32_t d,
                                 uint8_t* __restrict__ out, float* __restrict__ scale) {
    const uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* src = x + (size_t)row * d;
    float m = 0.0f;
    for (uint32_t i = lane; i < d; i += 32) m = fmaxf(m, fabsf(src[i]));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
    const float s = (m > 0.0f) ? m / 448.0f : 1.0f;
    const float inv = 1.0f / s;
    for (uint32_t i = lane; i < d; i += 32) {
        const __nv_fp8_e4m3 v(src[i] * inv);
        out[(size_t)row * d + i] = *reinterpret_cast<const uint8_t*>(&v);
    }
    if (lane == 0) scale[row] = s;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

template <int KIND, int EPI>
cudaError_t launch_kind(const GemmOperand& a, const GemmOperand& b, const GemmArgs& g, cudaStream_t st) {
    auto kern = (KIND == kGemmTF32x3 && EPI == kEpiStore) ? gemm_tf32x3_kernel : gemm_kernel<KIND, EPI>;
    constexpr uint32_t smem = gemm_smem_bytes<KIND>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const CUtensorMap& a1 = (KindTraits<KIND>::planes == 2) ? a.map[1] : a.map[0];
    const CUtensorMap& b1 = (KindTraits<KIND>::planes == 2) ? b.map[1] : b.map[0];
    dim3 grid((g.M + kTile - 1) / kTile, (g.N + kTile - 1) / kTile);
    const uint32_t threads = (KIND == kGemmTF32x3 && EPI == kEpiStore) ? kTF32x3Threads : 128u;
    kern<<<grid, threads, smem, st>>>(a.map[0], a1, b.map[0], b1, g);
    return cudaGetLastError();
}

}  // namespace

bool gemm_available() { return encode_fn() != nullptr; }

uint32_t gemm_elem_bytes(int kind) { return kind == kGemmTF32x3 ? 4u : (kind == kGemmBF16 ? 2u : 1u); }

bool gemm_shape_ok(int kind, uint32_t k) { return ((uint64_t)k * gemm_elem_bytes(kind)) % 16u == 0u; }

int make_gemm_operand(GemmOperand& op, int kind, const void* plane0, const void* plane1, uint32_t rows,
                      uint32_t k) {
    std::memset(&op, 0, sizeof(op));
    auto fn = encode_fn();
    if (!fn || !gemm_shape_ok(kind, k) || rows == 0 || k == 0) return -1;
    const uint32_t es = gemm_elem_bytes(kind);
    const CUtensorMapDataType dt = kind == kGemmTF32x3 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : kind == kGemmBF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                       : CU_TENSOR_MAP_DATA_TYPE_UINT8;
    const cuuint64_t dims[2] = {k, rows};
    const cuuint64_t strides[1] = {(cuuint64_t)k * es};
    const cuuint32_t box[2] = {kRowBytes / es, kTile};
    const cuuint32_t estr[2] = {1, 1};
    const void* planes[2] = {plane0, plane1};
    for (int i = 0; i < 2; ++i) {
        if (!planes[i]) continue;
        if (reinterpret_cast<uintptr_t>(planes[i]) % 16u) return -1;
        CUresult r = fn(&op.map[i], dt, 2, const_cast<void*>(planes[i]), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return -1;
    }
    op.kind = kind;
    op.rows = rows;
    op.k = k;
    return 0;
}

cudaError_t launch_gemm(const GemmOperand& a, const GemmOperand& b, int epi, const GemmArgs& g,
                        cudaStream_t st) {
    if (a.kind != b.kind || a.k != b.k || g.K != a.k || g.M > a.rows || g.N > b.rows)
        return cudaErrorInvalidValue;
    if (g.M == 0 || g.N == 0) return cudaSuccess;
    if (epi == kEpiDist && !g.col_add) return cudaErrorInvalidValue;
    switch (a.kind * 2 + epi) {
        case kGemmTF32x3 * 2 + kEpiStore: return launch_kind<kGemmTF32x3, kEpiStore>(a, b, g, st);
        case kGemmBF16 * 2 + kEpiStore: return launch_kind<kGemmBF16, kEpiStore>(a, b, g, st);
        case kGemmBF16 * 2 + kEpiDist: return launch_kind<kGemmBF16, kEpiDist>(a, b, g, st);
        case kGemmE4M3 * 2 + kEpiDist: return launch_kind<kGemmE4M3, kEpiDist>(a, b, g, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_split_rows(const float* q, uint32_t nq, uint32_t d, bool normalize, float* hi, float* lo,
                              cudaStream_t st) {
    if (nq == 0) return cudaSuccess;
    split_rows_kernel<<<(nq * 32 + 255) / 256, 256, 0, st>>>(q, nq, d, normalize ? 1 : 0, hi, lo);
    return cudaGetLastError();
}

cudaError_t launch_bf16_rows(const float* q, uint32_t nq, uint32_t d, bool normalize, void* out,
                             cudaStream_t st) {
    if (nq == 0) return cudaSuccess;
    bf16_rows_kernel<<<(nq * 32 + 255) / 256, 256, 0, st>>>(q, nq, d, normalize ? 1 : 0,
                                                            static_cast<__nv_bfloat16*>(out));
    return cudaGetLastError();
}

cudaError_t launch_e4m3_rows(const float* x, uint32_t n, uint32_t d, void* out, float* scale, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    e4m3_rows_kernel<<<(n * 32 + 255) / 256, 256, 0, st>>>(x, n, d, static_cast<uint8_t*>(out), scale);
    return cudaGetLastError();
}

}  // namespace pdxg
