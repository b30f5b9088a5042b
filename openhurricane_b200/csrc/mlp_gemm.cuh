// BF16 tensor-core GEMM for the surrogate network, sm_100a (tcgen05 + TMA).
//
//   D[M][N] = A[M][K] * B[N][K]^T       (both operands K-major, bf16)
//
// accumulated in FP32 in tensor memory, with a fused epilogue (bias, GELU,
// GELU' gating, bf16 / f32 stores, transposed bf16 store). One CTA computes a
// 128 x BN tile: warp 0 (one thread) streams 128x64 / BNx64 operand tiles
// with TMA (128-byte swizzle) through a STAGES-deep shared-memory ring, warp 1
// (one thread) issues tcgen05.mma (M = 128, N = BN, K = 16 per instruction,
// four per 64-wide K block) and commits each stage back to the producer, and
// after the last commit all four warps read the accumulator from tensor
// memory (warp w owns lanes 32w..32w+31 = tile rows) and run the epilogue.
// Shapes: M % 128 == 0, N % BN == 0, K % 64 == 0 (callers zero-pad).
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "sm100.cuh"

namespace hc {

struct GemmEpilogue {
    const float *bias;             // [N] or null
    int act;                       // 0 identity, 1 GELU
    const __nv_bfloat16 *gate_z;   // backward: D *= GELU'(gate_z[row][col]) (null: off)
    int ld_gz;
    float *out_f32;                // row-major [M][ld_f32] (null: off)
    int ld_f32;
    __nv_bfloat16 *out_bf;         // row-major [M][ld_bf]
    int ld_bf;
    __nv_bfloat16 *out_bt;         // transposed [N][ld_bt]
    int ld_bt;
    __nv_bfloat16 *z_out;          // pre-activation, row-major [M][ld_zo]
    int ld_zo;
};

constexpr uint32_t kWaitLimit = 1u << 22;
constexpr int kGemmBM = 128;
constexpr int kGemmBK = 64;

__device__ __forceinline__ float gelu_f(float z) {
    return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}

__device__ __forceinline__ float gelu_grad_f(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
           z * 0.39894228040143268f * expf(-0.5f * z * z);
}

template <int BN>
struct GemmSmem {
    static constexpr int kA = kGemmBM * kGemmBK * 2;  // 16 KiB
    static constexpr int kB = BN * kGemmBK * 2;
    static constexpr int kStage = kA + kB;            // multiple of 1024
    static constexpr int kTmemCols = BN < 32 ? 32 : BN;
};

template <int BN, int STAGES>
__global__ void __launch_bounds__(128, 1)
gemm_bf16_tn_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    int K, const __grid_constant__ GemmEpilogue ep, int *err) {
    using S = GemmSmem<BN>;
    static_assert(BN % 32 == 0 && BN >= 32 && BN <= 256, "BN");
    static_assert(S::kStage % 1024 == 0, "stage alignment");
    extern __shared__ uint8_t gemm_smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(gemm_smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * S::kStage);
    uint64_t *empty = full + STAGES;
    uint64_t *done = empty + STAGES;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kGemmBM, n0 = blockIdx.y * BN;
    const int nk = K / kGemmBK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            sm100::mbar_init(&full[s], 1);
            sm100::mbar_init(&empty[s], 1);
        }
        sm100::mbar_init(done, 1);
        *abort_flag = 0;
        sm100::fence_mbar_init();
    }
    if (warp == 2) {
        sm100::tmem_alloc(tmem_slot, S::kTmemCols);
        sm100::tmem_relinquish();
    }
    sm100::tc_fence_before();
    __syncthreads();
    sm100::tc_fence_after();
    const uint32_t taddr = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // producer
        sm100::tma_prefetch_desc(&tmA);
        sm100::tma_prefetch_desc(&tmB);
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % STAGES, it = kb / STAGES;
            if (kb >= STAGES && !sm100::mbar_wait(&empty[s], (it - 1) & 1, kWaitLimit)) {
                *abort_flag = 1;
                atomicExch(err, 1);
                break;
            }
            uint8_t *a = smem + s * S::kStage;
            uint8_t *b = a + S::kA;
            sm100::mbar_arrive_expect_tx(&full[s], S::kStage);
            sm100::tma_load_2d(a, &tmA, &full[s], kb * kGemmBK, m0);
            sm100::tma_load_2d(b, &tmB, &full[s], kb * kGemmBK, n0);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        constexpr uint32_t idesc = sm100::idesc_bf16_f32(kGemmBM, BN);
        bool ok = true;
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % STAGES, it = kb / STAGES;
            if (!sm100::mbar_wait(&full[s], it & 1, kWaitLimit)) {
                *abort_flag = 1;
                atomicExch(err, 2);
                ok = false;
                break;
            }
            sm100::tc_fence_after();
            const uint32_t a = sm100::smem_u32(smem + s * S::kStage);
            const uint32_t b = a + S::kA;
#pragma unroll
            for (int k = 0; k < kGemmBK / 16; ++k) {
                // K advance inside the 128-byte swizzle atom: 16 bf16 = 32 bytes
                sm100::mma_bf16(taddr, sm100::desc_kmajor_sw128(a + 32 * k),
                                sm100::desc_kmajor_sw128(b + 32 * k), idesc,
                                (kb | k) != 0 ? 1u : 0u);
            }
            sm100::mma_commit(&empty[s]);
        }
        (void)ok;
        sm100::mma_commit(done);
    }
    __syncwarp();

    // epilogue: every thread owns one tile row
    const bool got = sm100::mbar_wait(done, 0, kWaitLimit);
    if (!got) atomicExch(err, 3);
    sm100::tc_fence_after();
    // warp-uniform decision: the tensor-memory loads below are .sync.aligned
    const bool run = __all_sync(0xffffffffu, got && *abort_flag == 0);
    if (run) {
        const int row = m0 + warp * 32 + lane;
        const uint32_t lane_base = taddr + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 32) {
            uint32_t r[32];
            sm100::tmem_ld_32x32b_x32(lane_base + (uint32_t)c0, r);
            sm100::tmem_ld_wait();
            float v[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
            const int col0 = n0 + c0;
            if (ep.bias) {
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] += __ldg(&ep.bias[col0 + j]);
            }
            if (ep.z_out) {
                __nv_bfloat16 *zp = ep.z_out + (size_t)row * ep.ld_zo + col0;
#pragma unroll
                for (int j = 0; j < 32; j += 8) {
                    __align__(16) __nv_bfloat16 t[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) t[q] = __float2bfloat16_rn(v[j + q]);
                    *reinterpret_cast<uint4 *>(zp + j) = *reinterpret_cast<const uint4 *>(t);
                }
            }
            if (ep.act == 1) {
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] = gelu_f(v[j]);
            }
            if (ep.gate_z) {
                const __nv_bfloat16 *zp = ep.gate_z + (size_t)row * ep.ld_gz + col0;
#pragma unroll
                for (int j = 0; j < 32; ++j) v[j] *= gelu_grad_f(__bfloat162float(zp[j]));
            }
            if (ep.out_f32) {
                float *op = ep.out_f32 + (size_t)row * ep.ld_f32 + col0;
#pragma unroll
                for (int j = 0; j < 32; j += 4)
                    *reinterpret_cast<float4 *>(op + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
            }
            if (ep.out_bf) {
                __nv_bfloat16 *op = ep.out_bf + (size_t)row * ep.ld_bf + col0;
#pragma unroll
                for (int j = 0; j < 32; j += 8) {
                    __align__(16) __nv_bfloat16 t[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) t[q] = __float2bfloat16_rn(v[j + q]);
                    *reinterpret_cast<uint4 *>(op + j) = *reinterpret_cast<const uint4 *>(t);
                }
            }
            if (ep.out_bt) {
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    ep.out_bt[(size_t)(col0 + j) * ep.ld_bt + row] = __float2bfloat16_rn(v[j]);
            }
        }
    }
    sm100::tc_fence_before();
    __syncthreads();
    if (warp == 2) sm100::tmem_dealloc(taddr, S::kTmemCols);
}

}  // namespace hc
