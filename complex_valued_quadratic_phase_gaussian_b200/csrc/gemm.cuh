// Internal interface of the BF16 tensor-core GEMM (gemm.cu) used by the
// per-tile MLP of the learned initialiser (mlp.cu).
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace cvqpg {

constexpr int kGemmBM = 128;  // rows of C per CTA (TMEM lanes)
constexpr int kGemmBN = 128;  // columns of C per CTA (TMEM columns)
constexpr int kGemmBK = 64;   // K per pipeline stage (one 128-byte swizzle row of BF16)

// What the epilogue does with the FP32 accumulator tile (CVQPG_GEMM_EPI_* in cvqpg.h).
struct GemmEpi {
    int mode;
    int valid_n;               // columns >= valid_n are written as 0 in the BF16 outputs
    const float* bias;         // [N]
    const float* zin;          // [M][ld_z] pre-activation for the GELU derivative
    int ld_z;
    float* out_f32;            // [M][ld_f32] (+ split * split_stride)
    int ld_f32;
    long long split_stride;
    __nv_bfloat16* out_bf16;   // [M][ld_bf16], may be null
    int ld_bf16;
    __nv_bfloat16* out_bf16_t; // [N][ld_t] transposed copy, may be null
    int ld_t;
};

// C[M,N] = A[M,K] * B[N,K]^T with A, B BF16 row-major (K contiguous), FP32
// accumulation; K split `splits` ways along blockIdx.z (EPI_F32 only, each
// split to its own slab). Requirements: M, N multiples of 128, K a multiple of
// 64 * splits, lda, ldb multiples of 8, A and B 16-byte aligned.
int tc_gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K,
            const GemmEpi& epi, int splits, int* status, cudaStream_t stream);

}  // namespace cvqpg
