// BF16 GEMM on the sm_100a tensor cores: TMA -> shared memory (3-stage ring,
// 128-byte swizzle) -> tcgen05.mma into a TMEM accumulator -> tcgen05.ld ->
// fused epilogue (bias, GELU, GELU derivative, BF16 row-major and transposed
// copies, split-K slabs).
//
// One CTA computes one 128 x 128 tile of C with 8 warps, two CTAs per SM:
//   warp 0, lane 0: TMA producer (waits for a free stage, arms its mbarrier with
//                   the byte count, issues the A and B tile loads);
//   warp 1, lane 0: MMA issuer (waits for a full stage, issues 4 MMAs of K = 16,
//                   commits to the stage's "empty" barrier; after the last stage
//                   commits to the "done" barrier); warp 1 also owns the TMEM
//                   allocation (128 columns);
//   all 8 warps:    epilogue; warp w reads TMEM lanes 32 (w % 4) .. +31 (= rows of C),
//                   warps w and w + 4 take the two halves of the columns.
// Each thread of the epilogue owns one row of C, so stores of the transposed
// copy (column-major) are coalesced across the warp.
//
// Waits are bounded (tcgen05.cuh): a timeout sets status[0], the roles stop
// issuing, copies already in flight are waited for (bounded) and the TMEM
// allocation is released before the kernel returns.
#include <mutex>

#include "gemm.cuh"
#include "tcgen05.cuh"

namespace cvqpg {

// 3 stages of 32 KB let two CTAs share an SM, so one CTA's epilogue overlaps the other's main
// loop (measured on the MLP's 8192-row GEMMs: 4 stages at one CTA per SM took 44 / 38 us for the
// 1024- / 512-deep forward layers, 3 stages at two CTAs 32 / 28 us, with 8 warps 29 / 25 us)
#ifndef CVQPG_GEMM_STAGES
#define CVQPG_GEMM_STAGES 3
#endif
#ifndef CVQPG_GEMM_CTAS_PER_SM
#define CVQPG_GEMM_CTAS_PER_SM 2
#endif
#ifndef CVQPG_GEMM_THREADS
#define CVQPG_GEMM_THREADS 256
#endif
constexpr int kGemmStages = CVQPG_GEMM_STAGES;
constexpr int kGemmThreads = CVQPG_GEMM_THREADS;  // 128 or 256: warps w and w + 4 share TMEM lane quadrant w
constexpr int kEpiGroups = kGemmThreads / 128;     // column groups of the epilogue
static_assert(kGemmThreads == 128 || kGemmThreads == 256, "one or two warps per TMEM lane quadrant");
constexpr uint32_t kStageBytesA = kGemmBM * kGemmBK * 2;  // 16 KB
constexpr uint32_t kStageBytesB = kGemmBN * kGemmBK * 2;  // 16 KB
constexpr size_t kGemmSmem = 1024 /* alignment slack */ + kGemmStages * (kStageBytesA + kStageBytesB) + 256;

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * __expf(-0.5f * z * z);
}

// Epilogue of 16 consecutive columns n0..n0+15 of row m.
__device__ __forceinline__ void gemm_epilogue16(const GemmEpi& e, int m, int n0, int split, float (&v)[16]) {
    if (e.mode == CVQPG_GEMM_EPI_F32 || e.mode == CVQPG_GEMM_EPI_BIAS) {
        if (e.mode == CVQPG_GEMM_EPI_BIAS) {
#pragma unroll
            for (int j = 0; j < 16; j++) v[j] += __ldg(&e.bias[n0 + j]);
        }
        float* dst = e.out_f32 + (size_t)split * e.split_stride + (size_t)m * e.ld_f32 + n0;
#pragma unroll
        for (int j = 0; j < 16; j += 4) *(float4*)(dst + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        return;
    }
    float h[16];
    if (e.mode == CVQPG_GEMM_EPI_BIAS_GELU) {
        float* zdst = e.out_f32 ? e.out_f32 + (size_t)m * e.ld_f32 + n0 : nullptr;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const float z = v[j] + __ldg(&e.bias[n0 + j]);
            v[j] = z;
            h[j] = (n0 + j < e.valid_n) ? gelu_f(z) : 0.0f;
        }
        if (zdst) {
#pragma unroll
            for (int j = 0; j < 16; j += 4) *(float4*)(zdst + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        }
    } else {  // CVQPG_GEMM_EPI_DGELU: dZ = acc * gelu'(Z)
        const float* z = e.zin + (size_t)m * e.ld_z + n0;
        float zz[16];
        if (((e.ld_z & 3) | (int)((uintptr_t)e.zin & 15)) == 0) {  // the lane's 16 values as four float4 loads
#pragma unroll
            for (int j = 0; j < 16; j += 4) {
                const float4 q = __ldg(reinterpret_cast<const float4*>(z + j));
                zz[j] = q.x;
                zz[j + 1] = q.y;
                zz[j + 2] = q.z;
                zz[j + 3] = q.w;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 16; j++) zz[j] = __ldg(&z[j]);
        }
#pragma unroll
        for (int j = 0; j < 16; j++) h[j] = (n0 + j < e.valid_n) ? v[j] * gelu_grad(zz[j]) : 0.0f;
    }
    if (e.out_bf16) {
        __align__(16) __nv_bfloat16 b[16];
#pragma unroll
        for (int j = 0; j < 16; j++) b[j] = __float2bfloat16_rn(h[j]);
        uint4* dst = (uint4*)(e.out_bf16 + (size_t)m * e.ld_bf16 + n0);
        dst[0] = *(const uint4*)&b[0];
        dst[1] = *(const uint4*)&b[8];
    }
    if (e.out_bf16_t) {
#pragma unroll
        for (int j = 0; j < 16; j++) e.out_bf16_t[(size_t)(n0 + j) * e.ld_t + m] = __float2bfloat16_rn(h[j]);
    }
}

__global__ void __launch_bounds__(kGemmThreads, CVQPG_GEMM_CTAS_PER_SM) tc_gemm_kernel(const __grid_constant__ CUtensorMap map_a,
                                                                  const __grid_constant__ CUtensorMap map_b,
                                                                  int kblocks, GemmEpi epi, int* status) {
    extern __shared__ uint8_t gsm_raw[];
    uint8_t* base = (uint8_t*)(((uintptr_t)gsm_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* sA = base;
    uint8_t* sB = base + kGemmStages * kStageBytesA;
    uint64_t* bars = (uint64_t*)(sB + kGemmStages * kStageBytesB);  // full[S], empty[S], done
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * kGemmStages + 1);
    int* counters = (int*)(tmem_slot + 1);  // [0] stages issued, [1] stages consumed
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n0 = blockIdx.x * kGemmBN, m0 = blockIdx.y * kGemmBM;
    const int kb0 = blockIdx.z * kblocks;
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kGemmStages),
                   done = smem_u32(bars + 2 * kGemmStages);

    if (threadIdx.x == 0) {
        for (int s = 0; s < kGemmStages; s++) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done, 1);
        mbar_fence_init();
        counters[0] = 0;
        counters[1] = 0;
    }
    if (warp == 1) {
        tmem_alloc(smem_u32(tmem_slot), kGemmBN);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        int issued = 0;
        for (int i = 0; i < kblocks; ++i) {
            const int s = i % kGemmStages;
            const uint32_t ph = (uint32_t)(i / kGemmStages) & 1u;
            if (i >= kGemmStages && !mbar_wait(empty0 + 8 * s, ph ^ 1u)) {
                atomicExch(status, 1);
                break;
            }
            mbar_expect_tx(full0 + 8 * s, kStageBytesA + kStageBytesB);
            tma_load_2d(smem_u32(sA + s * kStageBytesA), &map_a, full0 + 8 * s, (kb0 + i) * kGemmBK, m0);
            tma_load_2d(smem_u32(sB + s * kStageBytesB), &map_b, full0 + 8 * s, (kb0 + i) * kGemmBK, n0);
            ++issued;
        }
        counters[0] = issued;
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = bf16_instr_desc(kGemmBM, kGemmBN);
        int consumed = 0;
        for (int i = 0; i < kblocks; ++i) {
            const int s = i % kGemmStages;
            const uint32_t ph = (uint32_t)(i / kGemmStages) & 1u;
            if (!mbar_wait(full0 + 8 * s, ph)) {
                atomicExch(status, 2);
                break;
            }
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA + s * kStageBytesA), b0 = smem_u32(sB + s * kStageBytesB);
#pragma unroll
            for (int kk = 0; kk < kGemmBK / 16; ++kk)
                tc_mma_bf16(tmem, sw128_kmajor_desc(a0 + 32 * kk), sw128_kmajor_desc(b0 + 32 * kk), idesc,
                            (i | kk) != 0 ? 1u : 0u);
            tc_commit(empty0 + 8 * s);  // stage s is free once these MMAs have read it
            ++consumed;
        }
        tc_commit(done);
        counters[1] = consumed;
    }
    __syncwarp();
    __syncthreads();  // the role lanes' counters are visible to every thread from here
    const bool complete = counters[1] == kblocks;

    if (!mbar_wait(done, 0)) atomicExch(status, 3);
    tc_fence_after();
    // warp w reads TMEM lanes 32 (w % 4) .. +31 (its quadrant); with 8 warps the two warps of a
    // quadrant take alternate halves of the columns
    const int quad = warp & 3, cg = warp >> 2;
    const int m = m0 + quad * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(quad * 32) << 16);
    if (complete) {
#pragma unroll 1
        for (int c0 = cg * (kGemmBN / kEpiGroups); c0 < (cg + 1) * (kGemmBN / kEpiGroups); c0 += 16) {
            float v[16];
            tmem_ld16(trow + (uint32_t)c0, v);
            gemm_epilogue16(epi, m, n0 + c0, blockIdx.z, v);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0 && lane == 0) {
        // only after an error: wait (bounded) for tile loads that were issued but never consumed
        for (int i = counters[1]; i < counters[0]; ++i)
            if (!mbar_wait(full0 + 8 * (i % kGemmStages), (uint32_t)(i / kGemmStages) & 1u)) break;
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, kGemmBN);
    }
}

// ---------------------------------------------------------------------------
// host: tensor maps through the driver entry point (no link-time libcuda)
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    });
    return fn;
}

// rows x cols BF16 matrix, row stride ld elements; box 64 (cols) x 128 (rows), 128-byte swizzle.
static bool make_tile_map(CUtensorMap* map, const __nv_bfloat16* ptr, int rows, int cols, int ld, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)kGemmBK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)ptr, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int tc_gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K,
            const GemmEpi& epi, int splits, int* status, cudaStream_t stream) {
    if (!A || !B || !status || M <= 0 || N <= 0 || K <= 0 || splits < 1) return CVQPG_ERR_ARG;
    if (M % kGemmBM || N % kGemmBN || K % (kGemmBK * splits) || lda % 8 || ldb % 8 || lda < K || ldb < K)
        return CVQPG_ERR_UNSUPPORTED;
    if (((uintptr_t)A | (uintptr_t)B) & 15) return CVQPG_ERR_UNSUPPORTED;
    if (splits > 1 && epi.mode != CVQPG_GEMM_EPI_F32) return CVQPG_ERR_UNSUPPORTED;
    switch (epi.mode) {
        case CVQPG_GEMM_EPI_F32:
            if (!epi.out_f32 || epi.ld_f32 < N || epi.ld_f32 % 4 || epi.split_stride % 4) return CVQPG_ERR_ARG;
            if (splits > 1 && epi.split_stride < (long long)M * epi.ld_f32) return CVQPG_ERR_ARG;
            break;
        case CVQPG_GEMM_EPI_BIAS:
            if (!epi.out_f32 || !epi.bias || epi.ld_f32 < N || epi.ld_f32 % 4) return CVQPG_ERR_ARG;
            break;
        case CVQPG_GEMM_EPI_BIAS_GELU:
            if (!epi.bias || (epi.out_f32 && (epi.ld_f32 < N || epi.ld_f32 % 4))) return CVQPG_ERR_ARG;
            break;
        case CVQPG_GEMM_EPI_DGELU:
            if (!epi.zin || epi.ld_z < N) return CVQPG_ERR_ARG;
            break;
        default:
            return CVQPG_ERR_ARG;
    }
    if (epi.out_f32 && ((uintptr_t)epi.out_f32 & 15)) return CVQPG_ERR_ARG;
    if (epi.mode == CVQPG_GEMM_EPI_BIAS_GELU || epi.mode == CVQPG_GEMM_EPI_DGELU) {
        if (epi.out_bf16 && (epi.ld_bf16 < N || epi.ld_bf16 % 8 || ((uintptr_t)epi.out_bf16 & 15)))
            return CVQPG_ERR_ARG;
        if (epi.out_bf16_t && epi.ld_t < M) return CVQPG_ERR_ARG;
    }
    CUtensorMap ma, mb;
    if (!make_tile_map(&ma, A, M, K, lda, kGemmBM) || !make_tile_map(&mb, B, N, K, ldb, kGemmBN))
        return CVQPG_ERR_CUDA;
    cudaFuncSetAttribute(tc_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem);
    const dim3 grid(N / kGemmBN, M / kGemmBM, splits);
    tc_gemm_kernel<<<grid, kGemmThreads, kGemmSmem, stream>>>(ma, mb, K / kGemmBK / splits, epi, status);
    return launch_status();
}

}  // namespace cvqpg

// ===========================================================================
// C ABI
// ===========================================================================
using namespace cvqpg;

extern "C" int cvqpg_gemm_bf16_tn(const void* A, int lda, const void* B, int ldb, int M, int N, int K,
                                  const cvqpg_gemm_epilogue* e, int splits, int* status, void* stream) {
    if (!e) return CVQPG_ERR_ARG;
    GemmEpi g;
    g.mode = e->mode;
    g.valid_n = e->valid_n > 0 ? e->valid_n : N;
    g.bias = e->bias;
    g.zin = e->zin;
    g.ld_z = e->ld_z;
    g.out_f32 = e->out_f32;
    g.ld_f32 = e->ld_f32;
    g.split_stride = e->split_stride;
    g.out_bf16 = (__nv_bfloat16*)e->out_bf16;
    g.ld_bf16 = e->ld_bf16;
    g.out_bf16_t = (__nv_bfloat16*)e->out_bf16_t;
    g.ld_t = e->ld_t;
    return tc_gemm((const __nv_bfloat16*)A, lda, (const __nv_bfloat16*)B, ldb, M, N, K, g, splits, status,
                   (cudaStream_t)stream);
}

// Self-check of the bounded wait: one thread waits on a shared-memory mbarrier
// (count 1) with the polling loop every tcgen05 kernel here uses. With arrive = 0
// nothing ever arrives, so the wait must give up after `limit` polls and report it.
__global__ void wait_probe_kernel(int arrive, uint32_t limit, int* status) {
    __shared__ __align__(8) uint64_t bar;
    const uint32_t b = cvqpg::smem_u32(&bar);
    cvqpg::mbar_init(b, 1);
    cvqpg::mbar_fence_init();
    if (arrive) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(b) : "memory");
    status[0] = cvqpg::mbar_wait_n(b, 0, limit) ? 0 : 4;
}

extern "C" int cvqpg_wait_probe(int arrive, unsigned spin_limit, int* status, void* stream) {
    if (!status || spin_limit == 0) return CVQPG_ERR_ARG;
    wait_probe_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(arrive, spin_limit, status);
    return cvqpg::launch_status();
}
