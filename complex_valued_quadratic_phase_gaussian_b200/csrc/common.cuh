// Shared device helpers for the CVQPG B200 kernels (sm_100a).
//
// Everything here is header-only and used by several translation units:
// status codes, launch helpers, complex arithmetic, the range-reduced sincos
// used by the splat, and a counter-based normal generator for the loss noise.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "cvqpg.h"

namespace cvqpg {

constexpr int kTile = 16;                 // splat tile edge in pixels (cuda/config.h BLOCK_X/Y)
constexpr int kTilePixels = kTile * kTile;
constexpr int kMaxChannels = 3;

// Launch-error check used by every C-ABI entry point after its launches.
static inline int launch_status() {
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CVQPG_OK : CVQPG_ERR_CUDA;
}

static inline unsigned ceil_div(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// Bump-pointer carving of a caller-provided workspace into 256-byte aligned slices.
struct Carver {
    char* base;
    size_t off;
    size_t cap;
    explicit Carver(void* p, size_t c) : base((char*)p), off(0), cap(c) {}
    template <typename T>
    T* take(size_t count) {
        off = (off + 255) & ~(size_t)255;
        T* p = base ? (T*)(base + off) : nullptr;
        off += count * sizeof(T);
        return p;
    }
    bool fits() const { return off <= cap; }
};

// ---------------------------------------------------------------------------
// complex helpers (float2 = re, im)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// ---------------------------------------------------------------------------
// sincos with an FMA Cody-Waite reduction modulo 2*pi.
//
// Method: W. J. Cody and W. Waite, "Software Manual for the Elementary
// Functions" (1980), additive range reduction with a two-term constant; the
// FMA form follows J.-M. Muller, "Elementary Functions" (3rd ed., 2016), sec. 11.
// The reduced argument lies in [-pi, pi], where the hardware sin/cos
// approximations (MUFU) have an absolute error below 2^-21.4. The splat phase
// phi + k*base is unbounded, so reducing first keeps the error at ~1e-7 rad for
// any |x| below ~1e6 instead of growing with |x|.
// ---------------------------------------------------------------------------
// n = an integer nearest to x/(2 pi): x/(2 pi) + 1.5 * 2^23 in one FMA (rounded
// to an integer there, for |x/(2 pi)| < 2^22), minus 1.5 * 2^23. A half-way
// case may round the other way than rintf(x * (1/2 pi)) would; then r moves by
// one turn to just outside [-pi, pi], which leaves sin and cos unchanged.
__device__ __forceinline__ void sincos_reduced(float x, float* s, float* c) {
    const float kInv2Pi = 0.15915494309189535f;
    const float k2PiHi = 6.28318548202514648f;       // float(2*pi)
    const float k2PiLo = -1.7484555314695172e-07f;   // 2*pi - float(2*pi)
    const float kRound = 12582912.0f;                 // 1.5 * 2^23
    const float n = __fsub_rn(__fmaf_rn(x, kInv2Pi, kRound), kRound);
    float r = fmaf(-n, k2PiHi, x);
    r = fmaf(-n, k2PiLo, r);
    __sincosf(r, s, c);
}

// The same SFU approximations through the PTX .ftz forms (ex2/sin/cos.approx.ftz.f32):
// without .ftz the hardware approximations need fix-up instructions for denormal
// arguments and results, which the splat paths never produce (|r| <= pi, and the
// Gaussian factor is at least exp(-20) under the Mahalanobis cut).
__device__ __forceinline__ float ex2_ftz(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ void sincos_reduced_ftz(float x, float* s, float* c) {
    const float kInv2Pi = 0.15915494309189535f;
    const float k2PiHi = 6.28318548202514648f;
    const float k2PiLo = -1.7484555314695172e-07f;
    const float kRound = 12582912.0f;
    const float n = __fsub_rn(__fmaf_rn(x, kInv2Pi, kRound), kRound);
    float r = fmaf(-n, k2PiHi, x);
    r = fmaf(-n, k2PiLo, r);
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(*s) : "f"(r));
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(*c) : "f"(r));
}

__device__ __forceinline__ float rcp_ftz(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Asynchronous 16-byte global -> shared copies (cp.async, completion by wait_group).
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// exp(-m / 2) = 2^(-m / (2 ln 2))
constexpr float kNegHalfLog2e = -0.72134752044448170368f;

// ---------------------------------------------------------------------------
// Philox4x32-10 counter-based generator (J. K. Salmon, M. A. Moraes, R. O. Dror,
// D. E. Shaw, "Parallel Random Numbers: As Easy as 1, 2, 3", SC 2011) and a
// Box-Muller transform to standard normals (four per call). Used for the fresh target noise of
// the multi-plane loss; the oracle restates the same generator.
// ---------------------------------------------------------------------------
struct Philox4 {
    uint32_t v[4];
};

__host__ __device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                         uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)M0 * c0;
        uint64_t p1 = (uint64_t)M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n1 = lo1;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        uint32_t n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += W0; k1 += W1;
    }
    Philox4 o;
    o.v[0] = c0; o.v[1] = c1; o.v[2] = c2; o.v[3] = c3;
    return o;
}

// Uniform in (0, 1]: (u + 1) * 2^-32 rounded to float once. u + 1 <= 2^32 is
// converted from 64 bits with one rounding and the scale is a power of two, so
// this equals the double-precision evaluation rounded to float.
__device__ __forceinline__ float u32_to_open01(uint32_t u) {
    return __ull2float_rn((unsigned long long)u + 1ull) * 2.3283064365386963e-10f;
}

// Four standard normals for counter `q` of stream (`seed`, `offset`): Box-Muller
// on the word pairs (w0, w1) and (w2, w3), z = sqrt(-2 ln u) * (cos, sin)(2 pi u').
// The logarithm and the sine/cosine use the hardware approximations (absolute
// error ~1e-6 in z against the float64 restatement; the noise enters the loss
// scaled by 1e-3 of the target range).
__device__ __forceinline__ float4 normal4_at(uint64_t seed, uint64_t offset, uint64_t q) {
    Philox4 r = philox4x32_10((uint32_t)q, (uint32_t)(q >> 32), (uint32_t)offset, (uint32_t)(offset >> 32),
                              (uint32_t)seed, (uint32_t)(seed >> 32));
    const float r01 = sqrtf(-2.0f * __logf(u32_to_open01(r.v[0])));
    const float r23 = sqrtf(-2.0f * __logf(u32_to_open01(r.v[2])));
    float s1, c1, s3, c3;
    sincos_reduced(6.28318530717958648f * u32_to_open01(r.v[1]), &s1, &c1);
    sincos_reduced(6.28318530717958648f * u32_to_open01(r.v[3]), &s3, &c3);
    return make_float4(r01 * c1, r01 * s1, r23 * c3, r23 * s3);
}

}  // namespace cvqpg
