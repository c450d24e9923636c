// Column kernels of the BLASM passes that transform four adjacent columns per
// CTA, for column lengths N = 16 x R2 x 16 (the 1080p grid: 2816 = 16 x 11 x 16).
//
// Why four columns: the intermediates are row-major ([C][rows][NW] complex64),
// so one column is one 8-byte element per 35 KB row. Four adjacent columns
// (kx0 = 4m .. 4m+3) are one 32-byte sector per row, and the thread mapping
// below makes every warp access 8 rows x 4 columns: each global load or store
// instruction of a warp moves eight whole sectors. The four transforms share
// the CTA: shared memory holds them interleaved (element e of column g at
// (e + e/16) * G + g, conflict-free for the passes' strides), and every pass
// is one barrier for all four.
//
// Plan (Stockham, natural-order output, see fft.cuh): forward 16 (first pass,
// input nonzero only in the middle half: 2x zero padding), R2, 16 (kept in
// registers); the inverse starts from those registers with a radix-16 pass
// (stride 1), then R2, then 16 whose output is pruned to the middle half (the
// crops are at most the padded height). The forward kernel multiplies the
// register spectrum by each plane's transfer function and inverts it per
// plane; the adjoint kernel transforms each plane's gradient forward,
// accumulates x conj(transfer) in registers and inverts once.
//
// Threads: TPC = 176 / BPT per column; each thread owns butterflies u + b TPC
// (b < BPT) of the radix-16 passes (176 = N/16 per column) and u + b TPC
// (< 256) of the radix-R2 pass (256 = N/R2 per column). Measured on B200 at
// 2816 x 4480 (forward / adjoint column stage): G = 4, BPT = 1 (704 threads,
// 80 registers, one CTA per SM) 0.670 / 0.746 ms; G = 4, BPT = 2 (352 threads,
// 168 registers) 0.750 / 0.797 ms; G = 2, BPT = 1 (two CTAs per SM) 0.700 /
// 0.740 ms; the one-column kernels 0.795 / 0.753 ms. Recomputing the transfer
// excess per plane instead of holding it in registers: 0.762 / 0.849 ms.
#pragma once

#include "blasm_cols.cuh"

namespace cvqpg {

#ifndef CVQPG_COLS4_BPT
#define CVQPG_COLS4_BPT 1
#endif
#ifndef CVQPG_COLS4_G
#define CVQPG_COLS4_G 4
#endif
#ifdef CVQPG_COLS4_MAXNREG
#define CVQPG_C4_BOUNDS(nt, mb) __maxnreg__(CVQPG_COLS4_MAXNREG)
#else
#define CVQPG_C4_BOUNDS(nt, mb) __launch_bounds__(nt, mb)
#endif
constexpr int kC4G = CVQPG_COLS4_G;      // adjacent columns per CTA
constexpr int kC4Bpt = CVQPG_COLS4_BPT;  // radix-16 butterflies per thread

template <int R2>
struct Cols4Plan {
    static constexpr int N = 16 * R2 * 16;
    static constexpr int NB16 = N / 16;  // butterflies of a radix-16 pass per column
    static constexpr int NBR = N / R2;   // butterflies of the radix-R2 pass per column (256)
    static constexpr int BPT = kC4Bpt;
    static constexpr int TPC = NB16 / BPT;  // threads per column
    static constexpr int NT = kC4G * TPC;
    static constexpr int RB = (NBR + TPC - 1) / TPC;  // radix-R2 butterflies per thread (rounds)
    static constexpr int LD = (N - 1 + ((N - 1) >> 4) + 1) * kC4G;  // float2 per shared buffer
    static constexpr int NTW = 256;  // twiddle prefix used (indices < 16 * 16 and < NB16)
    static constexpr size_t kSmem = (size_t)(2 * LD + NTW) * sizeof(float2);
    static constexpr int kMinBlocks = kC4G == 2 ? 2 : 1;  // CTAs per SM the shared memory allows
};

__device__ __forceinline__ int c4_addr(int e, int g) { return (e + (e >> 4)) * kC4G + g; }

// Radix-R2 pass (stride 16) over one shared buffer into another; both directions.
template <int R2, bool INV>
__device__ __forceinline__ void c4_pass_mid(const float2* __restrict__ in, float2* __restrict__ out,
                                            const float2* __restrict__ tw, int u, int g) {
    using PL = Cols4Plan<R2>;
#pragma unroll
    for (int b = 0; b < PL::RB; b++) {
        const int j = u + b * PL::TPC;
        if (b * PL::TPC + PL::TPC <= PL::NBR || j < PL::NBR) {
            const int k = j & 15, q = j >> 4;
            float2 v[R2];
#pragma unroll
            for (int r = 0; r < R2; r++) v[r] = in[c4_addr(j + r * PL::NBR, g)];
            float2 w = tw[16 * k];
            if (INV) w.y = -w.y;
            apply_twiddles<R2>(v, w);
            dft<R2>(v, INV);
            const int o = q * (16 * R2) + k;
#pragma unroll
            for (int r = 0; r < R2; r++) out[c4_addr(o + 16 * r, g)] = v[r];
        }
    }
}

// Radix-16 pass with stride 1 (inverse start): v holds x[j + r NB16]; writes y[16 j + r].
__device__ __forceinline__ void c4_store16_stride1(float2* __restrict__ out, int j, int g, const float2 (&v)[16]) {
    float2* p = out + c4_addr(16 * j, g);  // 16 j .. 16 j + 15 share one padding block
#pragma unroll
    for (int r = 0; r < 16; r++) p[r * kC4G] = v[r];
}

// Last forward pass (radix 16, stride NB16) read from shared memory: v = X[j + r NB16].
template <int R2, bool INV>
__device__ __forceinline__ void c4_last16(const float2* __restrict__ in, const float2* __restrict__ tw, int j, int g,
                                          float2 (&v)[16]) {
    using PL = Cols4Plan<R2>;
#pragma unroll
    for (int r = 0; r < 16; r++) v[r] = in[c4_addr(j + r * PL::NB16, g)];
    float2 w = tw[j];
    if (INV) w.y = -w.y;
    apply_twiddles<16>(v, w);
}

// Plane-independent transfer excess of the elements a thread holds (-1: no plane
// propagates it), kept in registers for all planes.
template <int R2>
__device__ __forceinline__ void c4_excess(const BlasmDev& d, int c, int ci, float bcol, int u,
                                          float (&E)[kC4Bpt][16]) {
    using PL = Cols4Plan<R2>;
#pragma unroll
    for (int b = 0; b < PL::BPT; b++) {
        const int j = u + b * PL::TPC;
#pragma unroll
        for (int r = 0; r < 16; r++) {
            int jj = j + r * PL::NB16 + PL::N / 2;
            if (jj >= PL::N) jj -= PL::N;
            float e;
            E[b][r] = transfer_excess(d, c, jj, ci, bcol, &e) ? e : -1.0f;
        }
    }
}

// transfer value of element (b, r) for plane pp, zero where the plane does not propagate it
template <int R2>
__device__ __forceinline__ float2 c4_transfer(const PCParam& pp, bool col_ok, float E, int e, float scale) {
    using PL = Cols4Plan<R2>;
    int jj = e + PL::N / 2;
    if (jj >= PL::N) jj -= PL::N;
    const bool on = col_ok && E >= 0.0f && jj >= pp.j0 && jj < pp.j1;
    return on ? transfer_from_excess(pp, E, scale) : make_float2(0.f, 0.f);
}

// Last inverse pass: radix 16 at stride NB16, only the middle half of the outputs
// (r = 4..11, rows [N/4, 3N/4)) formed; rows in [row0, row0 + nrows) are stored.
template <int R2>
__device__ __forceinline__ void c4_out16(const float2* __restrict__ in, const float2* __restrict__ tw, int u, int g,
                                         float2* __restrict__ dst, size_t ld, int row0, int nrows) {
    using PL = Cols4Plan<R2>;
#pragma unroll
    for (int b = 0; b < PL::BPT; b++) {
        const int j = u + b * PL::TPC;
        float2 v[16];
        c4_last16<R2, true>(in, tw, j, g, v);
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) dft4(v[n2], v[4 + n2], v[8 + n2], v[12 + n2], true);
        dft16_twiddle_rows<true>(v, true);
#pragma unroll
        for (int r = 4; r < 12; r++) {
            const int y = j + r * PL::NB16 - row0;
            if ((unsigned)y < (unsigned)nrows) dst[(size_t)y * ld + g] = v[r];
        }
    }
}

// First forward pass: radix 16, stride 1, inputs nonzero only at r = 4..11 (rows
// [N/4, 3N/4)), read from global rows y = e - row0 when 0 <= y < nrows.
template <int R2>
__device__ __forceinline__ void c4_in16(const float2* __restrict__ src, size_t ld, int row0, int nrows,
                                        float2* __restrict__ out, int u, int g) {
    using PL = Cols4Plan<R2>;
    float2 m[PL::BPT][8];
#pragma unroll
    for (int b = 0; b < PL::BPT; b++) {
        const int j = u + b * PL::TPC;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int y = j + (4 + i) * PL::NB16 - row0;
            m[b][i] = (unsigned)y < (unsigned)nrows ? __ldg(&src[(size_t)y * ld + g]) : make_float2(0.f, 0.f);
        }
    }
#pragma unroll
    for (int b = 0; b < PL::BPT; b++) {
        float2 v[16];
#pragma unroll
        for (int i = 0; i < 8; i++) v[4 + i] = m[b][i];
        dft16_mid_in(v, false);
        c4_store16_stride1(out, u + b * PL::TPC, g, v);
    }
}

// The adjoint's per-plane input block (the out_h kept rows x four columns, row-major, 32 B per
// row) is copied into a shared staging buffer with cp.async while the previous plane computes.
constexpr int kC4StageRows = 1216;  // staging capacity in rows (the shared memory left by the two buffers)

__device__ __forceinline__ void c4_stage_async(float2* __restrict__ stage, const float2* __restrict__ src, size_t ld,
                                               int nrows, int t, int nt) {
    // 16-byte chunks: two per row (columns g = 0,1 and 2,3)
    for (int i = t; i < 2 * nrows; i += nt) {
        const int y = i >> 1, h = i & 1;
        cp_async16(stage + 4 * y + 2 * h, src + (size_t)y * ld + 2 * h);
    }
    cp_async_commit();
}

__device__ __forceinline__ void c4_stage_wait() { cp_async_wait_all(); }

// c4_in16 reading the staged block (rows y = e - row0 in [0, nrows) at stage[4 y + g]).
template <int R2>
__device__ __forceinline__ void c4_in16_staged(const float2* __restrict__ stage, int row0, int nrows,
                                               float2* __restrict__ out, int u, int g) {
    using PL = Cols4Plan<R2>;
#pragma unroll
    for (int b = 0; b < PL::BPT; b++) {
        const int j = u + b * PL::TPC;
        float2 v[16];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int y = j + (4 + i) * PL::NB16 - row0;
            v[4 + i] = (unsigned)y < (unsigned)nrows ? stage[4 * y + g] : make_float2(0.f, 0.f);
        }
        dft16_mid_in(v, false);
        c4_store16_stride1(out, j, g, v);
    }
}

// Forward: four columns of A [C][pH][NW] -> spectrum x transfer -> inverse per
// plane -> the kept rows of B [P*C][out_h][NW].
template <int R2>
__global__ void CVQPG_C4_BOUNDS(Cols4Plan<R2>::NT, Cols4Plan<R2>::kMinBlocks) blasm_cols4_fwd_kernel(BlasmDev d,
                                                                              const float2* __restrict__ A,
                                                                              float2* __restrict__ B) {
    using PL = Cols4Plan<R2>;
    extern __shared__ float2 sm[];
    float2* b0 = sm;
    float2* b1 = sm + PL::LD;
    float2* tw = sm + 2 * PL::LD;
    const int t = threadIdx.x, g = t & (kC4G - 1), u = t / kC4G;
    const int NW = d.NW, groups = NW / kC4G;
    const int c = blockIdx.x / groups, kx0 = (blockIdx.x - c * groups) * kC4G;
    for (int i = t; i < PL::NTW; i += PL::NT) tw[i] = __ldg(&d.col.tw[i]);
    // forward pass 1 straight from global (the padded field sits in rows [N/4, 3N/4))
    c4_in16<R2>(A + (size_t)c * d.pH * NW + kx0, NW, PL::N / 2 - d.pH / 2, d.pH, b0, u, g);
    __syncthreads();
    c4_pass_mid<R2, false>(b0, b1, tw, u, g);
    __syncthreads();
    int ci = kx0 + g + (NW >> 1);
    if (ci >= NW) ci -= NW;
    const float bcol = __ldg(&d.b_col[c * NW + ci]);
    float2 spec[PL::BPT][16];
#pragma unroll
    for (int b = 0; b < PL::BPT; b++) {
        c4_last16<R2, false>(b1, tw, u + b * PL::TPC, g, spec[b]);
        dft<16>(spec[b], false);
    }
    float E[PL::BPT][16];
    c4_excess<R2>(d, c, ci, bcol, u, E);
    const int row0 = PL::N / 2 - d.out_h / 2, oh = d.out_h;
    for (int p = 0; p < d.P; p++) {
        const int pc = p * d.C + c;
        const PCParam pp = d.pcp[pc];
        const bool col_ok = ci >= pp.i0 && ci < pp.i1;
#pragma unroll
        for (int b = 0; b < PL::BPT; b++) {
            const int j = u + b * PL::TPC;
            float2 v[16];
#pragma unroll
            for (int r = 0; r < 16; r++)
                v[r] = cmul(spec[b][r], c4_transfer<R2>(pp, col_ok, E[b][r], j + r * PL::NB16, d.scale));
            dft<16>(v, true);
            c4_store16_stride1(b0, j, g, v);
        }
        __syncthreads();
        c4_pass_mid<R2, true>(b0, b1, tw, u, g);
        __syncthreads();
        c4_out16<R2>(b1, tw, u, g, B + (size_t)pc * oh * NW + kx0, NW, row0, oh);
    }
}

// Adjoint: per plane the forward transform of four columns of Bt [P*C][out_h][NW],
// x conj(transfer) accumulated in registers; one inverse -> Ab [C][in_h][NW].
template <int R2>
__global__ void CVQPG_C4_BOUNDS(Cols4Plan<R2>::NT, Cols4Plan<R2>::kMinBlocks) blasm_cols4_adj_kernel(BlasmDev d,
                                                                              const float2* __restrict__ Bt,
                                                                              float2* __restrict__ Ab) {
    using PL = Cols4Plan<R2>;
    extern __shared__ float2 sm[];
    float2* b0 = sm;
    float2* b1 = sm + PL::LD;
    float2* tw = sm + 2 * PL::LD;
    const int t = threadIdx.x, g = t & (kC4G - 1), u = t / kC4G;
    const int NW = d.NW, groups = NW / kC4G;
    const int c = blockIdx.x / groups, kx0 = (blockIdx.x - c * groups) * kC4G;
    for (int i = t; i < PL::NTW; i += PL::NT) tw[i] = __ldg(&d.col.tw[i]);
    int ci = kx0 + g + (NW >> 1);
    if (ci >= NW) ci -= NW;
    const float bcol = __ldg(&d.b_col[c * NW + ci]);
    float E[PL::BPT][16];
    c4_excess<R2>(d, c, ci, bcol, u, E);
    float2 acc[PL::BPT][16];
#pragma unroll
    for (int b = 0; b < PL::BPT; b++)
#pragma unroll
        for (int r = 0; r < 16; r++) acc[b][r] = make_float2(0.f, 0.f);
    const int row0 = PL::N / 2 - d.out_h / 2, oh = d.out_h;
    // the next plane's input is staged while this plane computes (when its rows fit)
    float2* stage = sm + 2 * PL::LD + PL::NTW;
    const bool staged = oh <= kC4StageRows;
    if (staged) c4_stage_async(stage, Bt + (size_t)c * oh * NW + kx0, NW, oh, t, PL::NT);
    for (int p = 0; p < d.P; p++) {
        const int pc = p * d.C + c;
        // b0 was last read by the previous plane's radix-R2 pass, before its closing barrier
        if (staged) {
            c4_stage_wait();
            __syncthreads();
            c4_in16_staged<R2>(stage, row0, oh, b0, u, g);
        } else {
            c4_in16<R2>(Bt + (size_t)pc * oh * NW + kx0, NW, row0, oh, b0, u, g);
        }
        __syncthreads();
        if (staged && p + 1 < d.P)  // every thread has read the stage (barrier above)
            c4_stage_async(stage, Bt + (size_t)(pc + d.C) * oh * NW + kx0, NW, oh, t, PL::NT);
        c4_pass_mid<R2, false>(b0, b1, tw, u, g);
        __syncthreads();
        const PCParam pp = d.pcp[pc];
        const bool col_ok = ci >= pp.i0 && ci < pp.i1;
#pragma unroll
        for (int b = 0; b < PL::BPT; b++) {
            const int j = u + b * PL::TPC;
            float2 v[16];
            c4_last16<R2, false>(b1, tw, j, g, v);
            dft<16>(v, false);
#pragma unroll
            for (int r = 0; r < 16; r++)
                acc[b][r] = cadd(acc[b][r], cmulc(v[r], c4_transfer<R2>(pp, col_ok, E[b][r], j + r * PL::NB16,
                                                                          d.scale)));
        }
    }
#pragma unroll
    for (int b = 0; b < PL::BPT; b++) {
        dft<16>(acc[b], true);
        c4_store16_stride1(b0, u + b * PL::TPC, g, acc[b]);
    }
    __syncthreads();
    c4_pass_mid<R2, true>(b0, b1, tw, u, g);
    __syncthreads();
    const int in_h = d.input_mode == 0 ? d.H : d.pH;
    c4_out16<R2>(b1, tw, u, g, Ab + (size_t)c * in_h * NW + kx0, NW, PL::N / 2 - in_h / 2, in_h);
}

// Launch for a grid whose column length is 16 x R2 x 16 and whose width is a multiple of 4.
template <int R2>
void launch_cols4_t(bool adjoint, const BlasmDev& d, const float2* in, float2* out, cudaStream_t s) {
    using PL = Cols4Plan<R2>;
    const unsigned grid = (unsigned)(d.C * (d.NW / kC4G));
    if (!adjoint) {
        cudaFuncSetAttribute(blasm_cols4_fwd_kernel<R2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PL::kSmem);
        blasm_cols4_fwd_kernel<R2><<<grid, PL::NT, PL::kSmem, s>>>(d, in, out);
    } else {
        const size_t smem = PL::kSmem + (size_t)kC4StageRows * kC4G * sizeof(float2);
        cudaFuncSetAttribute(blasm_cols4_adj_kernel<R2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        blasm_cols4_adj_kernel<R2><<<grid, PL::NT, smem, s>>>(d, in, out);
    }
}

}  // namespace cvqpg
