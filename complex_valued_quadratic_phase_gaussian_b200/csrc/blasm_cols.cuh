// Device helpers and the register-spectrum column kernels of the BLASM passes,
// shared by blasm.cu and the per-radix instantiation units blasm_cols_r*.cu.
#pragma once

#include <initializer_list>

#include "blasm.cuh"

namespace cvqpg {

constexpr int kRowThreads = 256;
constexpr int kColThreads = 256;
constexpr int kColPad = 4;  // shared-memory padding shift of the register-spectrum column kernels

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------
// Phase of the band-limited transfer function relative to theta0:
//   2 pi z sqrt(1/lambda^2 - f^2) = theta0 - K u / (1 + sqrt(1 - u)),   u = lambda^2 f^2,
// with u / (1 + sqrt(1-u)) = u/2 + u^2/8 + u^3/16 + 5u^4/128 + 7u^5/256 + O(u^6) for small u
// (truncation below 3e-8 rad for u < 0.02 at K = 2e4).
__device__ __forceinline__ float blasm_excess(float u) {
    if (u < 0.02f) return u * fmaf(u, fmaf(u, fmaf(u, fmaf(u, 0.02734375f, 0.0390625f), 0.0625f), 0.125f), 0.5f);
    return u / (1.0f + sqrtf(1.0f - u));
}

// Transfer function times 1/(NH*NW) at centred indices (j, i), column terms hoisted.
__device__ __forceinline__ float2 transfer_ji(const BlasmDev& d, const PCParam& pp, int c, int j, int i, float bcol) {
    if (j < pp.j0 || j >= pp.j1) return make_float2(0.f, 0.f);
    const int2 ap = d.aperture[j];
    if (i < ap.x || i >= ap.y) return make_float2(0.f, 0.f);
    const float u = __ldg(&d.a_row[c * d.NH + j]) + bcol;
    if (!(u < 1.0f)) return make_float2(0.f, 0.f);  // evanescent: excluded
    float sn, cs;
    sincos_reduced(pp.theta0 - pp.K * blasm_excess(u), &sn, &cs);
    return make_float2(cs * d.scale, sn * d.scale);
}

// ... at natural FFT index (ky, kx)
__device__ __forceinline__ float2 transfer(const BlasmDev& d, const PCParam& pp, int c, int ky, int kx) {
    int j = ky + (d.NH >> 1);
    if (j >= d.NH) j -= d.NH;
    int i = kx + (d.NW >> 1);
    if (i >= d.NW) i -= d.NW;
    if (i < pp.i0 || i >= pp.i1) return make_float2(0.f, 0.f);
    return transfer_ji(d, pp, c, j, i, __ldg(&d.b_col[c * d.NW + i]));
}

// Plane-independent part of the transfer function at centred indices (j, i):
// false where every plane's transfer is zero (outside the aperture, or
// evanescent); otherwise *E = u / (1 + sqrt(1 - u)), so that plane (p, c) has
// phase theta0 - K * E and only a band check and a sincos remain per plane.
__device__ __forceinline__ bool transfer_excess(const BlasmDev& d, int c, int j, int i, float bcol, float* E) {
    const int2 ap = __ldg(&d.aperture[j]);
    const float u = __ldg(&d.a_row[c * d.NH + j]) + bcol;
    const bool live = i >= ap.x && i < ap.y && u < 1.0f;
    *E = live ? blasm_excess(u) : 0.0f;
    return live;
}

// Transfer value of one plane from the hoisted excess (scale 1/(NH*NW) included).
__device__ __forceinline__ float2 transfer_from_excess(const PCParam& pp, float E, float scale) {
    float sn, cs;
    sincos_reduced(pp.theta0 - pp.K * E, &sn, &cs);
    return make_float2(cs * scale, sn * scale);
}

// amplitude clamp to 1 keeping the phase (reference: generate_complex_field(clamp(|U|,0,1), angle(U)))
__device__ __forceinline__ float2 clamp_amplitude(float2 u) {
    const float r2 = u.x * u.x + u.y * u.y;
    if (r2 <= 1.0f) return u;
    const float inv = rsqrtf(r2);
    return make_float2(u.x * inv, u.y * inv);
}

// adjoint of clamp_amplitude at u for the incoming gradient g (torch convention)
__device__ __forceinline__ float2 clamp_amplitude_adjoint(float2 u, float2 g) {
    const float r2 = u.x * u.x + u.y * u.y;
    if (r2 == 0.0f) return make_float2(0.f, 0.f);
    if (r2 <= 1.0f) return g;
    const float r = sqrtf(r2);
    const float c = u.x / r, s = u.y / r;
    const float gphi = -g.x * s + g.y * c;
    return make_float2(-gphi * u.y / r2, gphi * u.x / r2);
}

// Column plan split for the register-held spectrum: the last forward radix RL
// (compile time) and the remaining passes (`head`), used both after the first
// inverse pass and before the last forward pass.
struct ColSplit {
    unsigned long long head_code;
    int head_npass;
    int rl;
    int mb;
    int ntw;  // twiddle-table prefix the passes read (n / smallest radix), copied to shared memory
};

// ---------------------------------------------------------------------------
// Head passes of the column FFT: every pass of the plan except the radix held
// in registers. HeadRuntime follows the plan read at run time (any supported
// length); HeadCT<N, R...> is a head fixed at compile time
// (N = R... * RL), so its strides, index splits and padded shared-memory
// addresses fold into constants and no per-pass radix dispatch is compiled in.
// ---------------------------------------------------------------------------
struct HeadRuntime {
    static constexpr int kN = 0;
    static constexpr bool kEvenPasses = false;  // not known at compile time: every barrier is kept
    // forward head from stride 1 (first pass reads through src); returns the result buffer
    template <typename Src>
    __device__ static __forceinline__ float2* forward(Src src, float2* b0, float2* b1, int ld, int n,
                                                      const ColSplit& cs, const float2* tw) {
        return fft_run_passes<kColPad>(src, b0, b1, ld, 0, n, cs.head_code, cs.head_npass, 1, tw, false);
    }
    // inverse head from stride rl, input in b0, last pass through sink
    template <typename Sink>
    __device__ static __forceinline__ void inverse(Sink sink, float2* b0, float2* b1, int ld, int n, int rl,
                                                   const ColSplit& cs, const float2* tw) {
        fft_run_passes_to<kColPad>([b0](int, int e) { return b0[fft_padT<kColPad>(e)]; }, sink, b1, b0, ld, 0, n,
                                   cs.head_code, cs.head_npass, rl, tw, true);
    }
};

// The BLASM columns are zero-padded 2x: a forward column FFT's input is zero
// outside rows [N/4, 3N/4), and only rows inside [N/4, 3N/4) of an inverse one
// are kept (the output crop is at most the padded height). So a radix-16 first
// forward pass loads 8 of its 16 inputs and a radix-16 last inverse pass forms
// 8 of its 16 outputs (ct_pass MID_IN / MID_OUT).
template <int... R>
struct PassList;
template <int R0, int... Rest>
struct PassList<R0, Rest...> {
    static constexpr int first = R0;
    static constexpr int last = sizeof...(Rest) == 0 ? R0 : PassList<Rest...>::last;
    static constexpr int prod = R0 * PassList<Rest...>::prod;
};
template <>
struct PassList<> {
    static constexpr int first = 0, last = 0, prod = 1;
};

template <int N, int... R>
struct HeadCT {
    static constexpr int kN = N;
    static constexpr int kPasses = (int)sizeof...(R);
    static constexpr bool kEvenPasses = kPasses % 2 == 0;
    static constexpr int kRL = N / PassList<R...>::prod;
    template <typename Src>
    __device__ static __forceinline__ float2* forward(Src src, float2* b0, float2* b1, int, int, const ColSplit&,
                                                      const float2* tw) {
        float2* res = (kPasses % 2 == 1) ? b0 : b1;  // the buffer the last pass does not read
        CtFft<kColPad, kColThreads, N, false, 1, PassList<R...>::first == 16, false, true, R...>::run(
            ElemLoadF<Src>{src}, SmemStoreF<kColPad>{res}, b0, b1, tw);
        return res;
    }
    template <typename Sink>
    __device__ static __forceinline__ void inverse(Sink sink, float2* b0, float2* b1, int, int, int,
                                                   const ColSplit&, const float2* tw) {
        // With an even number of passes the last one reads b1, and the caller's next write
        // of b1 (the second pass of the next plane) comes after that plane's first barrier:
        // the closing barrier is left out.
        CtFft<kColPad, kColThreads, N, true, kRL, false, PassList<R...>::last == 16, !kEvenPasses, R...>::run(
            SmemLoadF<kColPad>{b0}, ElemStoreF<Sink>{sink}, b1, b0, tw);
    }
};

// v[r] = buf[j + r nbL], the input of the register-held pass
template <class Head, int RL>
__device__ __forceinline__ void load_rl(const float2* buf, int j, int nbL, float2 (&v)[RL]) {
    if constexpr (Head::kN > 0) {
        SmemLoadF<kColPad>{buf}.template get<Head::kN, RL>(j, v);
    } else {
#pragma unroll
        for (int r = 0; r < RL; r++) v[r] = buf[fft_padT<kColPad>(j + r * nbL)];
    }
}

// K2 (register-spectrum variant): one column per CTA. Forward column FFT;
// the last forward pass leaves its butterflies in registers together with the
// plane-independent transfer excess E of each element; for each plane the first
// inverse pass (same radix, same elements) multiplies by that plane's transfer
// function straight from registers, and the last inverse pass writes the kept
// rows to global memory. Shared memory: two FFT buffers, the twiddle prefix and
// the excess of every element (-1 where no plane propagates it).
template <int RL, int MB, class Head = HeadRuntime>
__global__ void __launch_bounds__(kColThreads, 3) blasm_cols_fwd_reg_kernel(BlasmDev d, ColSplit cs,
                                                                         const float2* __restrict__ A,
                                                                         float2* __restrict__ B) {
    extern __shared__ float2 sm[];
    const int NH = Head::kN > 0 ? Head::kN : d.NH, NW = d.NW, ld = fft_ldT<kColPad>(NH);
    float2* b0 = sm;
    float2* b1 = sm + ld;
    float2* tw = sm + 2 * ld;
    float* sE = (float*)(tw + cs.ntw);
    for (int t = threadIdx.x; t < cs.ntw; t += blockDim.x) tw[t] = __ldg(&d.col.tw[t]);
    __syncthreads();
    const int c = blockIdx.x / NW, kx = blockIdx.x - c * NW;
    const int y0 = (NH >> 1) - (d.pH >> 1), pH = d.pH;
    const float2* src = A + (size_t)c * pH * NW + kx;
    float2* buf = Head::forward(
        [=](int, int e) {
            const int y = e - y0;
            return (y < 0 || y >= pH) ? make_float2(0.f, 0.f) : __ldg(&src[(size_t)y * NW]);
        },
        b0, b1, ld, NH, cs, tw);
    const int nbL = NH / RL;  // = stride Ns of the last pass; k = j, twiddle stride 1
    int ci = kx + (NW >> 1);
    if (ci >= NW) ci -= NW;
    const float bcol = __ldg(&d.b_col[c * NW + ci]);
    float2 spec[MB][RL];
#pragma unroll
    for (int b = 0; b < MB; b++) {
        const int j = threadIdx.x + b * blockDim.x;
        if (j < nbL) {
            float2 v[RL];
            load_rl<Head, RL>(buf, j, nbL, v);
            apply_twiddles<RL>(v, tw[j]);
            dft<RL>(v, false);
#pragma unroll
            for (int r = 0; r < RL; r++) {
                spec[b][r] = v[r];
                int jj = j + r * nbL + (NH >> 1);
                if (jj >= NH) jj -= NH;
                float E;
                sE[j + r * nbL] = transfer_excess(d, c, jj, ci, bcol, &E) ? E : -1.0f;
            }
        }
    }
    // Each thread reads back only its own excess entries below. With an even number of head
    // passes `buf` is b1 and the plane loop first writes b0, so no barrier is needed here.
    if (!Head::kEvenPasses) __syncthreads();
    const int row0 = (NH >> 1) - (d.out_h >> 1), oh = d.out_h;
    for (int p = 0; p < d.P; p++) {
        const int pc = p * d.C + c;
        const PCParam pp = d.pcp[pc];
        const bool col_ok = ci >= pp.i0 && ci < pp.i1;
#pragma unroll
        for (int b = 0; b < MB; b++) {
            const int j = threadIdx.x + b * blockDim.x;
            if (j < nbL) {
                float2 v[RL];
#pragma unroll
                for (int r = 0; r < RL; r++) {
                    int jj = j + r * nbL + (NH >> 1);
                    if (jj >= NH) jj -= NH;
                    const float E = sE[j + r * nbL];
                    const bool on = col_ok && E >= 0.0f && jj >= pp.j0 && jj < pp.j1;
                    v[r] = on ? cmul(spec[b][r], transfer_from_excess(pp, E, d.scale)) : make_float2(0.f, 0.f);
                }
                dft<RL>(v, true);
                SmemStoreF<kColPad>{b0}.template put<1, RL>(j * RL, v);
            }
        }
        __syncthreads();
        float2* dst = B + (size_t)pc * oh * NW + kx;
        Head::inverse(
            [=](int, int a, float2 v) {
                const int y = a - row0;
                if ((unsigned)y < (unsigned)oh) dst[(size_t)y * NW] = v;
            },
            b0, b1, ld, NH, RL, cs, tw);
    }
}

// K2b (register variant): per plane forward column FFT whose last pass leaves
// its butterflies in registers, multiplied by conj(transfer) and accumulated
// there; then the first inverse pass starts from the accumulator and the last
// one writes the kept rows to global memory.
template <int RL, int MB, class Head = HeadRuntime>
__global__ void __launch_bounds__(kColThreads, 3) blasm_cols_adj_reg_kernel(BlasmDev d, ColSplit cs,
                                                                         const float2* __restrict__ Bt,
                                                                         float2* __restrict__ Ab) {
    extern __shared__ float2 sm[];
    const int NH = Head::kN > 0 ? Head::kN : d.NH, NW = d.NW, ld = fft_ldT<kColPad>(NH);
    float2* b0 = sm;
    float2* b1 = sm + ld;
    float2* tw = sm + 2 * ld;
    float* sE = (float*)(tw + cs.ntw);
    for (int t = threadIdx.x; t < cs.ntw; t += blockDim.x) tw[t] = __ldg(&d.col.tw[t]);
    const int c = blockIdx.x / NW, kx = blockIdx.x - c * NW;
    const int row0 = (NH >> 1) - (d.out_h >> 1), oh = d.out_h;
    const int nbL = NH / RL;
    int ci = kx + (NW >> 1);
    if (ci >= NW) ci -= NW;
    const float bcol = __ldg(&d.b_col[c * NW + ci]);
    for (int e = threadIdx.x; e < NH; e += blockDim.x) {
        int jj = e + (NH >> 1);
        if (jj >= NH) jj -= NH;
        float E;
        sE[e] = transfer_excess(d, c, jj, ci, bcol, &E) ? E : -1.0f;
    }
    __syncthreads();
    float2 acc[MB][RL];
#pragma unroll
    for (int b = 0; b < MB; b++)
#pragma unroll
        for (int r = 0; r < RL; r++) acc[b][r] = make_float2(0.f, 0.f);
    for (int p = 0; p < d.P; p++) {
        const int pc = p * d.C + c;
        const float2* src = Bt + (size_t)pc * oh * NW + kx;
        float2* buf = Head::forward(
            [=](int, int e) {
                const int y = e - row0;
                return (y < 0 || y >= oh) ? make_float2(0.f, 0.f) : __ldg(&src[(size_t)y * NW]);
            },
            b0, b1, ld, NH, cs, tw);
        const PCParam pp = d.pcp[pc];
        const bool col_ok = ci >= pp.i0 && ci < pp.i1;
#pragma unroll
        for (int b = 0; b < MB; b++) {
            const int j = threadIdx.x + b * blockDim.x;
            if (j < nbL) {
                float2 v[RL];
                load_rl<Head, RL>(buf, j, nbL, v);
                apply_twiddles<RL>(v, tw[j]);
                dft<RL>(v, false);
                if (col_ok) {
#pragma unroll
                    for (int r = 0; r < RL; r++) {
                        int jj = j + r * nbL + (NH >> 1);
                        if (jj >= NH) jj -= NH;
                        const float E = sE[j + r * nbL];
                        if (E >= 0.0f && jj >= pp.j0 && jj < pp.j1)
                            acc[b][r] = cadd(acc[b][r], cmulc(v[r], transfer_from_excess(pp, E, d.scale)));
                    }
                }
            }
        }
        // The pass above read `buf`. With an even number of head passes that is b1, which the
        // next plane first writes in its second pass, after its first pass's barrier; and the
        // final inverse below first writes b0. Otherwise buf is b0 and this barrier is needed.
        if (!Head::kEvenPasses) __syncthreads();
    }
#pragma unroll
    for (int b = 0; b < MB; b++) {
        const int j = threadIdx.x + b * blockDim.x;
        if (j < nbL) {
            float2 v[RL];
#pragma unroll
            for (int r = 0; r < RL; r++) v[r] = acc[b][r];
            dft<RL>(v, true);
            SmemStoreF<kColPad>{b0}.template put<1, RL>(j * RL, v);
        }
    }
    __syncthreads();
    const int in_h = d.input_mode == 0 ? d.H : d.pH;
    const int r0 = (NH >> 1) - (in_h >> 1);
    float2* dst = Ab + (size_t)c * in_h * NW + kx;
    Head::inverse(
        [=](int, int a, float2 v) {
            const int y = a - r0;
            if ((unsigned)y < (unsigned)in_h) dst[(size_t)y * NW] = v;
        },
        b0, b1, ld, NH, RL, cs, tw);
}


void launch_cols_reg_r3(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                        cudaStream_t s);
void launch_cols_reg_r5(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                        cudaStream_t s);
void launch_cols_reg_r7(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                        cudaStream_t s);
void launch_cols_reg_r8(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                        cudaStream_t s);
void launch_cols_reg_r11(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                         cudaStream_t s);
void launch_cols_reg_r13(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                         cudaStream_t s);
void launch_cols_reg_r16(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                         cudaStream_t s);

template <int RL, int MB, class Head>
void launch_cols_reg_t(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                       cudaStream_t s) {
    const size_t sm = ((size_t)2 * fft_ldT<kColPad>(d.NH) + cs.ntw) * sizeof(float2) + (size_t)d.NH * sizeof(float);
    if (!adjoint) {
        cudaFuncSetAttribute(blasm_cols_fwd_reg_kernel<RL, MB, Head>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
        blasm_cols_fwd_reg_kernel<RL, MB, Head><<<d.C * d.NW, kColThreads, sm, s>>>(d, cs, in, out);
    } else {
        cudaFuncSetAttribute(blasm_cols_adj_reg_kernel<RL, MB, Head>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
        blasm_cols_adj_reg_kernel<RL, MB, Head><<<d.C * d.NW, kColThreads, sm, s>>>(d, cs, in, out);
    }
}

// Column kernels with a compile-time head for the grids the fits use most; false
// when (d, cs) is not one of them (the run-time plan variants apply). One
// translation unit per grid (blasm_cols_ct*.cu).
bool launch_cols_ct(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                    cudaStream_t s);
bool launch_cols_ct_1664(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                         cudaStream_t s);
bool launch_cols_ct_2176(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                         cudaStream_t s);
bool launch_cols_ct_1152(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                         cudaStream_t s);

// the split (register radix, butterflies per thread, head radices in order) of a column plan
inline bool col_split_is(const ColSplit& cs, int rl, int mb, std::initializer_list<int> head) {
    if (cs.rl != rl || cs.mb != mb || cs.head_npass != (int)head.size()) return false;
    int p = 0;
    for (int r : head)
        if ((int)((cs.head_code >> (5 * p++)) & 31ull) != r) return false;
    return true;
}

// Instantiate the forward and adjoint register-spectrum kernels for one radix.
#define CVQPG_DEFINE_COLS_REG(RL)                                                                                  \
    void launch_cols_reg_r##RL(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out, \
                               cudaStream_t s) {                                                                   \
        if (cs.mb == 1)                                                                                            \
            launch_cols_reg_t<RL, 1, HeadRuntime>(adjoint, d, cs, in, out, s);                                     \
        else                                                                                                       \
            launch_cols_reg_t<RL, 2, HeadRuntime>(adjoint, d, cs, in, out, s);                                     \
    }

}  // namespace cvqpg
