// Shared-memory mixed-radix FFT engine (Stockham autosort, radices 2..17).
//
// A CTA transforms `ntrans` sequences of length n that live in shared memory
// (sequence t at buf + t*ld, element a at index fft_pad(a)). Passes are out of
// place between two buffers, so a thread only ever holds one butterfly in
// registers. The padding (one slot every 32 elements) breaks the power-of-two
// strides of the early passes into distinct banks.
//
// Pass s with radix R and Ns = product of the previous radices computes, for
// every butterfly j in [0, n/R):   k = j mod Ns,
//   v_r = x[j + r*n/R] * W_n^(r*k*n/(Ns*R)),  V = DFT_R(v),
//   y[(j/Ns)*Ns*R + k + r*Ns] = V_r
// (the textbook Stockham formulation, e.g. C. Van Loan, "Computational
// Frameworks for the Fast Fourier Transform", SIAM 1992, sec. 1.7). Forward
// transforms use W_n = exp(-2 pi i / n) (the numpy/torch fft sign), inverse
// ones exp(+2 pi i / n) without the 1/n factor.
#pragma once

#include "common.cuh"
#include "dft_tables.cuh"

namespace cvqpg {

constexpr int kMaxPasses = 8;

struct FftPlan {
    int n;
    int npass;
    unsigned long long code;  // radix of pass p in bits [5p, 5p+5)
    const float2* tw;         // device table W_n^m = exp(-2 pi i m / n), m in [0, n)
};

// Padded index: one spare slot every 2^PS elements (PS = 5 by default; the
// column kernels use 4, which also keeps the stride-16 stores of a first
// radix-16 pass on distinct banks).
template <int PS = 5>
__host__ __device__ __forceinline__ int fft_padT(int i) { return i + (i >> PS); }
template <int PS = 5>
__host__ __device__ __forceinline__ int fft_ldT(int n) { return fft_padT<PS>(n - 1) + 2; }
__host__ __device__ __forceinline__ int fft_pad(int i) { return fft_padT<5>(i); }
__host__ __device__ __forceinline__ int fft_ld(int n) { return fft_ldT<5>(n); }

// ---------------------------------------------------------------------------
// small DFTs on registers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 mul_i(float2 a, bool neg) {  // neg ? -i*a : +i*a
    return neg ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

__device__ __forceinline__ void dft4(float2& x0, float2& x1, float2& x2, float2& x3, bool inv) {
    const float2 t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), t3 = csub(x1, x3);
    const float2 r = mul_i(t3, !inv);  // forward: -i*t3
    x0 = cadd(t0, t2);
    x2 = csub(t0, t2);
    x1 = cadd(t1, r);
    x3 = csub(t1, r);
}

// Second half of the 4 x 4 DFT-16 (twiddle W16^(n2 k1), row DFTs over n2,
// transpose). MID_OUT: only the outputs 4..11 are formed (rows k2 = 1, 2 of
// each row DFT); the others are left undefined.
template <bool MID_OUT = false>
__device__ __forceinline__ void dft16_twiddle_rows(float2 (&v)[16], bool inv) {
#pragma unroll
    for (int n2 = 1; n2 < 4; n2++)
#pragma unroll
        for (int k1 = 1; k1 < 4; k1++) {
            const int q = (n2 * k1) & 15;
            const float2 w = make_float2(DftTab<16>::c(q), inv ? DftTab<16>::s(q) : -DftTab<16>::s(q));
            v[4 * k1 + n2] = cmul(v[4 * k1 + n2], w);
        }
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
        if constexpr (!MID_OUT) {
            dft4(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3], inv);
        } else {  // the k2 = 1, 2 outputs of dft4 only
            const float2 x0 = v[4 * k1], x1 = v[4 * k1 + 1], x2 = v[4 * k1 + 2], x3 = v[4 * k1 + 3];
            const float2 t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), t3 = csub(x1, x3);
            v[4 * k1 + 1] = cadd(t1, mul_i(t3, !inv));
            v[4 * k1 + 2] = csub(t0, t2);
        }
    }
    float2 x[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++)
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) x[k1 + 4 * k2] = v[4 * k1 + k2];
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = x[k];
}

// DFT-16 whose inputs other than 4..11 are zero: the column DFTs over n1 have
// x0 = x3 = 0 (same values as dft<16> on the zero-filled input).
__device__ __forceinline__ void dft16_mid_in(float2 (&v)[16], bool inv) {
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
        const float2 a = v[4 + n2], b = v[8 + n2];
        const float2 r = mul_i(a, !inv);
        v[n2] = cadd(b, a);
        v[8 + n2] = csub(b, a);
        v[4 + n2] = csub(r, b);
        v[12 + n2] = make_float2(-b.x - r.x, -b.y - r.y);
    }
    dft16_twiddle_rows(v, inv);
}

template <int R>
__device__ __forceinline__ void dft(float2 (&v)[R], bool inv) {
    if constexpr (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        dft4(v[0], v[1], v[2], v[3], inv);
    } else if constexpr (R == 8) {
        // radix-2 x 4, in place: evens and odds transformed where they sit
        dft4(v[0], v[2], v[4], v[6], inv);
        dft4(v[1], v[3], v[5], v[7], inv);
        float2 x[8];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float2 w = make_float2(DftTab<8>::c(k), inv ? DftTab<8>::s(k) : -DftTab<8>::s(k));
            const float2 t = k == 0 ? v[1] : cmul(v[2 * k + 1], w);
            x[k] = cadd(v[2 * k], t);
            x[k + 4] = csub(v[2 * k], t);
        }
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = x[k];
    } else if constexpr (R == 16) {
        // 4 x 4 in place: column DFTs over n1, twiddle W16^(n2 k1), row DFTs over n2,
        // then the 4x4 transpose is a compile-time renaming of registers.
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) dft4(v[n2], v[4 + n2], v[8 + n2], v[12 + n2], inv);
        dft16_twiddle_rows(v, inv);
    } else {
        // odd R: X_k = x0 + sum_m (x_m + x_{R-m}) cos(2 pi m k/R) -/+ i (x_m - x_{R-m}) sin(2 pi m k/R);
        // the inputs are folded into a[], b[] first, then the outputs overwrite v.
        static_assert(R % 2 == 1, "odd radix expected");
        constexpr int h = (R - 1) / 2;
        float2 a[h], b[h];
        const float2 x0 = v[0];
        float2 sum = x0;
#pragma unroll
        for (int m = 1; m <= h; m++) {
            a[m - 1] = cadd(v[m], v[R - m]);
            b[m - 1] = csub(v[m], v[R - m]);
            sum = cadd(sum, a[m - 1]);
        }
        v[0] = sum;
#pragma unroll
        for (int k = 1; k <= h; k++) {
            float2 A = x0, B = make_float2(0.f, 0.f);
#pragma unroll
            for (int m = 1; m <= h; m++) {
                const int q = (m * k) % R;
                A.x = fmaf(a[m - 1].x, DftTab<R>::c(q), A.x);
                A.y = fmaf(a[m - 1].y, DftTab<R>::c(q), A.y);
                B.x = fmaf(b[m - 1].x, DftTab<R>::s(q), B.x);
                B.y = fmaf(b[m - 1].y, DftTab<R>::s(q), B.y);
            }
            if (!inv) {
                v[k] = make_float2(A.x + B.y, A.y - B.x);
                v[R - k] = make_float2(A.x - B.y, A.y + B.x);
            } else {
                v[k] = make_float2(A.x - B.y, A.y + B.x);
                v[R - k] = make_float2(A.x + B.y, A.y - B.x);
            }
        }
    }
}

// v[r] *= w^r for r = 1..R-1 from one table value w = w^1. The powers come
// from a product tree, w^r = w^(2^k) * w^(r - 2^k) with 2^k the highest power
// of two in r (and w^(2^k) = (w^(2^(k-1)))^2): R-2 products as in a running
// product, but a dependency depth of about log2(R) instead of R-2, so the
// butterfly does not wait on a serial chain, and at most ~2 log2(R) roundings.
__device__ __forceinline__ float2 csqr(float2 a) {
    return make_float2(fmaf(a.x, a.x, -a.y * a.y), 2.0f * a.x * a.y);
}
// TREE = false forms the powers by a running product instead (two live values
// rather than R-1: for register-bound kernels).
template <int R, bool TREE = true>
__device__ __forceinline__ void apply_twiddles(float2 (&v)[R], float2 w1) {
    if constexpr (TREE) {
        float2 pw[R];
        pw[1] = w1;
#pragma unroll
        for (int r = 2; r < R; r++) {
            int hb = 1;
            while (hb * 2 <= r) hb *= 2;
            pw[r] = (r == hb) ? csqr(pw[r / 2]) : cmul(pw[hb], pw[r - hb]);
        }
#pragma unroll
        for (int r = 1; r < R; r++) v[r] = cmul(v[r], pw[r]);
    } else {
        float2 w = w1;
#pragma unroll
        for (int r = 1; r < R; r++) {
            v[r] = cmul(v[r], w);
            if (r + 1 < R) w = cmul(w, w1);
        }
    }
}

// Decompose a butterfly index j of a pass with stride Ns: q = j / Ns, k = j % Ns.
// floor((j + 1/2) / Ns) evaluated in float is exact for j < 2^22: the true value
// is at least 1/(2 Ns) from an integer and the float error is below j 2^-23 / Ns.
__device__ __forceinline__ void split_index(int j, int Ns, float inv_ns, int& q, int& k) {
    q = __float2int_rz(fmaf((float)j, inv_ns, 0.5f * inv_ns));
    k = j - q * Ns;
}

// ---------------------------------------------------------------------------
// one out-of-place Stockham pass over 2^tshift interleaved sequences. `src(t, a)`
// returns element a of sequence t (a shared-memory read, or for the first pass a
// global read with a pointwise operation fused into it); `sink(t, a, v)` stores
// element a of the result (a shared-memory write, or for the last pass a global
// write of the kept elements). Each thread holds a single butterfly at a time,
// so the register footprint is one radix. `tw` may point to shared or global memory.
// ---------------------------------------------------------------------------
template <int PS = 5>
struct SmemSinkT {
    float2* out;
    int ld;
    __device__ __forceinline__ void operator()(int t, int a, float2 v) const { out[t * ld + fft_padT<PS>(a)] = v; }
};
using SmemSink = SmemSinkT<5>;

template <int R, typename Src, typename Sink>
__device__ __forceinline__ void fft_pass(Src src, Sink sink, int tshift, int n, int Ns, const float2* tw, bool inv) {
    const int nb = n / R;
    const int total = nb << tshift;
    const int stride = n / (Ns * R);
    const float inv_ns = 1.0f / (float)Ns;
    const int tmask = (1 << tshift) - 1;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int t = idx & tmask, j = idx >> tshift;
        int q, k;
        split_index(j, Ns, inv_ns, q, k);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = src(t, j + r * nb);
        if (Ns > 1) {
            float2 w = tw[k * stride];
            if (inv) w.y = -w.y;
            apply_twiddles<R>(v, w);
        }
        dft<R>(v, inv);
        const int o = q * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; r++) sink(t, o + r * Ns, v[r]);
    }
    __syncthreads();
}

template <typename Src, typename Sink>
__device__ __forceinline__ void fft_pass_dispatch(int R, Src src, Sink sink, int tshift, int n, int Ns,
                                                  const float2* tw, bool inv) {
    switch (R) {
        case 16: fft_pass<16>(src, sink, tshift, n, Ns, tw, inv); break;
        case 8: fft_pass<8>(src, sink, tshift, n, Ns, tw, inv); break;
        case 4: fft_pass<4>(src, sink, tshift, n, Ns, tw, inv); break;
        case 2: fft_pass<2>(src, sink, tshift, n, Ns, tw, inv); break;
        case 3: fft_pass<3>(src, sink, tshift, n, Ns, tw, inv); break;
        case 5: fft_pass<5>(src, sink, tshift, n, Ns, tw, inv); break;
        case 7: fft_pass<7>(src, sink, tshift, n, Ns, tw, inv); break;
        case 11: fft_pass<11>(src, sink, tshift, n, Ns, tw, inv); break;
        case 13: fft_pass<13>(src, sink, tshift, n, Ns, tw, inv); break;
        case 17: fft_pass<17>(src, sink, tshift, n, Ns, tw, inv); break;
        default: break;
    }
}

// Run `npass` passes (radices packed 5 bits each in `code`, first one in the low
// bits) starting at stride Ns0. The first pass reads through `first`; passes
// ping-pong between the shared buffers a and b; the last pass stores through
// `last` instead. The caller must synchronise before `first` reads shared data
// written earlier; ends with a barrier.
template <int PS = 5, typename First, typename Last>
__device__ __forceinline__ void fft_run_passes_to(First first, Last last, float2* a, float2* b, int ld, int tshift,
                                                  int n, unsigned long long code, int npass, int Ns0,
                                                  const float2* tw, bool inv) {
    int Ns = Ns0;
    int R = (int)(code & 31ull);
    if (npass == 1) {
        fft_pass_dispatch(R, first, last, tshift, n, Ns, tw, inv);
        return;
    }
    fft_pass_dispatch(R, first, SmemSinkT<PS>{a, ld}, tshift, n, Ns, tw, inv);
    Ns *= R;
    float2* cur = a;
    float2* nxt = b;
    for (int p = 1; p < npass; p++) {
        R = (int)((code >> (5 * p)) & 31ull);
        const float2* in = cur;
        auto src = [in, ld](int t, int e) { return in[t * ld + fft_padT<PS>(e)]; };
        if (p + 1 < npass)
            fft_pass_dispatch(R, src, SmemSinkT<PS>{nxt, ld}, tshift, n, Ns, tw, inv);
        else
            fft_pass_dispatch(R, src, last, tshift, n, Ns, tw, inv);
        Ns *= R;
        float2* tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
}

// Same, with the result left in shared memory; returns the buffer holding it.
template <int PS = 5, typename First>
__device__ __forceinline__ float2* fft_run_passes(First first, float2* a, float2* b, int ld, int tshift, int n,
                                                  unsigned long long code, int npass, int Ns0, const float2* tw,
                                                  bool inv) {
    float2* res = (npass & 1) ? a : b;
    fft_run_passes_to<PS>(first, SmemSinkT<PS>{res, ld}, a, b, ld, tshift, n, code, npass, Ns0, tw, inv);
    return res;
}

// Full transform of 2^tshift sequences (all passes of the plan from stride 1).
template <typename First>
__device__ __forceinline__ float2* fft_run(First first, float2* a, float2* b, int ld, int tshift, FftPlan plan,
                                           bool inv) {
    return fft_run_passes(first, a, b, ld, tshift, plan.n, plan.code, plan.npass, 1, plan.tw, inv);
}

// Full transform whose last pass stores through `last`.
template <typename First, typename Last>
__device__ __forceinline__ void fft_run_to(First first, Last last, float2* a, float2* b, int ld, int tshift,
                                           FftPlan plan, bool inv) {
    fft_run_passes_to(first, last, a, b, ld, tshift, plan.n, plan.code, plan.npass, 1, plan.tw, inv);
}

// ---------------------------------------------------------------------------
// Compile-time plans: the same Stockham passes with the length, the radices and
// the strides as template constants, so a kernel instantiated for one grid has
// no per-pass radix dispatch and its index splits, strides and padded
// addresses fold into constants. NT = threads of the CTA.
//   load.get<N, R>(j, v):   v[r] = x[j + r N/R]
//   store.put<NS, R>(o, v): y[o + r NS] = v[r]
// ---------------------------------------------------------------------------
template <int PS>
struct SmemLoadF {  // padded shared buffer (fft_padT<PS>)
    const float2* in;
    template <int N, int R>
    __device__ __forceinline__ void get(int j, float2 (&v)[R]) const {
        constexpr int nb = N / R, blk = 1 << PS;
        if constexpr (nb % blk == 0) {  // (j + r nb) >> PS = (j >> PS) + r nb / blk
            const float2* p = in + fft_padT<PS>(j);
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = p[r * (nb + nb / blk)];
        } else {
#pragma unroll
            for (int r = 0; r < R; r++) v[r] = in[fft_padT<PS>(j + r * nb)];
        }
    }
};

template <int PS>
struct SmemStoreF {
    float2* out;
    template <int NS, int R>
    __device__ __forceinline__ void put(int o, const float2 (&v)[R]) const {
        constexpr int blk = 1 << PS;
        if constexpr (NS % blk == 0) {
            float2* p = out + fft_padT<PS>(o);
#pragma unroll
            for (int r = 0; r < R; r++) p[r * (NS + NS / blk)] = v[r];
        } else if constexpr (NS == 1 && blk % R == 0) {  // o is a multiple of R: o..o+R-1 share a block
            float2* p = out + fft_padT<PS>(o);
#pragma unroll
            for (int r = 0; r < R; r++) p[r] = v[r];
        } else {
#pragma unroll
            for (int r = 0; r < R; r++) out[fft_padT<PS>(o + r * NS)] = v[r];
        }
    }
};

template <typename Src>
struct ElemLoadF {  // element reads through src(0, e) (global loads with a fused pointwise op)
    Src src;
    template <int N, int R>
    __device__ __forceinline__ void get(int j, float2 (&v)[R]) const {
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = src(0, j + r * (N / R));
    }
};

template <typename Sink>
struct ElemStoreF {  // element writes through sink(0, a, v)
    Sink sink;
    template <int NS, int R>
    __device__ __forceinline__ void put(int o, const float2 (&v)[R]) const {
#pragma unroll
        for (int r = 0; r < R; r++) sink(0, o + r * NS, v[r]);
    }
};

// MID_IN (first pass, NS = 1): the input is zero outside its middle half
// [N/4, 3N/4), i.e. outside r in [R/4, 3R/4); only those elements are loaded.
// MID_OUT (last pass, NS = N/R): only the middle half of the output is used;
// only r in [R/4, 3R/4) is formed and stored. Both for R = 16.
// SYNC = false leaves out the closing barrier, for a caller that has shown the
// next writes of the buffers this pass reads come after another barrier.
template <int NT, int N, int R, int NS, bool INV, bool MID_IN = false, bool MID_OUT = false, bool SYNC = true,
          typename Load, typename Store>
__device__ __forceinline__ void ct_pass(const Load& load, const Store& store, const float2* tw) {
    static_assert(!(MID_IN || MID_OUT) || R == 16, "middle-half pruning is written for radix 16");
    static_assert(!MID_IN || NS == 1, "input pruning applies to the first pass");
    static_assert(!MID_OUT || NS * R == N, "output pruning applies to the last pass");
    constexpr int nb = N / R;
    constexpr int stride = N / (NS * R);
    for (int j = threadIdx.x; j < nb; j += NT) {
        const int q = j / NS, k = j - q * NS;
        float2 v[R];
        if constexpr (MID_IN) {
            float2 m[R / 2];
            load.template get<N / 2, R / 2>(j + N / 4, m);  // m[i] = x[j + N/4 + i N/R]
#pragma unroll
            for (int i = 0; i < R / 2; i++) v[R / 4 + i] = m[i];
#pragma unroll
            for (int i = 0; i < R / 4; i++) v[i] = v[3 * R / 4 + i] = make_float2(0.f, 0.f);
        } else {
            load.template get<N, R>(j, v);
        }
        if constexpr (NS > 1) {
            float2 w = tw[k * stride];
            if (INV) w.y = -w.y;
            apply_twiddles<R>(v, w);
        }
        if constexpr (MID_IN) {
            dft16_mid_in(reinterpret_cast<float2(&)[16]>(v), INV);
        } else if constexpr (MID_OUT) {
#pragma unroll
            for (int n2 = 0; n2 < 4; n2++) dft4(v[n2], v[4 + n2], v[8 + n2], v[12 + n2], INV);
            dft16_twiddle_rows<true>(reinterpret_cast<float2(&)[16]>(v), INV);
        } else {
            dft<R>(v, INV);
        }
        if constexpr (MID_OUT) {
            float2 m[R / 2];
#pragma unroll
            for (int i = 0; i < R / 2; i++) m[i] = v[R / 4 + i];
            store.template put<NS, R / 2>(q * NS * R + k + (R / 4) * NS, m);
        } else {
            store.template put<NS, R>(q * NS * R + k, v);
        }
    }
    if constexpr (SYNC) __syncthreads();
}

// Passes R, Rest... of length N from stride NS: the first reads through `load`,
// the intermediate ones ping-pong a -> b -> a ..., the last writes through `last`
// (which must not be the buffer the last pass reads: buffer (passes - 2) % 2).
// MI / MO: middle-half pruning of the first / last pass (ct_pass MID_IN / MID_OUT);
// LS: the last pass ends with a barrier (ct_pass SYNC).
template <int PS, int NT, int N, bool INV, int NS, bool MI, bool MO, bool LS, int R, int... Rest>
struct CtFft {
    static constexpr int kPasses = 1 + (int)sizeof...(Rest);
    template <typename Load, typename Store>
    __device__ static __forceinline__ void run(const Load& load, const Store& last, float2* a, float2* b,
                                               const float2* tw) {
        if constexpr (sizeof...(Rest) == 0) {
            ct_pass<NT, N, R, NS, INV, MI, MO, LS>(load, last, tw);
        } else {
            ct_pass<NT, N, R, NS, INV, MI, false>(load, SmemStoreF<PS>{a}, tw);
            CtFft<PS, NT, N, INV, NS * R, false, MO, LS, Rest...>::run(SmemLoadF<PS>{a}, last, b, a, tw);
        }
    }
};

// Host: factor n into supported radices in one of four orders (0: 16/8/4/2
// first, then 3..17; 1: odd radices first, largest first, then 16/8/4/2;
// 2: 8/4/2 only, then odd; 3: odd first, then 8/4/2). Returns false when n has
// a prime factor above 17 or needs more than kMaxPasses passes.
bool make_fft_plan(int n, FftPlan* plan, int order = 0);

}  // namespace cvqpg
