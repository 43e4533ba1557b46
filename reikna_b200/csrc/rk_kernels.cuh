// Device side of the FFT passes.
//
// A pass transforms a tile of NL lines of length L held by one CTA.  The line FFT is
// a Stockham autosort decomposition (natural-order output, no bit reversal): stage s
// with radix R and P = product of the earlier radices takes, for butterfly b, the R
// inputs at positions b + (L/R) m, applies an R-point register DFT, multiplies output
// m' by W_{L/P}^{j1 m'} (j1 = b / P) and writes it to position (b % P) + P (m' + R j1).
// The first stage reads HBM directly (positions are consecutive across threads, so
// the loads coalesce) and the last stage writes HBM directly; only the stages in
// between go through shared memory.  This is the role of reikna's fft_local /
// fft_global passes (reikna/fft/fft.mako:750-1038), re-derived for sm_100a:
// fixed compile-time radix plans, FP64-generated twiddle tables instead of per-element
// sin/cos (reikna/fft/fft.mako:636-649), and transformations applied on the first
// load and the last store (reikna/core/transformation_modules.py:260-318).
#pragma once
#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stdint.h>
#endif

#include "rk_dft.cuh"
#include "rk_params.h"

namespace rk {

// ------------------------------------------------------------------------------
// radix plans: RT elements per thread, NS stages with radices R[]
// ------------------------------------------------------------------------------
template <typename T, int L> struct Radix;
#define RK_RADIX(TY, LL, RTV, ...)                                  \
    template <> struct Radix<TY, LL> {                              \
        static constexpr int RT = RTV;                              \
        static constexpr int R[] = {__VA_ARGS__};                   \
        static constexpr int NS = sizeof(R) / sizeof(int);          \
    };
RK_RADIX(float, 1, 1, 1)
RK_RADIX(float, 2, 2, 2)
RK_RADIX(float, 4, 4, 4)
RK_RADIX(float, 8, 8, 8)
RK_RADIX(float, 16, 16, 16)
RK_RADIX(float, 32, 8, 8, 4)
RK_RADIX(float, 64, 8, 8, 8)
RK_RADIX(float, 128, 16, 16, 8)
RK_RADIX(float, 256, 16, 16, 16)
RK_RADIX(float, 512, 16, 16, 16, 2)
RK_RADIX(float, 1024, 16, 16, 16, 4)
RK_RADIX(float, 2048, 16, 16, 16, 8)
RK_RADIX(float, 4096, 16, 16, 16, 16)
RK_RADIX(float, 8192, 32, 32, 16, 16)
RK_RADIX(float, 16384, 32, 32, 32, 16)
RK_RADIX(double, 1, 1, 1)
RK_RADIX(double, 2, 2, 2)
RK_RADIX(double, 4, 4, 4)
RK_RADIX(double, 8, 8, 8)
RK_RADIX(double, 16, 16, 16)
RK_RADIX(double, 32, 8, 8, 4)
RK_RADIX(double, 64, 8, 8, 8)
RK_RADIX(double, 128, 16, 16, 8)
RK_RADIX(double, 256, 16, 16, 16)
RK_RADIX(double, 512, 8, 8, 8, 8)
RK_RADIX(double, 1024, 16, 16, 16, 4)
RK_RADIX(double, 2048, 16, 16, 16, 8)
RK_RADIX(double, 4096, 16, 16, 16, 16)
RK_RADIX(double, 8192, 16, 16, 16, 16, 2)
#undef RK_RADIX

// Radix plan PL of a length: 0 = the table above; 1 = sixteen elements a thread where
// the table holds 32 (8192-point float32 lines on 512 threads, the 16-element
// stages {16, 16, 16, 2}: half the registers a thread, twice the warps a line).
// Line-pass variant codes carry the plan in bit 4 (VAR = variant + 16 PL).
template <typename T, int L, int PL = 0> struct RadixP : Radix<T, L> {};
template <> struct RadixP<float, 8192, 1> {
    static constexpr int RT = 16;
    static constexpr int R[] = {16, 16, 16, 2};
    static constexpr int NS = 4;
};

// Stage twiddle tables of a length-L line: stage s (radix R, P = product of the
// earlier radices, J = L / (P R) butterfly groups) needs W_{L/P}^(j1 m) for
// 1 <= m < R, j1 < J, stored as [m - 1][j1]; the stages follow each other and the
// last stage needs none.  Generated in FP64 on the device (rk_lib.cu).
template <typename T, int L, int PL = 0> struct TwLayout {
    using RC = RadixP<T, L, PL>;
    static constexpr int size_of(int s) {
        int P = 1;
        for (int i = 0; i < s; ++i) P *= RC::R[i];
        return (RC::R[s] - 1) * (L / (P * RC::R[s]));
    }
    static constexpr int offset(int s) {
        int o = 0;
        for (int i = 0; i < s; ++i) o += size_of(i);
        return o;
    }
    static constexpr int total() { return RC::NS > 1 ? offset(RC::NS - 1) : 0; }
};

template <typename T> struct Vec;   // lanes per 128-byte segment
template <> struct Vec<float> { static constexpr int N = 16; };
template <> struct Vec<double> { static constexpr int N = 8; };

template <typename T, int L, int MODE, int PL = 0> struct LineCfg {
    using RC = RadixP<T, L, PL>;
    static constexpr int RT = RC::RT;
    static constexpr int TPL = L / RT;
    static constexpr int ESZ = 2 * sizeof(T);
    static constexpr int NL_POS = TPL >= 256 ? 1 : 256 / TPL;
    static constexpr int NL_LANE_A = (256 / TPL) > Vec<T>::N ? (256 / TPL) : Vec<T>::N;
    static constexpr int NL_LANE_B = 65536 / (L * ESZ);
    static constexpr int NL_LANE = NL_LANE_A < NL_LANE_B ? NL_LANE_A : NL_LANE_B;
    static constexpr int NL = MODE == MODE_POS ? NL_POS : NL_LANE;
    static constexpr int NT = NL * TPL;
    static constexpr int LS = L + L / 16;   // padded line stride (position mode)
};

// ------------------------------------------------------------------------------
// integer helpers
// ------------------------------------------------------------------------------
__device__ __forceinline__ void divmod64(int64_t a, int64_t b, int64_t& q, int64_t& r) {
    if (((uint64_t)a | (uint64_t)b) >> 32 == 0) {
        uint32_t qa = (uint32_t)a / (uint32_t)b;
        q = qa;
        r = (uint32_t)a - qa * (uint32_t)b;
    } else {
        q = a / b;
        r = a - q * b;
    }
}

// flat element offset of a line on one side, plus validity
struct LineAddr {
    int64_t base;
    int64_t c;
    bool ok;
};

__device__ __forceinline__ int64_t dims_base(int nd, const int64_t* shape, const int64_t* stride,
                                             const int64_t* bound, const int32_t* shift, int64_t idx,
                                             bool& ok) {
    int64_t base = 0;
    for (int d = nd - 1; d >= 0; --d) {
        int64_t q, r;
        divmod64(idx, shape[d], q, r);
        idx = q;
        if (shift[d]) {
            r += shift[d];
            if (r >= shape[d]) r -= shape[d];
        }
        ok = ok && (r < bound[d]);
        base += r * stride[d];
    }
    return base;
}

__device__ __forceinline__ LineAddr line_addr(const Side& s, int64_t line, int64_t C, int64_t I, bool lok) {
    LineAddr la;
    int64_t ci = C * I;
    int64_t o, rem, c, i;
    divmod64(line, ci, o, rem);
    divmod64(rem, I, c, i);
    bool ok = lok;
    int64_t base = s.offset;
    base += dims_base(s.nd_o, s.o_shape, s.o_stride, s.o_bound, s.o_shift, o, ok);
    base += dims_base(s.nd_i, s.i_shape, s.i_stride, s.i_bound, s.i_shift, i, ok);
    la.base = base;
    la.c = c;
    la.ok = ok;
    return la;
}

// ------------------------------------------------------------------------------
// element load / store with the fused value ops
// ------------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T hann(int64_t u, int32_t w) {
    if (u >= w) return T(1);
    // 0.5 * (1 - cos(2 pi u / (w - 1)))
    T x = T(2) * T(u) / T(w - 1);
    return T(0.5) * (T(1) - cospi(x));
}

// Square root for magnitudes (|z| = sqrt(re^2 + im^2), the norm post-operation of
// order 1): the hardware's approximate single-precision square root (relative error
// about 2^-23, below the transform's own rounding) for float, the correctly rounded
// one for double.
template <typename T> __device__ __forceinline__ T mag_sqrt(T x) { return sqrt(x); }
template <> __device__ __forceinline__ float mag_sqrt<float>(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// RP: compile the pair-read branch in (only the half-length route's passes set
// SF_RPAIR; other kernels leave it out to keep their registers)
template <typename T, bool RP = true>
__device__ __forceinline__ cplx<T> side_load(const Side& s, const LineAddr& la, int64_t j) {
    using V = cplx<T>;
    V v = cmk<V>(T(0), T(0));
    const int64_t a = la.c * s.cA + j * s.jB;
    bool inb = false;  // an element of the user's array (not padding)
    if (la.ok && a < s.ax_len) {
        int64_t u = a + s.ax_shift;
        if (u >= s.ax_len) u -= s.ax_len;
        inb = u < s.ax_bound;
        if (RP && (s.flags & SF_RPAIR) && u < s.ax_bound) {
            // a real signal read as sample pairs (x[2u], x[2u+1]); a window covers the
            // sample index 2u / 2u + 1
            const int64_t off = la.base + 2 * u * s.ax_stride;
            T x0, x1;
            if (s.fmt == RK_FMT_F64) {
                x0 = (T)reinterpret_cast<const double*>(s.ptr)[off];
                x1 = (T)reinterpret_cast<const double*>(s.ptr)[off + s.ax_stride];
            } else {
                x0 = (T)reinterpret_cast<const float*>(s.ptr)[off];
                x1 = (T)reinterpret_cast<const float*>(s.ptr)[off + s.ax_stride];
            }
            if (s.flags & SF_WINDOW) {
                const T* wt = reinterpret_cast<const T*>(s.win);
                x0 *= wt ? (2 * u < s.win_len ? wt[2 * u] : T(1)) : hann<T>(2 * u, s.win_len);
                x1 *= wt ? (2 * u + 1 < s.win_len ? wt[2 * u + 1] : T(1)) : hann<T>(2 * u + 1, s.win_len);
            }
            v = cmk<V>(x0, x1);
        } else if (u < s.ax_bound) {
            const int64_t off = la.base + u * s.ax_stride;
            switch (s.fmt) {
                case RK_FMT_C64: {
                    float2 t = reinterpret_cast<const float2*>(s.ptr)[off];
                    v = cmk<V>((T)t.x, (T)t.y);
                } break;
                case RK_FMT_C128: {
                    double2 t = reinterpret_cast<const double2*>(s.ptr)[off];
                    v = cmk<V>((T)t.x, (T)t.y);
                } break;
                case RK_FMT_F32:
                    v.x = (T)reinterpret_cast<const float*>(s.ptr)[off];
                    break;
                case RK_FMT_F64:
                    v.x = (T)reinterpret_cast<const double*>(s.ptr)[off];
                    break;
                case RK_FMT_F32_PAIR:
                    v.x = (T)reinterpret_cast<const float*>(s.ptr)[off];
                    v.y = (T)reinterpret_cast<const float*>(s.ptr2)[off - s.offset + s.offset2];
                    break;
                case RK_FMT_F64_PAIR:
                    v.x = (T)reinterpret_cast<const double*>(s.ptr)[off];
                    v.y = (T)reinterpret_cast<const double*>(s.ptr2)[off - s.offset + s.offset2];
                    break;
#ifdef RK_USER_LOAD
                case RK_FMT_USER:
                    // transformation code compiled with this kernel: off is the flat
                    // C-order index of the element in the FFT array
                    v = RK_USER_LOAD<T>(s, off);
                    break;
#endif
                default:
                    break;
            }
            if (s.flags & SF_WINDOW) {
                // the plan's FP64-generated table when present (the window ends at win_len)
                const T w = s.win ? (u < s.win_len ? reinterpret_cast<const T*>(s.win)[u] : T(1)) : hann<T>(u, s.win_len);
                v = cscale(v, w);
            }
        }
    }
    const int32_t f = s.flags;
    if (f & SF_SCALE) v = cmul(v, cmk<V>((T)s.scale_re, (T)s.scale_im));
    if ((f & SF_ADD) && inb) {
        v.x += (T)s.add_re;
        v.y += (T)s.add_im;
    }
    if (f & SF_PRE_CONJ) v = cconj(v);
    // the tables hold ax_len entries; beyond that the element is the zero padding
    if (a < s.ax_len) {
        if (f & SF_CHIRP) v = cmul(v, reinterpret_cast<const V*>(s.chirp)[a]);
        if (f & SF_TAB) v = cmul(v, reinterpret_cast<const V*>(s.tab)[a]);
    }
    if (f & SF_POST_CONJ) v = cconj(v);
    return v;
}

// W_{tw4N}^(e) for e < tw4N via the two-level 2^24 table, formed in FP64 from the
// FP64 tables and rounded once to the pass precision
template <typename T>
__device__ __forceinline__ cplx<T> tw4(const PassParams& p, int64_t e) {
    using V = cplx<T>;
    // tw4_N is a power of two <= 2^TW4_LOG: scale the exponent by a shift
    const int sh = TW4_LOG - (63 - __clzll((unsigned long long)p.tw4_N));
    const int64_t k = (e & (p.tw4_N - 1)) << sh;
    const double2 hi = __ldg(reinterpret_cast<const double2*>(p.tw4_hi) + (k >> 12));
    const double2 lo = __ldg(reinterpret_cast<const double2*>(p.tw4_lo) + (k & (TW4_HALF - 1)));
    const double2 w = cmul(hi, lo);
    return cmk<V>((T)w.x, (T)w.y);
}

template <typename T>
__device__ __forceinline__ void side_store(const Side& s, const PassParams& p, const LineAddr& la, int64_t j,
                                           cplx<T> v) {
    using V = cplx<T>;
    const int64_t a = la.c * s.cA + j * s.jB;
    const int32_t f = s.flags;
    if (f & SF_TW4) v = cmul(v, tw4<T>(p, la.c * j));
    if (f & SF_PRE_CONJ) v = cconj(v);
    if (!(la.ok && a < s.ax_len)) return;
    if (f & SF_CHIRP) v = cmul(v, reinterpret_cast<const V*>(s.chirp)[a]);
    if (f & SF_POST_CONJ) v = cconj(v);
    if (f & SF_SCALE) v = cmul(v, cmk<V>((T)s.scale_re, (T)s.scale_im));
    if (f & SF_ADD) {
        v.x += (T)s.add_re;
        v.y += (T)s.add_im;
    }
    int64_t u = a + s.ax_shift;
    if (u >= s.ax_len) u -= s.ax_len;
    if (u >= s.ax_bound) return;
    const int64_t off = la.base + u * s.ax_stride;
    T nrm = T(0);
    if (f & SF_NORM) {
        nrm = v.x * v.x + v.y * v.y;
        // |v|^order: the square root for the magnitude, no power for order 2
        if (s.post_param == 1.0)
            nrm = mag_sqrt<T>(nrm);
        else if (s.post_param != 2.0)
            nrm = pow(nrm, (T)(s.post_param * 0.5));
    }
    switch (s.fmt) {
        case RK_FMT_C64:
            reinterpret_cast<float2*>(s.ptr)[off] = make_float2((float)v.x, (float)v.y);
            break;
        case RK_FMT_C128:
            reinterpret_cast<double2*>(s.ptr)[off] = make_double2((double)v.x, (double)v.y);
            break;
        case RK_FMT_F32:
            reinterpret_cast<float*>(s.ptr)[off] = (float)((f & SF_NORM) ? nrm : v.x);
            break;
        case RK_FMT_F64:
            reinterpret_cast<double*>(s.ptr)[off] = (double)((f & SF_NORM) ? nrm : v.x);
            break;
        case RK_FMT_F32_PAIR:
            reinterpret_cast<float*>(s.ptr)[off] = (float)v.x;
            reinterpret_cast<float*>(s.ptr2)[off - s.offset + s.offset2] = (float)v.y;
            break;
        case RK_FMT_F64_PAIR:
            reinterpret_cast<double*>(s.ptr)[off] = (double)v.x;
            reinterpret_cast<double*>(s.ptr2)[off - s.offset + s.offset2] = (double)v.y;
            break;
#ifdef RK_USER_STORE
        case RK_FMT_USER:
            RK_USER_STORE<T>(s, off, v);
            break;
#endif
        default:
            break;
    }
}

// ------------------------------------------------------------------------------
// per-thread block load / store: the N elements a thread holds on one line.
// SF_FAST sides (set by the planner when the side is the pass dtype, the axis
// index is the position, no padding or cropping along the axis, and only scale /
// conjugation ops) use one line pointer, 32-bit strided offsets and a power-of-two
// mask for the index remap; the value ops run once per block with hoisted flags.
// ------------------------------------------------------------------------------
// the side's constant scale on a thread's block; a real scale (the usual 1/N) takes
// two multiplications an element instead of a complex product (same results)
template <typename T, int N>
__device__ __forceinline__ void scale_block(const Side& s, cplx<T>* v) {
    const cplx<T> c = cmk<cplx<T>>((T)s.scale_re, (T)s.scale_im);
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = cmul(v[i], c);
}

// The value ops of a pass-dtype side without tables, for an element read outside the
// block load (the Nyquist bin of an inverse real transform).
template <typename T>
__device__ __forceinline__ cplx<T> edge_value(const Side& s, cplx<T> v) {
    if (s.flags & SF_SCALE) {
        if (s.scale_im == 0.0) {
            v.x *= (T)s.scale_re;
            v.y *= (T)s.scale_re;
        } else {
            v = cmul(v, cmk<cplx<T>>((T)s.scale_re, (T)s.scale_im));
        }
    }
    if (((s.flags & SF_PRE_CONJ) != 0) != ((s.flags & SF_POST_CONJ) != 0)) v.y = -v.y;
    return v;
}

// The Nyquist bin X[L] of a real-spectrum store at element offset off: the side's
// scale, then the complex value or, for a real output, |X|^post_param (SF_NORM) or
// its real part.
template <typename T>
__device__ __forceinline__ void store_nyquist(const Side& s, int64_t off, cplx<T> x) {
    using V = cplx<T>;
    if (s.flags & SF_SCALE) x = cmul(x, cmk<V>((T)s.scale_re, (T)s.scale_im));
    if (s.fmt == RK_FMT_C64 || s.fmt == RK_FMT_C128) {
        reinterpret_cast<V*>(s.ptr)[off] = x;
        return;
    }
    T r = x.x;
    if (s.flags & SF_NORM) {
        r = x.x * x.x + x.y * x.y;
        if (s.post_param == 1.0)
            r = mag_sqrt<T>(r);
        else if (s.post_param != 2.0)
            r = pow(r, (T)(s.post_param * 0.5));
    }
    reinterpret_cast<T*>(s.ptr)[off] = r;
}

// Bins of the pairwise real-signal step owned by thread tb of a line: slot q < RT/2
// holds bin k_q = tb + TPL q (every k_q < L/2), slot RT/2 + q its mirror
// L - k_q - rodd; without rodd the mirror of bin 0 is bin L (kept apart), so slot
// RT/2 of thread 0 holds the self-mirrored bin L/2 instead.
template <int L, int RT, int TPL>
__device__ __forceinline__ int pair_pos(int tb, int i, int rodd) {
    if (i < RT / 2) return tb + TPL * i;
    const int k = tb + TPL * (i - RT / 2);
    return (!rodd && k == 0) ? L / 2 : L - k - rodd;
}

// The step y[k] A_k + conj(y[m]) B_k for bin k and its mirror m at once: with
// P = y[k], Q = conj(y[m]), S = h (P + Q) and D = -i h w_k (P - Q), bin k gets S + D
// and bin m gets conj(S - D) (A_m = conj(A_k), B_m = conj(B_k) since w_m = -conj(w_k))
template <typename T>
__device__ __forceinline__ void real_pair(cplx<T> y, cplx<T> ym, cplx<T> w, T h, cplx<T>& ok, cplx<T>& om) {
    using V = cplx<T>;
    const V q = cconj(ym);
    const V s = cmk<V>(h * (y.x + q.x), h * (y.y + q.y));
    const V d = cmul(cmk<V>(y.x - q.x, y.y - q.y), cmk<V>(h * w.y, -h * w.x));
    ok = cmk<V>(s.x + d.x, s.y + d.y);
    om = cmk<V>(s.x - d.x, d.y - s.y);
}

// Forward step after the FFT: v[] (pair_pos order) from the half-length spectrum Z
// read through zat(k); returns the Nyquist bin X[L] for thread 0 without rodd.
template <typename T, int L, int RT, int TPL, class ZAt>
__device__ __forceinline__ cplx<T> real_pairs_out(const PassParams& p, int tb, ZAt zat, cplx<T>* v) {
    using V = cplx<T>;
    const V* wk = reinterpret_cast<const V*>(p.rmix);
    const T h = (T)p.rh;
#pragma unroll
    for (int q = 0; q < RT / 2; ++q) {
        const int k = tb + TPL * q;
        real_pair<T>(zat(k), zat((L - k - p.rodd) & (L - 1)), __ldg(wk + k), h, v[q], v[RT / 2 + q]);
    }
    V nyq = cmk<V>(T(0), T(0));
    if (!p.rodd && tb == 0) {
        nyq = v[RT / 2];
        V unused;
        const V zh = zat(L / 2);
        real_pair<T>(zh, zh, __ldg(wk + L / 2), h, v[RT / 2], unused);
    }
    return nyq;
}

// Inverse step before the FFT, in place on v[] (pair_pos order: the raw bins y);
// yl is bin L of the input row (the mirror of bin 0 without rodd).
template <typename T, int L, int RT, int TPL>
__device__ __forceinline__ void real_pairs_in(const PassParams& p, int tb, cplx<T> yl, cplx<T>* v) {
    using V = cplx<T>;
    const V* wk = reinterpret_cast<const V*>(p.rmix);
    const T h = (T)p.rh;
    const bool special = !p.rodd && tb == 0;
    const V yh = v[RT / 2];  // bin L/2 in thread 0's slot RT/2 when special
#pragma unroll
    for (int q = 0; q < RT / 2; ++q) {
        const int k = tb + TPL * q;
        V y = v[q], ym = v[RT / 2 + q];
        if (q == 0 && special) {
            ym = yl;
            if (p.rnyq) {
                y.y = T(0);
                ym.y = T(0);
            }
        }
        real_pair<T>(y, ym, __ldg(wk + k), h, v[q], v[RT / 2 + q]);
    }
    if (special) {
        V unused;
        real_pair<T>(yh, yh, __ldg(wk + L / 2), h, v[RT / 2], unused);
    }
}

// LPATHS: the lean load paths compiled in (LOAD_FAST | LOAD_FAST2 | LOAD_FASTR); RP:
// the sample-pair reads.  A side marked for a path left out takes the general path.
enum : int { LOAD_FAST = 1, LOAD_FAST2 = 2, LOAD_FASTR = 4, LOAD_ALL = 7 };

template <typename T, int N, bool RP = true, int LPATHS = LOAD_ALL, class PosF>
__device__ __forceinline__ void load_block(const Side& s, const LineAddr& la, PosF pos, cplx<T>* v) {
    using V = cplx<T>;
    const int32_t f = s.flags;
    if ((LPATHS & LOAD_FAST) && (f & SF_FAST)) {
        const V* lp = reinterpret_cast<const V*>(s.ptr) + la.base;
        const int st = (int)s.ax_stride, sh = s.ax_shift, mask = (int)s.ax_len - 1;
        if (la.ok) {
#pragma unroll
            for (int i = 0; i < N; ++i) v[i] = lp[((pos(i) + sh) & mask) * st];
        } else {
#pragma unroll
            for (int i = 0; i < N; ++i) v[i] = cmk<V>(T(0), T(0));
        }
        if (f & SF_SCALE) scale_block<T, N>(s, v);
        if (((f & SF_PRE_CONJ) != 0) != ((f & SF_POST_CONJ) != 0)) {
#pragma unroll
            for (int i = 0; i < N; ++i) v[i].y = -v[i].y;
        }
    } else if ((LPATHS & LOAD_FAST2) && (f & SF_FAST2)) {
        // pass-dtype side with an index map a = c cA + j jB (four-step, Bluestein
        // padding): one line pointer, 32-bit offsets, a bounds predicate, and the
        // chirp / table ops in side_load's order
        const int a0 = (int)(la.c * s.cA), jB = (int)s.jB, st = (int)s.ax_stride;
        const int bound = (int)s.ax_bound, alen = (int)s.ax_len;
        const V* lp = reinterpret_cast<const V*>(s.ptr) + la.base;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const int a = a0 + pos(i) * jB;
            v[i] = (la.ok && a < bound) ? lp[a * st] : cmk<V>(T(0), T(0));
        }
        if (f & SF_SCALE) scale_block<T, N>(s, v);
        if (f & SF_PRE_CONJ) {
#pragma unroll
            for (int i = 0; i < N; ++i) v[i].y = -v[i].y;
        }
        if (f & SF_CHIRP) {
            const V* ch = reinterpret_cast<const V*>(s.chirp);
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int a = a0 + pos(i) * jB;
                if (a < alen) v[i] = cmul(v[i], __ldg(ch + a));
            }
        }
        if (f & SF_TAB) {
            const V* tb = reinterpret_cast<const V*>(s.tab);
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int a = a0 + pos(i) * jB;
                if (a < alen) v[i] = cmul(v[i], __ldg(tb + a));
            }
        }
        if (f & SF_POST_CONJ) {
#pragma unroll
            for (int i = 0; i < N; ++i) v[i].y = -v[i].y;
        }
    } else if ((LPATHS & LOAD_FASTR) && (f & SF_FASTR)) {
        // real input of the pass precision (e.g. windowed signal frames): one line
        // pointer, 32-bit offsets, the window from the plan's table; SF_RPAIR reads the
        // samples 2a and 2a + 1 as one element (one vector load on a contiguous,
        // aligned line)
        const T* lp = reinterpret_cast<const T*>(s.ptr) + la.base;
        const T* wt = (f & SF_WINDOW) ? reinterpret_cast<const T*>(s.win) : nullptr;
        const int st = (int)s.ax_stride;
        if (RP && (f & SF_RPAIR)) {
            // the pair vector load needs the line's address aligned to the pair type
            if (!la.ok) {
#pragma unroll
                for (int i = 0; i < N; ++i) v[i] = cmk<V>(T(0), T(0));
            } else if (st == 1 && (reinterpret_cast<uintptr_t>(lp) % sizeof(V)) == 0) {
#pragma unroll
                for (int i = 0; i < N; ++i) v[i] = reinterpret_cast<const V*>(lp)[pos(i)];
            } else {
#pragma unroll
                for (int i = 0; i < N; ++i) v[i] = cmk<V>(lp[2 * pos(i) * st], lp[(2 * pos(i) + 1) * st]);
            }
            if (wt) {
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    const V w = __ldg(reinterpret_cast<const V*>(wt) + pos(i));
                    v[i].x *= w.x;
                    v[i].y *= w.y;
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int a = pos(i);
                T x = la.ok ? lp[a * st] : T(0);
                if (wt) x *= __ldg(wt + a);
                v[i] = cmk<V>(x, T(0));
            }
        }
        if (f & SF_SCALE) scale_block<T, N>(s, v);
        if (((f & SF_PRE_CONJ) != 0) != ((f & SF_POST_CONJ) != 0)) {
#pragma unroll
            for (int i = 0; i < N; ++i) v[i].y = -v[i].y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = side_load<T, RP>(s, la, pos(i));
    }
}

// PATHS: the lean paths compiled in (STORE_FAST | STORE_FAST2 | STORE_FASTR); a side
// marked for a path left out takes the general element path.  Kernels whose store
// sides only ever take SF_FAST compile the others out to keep their registers.
enum : int { STORE_FAST = 1, STORE_FAST2 = 2, STORE_FASTR = 4, STORE_ALL = 7 };

template <typename T, int N, int PATHS = STORE_ALL, class PosF>
__device__ __forceinline__ void store_block(const Side& s, const PassParams& p, const LineAddr& la, PosF pos,
                                            cplx<T>* v) {
    using V = cplx<T>;
    const int32_t f = s.flags;
    if ((PATHS & STORE_FAST) && (f & SF_FAST)) {
        if (((f & SF_PRE_CONJ) != 0) != ((f & SF_POST_CONJ) != 0)) {
#pragma unroll
            for (int i = 0; i < N; ++i) v[i].y = -v[i].y;
        }
        if (f & SF_SCALE) scale_block<T, N>(s, v);
        if (la.ok) {
            V* lp = reinterpret_cast<V*>(s.ptr) + la.base;
            const int st = (int)s.ax_stride, sh = s.ax_shift, mask = (int)s.ax_len - 1;
#pragma unroll
            for (int i = 0; i < N; ++i) lp[((pos(i) + sh) & mask) * st] = v[i];
        }
    } else if ((PATHS & STORE_FAST2) && (f & SF_FAST2)) {
        const int a0 = (int)(la.c * s.cA), jB = (int)s.jB, st = (int)s.ax_stride;
        const int bound = (int)s.ax_bound, alen = (int)s.ax_len;
        if (f & SF_TW4) {
#pragma unroll
            for (int i = 0; i < N; ++i) v[i] = cmul(v[i], tw4<T>(p, la.c * pos(i)));
        }
        if (f & SF_PRE_CONJ) {
#pragma unroll
            for (int i = 0; i < N; ++i) v[i].y = -v[i].y;
        }
        if (f & SF_CHIRP) {
            const V* ch = reinterpret_cast<const V*>(s.chirp);
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int a = a0 + pos(i) * jB;
                if (a < alen) v[i] = cmul(v[i], __ldg(ch + a));
            }
        }
        if (f & SF_POST_CONJ) {
#pragma unroll
            for (int i = 0; i < N; ++i) v[i].y = -v[i].y;
        }
        if (f & SF_SCALE) scale_block<T, N>(s, v);
        if (la.ok) {
            V* lp = reinterpret_cast<V*>(s.ptr) + la.base;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int a = a0 + pos(i) * jB;
                if (a < bound) lp[a * st] = v[i];
            }
        }
    } else if ((PATHS & STORE_FASTR) && (f & SF_FASTR)) {
        // real output of the pass precision (real part or |v|^order, e.g. magnitudes),
        // positions at or beyond the axis bound are cropped
        if (((f & SF_PRE_CONJ) != 0) != ((f & SF_POST_CONJ) != 0)) {
#pragma unroll
            for (int i = 0; i < N; ++i) v[i].y = -v[i].y;
        }
        if (f & SF_SCALE) scale_block<T, N>(s, v);
        if (la.ok) {
            T* lp = reinterpret_cast<T*>(s.ptr) + la.base;
            const int st = (int)s.ax_stride, bound = (int)s.ax_bound;
            const bool norm = f & SF_NORM;
            const T order = (T)s.post_param;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int a = pos(i);
                if (a >= bound) continue;
                T r = v[i].x;
                if (norm) {
                    r = v[i].x * v[i].x + v[i].y * v[i].y;
                    if (order == T(1))
                        r = mag_sqrt<T>(r);
                    else if (order != T(2))
                        r = pow(r, order * T(0.5));
                }
                lp[a * st] = r;
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) side_store<T>(s, p, la, pos(i), v[i]);
    }
}

// ------------------------------------------------------------------------------
// Stockham engine
// ------------------------------------------------------------------------------
template <typename T, int L, int MODE, int PL = 0, int NL_ = LineCfg<T, L, MODE, PL>::NL> struct Engine {
    using V = cplx<T>;
    using Cfg = LineCfg<T, L, MODE, PL>;
    using RC = RadixP<T, L, PL>;
    static constexpr int RT = Cfg::RT, TPL = Cfg::TPL, NL = NL_, NS = RC::NS;

    static __device__ __forceinline__ int sidx(int ln, int pos) {
        if constexpr (MODE == MODE_POS)
            return ln * Cfg::LS + pos + (pos >> 4);
        else
            return pos * NL + ln;
    }

    // TWS: the stage twiddle table `tw` is a copy in shared memory (plain loads;
    // the read-only global path must not address shared memory)
    template <int S, int P, bool TWS = false>
    static __device__ __forceinline__ void stages(V* v, V* sm, int ln, int tb, const V* tw) {
        if constexpr (S < NS) {
            constexpr int R = RC::R[S];
            constexpr int NB = RT / R;
            if constexpr (S + 1 < NS) {
                // twiddles W_{L/P}^(j1 m), 1 <= m < R, from the stage table laid out
                // [m - 1][j1] (TwLayout; each an FP64 value rounded once), loaded
                // before the butterfly so their latency overlaps its arithmetic
                constexpr int J = L / (P * R);
                const V* tws = tw + TwLayout<T, L, PL>::offset(S);
#pragma unroll
                for (int z = 0; z < NB; ++z) {
                    const int b = tb + TPL * z;
                    const int l = b % P, j1 = b / P;
                    // (plan 1 keeps to half the registers: twiddles after the butterfly)
                    if constexpr (R <= 16 && PL == 0) {
                        V w[R - 1];
#pragma unroll
                        for (int m = 1; m < R; ++m) w[m - 1] = TWS ? tws[(m - 1) * J + j1] : __ldg(tws + (m - 1) * J + j1);
                        dft<R>(v + z * R);
#pragma unroll
                        for (int m = 1; m < R; ++m) v[z * R + m] = cmul(v[z * R + m], w[m - 1]);
                    } else {
                        // radix 32: keep the register budget, load after the butterfly
                        dft<R>(v + z * R);
#pragma unroll
                        for (int m = 1; m < R; ++m)
                            v[z * R + m] = cmul(v[z * R + m], TWS ? tws[(m - 1) * J + j1] : __ldg(tws + (m - 1) * J + j1));
                    }
#pragma unroll
                    for (int m = 0; m < R; ++m) sm[sidx(ln, l + P * (m + R * j1))] = v[z * R + m];
                }
                __syncthreads();
                constexpr int R2 = RC::R[S + 1];
                constexpr int NB2 = RT / R2;
#pragma unroll
                for (int z = 0; z < NB2; ++z)
#pragma unroll
                    for (int m = 0; m < R2; ++m) v[z * R2 + m] = sm[sidx(ln, tb + TPL * z + (L / R2) * m)];
                __syncthreads();
                stages<S + 1, P * R, TWS>(v, sm, ln, tb, tw);
            } else {
#pragma unroll
                for (int z = 0; z < NB; ++z) dft<R>(v + z * R);
            }
        }
    }

    // v holds stage-0 inputs: v[z*R0 + m] = x[tb + TPL z + (L/R0) m];
    // afterwards v[z*Rl + m] = X[tb + TPL z + (L/Rl) m]
    template <bool TWS = false>
    static __device__ __forceinline__ void run(V* v, V* sm, int ln, int tb, const V* tw) {
        stages<0, 1, TWS>(v, sm, ln, tb, tw);
    }

    static constexpr int R0 = RC::R[0];
    static constexpr int RL = RC::R[NS - 1];
    static __device__ __forceinline__ int in_pos(int tb, int z, int m) { return tb + TPL * z + (L / R0) * m; }
    static __device__ __forceinline__ int out_pos(int tb, int z, int m) { return tb + TPL * z + (L / RL) * m; }
};

// ------------------------------------------------------------------------------
// line pass kernel (optionally a fused single-pass Bluestein convolution)
// ------------------------------------------------------------------------------
// VAR 0: plain pass; VAR 1: fused Bluestein convolution; VAR 2: position-mode
// compute with a lane-fastest store through shared memory (four-step second pass,
// whose output positions are strided by N1 while consecutive lines are adjacent).
// One CTA's tile (NL lines starting at line block * NL) of a line pass; shared by
// the per-pass kernel k_line and the persistent batch kernel (rk_batch.cu).
template <typename T, int L, int MODE, int VARC>
__device__ __forceinline__ void line_body(const PassParams& p, int64_t block, unsigned char* smem, int tid) {
    constexpr int VAR = VARC & 15, PL = VARC >> 4;   // variant, radix plan
    using V = cplx<T>;
    using E = Engine<T, L, MODE, PL>;
    using Cfg = LineCfg<T, L, MODE, PL>;
    constexpr int RT = Cfg::RT, TPL = Cfg::TPL, NL = Cfg::NL;
    constexpr int R0 = E::R0, RL = E::RL;
    V* sm = reinterpret_cast<V*>(smem);
    const V* tw = reinterpret_cast<const V*>(p.tw);

    const int ln = MODE == MODE_POS ? tid / TPL : tid % NL;
    const int tb = MODE == MODE_POS ? tid % TPL : tid / NL;
    const int64_t line = block * NL + ln;
    const bool lok = line < p.nlines;

    V v[RT];
    {
        const LineAddr la = line_addr(p.ld, line, p.C, p.I, lok);
        if constexpr (VAR == 4) {
            // half-length spectrum of a real signal from its bins y (the inverse real
            // transforms; y arrives conjugated, as the inverse FFT's first load), pair
            // by pair; with rnyq the mirror of bin 0 is bin L of the input row, and
            // bins 0 and L lose their imaginary parts
            static_assert(MODE == MODE_POS, "the real-signal step needs whole lines");
            load_block<T, RT, false>(p.ld, la, [&](int i) { return pair_pos<L, RT, TPL>(tb, i, p.rodd); }, v);
            V yl = cmk<V>(T(0), T(0));
            if (p.rnyq && la.ok) yl = edge_value<T>(p.ld, reinterpret_cast<const V*>(p.ld.ptr)[la.base + (int64_t)L * p.ld.ax_stride]);
            real_pairs_in<T, L, RT, TPL>(p, tb, yl, v);
#pragma unroll
            for (int i = 0; i < RT; ++i) sm[E::sidx(ln, pair_pos<L, RT, TPL>(tb, i, p.rodd))] = v[i];
            __syncthreads();
#pragma unroll
            for (int z = 0; z < RT / R0; ++z)
#pragma unroll
                for (int m = 0; m < R0; ++m) v[z * R0 + m] = sm[E::sidx(ln, E::in_pos(tb, z, m))];
            __syncthreads();
        } else {
            // sample-pair reads (SF_RPAIR) only occur on the half-length route's passes
            // (variants 5 and 6, whose loads are always real); the complex-input
            // real-spectrum pass (variant 3) never meets a real side
            constexpr bool half = VAR == 5 || VAR == 6;
            constexpr int lp = half ? LOAD_FASTR : (VAR == 3 ? (LOAD_FAST | LOAD_FAST2) : LOAD_ALL);
            load_block<T, RT, half, lp>(p.ld, la, [&](int i) { return E::in_pos(tb, i / R0, i % R0); }, v);
        }
    }
    // the fused Bluestein pass runs the same line FFT twice: one copy of its code,
    // looped (half the instruction footprint of two inlined copies)
    if constexpr (VAR != 1) E::run(v, sm, ln, tb, tw);
#pragma unroll 1
    for (int it = 0; it < (VAR == 1 ? 2 : 0); ++it) {
        E::run(v, sm, ln, tb, tw);
        if constexpr (VAR == 1) {
            if (it == 0) {
                // multiply by the kernel spectrum (1/M folded in) and conjugate, so
                // that a second forward FFT followed by a conjugation yields the
                // inverse FFT
                const V* K = reinterpret_cast<const V*>(p.blue_k);
#pragma unroll
                for (int z = 0; z < RT / RL; ++z)
#pragma unroll
                    for (int m = 0; m < RL; ++m) {
                        const int pos = E::out_pos(tb, z, m);
                        sm[E::sidx(ln, pos)] = cconj(cmul(v[z * RL + m], K[pos]));
                    }
                __syncthreads();
#pragma unroll
                for (int z = 0; z < RT / R0; ++z)
#pragma unroll
                    for (int m = 0; m < R0; ++m) v[z * R0 + m] = sm[E::sidx(ln, E::in_pos(tb, z, m))];
                __syncthreads();
            }
        }
    }
    if constexpr (VAR == 4) {
        // antiperiodic inverse: W_2L^m on the FFT's output, which the store then
        // conjugates (the inverse's last conjugation) into W_2L^-m on the result
        if (p.rtwid) {
            const V* tt = reinterpret_cast<const V*>(p.rtwid);
#pragma unroll
            for (int z = 0; z < RT / RL; ++z)
#pragma unroll
                for (int m = 0; m < RL; ++m) v[z * RL + m] = cmul(v[z * RL + m], __ldg(tt + E::out_pos(tb, z, m)));
        }
    }
    if constexpr (VAR == 3 || VAR == 5 || VAR == 6) {
        // real-signal spectrum from the half-length spectrum Z of this line (the line
        // holds x[2n] + i x[2n+1]): X[k] = Z[k] A_k + conj(Z[mirror k]) B_k with the
        // plan's FP64-generated w_k in rmix; with rnyq the Nyquist bin
        // X[L] = Re Z[0] - Im Z[0] is stored after the line's L positions.  Variant 5
        // then stores lane-fastest through shared memory, as variant 2 does.
        static_assert(MODE == MODE_POS, "the real-spectrum step needs whole lines");
#pragma unroll
        for (int z = 0; z < RT / RL; ++z)
#pragma unroll
            for (int m = 0; m < RL; ++m) sm[E::sidx(ln, E::out_pos(tb, z, m))] = v[z * RL + m];
        __syncthreads();
        const V nyq = real_pairs_out<T, L, RT, TPL>(p, tb, [&](int k) { return sm[E::sidx(ln, k)]; }, v);
        const LineAddr la = line_addr(p.st, line, p.C, p.I, lok);
        if (tb == 0 && la.ok && p.rnyq) store_nyquist<T>(p.st, la.base + (int64_t)L * p.st.ax_stride, nyq);
        if constexpr (VAR == 3 || VAR == 6) {
            // real-spectrum stores are complex bins or real magnitudes along the line:
            // the lean paths for those two only (others take the element path)
            store_block<T, RT, STORE_FAST | STORE_FASTR>(p.st, p, la,
                                                         [&](int i) { return pair_pos<L, RT, TPL>(tb, i, p.rodd); }, v);
        } else {
            __syncthreads();
            // the lane-fastest read-back takes a warp's 32 / NL positions of NL lines
            // at once: a line stride of L + 32 / NL (8-byte words; not the engine's
            // L + L / 16, a multiple of 16 words, which put all NL lines of a position
            // on one bank) spreads them over the banks; it fits the engine's buffer
            // whenever 32 / NL <= L / 16
            constexpr int D = NL >= 32 ? 1 : 32 / NL;
            constexpr bool PAD = D <= L / 16;
            auto ts = [&](int l, int pos) { return PAD ? l * (L + D) + pos : E::sidx(l, pos); };
#pragma unroll
            for (int i = 0; i < RT; ++i) sm[ts(ln, pair_pos<L, RT, TPL>(tb, i, p.rodd))] = v[i];
            __syncthreads();
            const int lane = tid % NL;
            const int p0 = tid / NL;
            const int64_t sline = block * NL + lane;
            const LineAddr ls = line_addr(p.st, sline, p.C, p.I, sline < p.nlines);
#pragma unroll
            for (int q = 0; q < RT; ++q) v[q] = sm[ts(lane, p0 + TPL * q)];
            store_block<T, RT, STORE_FAST | STORE_FASTR>(p.st, p, ls, [&](int q) { return p0 + TPL * q; }, v);
        }
    } else if constexpr (VAR == 2) {
        static_assert(MODE == MODE_POS, "transposed store needs position mode");
        // line stride L + 32 / NL for the lane-fastest read-back (as in variant 5)
        constexpr int D = NL >= 32 ? 1 : 32 / NL;
        constexpr bool PAD = D <= L / 16;
        auto ts = [&](int l, int pos) { return PAD ? l * (L + D) + pos : E::sidx(l, pos); };
#pragma unroll
        for (int z = 0; z < RT / RL; ++z)
#pragma unroll
            for (int m = 0; m < RL; ++m) sm[ts(ln, E::out_pos(tb, z, m))] = v[z * RL + m];
        __syncthreads();
        // thread t stores lane t % NL, positions t / NL + TPL * q
        const int lane = tid % NL;
        const int p0 = tid / NL;
        const int64_t sline = block * NL + lane;
        const LineAddr la = line_addr(p.st, sline, p.C, p.I, sline < p.nlines);
#pragma unroll
        for (int q = 0; q < RT; ++q) v[q] = sm[ts(lane, p0 + TPL * q)];
        store_block<T, RT>(p.st, p, la, [&](int q) { return p0 + TPL * q; }, v);
    } else {
        const LineAddr la = line_addr(p.st, line, p.C, p.I, lok);
        store_block<T, RT>(p.st, p, la, [&](int i) { return E::out_pos(tb, i / RL, i % RL); }, v);
    }
}

template <typename T, int L, int MODE, int VAR>
__global__ void __launch_bounds__(LineCfg<T, L, MODE, (VAR >> 4)>::NT) k_line(const PassParams p) {
    extern __shared__ __align__(16) unsigned char rk_smem[];
    line_body<T, L, MODE, VAR>(p, blockIdx.x, rk_smem, threadIdx.x);
}

// Fused Bluestein bodies with 16 elements a thread would take 160-180 registers;
// k_line_2 holds them to 128 so that two 256-thread CTAs share an SM.  The float32
// real-spectrum variants (3 to 6) of 256 to 1024 points run four CTAs an SM
// (k_line_4, 64 registers, a few spilled): the frame-major spectrogram pass went
// from 59 to 41 us with the paired loads split and the approximate square root.
// Other bodies keep the register count ptxas picks by itself (any minimum-blocks
// bound, 1 included, lets it spend registers up to the bound).
template <typename T, int L, int MODE, int VARC> struct LineMinBlocks {
    static constexpr int VAR = VARC & 15, PL = VARC >> 4;
    static constexpr int V = (VAR == 1 && RadixP<T, L, PL>::RT == 16 && L >= 512 && LineCfg<T, L, MODE, PL>::NT <= 256) ? 2
                             : (VAR >= 3 && sizeof(T) == 4 && L >= 256 && L <= 1024)                          ? 4
                                                                                                                : 1;
};

template <typename T, int L, int MODE, int VAR>
__global__ void __launch_bounds__(LineCfg<T, L, MODE, (VAR >> 4)>::NT, 2) k_line_2(const PassParams p) {
    extern __shared__ __align__(16) unsigned char rk_smem[];
    line_body<T, L, MODE, VAR>(p, blockIdx.x, rk_smem, threadIdx.x);
}

template <typename T, int L, int MODE, int VAR>
__global__ void __launch_bounds__(LineCfg<T, L, MODE, (VAR >> 4)>::NT, 4) k_line_4(const PassParams p) {
    extern __shared__ __align__(16) unsigned char rk_smem[];
    line_body<T, L, MODE, VAR>(p, blockIdx.x, rk_smem, threadIdx.x);
}

}  // namespace rk
