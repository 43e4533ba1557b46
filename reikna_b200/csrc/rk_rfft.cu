// Real-signal transforms through a half-length complex FFT (the reference's
// examples/demo_specialized_fft.py:156-331 and demo_specialized_fft.mako:1-62).
//
// A real x of even length N, read as the complex z[n] = x[2n] + i x[2n+1] of length
// H = N / 2, has Z = FFT_H(z) and
//     X[k] = Z[k] A[k] + conj(Z[(H - k) mod H]) B[k],   k = 0 .. H,
//     A[k] = (1 - i W^k) / 2,  B[k] = (1 + i W^k) / 2,  W = exp(-2 pi i / N);
// the inverse takes Z[k] = X[k] conj(A[k]) + conj(X[H - k]) conj(B[k]) and
// z = IFFT_H(Z).  W^k (k = 0 .. H) is tabulated once in FP64 and rounded to the
// working precision.  Both kernels are element-wise over (batch, k): one read of
// each input element pair and one write per output element.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "rk_internal.h"

namespace rk {

namespace {

template <typename V> struct Real;
template <> struct Real<float2> { using T = float; };
template <> struct Real<double2> { using T = double; };

template <typename V> __device__ __forceinline__ V mk(typename Real<V>::T x, typename Real<V>::T y) {
    V v;
    v.x = x;
    v.y = y;
    return v;
}

template <typename V> __device__ __forceinline__ V mulc(V a, V b) {
    return mk<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

template <typename V> __device__ __forceinline__ V conjc(V a) { return mk<V>(a.x, -a.y); }

// A[k] = (1 - i w) / 2, B[k] = (1 + i w) / 2 with w = W^k
template <typename V> __device__ __forceinline__ void ab(V w, V& a, V& b) {
    using T = typename Real<V>::T;
    a = mk<V>(T(0.5) * (T(1) + w.y), T(-0.5) * w.x);
    b = mk<V>(T(0.5) * (T(1) - w.y), T(0.5) * w.x);
}

template <typename V>
__global__ void k_rfft_twiddles(V* w, int64_t half) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k > half) return;
    double s, c;
    sincospi(-(double)k / (double)half, &s, &c);  // exp(-2 pi i k / N), N = 2 half
    w[k] = mk<V>((typename Real<V>::T)c, (typename Real<V>::T)s);
}

// one CTA a row at a time (grid-stride over rows), threads across the row: no
// per-element index division
template <typename V>
__global__ void k_rfft_post(V* __restrict__ out, const V* __restrict__ z, const V* __restrict__ w, int64_t half,
                            int64_t batch, int64_t out_len) {
    for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
        const V* zr = z + b * half;
        V* orow = out + b * out_len;
        for (int64_t k = threadIdx.x; k < out_len; k += blockDim.x) {
            const V zk = zr[k == half ? 0 : k];
            const V zc = conjc(zr[k == 0 ? 0 : half - k]);
            V a, bb;
            ab(__ldg(w + k), a, bb);
            const V x = mulc(zk, a);
            const V y = mulc(zc, bb);
            orow[k] = mk<V>(x.x + y.x, x.y + y.y);
        }
    }
}

template <typename V>
__global__ void k_irfft_pre(V* __restrict__ z, const V* __restrict__ x, const V* __restrict__ w, int64_t half,
                            int64_t batch) {
    for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
        const V* xr = x + b * (half + 1);
        V* zr = z + b * half;
        for (int64_t k = threadIdx.x; k < half; k += blockDim.x) {
            V xk = xr[k];
            V xc = xr[half - k];
            // a real signal's bins 0 and H are real: their imaginary parts are ignored,
            // as numpy's irfft does
            if (k == 0) {
                xk.y = 0;
                xc.y = 0;
            }
            xc = conjc(xc);
            V a, bb;
            ab(__ldg(w + k), a, bb);
            const V p = mulc(xk, conjc(a));
            const V q = mulc(xc, conjc(bb));
            zr[k] = mk<V>(p.x + q.x, p.y + q.y);
        }
    }
}

// Antiperiodic real signals (x[n + 2L] = -x[n], length 4L, first half x[0 .. 2L)):
// only the odd harmonics F[k] = X[2k + 1], k < L, are non-zero, and with
// c[m] = (x[2m] + i x[2m+1]) W_2L^m, C = FFT_L(c), w_k = exp(-i pi (2k + 1) / 2L):
//     F[k] = C[k] (1 - i w_k) + conj(C[L - 1 - k]) (1 + i w_k),
//     C[k] = (F[k] conj(1 - i w_k) + conj(F[L - 1 - k]) conj(1 + i w_k)) / 4,
// the second inverting the first pairwise (k, L - 1 - k).  The table holds w_k for
// k < L followed by W_2L^m for m < L.
template <typename V>
__global__ void k_aprfft_twiddles(V* t, int64_t half) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= half) return;
    double s, c;
    sincospi(-(double)(2 * k + 1) / (double)(2 * half), &s, &c);
    t[k] = mk<V>((typename Real<V>::T)c, (typename Real<V>::T)s);
    sincospi(-(double)k / (double)half, &s, &c);
    t[half + k] = mk<V>((typename Real<V>::T)c, (typename Real<V>::T)s);
}

template <typename V>
__global__ void k_aprfft_post(V* __restrict__ out, const V* __restrict__ z, const V* __restrict__ w, int64_t half,
                              int64_t batch) {
    using T = typename Real<V>::T;
    for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
        const V* zr = z + b * half;
        V* orow = out + b * half;
        for (int64_t k = threadIdx.x; k < half; k += blockDim.x) {
            const V wk = __ldg(w + k);
            const V x = mulc(zr[k], mk<V>(T(1) + wk.y, -wk.x));
            const V y = mulc(conjc(zr[half - 1 - k]), mk<V>(T(1) - wk.y, wk.x));
            orow[k] = mk<V>(x.x + y.x, x.y + y.y);
        }
    }
}

template <typename V>
__global__ void k_iaprfft_pre(V* __restrict__ z, const V* __restrict__ x, const V* __restrict__ w, int64_t half,
                              int64_t batch) {
    using T = typename Real<V>::T;
    for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
        const V* xr = x + b * half;
        V* zr = z + b * half;
        for (int64_t k = threadIdx.x; k < half; k += blockDim.x) {
            const V wk = __ldg(w + k);
            const V p = mulc(xr[k], mk<V>(T(0.25) * (T(1) + wk.y), T(0.25) * wk.x));
            const V q = mulc(conjc(xr[half - 1 - k]), mk<V>(T(0.25) * (T(1) - wk.y), T(-0.25) * wk.x));
            zr[k] = mk<V>(p.x + q.x, p.y + q.y);
        }
    }
}

// rows times W_2L^m (inverse: its conjugate); in place allowed
template <typename V>
__global__ void k_aprfft_twiddle(V* out, const V* in, const V* t, int64_t half, int64_t batch, int inverse) {
    for (int64_t b = blockIdx.x; b < batch; b += gridDim.x) {
        for (int64_t m = threadIdx.x; m < half; m += blockDim.x) {
            V tm = __ldg(t + m);
            if (inverse) tm = conjc(tm);
            out[b * half + m] = mulc(in[b * half + m], tm);
        }
    }
}

// CTAs for a row-per-CTA kernel: the rows, at most 16 waves of one CTA per SM
int grid_for(int64_t rows) {
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (!nsm) nsm = 148;
    }
    return (int)(rows < (int64_t)nsm * 16 ? (rows > 0 ? rows : 1) : (int64_t)nsm * 16);
}

int check_fmt(int32_t fmt, const char* who) {
    if (fmt != RK_FMT_C64 && fmt != RK_FMT_C128) {
        set_error(std::string(who) + ": format must be RK_FMT_C64 or RK_FMT_C128");
        return RK_ERR_INVALID;
    }
    return RK_OK;
}

int finish(const char* who) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string(who) + ": " + cudaGetErrorString(e));
        return RK_ERR_CUDA;
    }
    return RK_OK;
}

}  // namespace

}  // namespace rk

using namespace rk;

extern "C" int rk_rfft_twiddles(void* table, int32_t fmt, int64_t half, void* stream) {
    if (int rc = check_fmt(fmt, "rk_rfft_twiddles")) return rc;
    if (!table || half < 1) {
        set_error("rk_rfft_twiddles: null table or half length < 1");
        return RK_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned g = (unsigned)((half + 256) / 256);
    if (fmt == RK_FMT_C64)
        k_rfft_twiddles<float2><<<g, 256, 0, st>>>((float2*)table, half);
    else
        k_rfft_twiddles<double2><<<g, 256, 0, st>>>((double2*)table, half);
    return finish("rk_rfft_twiddles");
}

extern "C" int rk_rfft_post(void* out, const void* z, const void* table, int32_t fmt, int64_t half, int64_t batch,
                            int32_t store_last, void* stream) {
    if (int rc = check_fmt(fmt, "rk_rfft_post")) return rc;
    if (!out || !z || !table || half < 1 || batch < 1) {
        set_error("rk_rfft_post: null pointer or non-positive size");
        return RK_ERR_INVALID;
    }
    if (out == z) {
        set_error("rk_rfft_post: output may not alias the half-length spectrum");
        return RK_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t out_len = half + (store_last ? 1 : 0);
    const int g = grid_for(batch);
    if (fmt == RK_FMT_C64)
        k_rfft_post<float2><<<g, 256, 0, st>>>((float2*)out, (const float2*)z, (const float2*)table, half, batch, out_len);
    else
        k_rfft_post<double2><<<g, 256, 0, st>>>((double2*)out, (const double2*)z, (const double2*)table, half, batch,
                                                 out_len);
    return finish("rk_rfft_post");
}

extern "C" int rk_irfft_pre(void* z, const void* x, const void* table, int32_t fmt, int64_t half, int64_t batch,
                            void* stream) {
    if (int rc = check_fmt(fmt, "rk_irfft_pre")) return rc;
    if (!z || !x || !table || half < 1 || batch < 1) {
        set_error("rk_irfft_pre: null pointer or non-positive size");
        return RK_ERR_INVALID;
    }
    if (z == x) {
        set_error("rk_irfft_pre: output may not alias the spectrum");
        return RK_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int g = grid_for(batch);
    if (fmt == RK_FMT_C64)
        k_irfft_pre<float2><<<g, 256, 0, st>>>((float2*)z, (const float2*)x, (const float2*)table, half, batch);
    else
        k_irfft_pre<double2><<<g, 256, 0, st>>>((double2*)z, (const double2*)x, (const double2*)table, half, batch);
    return finish("rk_irfft_pre");
}

extern "C" int rk_aprfft_twiddles(void* table, int32_t fmt, int64_t half, void* stream) {
    if (int rc = check_fmt(fmt, "rk_aprfft_twiddles")) return rc;
    if (!table || half < 1) {
        set_error("rk_aprfft_twiddles: null table or half length < 1");
        return RK_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned g = (unsigned)((half + 255) / 256);
    if (fmt == RK_FMT_C64)
        k_aprfft_twiddles<float2><<<g, 256, 0, st>>>((float2*)table, half);
    else
        k_aprfft_twiddles<double2><<<g, 256, 0, st>>>((double2*)table, half);
    return finish("rk_aprfft_twiddles");
}

extern "C" int rk_aprfft_post(void* out, const void* z, const void* table, int32_t fmt, int64_t half, int64_t batch,
                              void* stream) {
    if (int rc = check_fmt(fmt, "rk_aprfft_post")) return rc;
    if (!out || !z || !table || half < 1 || batch < 1) {
        set_error("rk_aprfft_post: null pointer or non-positive size");
        return RK_ERR_INVALID;
    }
    if (out == z) {
        set_error("rk_aprfft_post: output may not alias the half-length spectrum");
        return RK_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int g = grid_for(batch);
    if (fmt == RK_FMT_C64)
        k_aprfft_post<float2><<<g, 256, 0, st>>>((float2*)out, (const float2*)z, (const float2*)table, half, batch);
    else
        k_aprfft_post<double2><<<g, 256, 0, st>>>((double2*)out, (const double2*)z, (const double2*)table, half, batch);
    return finish("rk_aprfft_post");
}

extern "C" int rk_iaprfft_pre(void* z, const void* x, const void* table, int32_t fmt, int64_t half, int64_t batch,
                              void* stream) {
    if (int rc = check_fmt(fmt, "rk_iaprfft_pre")) return rc;
    if (!z || !x || !table || half < 1 || batch < 1) {
        set_error("rk_iaprfft_pre: null pointer or non-positive size");
        return RK_ERR_INVALID;
    }
    if (z == x) {
        set_error("rk_iaprfft_pre: output may not alias the harmonics");
        return RK_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int g = grid_for(batch);
    if (fmt == RK_FMT_C64)
        k_iaprfft_pre<float2><<<g, 256, 0, st>>>((float2*)z, (const float2*)x, (const float2*)table, half, batch);
    else
        k_iaprfft_pre<double2><<<g, 256, 0, st>>>((double2*)z, (const double2*)x, (const double2*)table, half, batch);
    return finish("rk_iaprfft_pre");
}

extern "C" int rk_aprfft_twiddle(void* out, const void* in, const void* table, int32_t fmt, int64_t half,
                                 int64_t batch, int32_t inverse, void* stream) {
    if (int rc = check_fmt(fmt, "rk_aprfft_twiddle")) return rc;
    if (!out || !in || !table || half < 1 || batch < 1) {
        set_error("rk_aprfft_twiddle: null pointer or non-positive size");
        return RK_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int g = grid_for(batch);
    // the table's second half holds W_2L^m
    if (fmt == RK_FMT_C64)
        k_aprfft_twiddle<float2><<<g, 256, 0, st>>>((float2*)out, (const float2*)in, (const float2*)table + half, half,
                                                    batch, inverse ? 1 : 0);
    else
        k_aprfft_twiddle<double2><<<g, 256, 0, st>>>((double2*)out, (const double2*)in, (const double2*)table + half,
                                                     half, batch, inverse ? 1 : 0);
    return finish("rk_aprfft_twiddle");
}
