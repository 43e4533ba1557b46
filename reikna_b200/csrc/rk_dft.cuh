// Complex arithmetic and register-resident small DFTs for the FFT kernels.
//
// Every kernel computes the forward transform X[k] = sum_n x[n] exp(-2 pi i n k / N)
// (reikna's direction = -1, reikna/fft/fft.mako:741-745); the inverse is obtained by
// conjugating on the first load and on the last store, so one set of kernels serves
// both directions (reikna instead passes `inverse` as a runtime sign into every
// butterfly, reikna/fft/fft.mako:64-193).
//
// dft<R, S>(a) transforms a[0], a[S], ..., a[(R-1)S] in place into natural order.
// Sizes above 4 are split as R = A*B (A in {2,4}): A-point DFTs on stride B, a
// twiddle by W_R^(n2*k1), B-point DFTs on contiguous groups, then a register
// permutation that the compiler resolves to renaming.
#pragma once
#ifndef __CUDACC_RTC__
#include <cuda_runtime.h>
#include <stdint.h>
#endif

namespace rk {

template <typename T> struct cplx_t;
template <> struct cplx_t<float> { using type = float2; };
template <> struct cplx_t<double> { using type = double2; };
template <typename T> using cplx = typename cplx_t<T>::type;

template <typename V> __device__ __forceinline__ V cmk(decltype(V().x) x, decltype(V().x) y) {
    V r; r.x = x; r.y = y; return r;
}
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
    V r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
// a * conj(b)
template <typename V> __device__ __forceinline__ V cmulc(V a, V b) {
    V r;
    r.x = a.x * b.x + a.y * b.y;
    r.y = a.y * b.x - a.x * b.y;
    return r;
}
template <typename V> __device__ __forceinline__ V cconj(V a) { a.y = -a.y; return a; }
template <typename V, typename T> __device__ __forceinline__ V cscale(V a, T s) { a.x *= s; a.y *= s; return a; }

// cos and sin of 2*pi*m/32 for m in [0, 8], as exact-to-double literals.
__host__ __device__ constexpr double k_cos32(int m) {
    return m == 0 ? 1.0 : m == 1 ? 0.98078528040323044912618223613424 :
           m == 2 ? 0.92387953251128675612818318939679 : m == 3 ? 0.83146961230254523707878837761791 :
           m == 4 ? 0.70710678118654752440084436210485 : m == 5 ? 0.55557023301960222474283081394853 :
           m == 6 ? 0.38268343236508977172845998403040 : m == 7 ? 0.19509032201612826784828486847702 : 0.0;
}
// cos(2 pi m / 32), sin(2 pi m / 32) for any integer m
__host__ __device__ constexpr double k_c32(int m) {
    m = ((m % 32) + 32) % 32;
    return m <= 8 ? k_cos32(m) : m <= 16 ? -k_cos32(16 - m) : m <= 24 ? -k_cos32(m - 16) : k_cos32(32 - m);
}
__host__ __device__ constexpr double k_s32(int m) { return k_c32(8 - m); }

// multiply v by W_R^k = exp(-2 pi i k / R), R | 32, with cheap special cases
template <int R, int K, typename V> __device__ __forceinline__ V mul_w(V v) {
    static_assert(32 % R == 0, "twiddle radix must divide 32");
    constexpr int m = ((K * (32 / R)) % 32 + 32) % 32;
    using T = decltype(v.x);
    if constexpr (m == 0) return v;
    else if constexpr (m == 8) return cmk<V>(v.y, -v.x);        // -i
    else if constexpr (m == 16) return cmk<V>(-v.x, -v.y);      // -1
    else if constexpr (m == 24) return cmk<V>(-v.y, v.x);       // +i
    else if constexpr (m == 4) { constexpr T h = (T)k_cos32(4); return cmk<V>((v.x + v.y) * h, (v.y - v.x) * h); }
    else if constexpr (m == 12) { constexpr T h = (T)k_cos32(4); return cmk<V>((v.y - v.x) * h, -(v.x + v.y) * h); }
    else if constexpr (m == 20) { constexpr T h = (T)k_cos32(4); return cmk<V>(-(v.x + v.y) * h, (v.x - v.y) * h); }
    else if constexpr (m == 28) { constexpr T h = (T)k_cos32(4); return cmk<V>((v.x - v.y) * h, (v.x + v.y) * h); }
    else {
        constexpr T c = (T)k_c32(m);
        constexpr T s = (T)k_s32(m);
        // (x + iy)(c - is)
        return cmk<V>(v.x * c + v.y * s, v.y * c - v.x * s);
    }
}

template <int R, int S, typename V> struct Dft;

template <int S, typename V> struct Dft<1, S, V> {
    static __device__ __forceinline__ void run(V*) {}
};
template <int S, typename V> struct Dft<2, S, V> {
    static __device__ __forceinline__ void run(V* a) {
        V t = a[0];
        a[0] = t + a[S];
        a[S] = t - a[S];
    }
};
template <int S, typename V> struct Dft<4, S, V> {
    static __device__ __forceinline__ void run(V* a) {
        V s02 = a[0] + a[2 * S], d02 = a[0] - a[2 * S];
        V s13 = a[S] + a[3 * S], d13 = a[S] - a[3 * S];
        // -i * d13 = (d13.y, -d13.x)
        V md = cmk<V>(d13.y, -d13.x);
        a[0] = s02 + s13;
        a[2 * S] = s02 - s13;
        a[S] = d02 + md;
        a[3 * S] = d02 - md;
    }
};

template <int R, int S, typename V> struct Dft {
    static constexpr int A = (R > 8 && R % 4 == 0) ? 4 : 2;
    static constexpr int B = R / A;
    template <int N2> static __device__ __forceinline__ void step1(V* a) {
        if constexpr (N2 < B) {
            Dft<A, B * S, V>::run(a + N2 * S);
            step1<N2 + 1>(a);
        }
    }
    template <int I> static __device__ __forceinline__ void step2(V* a) {
        if constexpr (I < R) {
            constexpr int k1 = I / B, n2 = I % B;
            a[I * S] = mul_w<R, k1 * n2>(a[I * S]);
            step2<I + 1>(a);
        }
    }
    template <int K1> static __device__ __forceinline__ void step3(V* a) {
        if constexpr (K1 < A) {
            Dft<B, S, V>::run(a + B * K1 * S);
            step3<K1 + 1>(a);
        }
    }
    static __device__ __forceinline__ void run(V* a) {
        step1<0>(a);
        step2<0>(a);
        step3<0>(a);
        // slot B*k1 + k2 holds X[k1 + A*k2]
        V t[R];
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1)
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) t[k1 + A * k2] = a[(B * k1 + k2) * S];
#pragma unroll
        for (int i = 0; i < R; ++i) a[i * S] = t[i];
    }
};

template <int R, int S = 1, typename V> __device__ __forceinline__ void dft(V* a) { Dft<R, S, V>::run(a); }

}  // namespace rk
