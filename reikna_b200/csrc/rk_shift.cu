// Standalone FFTShift (reikna/fft/fftshift.py:14-110, fftshift.mako:1-84).
//
// Every shifted axis even: one kernel over the array with the first shifted axis
// halved swaps each element with its shifted partner (its own inverse), so it works
// in place.  Otherwise one out-of-place scatter out[(i + s) mod n] = in[i] with
// s = n // 2 (fftshift) or (n + 1) // 2 (ifftshift); when out aliases in, the scatter
// goes to `scratch` and is copied back.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <string>

#include "rk_internal.h"

namespace rk {

struct ShiftParams {
    int32_t nd;
    int64_t shape[MAXD];      // iteration shape
    int64_t full[MAXD];       // array shape
    int64_t stride[MAXD];     // element strides (contiguous)
    int64_t shift[MAXD];
    int32_t first_axis;       // in-place swap: axis whose iteration extent is halved
    int64_t total;            // iteration count
};

template <typename E>
__global__ void k_shift_swap(E* out, const E* in, const ShiftParams p) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= p.total) return;
    int64_t rem = t, a = 0, b = 0;
    for (int d = p.nd - 1; d >= 0; --d) {
        const int64_t i = rem % p.shape[d];
        rem /= p.shape[d];
        int64_t j = i + p.shift[d];
        if (j >= p.full[d]) j -= p.full[d];
        a += i * p.stride[d];
        b += j * p.stride[d];
    }
    const E va = in[a];
    const E vb = in[b];
    out[a] = vb;
    out[b] = va;
}

template <typename E>
__global__ void k_shift_scatter(E* out, const E* in, const ShiftParams p) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= p.total) return;
    int64_t rem = t, b = 0;
    for (int d = p.nd - 1; d >= 0; --d) {
        const int64_t i = rem % p.shape[d];
        rem /= p.shape[d];
        int64_t j = i + p.shift[d];
        if (j >= p.full[d]) j -= p.full[d];
        b += j * p.stride[d];
    }
    out[b] = in[t];
}

// Row-structured forms: the array is (rows, last axis); a block takes one row (or a
// part of it) of the iteration space, its threads compute the row's two offsets once
// and then move VEC-element vectors along the row (16-byte accesses for complex64
// when VEC = 2).  Used when the last axis' extent and shift are multiples of VEC, so
// a vector never wraps around the shifted last axis.
struct ShiftRows {
    int32_t nd;                // dims before the last one
    int64_t shape[MAXD];       // iteration extents of those dims
    int64_t full[MAXD];
    int64_t stride[MAXD];
    int64_t shift[MAXD];
    int64_t rows;              // product of shape[0 .. nd)
    int64_t w;                 // iterated extent of the last axis
    int64_t n_last, s_last;    // last axis length and shift (0 = not shifted)
};

template <typename E, int VEC> struct Vec2;
template <typename E> struct Vec2<E, 1> { using T = E; };
template <> struct Vec2<int2, 2> { using T = int4; };
template <> struct Vec2<int32_t, 2> { using T = int2; };
template <> struct Vec2<int32_t, 4> { using T = int4; };

template <typename E, int VEC, bool SWAP>
__global__ void k_shift_rows(E* out, const E* in, const ShiftRows p) {
    using VT = typename Vec2<E, VEC>::T;
    for (int64_t row = blockIdx.y; row < p.rows; row += gridDim.y) {
        int64_t rem = row, a = 0, b = 0;
        for (int d = p.nd - 1; d >= 0; --d) {
            const int64_t i = rem % p.shape[d];
            rem /= p.shape[d];
            int64_t j = i + p.shift[d];
            if (j >= p.full[d]) j -= p.full[d];
            a += i * p.stride[d];
            b += j * p.stride[d];
        }
        for (int64_t c = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * VEC; c < p.w;
             c += (int64_t)gridDim.x * blockDim.x * VEC) {
            int64_t cb = c + p.s_last;
            if (cb >= p.n_last) cb -= p.n_last;
            const VT va = *reinterpret_cast<const VT*>(in + a + c);
            if (SWAP) {
                const VT vb = *reinterpret_cast<const VT*>(in + b + cb);
                *reinterpret_cast<VT*>(out + a + c) = vb;
            }
            *reinterpret_cast<VT*>(out + b + cb) = va;
        }
    }
}

// true (and the launch made) when the row form applies
template <typename E>
static bool launch_rows(bool swap, void* out, const void* in, const ShiftParams& q, cudaStream_t st,
                        cudaError_t* err) {
    const int nd = q.nd;
    ShiftRows r;
    memset(&r, 0, sizeof(r));
    r.nd = nd - 1;
    r.rows = 1;
    for (int d = 0; d < nd - 1; ++d) {
        r.shape[d] = q.shape[d];
        r.full[d] = q.full[d];
        r.stride[d] = q.stride[d];
        r.shift[d] = q.shift[d];
        r.rows *= q.shape[d];
    }
    r.w = q.shape[nd - 1];
    r.n_last = q.full[nd - 1];
    r.s_last = q.shift[nd - 1];
    if (q.stride[nd - 1] != 1) return false;
    // vector accesses need every row start, shift and both base addresses aligned to
    // the vector (a view may start on an odd element)
    bool v2 = sizeof(E) <= 8 && r.w % 2 == 0 && r.n_last % 2 == 0 && r.s_last % 2 == 0 &&
              ((uintptr_t)in % (2 * sizeof(E))) == 0 && ((uintptr_t)out % (2 * sizeof(E))) == 0;
    for (int d = 0; d < nd - 1 && v2; ++d) v2 = q.stride[d] % 2 == 0;
    // blocks along a row so that each thread moves about eight vectors of it (the row
    // offsets are computed once a thread), rows on the y axis
    const int64_t per_block = 256 * (v2 ? 2 : 1) * 8;
    const int64_t bx = std::min<int64_t>((r.w + per_block - 1) / per_block, 65535);
    const int64_t by = std::min<int64_t>(r.rows, 65535);
    if (r.rows == 0 || r.w == 0) {
        *err = cudaSuccess;
        return true;
    }
    dim3 grid((unsigned)bx, (unsigned)by);
    bool done = false;
    if constexpr (sizeof(E) <= 8) {
        if (v2) {
            if (swap)
                k_shift_rows<E, 2, true><<<grid, 256, 0, st>>>((E*)out, (const E*)in, r);
            else
                k_shift_rows<E, 2, false><<<grid, 256, 0, st>>>((E*)out, (const E*)in, r);
            done = true;
        }
    }
    if (!done) {
        if (swap)
            k_shift_rows<E, 1, true><<<grid, 256, 0, st>>>((E*)out, (const E*)in, r);
        else
            k_shift_rows<E, 1, false><<<grid, 256, 0, st>>>((E*)out, (const E*)in, r);
    }
    *err = cudaGetLastError();
    return true;
}

template <typename E>
static cudaError_t launch_shift(bool swap, void* out, const void* in, const ShiftParams& p, cudaStream_t st) {
    if (p.total == 0) return cudaSuccess;
    // the row form for rows of at least a warp's worth of elements
    if (p.shape[p.nd - 1] >= 32) {
        cudaError_t e = cudaSuccess;
        if (launch_rows<E>(swap, out, in, p, st, &e)) return e;
    }
    const int64_t nb = (p.total + 255) / 256;
    if (swap)
        k_shift_swap<E><<<(unsigned)nb, 256, 0, st>>>((E*)out, (const E*)in, p);
    else
        k_shift_scatter<E><<<(unsigned)nb, 256, 0, st>>>((E*)out, (const E*)in, p);
    return cudaGetLastError();
}

}  // namespace rk

using namespace rk;

extern "C" int rk_fftshift_execute(void* out, const void* in, int32_t elem_bytes, int32_t ndim, const int64_t* shape,
                                   int32_t naxes, const int32_t* axes, int32_t inverse, void* scratch,
                                   void* stream) {
    if (!out || !in || !shape || ndim < 1 || ndim > RK_MAXD || naxes < 0 || naxes > ndim ||
        (naxes > 0 && !axes)) {
        set_error("rk_fftshift_execute: bad arguments");
        return RK_ERR_INVALID;
    }
    if (elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16) {
        set_error("rk_fftshift_execute: element size must be 4, 8 or 16 bytes");
        return RK_ERR_INVALID;
    }
    ShiftParams p;
    memset(&p, 0, sizeof(p));
    p.nd = ndim;
    int64_t st = 1, total = 1;
    for (int d = ndim - 1; d >= 0; --d) {
        if (shape[d] < 1) {
            set_error("rk_fftshift_execute: shape entries must be positive");
            return RK_ERR_INVALID;
        }
        p.full[d] = shape[d];
        p.shape[d] = shape[d];
        p.stride[d] = st;
        st *= shape[d];
    }
    total = st;
    bool all_even = true;
    int first = -1;
    bool seen[RK_MAXD] = {false};
    for (int i = 0; i < naxes; ++i) {
        const int a = axes[i];
        if (a < 0 || a >= ndim || seen[a]) {
            set_error("rk_fftshift_execute: bad axis");
            return RK_ERR_INVALID;
        }
        seen[a] = true;
        if (shape[a] % 2) all_even = false;
        if (first < 0 || a < first) first = a;
        p.shift[a] = inverse ? (shape[a] + 1) / 2 : shape[a] / 2;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = (size_t)total * elem_bytes;
    int64_t moved = 1;
    for (int i = 0; i < naxes; ++i) moved *= shape[axes[i]];
    if (naxes == 0 || moved == 1) {
        if (out != in) {
            cudaError_t e = cudaMemcpyAsync(out, in, bytes, cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) {
                set_error(std::string("rk_fftshift_execute: ") + cudaGetErrorString(e));
                return RK_ERR_CUDA;
            }
        }
        return RK_OK;
    }
    cudaError_t e;
    if (all_even) {
        p.shape[first] = shape[first] / 2;
        p.total = total / 2;
        p.first_axis = first;
        switch (elem_bytes) {
            case 4: e = launch_shift<int32_t>(true, out, in, p, s); break;
            case 8: e = launch_shift<int2>(true, out, in, p, s); break;
            default: e = launch_shift<int4>(true, out, in, p, s); break;
        }
    } else {
        p.total = total;
        void* dst = out;
        if (out == in) {
            if (!scratch) {
                set_error("rk_fftshift_execute: in-place shift of an odd axis needs scratch");
                return RK_ERR_INVALID;
            }
            dst = scratch;
        }
        switch (elem_bytes) {
            case 4: e = launch_shift<int32_t>(false, dst, in, p, s); break;
            case 8: e = launch_shift<int2>(false, dst, in, p, s); break;
            default: e = launch_shift<int4>(false, dst, in, p, s); break;
        }
        if (e == cudaSuccess && dst != out) e = cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToDevice, s);
    }
    if (e != cudaSuccess) {
        set_error(std::string("rk_fftshift_execute: ") + cudaGetErrorString(e));
        return RK_ERR_CUDA;
    }
    return RK_OK;
}
