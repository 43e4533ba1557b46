// Standalone FFTShift (reikna/fft/fftshift.py:14-110, fftshift.mako:1-84).
//
// Every shifted axis even: one kernel over the array with the first shifted axis
// halved swaps each element with its shifted partner (its own inverse), so it works
// in place.  Otherwise one out-of-place scatter out[(i + s) mod n] = in[i] with
// s = n // 2 (fftshift) or (n + 1) // 2 (ifftshift); when out aliases in, the scatter
// goes to `scratch` and is copied back.
#include <cuda_runtime.h>
#include <string.h>

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

template <typename E>
static cudaError_t launch_shift(bool swap, void* out, const void* in, const ShiftParams& p, cudaStream_t st) {
    if (p.total == 0) return cudaSuccess;
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
