// Batched transpose of the two trailing index groups of a C-order array:
// out[b][w][h] = in[b][h][w] (reikna/algorithms/transpose.py:157-201 swaps adjacent
// axis groups the same way; any permutation is a sequence of such swaps).
//
// 32 x 32 tiles staged in shared memory (one padding column against bank
// conflicts): both the reads and the writes are row segments of 32 elements, so an
// element size of 4 bytes moves 128-byte lines each way.  Pure HBM traffic: 2 x the
// array bytes per call.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>

#include "rk_internal.h"

namespace rk {

namespace {

constexpr int TT = 32;   // tile edge
constexpr int TR = 8;    // thread rows (32 x 8 threads, 4 elements each)

struct E16 {
    uint4 v;
};

template <typename E>
__global__ void __launch_bounds__(TT * TR) k_transpose(E* __restrict__ out, const E* __restrict__ in, int64_t batch,
                                                        int64_t H, int64_t W) {
    __shared__ E tile[TT][TT + 1];
    const int64_t tiles_w = (W + TT - 1) / TT, tiles_h = (H + TT - 1) / TT;
    const int64_t per = tiles_w * tiles_h;
    const int64_t total = per * batch;
    const int tx = threadIdx.x % TT, ty = threadIdx.x / TT;
    for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
        const int64_t b = t / per, r = t % per;
        const int64_t th = r / tiles_w, tw = r % tiles_w;
        const E* src = in + b * H * W;
        E* dst = out + b * H * W;
        const int64_t x = tw * TT + tx;
#pragma unroll
        for (int j = ty; j < TT; j += TR) {
            const int64_t y = th * TT + j;
            if (x < W && y < H) tile[j][tx] = src[y * W + x];
        }
        __syncthreads();
        const int64_t ox = th * TT + tx;   // output column = input row
#pragma unroll
        for (int j = ty; j < TT; j += TR) {
            const int64_t oy = tw * TT + j;  // output row = input column
            if (ox < H && oy < W) dst[oy * H + ox] = tile[tx][j];
        }
        __syncthreads();
    }
}

template <typename E> cudaError_t launch(void* out, const void* in, int64_t batch, int64_t H, int64_t W, cudaStream_t st) {
    static int grid = 0;
    if (grid == 0) {
        int per = 0, nsm = 0, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_transpose<E>, TT * TR, 0);
        grid = std::max(1, per) * nsm;
    }
    const int64_t total = ((W + TT - 1) / TT) * ((H + TT - 1) / TT) * batch;
    const int g = (int)std::min<int64_t>(grid, total);
    k_transpose<E><<<g, TT * TR, 0, st>>>(reinterpret_cast<E*>(out), reinterpret_cast<const E*>(in), batch, H, W);
    return cudaGetLastError();
}

}  // namespace

}  // namespace rk

using namespace rk;

extern "C" int rk_transpose_execute(void* out, const void* in, int32_t elem_bytes, int64_t batch, int64_t height,
                                    int64_t width, void* stream) {
    if (!out || !in || batch < 1 || height < 1 || width < 1) {
        set_error("rk_transpose_execute: null pointer or non-positive size");
        return RK_ERR_INVALID;
    }
    if (out == in) {
        set_error("rk_transpose_execute: output may not alias input");
        return RK_ERR_INVALID;
    }
    const uintptr_t align = (uintptr_t)(elem_bytes > 0 && elem_bytes <= 16 ? elem_bytes : 1);
    if (((uintptr_t)out | (uintptr_t)in) % align) {
        set_error("rk_transpose_execute: pointers must be aligned to the element size");
        return RK_ERR_INVALID;
    }
    const int64_t n = batch * height * width;
    if (n / batch / height != width) {
        set_error("rk_transpose_execute: size overflow");
        return RK_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    switch (elem_bytes) {
        case 1: e = launch<uint8_t>(out, in, batch, height, width, st); break;
        case 2: e = launch<uint16_t>(out, in, batch, height, width, st); break;
        case 4: e = launch<uint32_t>(out, in, batch, height, width, st); break;
        case 8: e = launch<uint2>(out, in, batch, height, width, st); break;
        case 16: e = launch<E16>(out, in, batch, height, width, st); break;
        default:
            set_error("rk_transpose_execute: element size must be 1, 2, 4, 8 or 16 bytes");
            return RK_ERR_INVALID;
    }
    if (e != cudaSuccess) {
        set_error(std::string("rk_transpose_execute: ") + cudaGetErrorString(e));
        return RK_ERR_CUDA;
    }
    return RK_OK;
}
