// Persistent line passes fed by the Tensor Memory Accelerator.
//
// Each CTA loops over tiles of NL lines.  Two shared-memory buffers alternate: while
// the CTA transforms tile k out of one buffer, the bulk-copy engine is already
// writing tile k+1 into the other (completion tracked by an mbarrier per buffer), so
// HBM latency overlaps the butterflies instead of stalling the warps that issued the
// loads.  The buffer of the current tile doubles as the Stockham exchange buffer
// once its stage-0 inputs are in registers.  Results are stored straight from
// registers (coalesced 128-byte rows), then the freed buffer receives tile k+2.
//
//  * position mode: a tile is NL contiguous lines -> one 1-D cp.async.bulk;
//  * lane mode: a tile is L rows of NL adjacent lines (128 bytes) at the axis
//    stride -> a 3-D tiled tensor copy whose box lands in shared memory exactly in
//    the lane-mode layout [position][lane].
#include <cuda.h>

#include <mutex>

#include "rk_tma.cuh"

namespace rk {

#define RK_TI(TY, LL, MODE) \
    if (L == LL && mode == MODE) { *out = TmaLauncher<TY, LL, MODE>::info(); return true; }

bool tma_info(int dbl, int L, int mode, TmaInfo* out) {
    if (!dbl) {
        RK_TI(float, 64, MODE_POS)
        RK_TI(float, 128, MODE_POS)
        RK_TI(float, 256, MODE_POS)
        RK_TI(float, 512, MODE_POS)
        RK_TI(float, 1024, MODE_POS)
        RK_TI(float, 2048, MODE_POS)
        RK_TI(float, 4096, MODE_POS)
        RK_TI(float, 8192, MODE_POS)
        RK_TI(float, 16, MODE_LANE)
        RK_TI(float, 32, MODE_LANE)
        RK_TI(float, 64, MODE_LANE)
        RK_TI(float, 128, MODE_LANE)
        RK_TI(float, 256, MODE_LANE)
        RK_TI(float, 512, MODE_LANE)
        RK_TI(float, 1024, MODE_LANE)
    } else {
        RK_TI(double, 64, MODE_POS)
        RK_TI(double, 128, MODE_POS)
        RK_TI(double, 256, MODE_POS)
        RK_TI(double, 512, MODE_POS)
        RK_TI(double, 1024, MODE_POS)
        RK_TI(double, 2048, MODE_POS)
        RK_TI(double, 4096, MODE_POS)
        RK_TI(double, 16, MODE_LANE)
        RK_TI(double, 32, MODE_LANE)
        RK_TI(double, 64, MODE_LANE)
        RK_TI(double, 128, MODE_LANE)
        RK_TI(double, 256, MODE_LANE)
        RK_TI(double, 512, MODE_LANE)
    }
    return false;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda)
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// 3-D map over (line-in-plane i, position, plane o) of a lane-mode load side:
// element (o, i, j) at base + (o * so + i + j * sj) elements.  Box {NL, rows, 1}.
bool encode_lane_map(void* base, int dbl, int64_t I, int64_t L, int64_t O, int64_t sj, int64_t so, int nl, int rows,
                     TensorMapBytes* out) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const int xs = dbl ? 2 : 1;  // complex128 as two doubles, complex64 as one 64-bit word
    const int64_t esz = dbl ? 8 : 8;
    cuuint64_t dims[3] = {(cuuint64_t)(I * xs), (cuuint64_t)L, (cuuint64_t)O};
    cuuint64_t strides[2] = {(cuuint64_t)(sj * xs * esz), (cuuint64_t)(so * xs * esz)};
    cuuint32_t box[3] = {(cuuint32_t)(nl * xs), (cuuint32_t)rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    if (strides[0] % 16 || strides[1] % 16 || ((uintptr_t)base) % 16) return false;
    CUtensorMap m;
    CUresult r = fn(&m, dbl ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, base, dims, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    static_assert(sizeof(CUtensorMap) == sizeof(TensorMapBytes), "tensor map size");
    memcpy(out, &m, sizeof(m));
    return true;
}

}  // namespace rk
