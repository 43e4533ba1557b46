// Row and column passes of the two innermost axes run as one persistent launch in
// plane order, so that a plane's intermediate never leaves L2.
//
// The plane (L1 rows of L2 contiguous elements) is transformed along its rows by a
// position-mode line pass (A) and along its columns by a lane-mode line pass (B), the
// same tile bodies as the stand-alone kernels.  Tasks are the tiles of both passes,
// ordered plane by plane: the A tiles of plane s, then the B tiles of plane s - lag.
// CTAs claim tasks from a counter (the next one while the current one runs); a B
// tile waits until every A tile of its plane is done (per-plane counters,
// release/acquire at GPU scope, clock-bounded with the status word on timeout).  The
// lag keeps the A tiles of a plane finished by the time its B tiles are claimed,
// while the lag planes in between stay far below the L2 size, so B reads what A
// wrote from L2 and HBM sees each element read once and written once for both axes
// (the clustered plane pass achieves the same with a distributed shared memory
// exchange, whose cluster scheduling leaves a quarter of the SM slots empty).
// Deadlock freedom: the lowest-index claimed unfinished task is always running,
// because everything it waits on has a lower index.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "rk_async.cuh"
#include "rk_internal.h"
#include "rk_kernels.cuh"

namespace rk {

namespace {

template <typename T, int LR, int LC> struct PairCfg {
    using A = LineCfg<T, LR, MODE_POS>;   // rows: L = LR along the contiguous axis
    using B = LineCfg<T, LC, MODE_LANE>;  // columns: L = LC along the strided axis
    static_assert(A::NT == B::NT, "both tile bodies run with the same block size");
    static constexpr int NT = A::NT;
    static constexpr size_t SA = (size_t)A::NL * A::LS * A::ESZ;
    static constexpr size_t SB = (size_t)B::NL * LC * B::ESZ;
    static constexpr size_t SMEM = SA > SB ? SA : SB;
};

struct PairArgs {
    PassParams a, b;
    const int32_t* tasks;        // bit 31: B tile; low bits: tile index within its pass
    int64_t ntasks;
    unsigned int* next;          // task counter
    unsigned int* rows_done;     // A tiles finished, per plane
    int32_t a_per_plane, b_per_plane;
    int32_t* status;
};

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <typename T, int LR, int LC>
__global__ void __launch_bounds__(PairCfg<T, LR, LC>::NT, 3) k_pair(const __grid_constant__ PairArgs a) {
    extern __shared__ __align__(16) unsigned char rk_smem[];
    __shared__ int s_task[2];
    bool healthy = true;
    if (threadIdx.x == 0) s_task[0] = (int)atomicAdd(a.next, 1u);
    __syncthreads();
    for (int cur = 0;; cur ^= 1) {
        const int t = s_task[cur];
        if (t >= a.ntasks) break;
        if (threadIdx.x == 0) s_task[cur ^ 1] = (int)atomicAdd(a.next, 1u);
        const int32_t code = a.tasks[t];
        const bool col = code < 0;
        const int tile = code & 0x7fffffff;
        if (col) {
            const int plane = tile / a.b_per_plane;
            if (threadIdx.x == 0) {
                const unsigned int need = (unsigned int)a.a_per_plane;
                bool ok = ld_acquire_u32(a.rows_done + plane) >= need;
                if (!ok && healthy) {
                    const long long t0 = clock64(), lim = wait_limit(a.status);
                    while (!(ok = ld_acquire_u32(a.rows_done + plane) >= need))
                        if (clock64() - t0 > lim) break;
                }
                if (!ok) {
                    healthy = false;
                    atomicOr(a.status, RK_STATUS_TIMEOUT);
                }
            }
            __syncthreads();
            __threadfence();
            line_body<T, LC, MODE_LANE, 0>(a.b, tile, rk_smem, threadIdx.x);
            __syncthreads();
        } else {
            line_body<T, LR, MODE_POS, 0>(a.a, tile, rk_smem, threadIdx.x);
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                atomicAdd(a.rows_done + tile / a.a_per_plane, 1u);
            }
        }
    }
}

template <typename T, int LR, int LC> struct PairLauncher {
    using C = PairCfg<T, LR, LC>;
    static int resident() {
        static int n = 0;
        if (n) return n;
        if (cudaFuncSetAttribute(k_pair<T, LR, LC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM) !=
            cudaSuccess)
            return 0;
        int per = 0, nsm = 0, dev = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pair<T, LR, LC>, C::NT, C::SMEM) != cudaSuccess)
            return 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        n = std::max(1, per) * nsm;
        return n;
    }
    static cudaError_t launch(const PairArgs& args, cudaStream_t st) {
        const int res = resident();
        if (!res) return cudaErrorInvalidConfiguration;
        const int grid = (int)std::min<int64_t>(res, args.ntasks);
        if (grid <= 0) return cudaSuccess;
        k_pair<T, LR, LC><<<grid, C::NT, C::SMEM, st>>>(args);
        return cudaGetLastError();
    }
    static PairInfo info() {
        return PairInfo{&launch_erased, &resident, C::A::NL, C::B::NL};
    }
    static cudaError_t launch_erased(const void* args, cudaStream_t st) {
        return launch(*reinterpret_cast<const PairArgs*>(args), st);
    }
};

}  // namespace

bool pair_info(int dbl, int LR, int LC, PairInfo* out) {
    if (dbl) return false;
    if (LR == 256 && LC == 256) { *out = PairLauncher<float, 256, 256>::info(); return true; }
    if (LR == 128 && LC == 128) { *out = PairLauncher<float, 128, 128>::info(); return true; }
    return false;
}

// Task table and counters of a pair of passes; returns RK_OK or an error code.
int pair_setup(PassRec& ra, PassRec& rb, const PairInfo& pi) {
    const PassParams& pa = ra.prm;
    const PassParams& pb = rb.prm;
    // the column pass runs over (plane, column) lines: its outer count is the planes
    const int64_t planes = pb.O;
    if (planes < 1 || pa.nlines % planes || pb.nlines % planes) return RK_ERR_UNSUPPORTED;
    const int64_t rows = pa.nlines / planes, cols = pb.nlines / planes;
    if (rows % pi.nl_rows || cols % pi.nl_cols) return RK_ERR_UNSUPPORTED;
    const int ta = (int)(rows / pi.nl_rows), tb = (int)(cols / pi.nl_cols);
    const int res = pi.resident();
    if (!res) return RK_ERR_UNSUPPORTED;  // the plan keeps the two passes separate
    // lag: the tasks claimed between a plane's last row tile and its first column
    // tile cover about 1.5 waves of resident CTAs
    const int64_t lag = std::max<int64_t>(1, (3 * (int64_t)res / 2 + ta + tb - 1) / (ta + tb));
    std::vector<int32_t> tasks;
    tasks.reserve((size_t)(planes * (ta + tb)));
    for (int64_t s = 0; s < planes + lag; ++s) {
        if (s < planes)
            for (int k = 0; k < ta; ++k) tasks.push_back((int32_t)(s * ta + k));
        const int64_t q = s - lag;
        if (q >= 0 && q < planes)
            for (int k = 0; k < tb; ++k) tasks.push_back((int32_t)((q * tb + k) | 0x80000000u));
    }
    if (tasks.size() > 0x7fffffff) return RK_ERR_UNSUPPORTED;
    ra.pair_ntasks = (int64_t)tasks.size();
    ra.pair_a = ta;
    ra.pair_b = tb;
    ra.pair_planes = planes;
    if (cudaMalloc(&ra.pair_tasks, tasks.size() * sizeof(int32_t)) != cudaSuccess) return RK_ERR_NOMEM;
    if (cudaMalloc(&ra.pair_counters, (size_t)(planes + 1) * sizeof(unsigned int)) != cudaSuccess)
        return RK_ERR_NOMEM;
    if (cudaMemcpy(ra.pair_tasks, tasks.data(), tasks.size() * sizeof(int32_t), cudaMemcpyHostToDevice) !=
        cudaSuccess)
        return RK_ERR_CUDA;
    ra.pair = pi;
    ra.pair_first = true;
    return RK_OK;
}

cudaError_t pair_launch(const PassRec& ra, const PassParams& pa, const PassParams& pb, int32_t* status,
                        cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(ra.pair_counters, 0, (size_t)(ra.pair_planes + 1) * sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    PairArgs args;
    args.a = pa;
    args.b = pb;
    args.tasks = reinterpret_cast<const int32_t*>(ra.pair_tasks);
    args.ntasks = ra.pair_ntasks;
    args.next = reinterpret_cast<unsigned int*>(ra.pair_counters);
    args.rows_done = reinterpret_cast<unsigned int*>(ra.pair_counters) + 1;
    args.a_per_plane = ra.pair_a;
    args.b_per_plane = ra.pair_b;
    args.status = status;
    return ra.pair.launch(&args, st);
}

}  // namespace rk
