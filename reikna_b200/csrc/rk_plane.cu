// Two-axis plane pass: a 2-D FFT over the last two axes of an array in one HBM
// round trip, using a thread-block cluster and distributed shared memory.
//
// A cluster of Q CTAs owns one L1 x L2 plane.  CTA q loads rows [q L1/Q, (q+1) L1/Q)
// (contiguous, coalesced) and transforms them along the last axis.  After a
// cluster barrier (every CTA is done with its own shared memory) each thread pushes
// its row spectra straight into the shared memory of the CTA that owns those
// columns (st.shared::cluster through map_shared_rank, laid out for the column
// phase), so no thread waits on a remote read.  After a second barrier every CTA
// transforms its L2/Q columns along the row axis and stores them (adjacent columns
// are adjacent in memory, so the stores coalesce).  A 256^3 complex64 transform is
// then two HBM passes (this one plus one strided pass) instead of reikna's five
// kernels (reikna/fft/fft.py:532-584 for the chain it builds).
#include <cooperative_groups.h>

#include "rk_internal.h"
#include "rk_kernels.cuh"

namespace cg = cooperative_groups;

namespace rk {

template <typename T, int L1, int L2, int Q> struct PlaneCfg {
    static constexpr int RT = Radix<T, L2>::RT;
    static_assert(Radix<T, L1>::RT == RT, "row and column plans must hold the same elements per thread");
    static constexpr int NLR = L1 / Q;   // rows per CTA
    static constexpr int NLC = L2 / Q;   // columns per CTA
    static constexpr int NT = NLR * (L2 / RT);
    static_assert(NT == NLC * (L1 / RT), "row and column phases must use the same thread count");
    static constexpr int ESZ = 2 * sizeof(T);
    static constexpr int LS2 = L2 + L2 / 16;
    static constexpr int A = NLR * LS2, B = NLC * L1;
    static constexpr size_t SMEM = (size_t)(A > B ? A : B) * ESZ;
    // resident CTAs per SM the register budget is sized for
    static constexpr int MINB = (sizeof(T) == 4 ? 1024 : 512) / NT > 0 ? (sizeof(T) == 4 ? 1024 : 512) / NT : 1;
};

template <typename T, int L1, int L2, int Q>
__global__ void __launch_bounds__(PlaneCfg<T, L1, L2, Q>::NT, PlaneCfg<T, L1, L2, Q>::MINB)
    k_plane(const PassParams p) {
    using V = cplx<T>;
    using C = PlaneCfg<T, L1, L2, Q>;
    using ER = Engine<T, L2, MODE_POS, C::NLR>;
    using EC = Engine<T, L1, MODE_LANE, C::NLC>;
    constexpr int RT = C::RT;
    extern __shared__ __align__(16) unsigned char rk_smem[];
    V* sm = reinterpret_cast<V*>(rk_smem);
    const V* tw = reinterpret_cast<const V*>(p.tw);
    const int tid = threadIdx.x;
    int q = 0;
    if constexpr (Q > 1) q = (int)cg::this_cluster().block_rank();
    const int64_t plane = blockIdx.x / Q;
    const bool pok = plane < p.O;

    V v[RT];
    // ---- rows: transform along the last axis
    const int ln = tid / ER::TPL, tb = tid % ER::TPL;
    {
        const int64_t line = plane * L1 + (int64_t)q * C::NLR + ln;
        const LineAddr la = line_addr(p.ld, line, 1, 1, pok);
        load_block<T, RT>(p.ld, la, [&](int i) { return ER::in_pos(tb, i / ER::R0, i % ER::R0); }, v);
        ER::run(v, sm, ln, tb, tw);
    }
    if constexpr (Q > 1)
        cg::this_cluster().sync();
    else
        __syncthreads();
    // ---- push row spectra into the owners of their columns (column-phase layout)
    {
        const int row = q * C::NLR + ln;
#pragma unroll
        for (int z = 0; z < RT / ER::RL; ++z)
#pragma unroll
            for (int m = 0; m < ER::RL; ++m) {
                const int col = ER::out_pos(tb, z, m);
                V* dst = sm;
                if constexpr (Q > 1) dst = cg::this_cluster().map_shared_rank(sm, col / C::NLC);
                dst[EC::sidx(col % C::NLC, row)] = v[z * ER::RL + m];
            }
    }
    if constexpr (Q > 1)
        cg::this_cluster().sync();
    else
        __syncthreads();
    // ---- columns: transform along the row axis
    const int lc = tid % C::NLC, tc = tid / C::NLC;
    const int col = q * C::NLC + lc;
#pragma unroll
    for (int z = 0; z < RT / EC::R0; ++z)
#pragma unroll
        for (int m = 0; m < EC::R0; ++m) v[z * EC::R0 + m] = sm[EC::sidx(lc, EC::in_pos(tc, z, m))];
    __syncthreads();
    EC::run(v, sm, lc, tc, reinterpret_cast<const V*>(p.tw2));
    {
        const int64_t line = plane * L2 + col;
        const LineAddr la = line_addr(p.st, line, 1, L2, pok);
        store_block<T, RT>(p.st, p, la, [&](int i) { return EC::out_pos(tc, i / EC::RL, i % EC::RL); }, v);
    }
}

template <typename T, int L1, int L2, int Q> struct PlaneLauncher {
    using C = PlaneCfg<T, L1, L2, Q>;
    static cudaError_t launch(const PassParams& p, int64_t nplanes, cudaStream_t st) {
        static bool attr_done = false;
        if (!attr_done) {
            cudaError_t e = cudaFuncSetAttribute(k_plane<T, L1, L2, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)C::SMEM);
            if (e != cudaSuccess) return e;
            if (Q > 8) {
                e = cudaFuncSetAttribute(k_plane<T, L1, L2, Q>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
                if (e != cudaSuccess) return e;
            }
            attr_done = true;
        }
        if (nplanes <= 0) return cudaSuccess;
        if (nplanes * Q > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(nplanes * Q), 1, 1);
        cfg.blockDim = dim3(C::NT, 1, 1);
        cfg.dynamicSmemBytes = C::SMEM;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = Q;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = Q > 1 ? 1 : 0;
        return cudaLaunchKernelEx(&cfg, k_plane<T, L1, L2, Q>, p);
    }
    static PlaneInfo info() { return PlaneInfo{&launch, Q, C::NT, C::SMEM}; }
};

// wide = 1 selects the 16-CTA cluster variant where one exists
bool plane_info(int dbl, int L1, int L2, int wide, PlaneInfo* out) {
    if (!dbl) {
        if (L1 == 256 && L2 == 256) {
            *out = wide ? PlaneLauncher<float, 256, 256, 16>::info() : PlaneLauncher<float, 256, 256, 8>::info();
            return true;
        }
        if (L1 == 128 && L2 == 128) {
            *out = wide ? PlaneLauncher<float, 128, 128, 4>::info() : PlaneLauncher<float, 128, 128, 2>::info();
            return true;
        }
        if (L1 == 64 && L2 == 64) { *out = PlaneLauncher<float, 64, 64, 1>::info(); return true; }
    } else {
        if (L1 == 128 && L2 == 128) {
            *out = wide ? PlaneLauncher<double, 128, 128, 8>::info() : PlaneLauncher<double, 128, 128, 4>::info();
            return true;
        }
        if (L1 == 64 && L2 == 64) { *out = PlaneLauncher<double, 64, 64, 1>::info(); return true; }
    }
    return false;
}

}  // namespace rk
