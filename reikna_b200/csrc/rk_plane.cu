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

#include "rk_async.cuh"
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
    using ER = Engine<T, L2, MODE_POS, 0, C::NLR>;
    using EC = Engine<T, L1, MODE_LANE, 0, C::NLC>;
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
        load_block<T, RT, false>(p.ld, la, [&](int i) { return ER::in_pos(tb, i / ER::R0, i % ER::R0); }, v);
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
        store_block<T, RT, STORE_FAST>(p.st, p, la, [&](int i) { return EC::out_pos(tc, i / EC::RL, i % EC::RL); }, v);
    }
}

// ------------------------------------------------------------------------------
// Persistent TMA-fed variant.  A cluster loops over planes; each CTA keeps two
// buffers: A receives its rows (one 1-D bulk copy of NLR contiguous rows) and then
// serves as the row-phase exchange area; B receives the pushed column data and
// serves as the column-phase exchange area.  As soon as a CTA's row transform is in
// registers it starts the bulk copy of its rows of the next plane into A, so the
// load overlaps the push, the column transform and the stores.
// Every CTA of a cluster runs the same number of iterations and reaches every
// cluster barrier; a timed-out copy wait records the status word and the loop
// carries on (skipping further waits) so no barrier is left unmatched.
// ------------------------------------------------------------------------------

template <typename T, int L1, int L2, int Q> struct PlaneTmaCfg {
    using C = PlaneCfg<T, L1, L2, Q>;
    static constexpr int A = C::NLR * C::LS2;   // rows (dense) / row exchange (padded)
    static constexpr int B = C::NLC * L1;       // columns
    // stage twiddle tables of the row and column lengths, copied to shared memory
    static constexpr int TW2 = TwLayout<T, L2>::total(), TW1 = TwLayout<T, L1>::total();
    static constexpr size_t SMEM = (size_t)(A + B + TW2 + TW1) * C::ESZ + 64;
    // resident CTAs per SM: as many as shared memory allows, capped by the plain config
    static constexpr int BY_SMEM = (int)((227 * 1024) / SMEM) > 0 ? (int)((227 * 1024) / SMEM) : 1;
    static constexpr int MINB = BY_SMEM < C::MINB ? BY_SMEM : C::MINB;
};

template <typename T, int L1, int L2, int Q>
__global__ void __launch_bounds__(PlaneCfg<T, L1, L2, Q>::NT, (PlaneTmaCfg<T, L1, L2, Q>::MINB))
    k_plane_tma(const __grid_constant__ PassParams p) {
    using V = cplx<T>;
    using C = PlaneCfg<T, L1, L2, Q>;
    using ER = Engine<T, L2, MODE_POS, 0, C::NLR>;
    using EC = Engine<T, L1, MODE_LANE, 0, C::NLC>;
    constexpr int RT = C::RT;
    extern __shared__ __align__(128) unsigned char rk_smem[];
    V* bufA = reinterpret_cast<V*>(rk_smem);
    V* bufB = bufA + PlaneTmaCfg<T, L1, L2, Q>::A;
    // bars[0]: rows of the plane arrived (TMA); bars[1]: column data arrived (st.async
    // bytes from every CTA); bars[2]: every receiver freed its column buffer
    uint64_t* bars = reinterpret_cast<uint64_t*>(bufB + PlaneTmaCfg<T, L1, L2, Q>::B);
    using TC = PlaneTmaCfg<T, L1, L2, Q>;
    // rows of 256 points on 16 lanes: the warp-local row transform below
    constexpr bool ROWL = L2 == 256 && Q > 1 && RT == 16 && ER::NS == 2 && ER::R0 == 16 && ER::TPL == 16;
    V* tw = reinterpret_cast<V*>(bars + 8);
    V* tw2 = tw + TC::TW2;
    const int tid = threadIdx.x;
    // the stage twiddles stay in shared memory for the kernel's life (every plane
    // uses the same ones; loads from there do not wait on L2)
    for (int i = tid; i < TC::TW2; i += C::NT) tw[i] = reinterpret_cast<const V*>(p.tw)[i];
    for (int i = tid; i < TC::TW1; i += C::NT) tw2[i] = reinterpret_cast<const V*>(p.tw2)[i];
    const int q = Q > 1 ? (int)cg::this_cluster().block_rank() : 0;
    const int64_t ncl = gridDim.x / Q;
    const int ln = tid / ER::TPL, tb = tid % ER::TPL;
    const int lc = tid % C::NLC, tc = tid / C::NLC;
    constexpr uint32_t ROW_BYTES = (uint32_t)(C::NLR * L2 * C::ESZ);
    constexpr uint32_t COL_BYTES = (uint32_t)(C::NLC * L1 * C::ESZ);

    auto issue = [&](int64_t plane) {
        mbar_arrive_expect_tx(&bars[0], ROW_BYTES);
        const V* src = reinterpret_cast<const V*>(p.ld.ptr) + p.ld.offset + plane * p.tile_stride +
                       (int64_t)q * C::NLR * L2;
        bulk_g2s(bufA, src, ROW_BYTES, &bars[0]);
    };
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], Q);
        fence_mbar_init();
    }
    // every CTA's barriers exist before anybody signals a remote one
    if constexpr (Q > 1) cg::this_cluster().sync(); else __syncthreads();
    const uint32_t bufB_s = smem_u32(bufB), full_s = smem_u32(&bars[1]), empty_s = smem_u32(&bars[2]);
    int64_t plane = blockIdx.x / Q;
    if (tid == 0 && plane < p.O) issue(plane);
    uint32_t pa = 0, pf = 0, pe = 0;
    bool healthy = true;
    for (; plane < p.O; plane += ncl) {
        const bool last = plane + ncl >= p.O;
        if (healthy) healthy = mbar_wait(&bars[0], pa, p.status);
        pa ^= 1;
        V v[RT];
        if constexpr (ROWL) {
#pragma unroll
            for (int m = 0; m < 16; ++m) v[m] = bufA[ln * L2 + tb + 16 * m];
        } else {
#pragma unroll
            for (int z = 0; z < RT / ER::R0; ++z)
#pragma unroll
                for (int m = 0; m < ER::R0; ++m) v[z * ER::R0 + m] = bufA[ln * L2 + ER::in_pos(tb, z, m)];
        }
        if (p.ld.flags & SF_SCALE) {
            const V c = cmk<V>((T)p.ld.scale_re, (T)p.ld.scale_im);
#pragma unroll
            for (int i = 0; i < RT; ++i) v[i] = cmul(v[i], c);
        }
        if (((p.ld.flags & SF_PRE_CONJ) != 0) != ((p.ld.flags & SF_POST_CONJ) != 0)) {
#pragma unroll
            for (int i = 0; i < RT; ++i) v[i].y = -v[i].y;
        }
        if constexpr (ROWL) {
            // the 16 lanes of a row are one half-warp: the row's exchange between its
            // two radix-16 stages stays inside the warp, in place in the row's own
            // landing area, position p at p ^ ((p >> 4) & 15) (no bank conflicts for
            // either order, no block barrier)
            V* row = bufA + ln * L2;
            V* rowt = row + 16 * tb;
            // stage twiddles from shared memory after the butterfly (short latency;
            // keeps them out of the live registers during the DFT)
            dft<16>(v);
#pragma unroll
            for (int m = 1; m < 16; ++m) v[m] = cmul(v[m], tw[(m - 1) * 16 + tb]);
            __syncwarp();
#pragma unroll
            for (int m = 0; m < 16; ++m) rowt[m ^ tb] = v[m];
            __syncwarp();
#pragma unroll
            for (int m = 0; m < 16; ++m) v[m] = row[16 * m + (tb ^ m)];
            dft<16>(v);
        } else {
            __syncthreads();
            ER::template run<true>(v, bufA, ln, tb, tw);
            if constexpr (ER::NS == 1) __syncthreads();
            if (tid == 0 && !last) {
                fence_proxy_async_smem();
                issue(plane + ncl);
            }
        }
        if constexpr (Q > 1) {
            if (tid == 0) mbar_arrive_expect_tx(&bars[1], COL_BYTES);
            // every receiver has consumed the previous plane's column data
            if (healthy) healthy = mbar_wait_cluster(&bars[2], pe ^ 1, p.status);
            pe ^= 1;
            const int row = q * C::NLR + ln;
#pragma unroll
            for (int z = 0; z < RT / ER::RL; ++z)
#pragma unroll
                for (int m = 0; m < ER::RL; ++m) {
                    const int col = ER::out_pos(tb, z, m);
                    const uint32_t owner = (uint32_t)(col / C::NLC);
                    const uint32_t off = (uint32_t)(EC::sidx(col % C::NLC, row) * C::ESZ);
                    st_async(mapa(bufB_s + off, owner), v[z * ER::RL + m], mapa(full_s, owner));
                }
            if (healthy) healthy = mbar_wait_cluster(&bars[1], pf, p.status);
            pf ^= 1;
        } else {
            // a single CTA owns the whole plane: the exchange is local (no cluster
            // instructions, which a launch without clusters may not execute)
#pragma unroll
            for (int z = 0; z < RT / ER::RL; ++z)
#pragma unroll
                for (int m = 0; m < ER::RL; ++m) bufB[EC::sidx(ER::out_pos(tb, z, m), ln)] = v[z * ER::RL + m];
            __syncthreads();
        }
#pragma unroll
        for (int z = 0; z < RT / EC::R0; ++z)
#pragma unroll
            for (int m = 0; m < EC::R0; ++m) v[z * EC::R0 + m] = bufB[EC::sidx(lc, EC::in_pos(tc, z, m))];
        __syncthreads();
        if constexpr (ROWL) {
            // every warp is past its rows: the next plane's rows may land in A
            if (tid == 0 && !last) {
                fence_proxy_async_smem();
                issue(plane + ncl);
            }
        }
        EC::template run<true>(v, bufB, lc, tc, tw2);
        if constexpr (EC::NS == 1) __syncthreads();
        // the column buffer is free again: tell every sender of the next plane
        if constexpr (Q > 1)
            if (!last && tid < Q) mbar_arrive_remote(mapa(empty_s, (uint32_t)tid));
        const int64_t line = plane * L2 + q * C::NLC + lc;
        const LineAddr la = line_addr(p.st, line, 1, L2, true);
        store_block<T, RT, STORE_FAST>(p.st, p, la, [&](int i) { return EC::out_pos(tc, i / EC::RL, i % EC::RL); }, v);
    }
    if (!healthy) mbar_wait(&bars[0], pa, nullptr);
    // no CTA leaves while another could still address its shared memory
    if constexpr (Q > 1) cg::this_cluster().sync();
}

template <typename T, int L1, int L2, int Q> struct PlaneTmaLauncher {
    using C = PlaneCfg<T, L1, L2, Q>;
    using TC = PlaneTmaCfg<T, L1, L2, Q>;
    static cudaError_t attr() {
        static bool done = false;
        if (done) return cudaSuccess;
        cudaError_t e =
            cudaFuncSetAttribute(k_plane_tma<T, L1, L2, Q>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC::SMEM);
        if (e != cudaSuccess) return e;
        if (Q > 8) {
            e = cudaFuncSetAttribute(k_plane_tma<T, L1, L2, Q>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (e != cudaSuccess) return e;
        }
        done = true;
        return cudaSuccess;
    }
    static cudaLaunchConfig_t config(int64_t nctas, cudaStream_t st, cudaLaunchAttribute* a) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)nctas, 1, 1);
        cfg.blockDim = dim3(C::NT, 1, 1);
        cfg.dynamicSmemBytes = TC::SMEM;
        cfg.stream = st;
        a[0].id = cudaLaunchAttributeClusterDimension;
        a[0].val.clusterDim.x = Q;
        a[0].val.clusterDim.y = 1;
        a[0].val.clusterDim.z = 1;
        cfg.attrs = a;
        cfg.numAttrs = Q > 1 ? 1 : 0;
        return cfg;
    }
    // nblocks = CTAs of the persistent grid (a multiple of Q)
    static cudaError_t launch(const PassParams& p, int64_t nblocks, cudaStream_t st) {
        cudaError_t e = attr();
        if (e != cudaSuccess) return e;
        if (nblocks <= 0) return cudaSuccess;
        cudaLaunchAttribute a[1];
        cudaLaunchConfig_t cfg = config(nblocks, st, a);
        return cudaLaunchKernelEx(&cfg, k_plane_tma<T, L1, L2, Q>, p);
    }
    // clusters that fit on the device at once
    static int clusters() {
        if (attr() != cudaSuccess) return 0;
        cudaLaunchAttribute a[1];
        cudaLaunchConfig_t cfg = config(Q * 256, nullptr, a);
        int n = 0;
        if (Q > 1) {
            if (cudaOccupancyMaxActiveClusters(&n, k_plane_tma<T, L1, L2, Q>, &cfg) != cudaSuccess) return 0;
        } else {
            int dev = 0, nsm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_plane_tma<T, L1, L2, Q>, C::NT, TC::SMEM);
            n *= nsm;
        }
        return n;
    }
    static PlaneTmaInfo info() { return PlaneTmaInfo{&launch, &clusters, Q, C::NT, TC::SMEM}; }
};

bool plane_tma_info(int dbl, int L1, int L2, PlaneTmaInfo* out) {
    if (!dbl) {
        if (L1 == 256 && L2 == 256) { *out = PlaneTmaLauncher<float, 256, 256, 16>::info(); return true; }
        if (L1 == 128 && L2 == 128) { *out = PlaneTmaLauncher<float, 128, 128, 4>::info(); return true; }
        if (L1 == 64 && L2 == 64) { *out = PlaneTmaLauncher<float, 64, 64, 1>::info(); return true; }
    } else {
        if (L1 == 128 && L2 == 128) { *out = PlaneTmaLauncher<double, 128, 128, 8>::info(); return true; }
    }
    return false;
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
