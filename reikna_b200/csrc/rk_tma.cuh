// Persistent TMA-fed line pass (the kernel template; instantiated by rk_tma.cu).
#pragma once
#include "rk_async.cuh"
#include "rk_internal.h"
#include "rk_kernels.cuh"

namespace rk {

template <typename T, int L, int MODE> struct TmaCfg {
    using Cfg = LineCfg<T, L, MODE>;
    static constexpr int ESZ = Cfg::ESZ;
    // lane mode: lines a CTA halved (down to half a 128-byte segment of lines) where a
    // tile exceeds 32 KB, so that its two buffers leave room for more than one CTA an SM
    // (complex128 128-point lines: 32 -> 16 lines, 133 -> 66 KB; complex64 512-point
    // lines: 16 -> 8, 64-byte rows)
    static constexpr int NL_HALF = Cfg::NL / 2 >= Vec<T>::N / 2 && Cfg::NL * L * ESZ > 32768 ? Cfg::NL / 2 : Cfg::NL;
    static constexpr int NL = MODE == MODE_LANE ? NL_HALF : Cfg::NL;
    static constexpr int NT = NL * Cfg::TPL;
    static constexpr int TILE = NL * L;                                           // elements copied
    static constexpr int BUF = MODE == MODE_POS ? NL * Cfg::LS : NL * L;          // elements per buffer
    static constexpr size_t SMEM0 = 2 * (size_t)BUF * ESZ + 64;                    // + mbarriers
    // the stage twiddles move to shared memory when that costs no resident CTA
    static constexpr int TWN = TwLayout<T, L>::total();
    static constexpr bool TWS =
        TWN > 0 && (227 * 1024) / (SMEM0 + (size_t)TWN * ESZ) == (227 * 1024) / SMEM0;
    static constexpr size_t SMEM = SMEM0 + (TWS ? (size_t)TWN * ESZ : 0);
};

template <typename T, int L, int MODE>
__global__ void __launch_bounds__(TmaCfg<T, L, MODE>::NT) k_line_tma(const __grid_constant__ PassParams p) {
    using V = cplx<T>;
    using C = TmaCfg<T, L, MODE>;
    using E = Engine<T, L, MODE, 0, C::NL>;
    constexpr int RT = E::RT, TPL = E::TPL, NL = E::NL, R0 = E::R0, RL = E::RL;
    extern __shared__ __align__(128) unsigned char rk_smem[];
    V* buf0 = reinterpret_cast<V*>(rk_smem);
    V* buf1 = buf0 + C::BUF;
    uint64_t* bars = reinterpret_cast<uint64_t*>(buf1 + C::BUF);
    const int tid = threadIdx.x;
    const V* tw = reinterpret_cast<const V*>(p.tw);
    if constexpr (C::TWS) {
        V* tws = reinterpret_cast<V*>(bars + 8);
        for (int i = tid; i < C::TWN; i += C::NT) tws[i] = tw[i];
        tw = tws;   // made visible by the barrier after the mbarrier set-up
    }
    const int ln = MODE == MODE_POS ? tid / TPL : tid % NL;
    const int tb = MODE == MODE_POS ? tid % TPL : tid / NL;

    auto issue = [&](int64_t t, int b) {
        V* dst = b ? buf1 : buf0;
        uint64_t* bar = bars + b;
        if (p.tma_mode == TMA_BULK) {
            const int64_t first = t * NL;
            const int64_t nl = (p.nlines - first) < NL ? (p.nlines - first) : NL;
            const uint32_t bytes = (uint32_t)(nl * L * C::ESZ);
            mbar_arrive_expect_tx(bar, bytes);
            const V* src = reinterpret_cast<const V*>(p.ld.ptr) + p.ld.offset + t * p.tile_stride;
            bulk_g2s(dst, src, bytes, bar);
        } else {
            const int64_t first = t * NL;
            const int64_t o = first / p.I, i = first % p.I;
            const int rows = L / p.tma_boxes;
            mbar_arrive_expect_tx(bar, (uint32_t)(C::TILE * C::ESZ));
            const int xs = sizeof(T) == 8 ? 2 : 1;  // complex128 maps as pairs of doubles
            for (int k = 0; k < p.tma_boxes; ++k)
                tma_g2s_3d(dst + (size_t)k * rows * NL, &p.tmap, (int)i * xs, k * rows, (int)o, bar);
        }
    };

    if (tid == 0) {
        mbar_init(bars + 0, 1);
        mbar_init(bars + 1, 1);
        fence_mbar_init();
    }
    __syncthreads();
    const int64_t stride = gridDim.x;
    int64_t t = blockIdx.x;
    if (tid == 0) {
        if (t < p.ntiles) issue(t, 0);
        if (t + stride < p.ntiles) issue(t + stride, 1);
    }
    uint32_t phase0 = 0, phase1 = 0;
    for (int k = 0; t < p.ntiles; t += stride, ++k) {
        const int b = k & 1;
        V* buf = b ? buf1 : buf0;
        const bool ok = mbar_wait(bars + b, b ? phase1 : phase0, p.status);
        if (b) phase1 ^= 1; else phase0 ^= 1;
        if (!ok) {
            // the status word records the timeout; before leaving, give the copy into
            // the other buffer (if one was issued) a bounded chance to land
            if (t + stride < p.ntiles) mbar_wait(bars + (b ^ 1), b ? phase0 : phase1, nullptr);
            break;
        }
        V v[RT];
#pragma unroll
        for (int z = 0; z < RT / R0; ++z)
#pragma unroll
            for (int m = 0; m < R0; ++m) {
                const int pos = E::in_pos(tb, z, m);
                v[z * R0 + m] = MODE == MODE_POS ? buf[ln * L + pos] : buf[pos * NL + ln];
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
        __syncthreads();  // the tile is in registers: the buffer becomes the exchange area
        E::template run<C::TWS>(v, buf, ln, tb, tw);
        if constexpr (E::NS == 1) __syncthreads();
        if (tid == 0 && t + 2 * stride < p.ntiles) {
            fence_proxy_async_smem();
            issue(t + 2 * stride, b);
        }
        const int64_t line = t * NL + ln;
        const LineAddr la = line_addr(p.st, line, p.C, p.I, line < p.nlines);
        // the planner takes this kernel only for SF_FAST store sides
        store_block<T, RT, STORE_FAST>(p.st, p, la, [&](int i) { return E::out_pos(tb, i / RL, i % RL); }, v);
    }
}

template <typename T, int L, int MODE> struct TmaLauncher {
    using C = TmaCfg<T, L, MODE>;
    static cudaError_t launch(const PassParams& p, int64_t nblocks, cudaStream_t st) {
        static bool attr_done = false;
        if (!attr_done) {
            cudaError_t e =
                cudaFuncSetAttribute(k_line_tma<T, L, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
            if (e != cudaSuccess) return e;
            attr_done = true;
        }
        if (nblocks <= 0) return cudaSuccess;
        k_line_tma<T, L, MODE><<<(unsigned)nblocks, C::NT, C::SMEM, st>>>(p);
        return cudaGetLastError();
    }
    static int per_sm() {
        int n = 0;
        cudaFuncSetAttribute(k_line_tma<T, L, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_line_tma<T, L, MODE>, C::NT, C::SMEM);
        return n;
    }
    static TmaInfo info() { return TmaInfo{&launch, &per_sm, C::NT, C::NL, C::SMEM}; }
};

}  // namespace rk
