// Persistent TMA-fed line pass (the kernel template; instantiated by rk_tma.cu for
// plain passes and by rk_tma_real.cu for the one-pass real transforms).
#pragma once
#include "rk_async.cuh"
#include "rk_internal.h"
#include "rk_kernels.cuh"

namespace rk {

template <typename T, int L, int MODE> struct TmaCfg {
    using Cfg = LineCfg<T, L, MODE>;
    static constexpr int NL = Cfg::NL, NT = Cfg::NT, ESZ = Cfg::ESZ;
    static constexpr int TILE = NL * L;                                           // elements copied
    static constexpr int BUF = MODE == MODE_POS ? NL * Cfg::LS : NL * L;          // elements per buffer
    static constexpr size_t SMEM = 2 * (size_t)BUF * ESZ + 64;                     // + 2 mbarriers
};

template <typename T, int L, int MODE, int VAR>
__global__ void __launch_bounds__(LineCfg<T, L, MODE>::NT) k_line_tma(const __grid_constant__ PassParams p) {
    using V = cplx<T>;
    using E = Engine<T, L, MODE>;
    using C = TmaCfg<T, L, MODE>;
    constexpr int RT = E::RT, TPL = E::TPL, NL = E::NL, R0 = E::R0, RL = E::RL;
    extern __shared__ __align__(128) unsigned char rk_smem[];
    V* buf0 = reinterpret_cast<V*>(rk_smem);
    V* buf1 = buf0 + C::BUF;
    uint64_t* bars = reinterpret_cast<uint64_t*>(buf1 + C::BUF);
    const V* tw = reinterpret_cast<const V*>(p.tw);
    const int tid = threadIdx.x;
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
        if constexpr (VAR == 4) {
            // inverse real transforms (rows of L bins, no Nyquist bin on this path): the
            // half-length spectrum from the tile pair by pair, reordered through the
            // buffer into the FFT's input order
            static_assert(MODE == MODE_POS, "the real-signal step needs whole lines");
#pragma unroll
            for (int i = 0; i < RT; ++i) v[i] = edge_value<T>(p.ld, buf[ln * L + pair_pos<L, RT, TPL>(tb, i, p.rodd)]);
            real_pairs_in<T, L, RT, TPL>(p, tb, cmk<V>(T(0), T(0)), v);
            __syncthreads();
#pragma unroll
            for (int i = 0; i < RT; ++i) buf[E::sidx(ln, pair_pos<L, RT, TPL>(tb, i, p.rodd))] = v[i];
            __syncthreads();
#pragma unroll
            for (int z = 0; z < RT / R0; ++z)
#pragma unroll
                for (int m = 0; m < R0; ++m) v[z * R0 + m] = buf[E::sidx(ln, E::in_pos(tb, z, m))];
        } else {
#pragma unroll
            for (int z = 0; z < RT / R0; ++z)
#pragma unroll
                for (int m = 0; m < R0; ++m) {
                    const int pos = E::in_pos(tb, z, m);
                    v[z * R0 + m] = MODE == MODE_POS ? buf[ln * L + pos] : buf[pos * NL + ln];
                }
            const int32_t f = p.ld.flags;
            if (f & SF_SCALE) scale_block<T, RT>(p.ld, v);
            if (f & SF_TAB) {
                // a per-position table (the antiperiodic forward transform's W_2L^m),
                // between the two conjugations as in the element path
                if (f & SF_PRE_CONJ) {
#pragma unroll
                    for (int i = 0; i < RT; ++i) v[i].y = -v[i].y;
                }
                const V* tab = reinterpret_cast<const V*>(p.ld.tab);
#pragma unroll
                for (int z = 0; z < RT / R0; ++z)
#pragma unroll
                    for (int m = 0; m < R0; ++m) v[z * R0 + m] = cmul(v[z * R0 + m], __ldg(tab + E::in_pos(tb, z, m)));
                if (f & SF_POST_CONJ) {
#pragma unroll
                    for (int i = 0; i < RT; ++i) v[i].y = -v[i].y;
                }
            } else if (((f & SF_PRE_CONJ) != 0) != ((f & SF_POST_CONJ) != 0)) {
#pragma unroll
                for (int i = 0; i < RT; ++i) v[i].y = -v[i].y;
            }
        }
        __syncthreads();  // the tile is in registers: the buffer becomes the exchange area
        E::run(v, buf, ln, tb, tw);
        if constexpr (E::NS == 1) __syncthreads();
        V nyq = cmk<V>(T(0), T(0));
        if constexpr (VAR == 3) {
            // real-signal spectrum X[k] = Z[k] A_k + conj(Z[mirror k]) B_k through the
            // exchange buffer, before the next copy lands in it
            static_assert(MODE == MODE_POS, "the real-spectrum step needs whole lines");
#pragma unroll
            for (int z = 0; z < RT / RL; ++z)
#pragma unroll
                for (int m = 0; m < RL; ++m) buf[E::sidx(ln, E::out_pos(tb, z, m))] = v[z * RL + m];
            __syncthreads();
            nyq = real_pairs_out<T, L, RT, TPL>(p, tb, [&](int k) { return buf[E::sidx(ln, k)]; }, v);
            __syncthreads();
        }
        if (tid == 0 && t + 2 * stride < p.ntiles) {
            fence_proxy_async_smem();
            issue(t + 2 * stride, b);
        }
        const int64_t line = t * NL + ln;
        const LineAddr la = line_addr(p.st, line, p.C, p.I, line < p.nlines);
        if constexpr (VAR == 3) {
            if (p.rnyq && tb == 0 && la.ok) store_nyquist<T>(p.st, la.base + (int64_t)L * p.st.ax_stride, nyq);
        }
        if constexpr (VAR == 3)
            store_block<T, RT>(p.st, p, la, [&](int i) { return pair_pos<L, RT, TPL>(tb, i, p.rodd); }, v);
        else
            store_block<T, RT>(p.st, p, la, [&](int i) { return E::out_pos(tb, i / RL, i % RL); }, v);
    }
}

template <typename T, int L, int MODE, int VAR> struct TmaLauncher {
    using C = TmaCfg<T, L, MODE>;
    static cudaError_t launch(const PassParams& p, int64_t nblocks, cudaStream_t st) {
        static bool attr_done = false;
        if (!attr_done) {
            cudaError_t e =
                cudaFuncSetAttribute(k_line_tma<T, L, MODE, VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
            if (e != cudaSuccess) return e;
            attr_done = true;
        }
        if (nblocks <= 0) return cudaSuccess;
        k_line_tma<T, L, MODE, VAR><<<(unsigned)nblocks, C::NT, C::SMEM, st>>>(p);
        return cudaGetLastError();
    }
    static int per_sm() {
        int n = 0;
        cudaFuncSetAttribute(k_line_tma<T, L, MODE, VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_line_tma<T, L, MODE, VAR>, C::NT, C::SMEM);
        return n;
    }
    static TmaInfo info() { return TmaInfo{&launch, &per_sm, C::NT, C::NL, C::SMEM}; }
};

}  // namespace rk
