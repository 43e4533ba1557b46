// Fused Bluestein pass on a two-CTA cluster a line (line-pass variant 7).
//
// Bluestein's convolution length M is a power of two with M >= 2N, so the chirped
// input a[n] = x[n] c[n] occupies less than half of the padded line (N <= M/2) and
// only outputs n < N <= M/2 are kept.  With L = M/2:
//   FFT_M(a)[2j + r] = FFT_L(a[n] W_M^(n r))[j],   r = 0, 1
// (the first radix-2 step of the M-point transform has zeros in its upper half), and
// for the inverse transform of Y = FFT_M(a) K,
//   y[n] = c_0[n] + W_M^(-n) c_1[n],  c_r = IFFT_L(Y[2j + r]),  n < L.
// CTA r of the cluster owns bins 2j + r: it loads the line (chirp applied by the load
// side, W_M^n for r = 1), runs the L-point FFT, multiplies by the kernel spectrum K
// (1/M folded in) and conjugates, runs the L-point FFT again (the inverse as a
// conjugated forward transform: u_r = FFT_L(conj(Y_r)), c_r = conj(u_r)), and keeps
// u_r (times W_M^n for r = 1) in its shared memory.  After a cluster barrier CTA r
// adds the peer's values for its half of the outputs, n in [r L/2, (r + 1) L/2),
// read through distributed shared memory; the store side conjugates and applies the
// chirp: conj(u_0 + W_M^n u_1) = c_0 + W_M^(-n) c_1.  A second cluster barrier keeps
// each CTA's shared memory alive until the peer has read it.
//
// Against one CTA a line (variant 1) each CTA holds half the line (16 elements a
// thread instead of 32), so two CTAs share an SM where one did: twice the warps to
// hide the FFT's latencies, for one exchange of L complex values a line.
#include <cooperative_groups.h>

#include "rk_internal.h"
#include "rk_kernels.cuh"

namespace cg = cooperative_groups;

namespace rk {

namespace {

template <typename T, int L>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(LineCfg<T, L, MODE_POS>::NT, 2)
    k_blue2(const __grid_constant__ PassParams p) {
    using V = cplx<T>;
    using E = Engine<T, L, MODE_POS>;
    using Cfg = LineCfg<T, L, MODE_POS>;
    constexpr int RT = Cfg::RT, TPL = Cfg::TPL, R0 = E::R0, RL = E::RL;
    constexpr int H = L / 2;       // outputs a CTA
    constexpr int NO = H / TPL;    // outputs a thread
    static_assert(Cfg::NL == 1 && Cfg::NT == TPL && H % TPL == 0, "one line a CTA");
    extern __shared__ __align__(16) unsigned char rk_smem[];
    V* sm = reinterpret_cast<V*>(rk_smem);
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int tb = (int)threadIdx.x;
    const int64_t line = blockIdx.x >> 1;
    const bool lok = line < p.nlines;
    const V* tw = reinterpret_cast<const V*>(p.tw);
    const V* wm = reinterpret_cast<const V*>(p.rtwid);   // W_M^n, n <= L
    const V* K = reinterpret_cast<const V*>(p.blue_k);    // kernel spectrum, M bins

    V v[RT];
    {
        const LineAddr la = line_addr(p.ld, line, p.C, p.I, lok);
        load_block<T, RT, false>(p.ld, la, [&](int i) { return E::in_pos(tb, i / R0, i % R0); }, v);
    }
    if (rank == 1) {
#pragma unroll
        for (int i = 0; i < RT; ++i) v[i] = cmul(v[i], __ldg(wm + E::in_pos(tb, i / R0, i % R0)));
    }
    // both L-point FFTs run one looped copy of the code (instruction-cache footprint)
#pragma unroll 1
    for (int it = 0; it < 2; ++it) {
        E::run(v, sm, 0, tb, tw);
        if (it == 0) {
            // bins 2j + rank times the kernel spectrum, conjugated, back to stage-0 order
#pragma unroll
            for (int z = 0; z < RT / RL; ++z)
#pragma unroll
                for (int m = 0; m < RL; ++m) {
                    const int pos = E::out_pos(tb, z, m);
                    sm[E::sidx(0, pos)] = cconj(cmul(v[z * RL + m], __ldg(K + 2 * pos + rank)));
                }
            __syncthreads();
#pragma unroll
            for (int z = 0; z < RT / R0; ++z)
#pragma unroll
                for (int m = 0; m < R0; ++m) v[z * R0 + m] = sm[E::sidx(0, E::in_pos(tb, z, m))];
            __syncthreads();
        }
    }
#pragma unroll
    for (int z = 0; z < RT / RL; ++z)
#pragma unroll
        for (int m = 0; m < RL; ++m) {
            const int pos = E::out_pos(tb, z, m);
            V u = v[z * RL + m];
            if (rank == 1) u = cmul(u, __ldg(wm + pos));
            sm[E::sidx(0, pos)] = u;
        }
    // both CTAs' halves are in shared memory
    cl.sync();
    const V* peer = cl.map_shared_rank(sm, rank ^ 1);
    V w[NO];
#pragma unroll
    for (int q = 0; q < NO; ++q) {
        const int s = E::sidx(0, H * rank + tb + TPL * q);
        const V a = sm[s], b = peer[s];
        w[q] = cmk<V>(a.x + b.x, a.y + b.y);
    }
    {
        const LineAddr ls = line_addr(p.st, line, p.C, p.I, lok);
        store_block<T, NO>(p.st, p, ls, [&](int q) { return H * rank + tb + TPL * q; }, w);
    }
    // the peer has read this CTA's shared memory
    cl.sync();
}

template <typename T, int L>
struct Blue2Launcher {
    using Cfg = LineCfg<T, L, MODE_POS>;
    static size_t smem() { return (size_t)Cfg::LS * Cfg::ESZ; }
    // nblocks = lines: two CTAs (one cluster) a line
    static cudaError_t launch(const PassParams& p, int64_t nblocks, cudaStream_t st) {
        static bool attr_done = false;
        if (!attr_done) {
            if (smem() > 48 * 1024) {
                cudaError_t e = cudaFuncSetAttribute(k_blue2<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)smem());
                if (e != cudaSuccess) return e;
            }
            attr_done = true;
        }
        if (nblocks <= 0) return cudaSuccess;
        if (nblocks > 0x3fffffffLL) return cudaErrorInvalidConfiguration;
        k_blue2<T, L><<<(unsigned)(2 * nblocks), Cfg::NT, smem(), st>>>(p);
        return cudaGetLastError();
    }
    static LineInfo info() { return LineInfo{&launch, Cfg::NT, 1, smem()}; }
};

}  // namespace

bool blue2_info(int dbl, int L, LineInfo* out) {
    if (!dbl && L == 4096) {
        *out = Blue2Launcher<float, 4096>::info();
        return true;
    }
    return false;
}

}  // namespace rk
