// Launch wrappers for the line-pass kernel instantiations.
#pragma once
#include "rk_internal.h"
#include "rk_kernels.cuh"

namespace rk {

template <typename T, int L, int MODE, int VAR> struct LineLauncher {
    using Cfg = LineCfg<T, L, MODE, (VAR >> 4)>;
    static size_t smem() {
        const bool need = RadixP<T, L, (VAR >> 4)>::NS > 1 || VAR != 0;
        return need ? (size_t)(MODE == MODE_POS ? Cfg::NL * Cfg::LS : Cfg::NL * L) * Cfg::ESZ : 0;
    }
    static constexpr auto kernel() {
        if constexpr (LineMinBlocks<T, L, MODE, VAR>::V == 2)
            return &k_line_2<T, L, MODE, VAR>;
        else if constexpr (LineMinBlocks<T, L, MODE, VAR>::V == 4)
            return &k_line_4<T, L, MODE, VAR>;
        else
            return &k_line<T, L, MODE, VAR>;
    }
    static cudaError_t launch(const PassParams& p, int64_t nblocks, cudaStream_t st) {
        static bool attr_done = false;
        const size_t sm = smem();
        if (!attr_done) {
            if (sm > 48 * 1024) {
                cudaError_t e = cudaFuncSetAttribute(kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
                if (e != cudaSuccess) return e;
            }
            attr_done = true;
        }
        if (nblocks <= 0) return cudaSuccess;
        if (nblocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
        kernel()<<<(unsigned)nblocks, Cfg::NT, sm, st>>>(p);
        return cudaGetLastError();
    }
    static LineInfo info() { return LineInfo{&launch, Cfg::NT, Cfg::NL, smem()}; }
};

}  // namespace rk
