// complex128 line-pass instantiations
#include "rk_launch.cuh"

namespace rk {

#define RK_LI(L, MODE, VAR) \
    if (L_ == L && mode == MODE && var == VAR) { *out = LineLauncher<double, L, MODE, VAR>::info(); return true; }

static bool lookup(int L_, int mode, int var, LineInfo* out) {
    RK_LI(1, MODE_POS, 0)
    RK_LI(2, MODE_POS, 0)
    RK_LI(4, MODE_POS, 0)
    RK_LI(8, MODE_POS, 0)
    RK_LI(16, MODE_POS, 0)
    RK_LI(32, MODE_POS, 0)
    RK_LI(64, MODE_POS, 0)
    RK_LI(128, MODE_POS, 0)
    RK_LI(256, MODE_POS, 0)
    RK_LI(512, MODE_POS, 0)
    RK_LI(1024, MODE_POS, 0)
    RK_LI(2048, MODE_POS, 0)
    RK_LI(4096, MODE_POS, 0)
    RK_LI(8192, MODE_POS, 0)
    RK_LI(2, MODE_LANE, 0)
    RK_LI(4, MODE_LANE, 0)
    RK_LI(8, MODE_LANE, 0)
    RK_LI(16, MODE_LANE, 0)
    RK_LI(32, MODE_LANE, 0)
    RK_LI(64, MODE_LANE, 0)
    RK_LI(128, MODE_LANE, 0)
    RK_LI(256, MODE_LANE, 0)
    RK_LI(512, MODE_LANE, 0)
    RK_LI(4, MODE_POS, 1)
    RK_LI(8, MODE_POS, 1)
    RK_LI(16, MODE_POS, 1)
    RK_LI(32, MODE_POS, 1)
    RK_LI(64, MODE_POS, 1)
    RK_LI(128, MODE_POS, 1)
    RK_LI(256, MODE_POS, 1)
    RK_LI(512, MODE_POS, 1)
    RK_LI(1024, MODE_POS, 1)
    RK_LI(2048, MODE_POS, 1)
    RK_LI(4096, MODE_POS, 1)
    RK_LI(8192, MODE_POS, 1)
    RK_LI(4, MODE_LANE, 1)
    RK_LI(8, MODE_LANE, 1)
    RK_LI(16, MODE_LANE, 1)
    RK_LI(32, MODE_LANE, 1)
    RK_LI(64, MODE_LANE, 1)
    RK_LI(128, MODE_LANE, 1)
    RK_LI(256, MODE_LANE, 1)
    RK_LI(512, MODE_LANE, 1)
    RK_LI(2, MODE_POS, 2)
    RK_LI(4, MODE_POS, 2)
    RK_LI(8, MODE_POS, 2)
    RK_LI(16, MODE_POS, 2)
    RK_LI(32, MODE_POS, 2)
    RK_LI(64, MODE_POS, 2)
    RK_LI(128, MODE_POS, 2)
    RK_LI(256, MODE_POS, 2)
    RK_LI(512, MODE_POS, 2)
    RK_LI(8, MODE_POS, 3)
    RK_LI(16, MODE_POS, 3)
    RK_LI(32, MODE_POS, 3)
    RK_LI(64, MODE_POS, 3)
    RK_LI(128, MODE_POS, 3)
    RK_LI(256, MODE_POS, 3)
    RK_LI(512, MODE_POS, 3)
    RK_LI(1024, MODE_POS, 3)
    RK_LI(2048, MODE_POS, 3)
    RK_LI(4096, MODE_POS, 3)
    return false;
}

bool line_info_f64(int L, int mode, int var, LineInfo* out) { return lookup(L, mode, var, out); }

}  // namespace rk
