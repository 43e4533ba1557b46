// TMA-fed line passes of the one-pass real transforms: the spectrum step after the
// FFT (variant 3: RFFT, APRFFT) or before it (variant 4: IAPRFFT; IRFFT rows of
// L + 1 bins are not whole tiles and take the plain kernel).
#include "rk_tma.cuh"

namespace rk {

#define RK_TR(TY, LL, VV) \
    if (L == LL && var == VV) { *out = TmaLauncher<TY, LL, MODE_POS, VV>::info(); return true; }

bool tma_info_real(int dbl, int L, int mode, int var, TmaInfo* out) {
    if (mode != MODE_POS) return false;
    if (!dbl) {
        RK_TR(float, 64, 3)
        RK_TR(float, 128, 3)
        RK_TR(float, 256, 3)
        RK_TR(float, 512, 3)
        RK_TR(float, 1024, 3)
        RK_TR(float, 2048, 3)
        RK_TR(float, 4096, 3)
        RK_TR(float, 8192, 3)
        RK_TR(float, 64, 4)
        RK_TR(float, 128, 4)
        RK_TR(float, 256, 4)
        RK_TR(float, 512, 4)
        RK_TR(float, 1024, 4)
        RK_TR(float, 2048, 4)
        RK_TR(float, 4096, 4)
        RK_TR(float, 8192, 4)
    } else {
        RK_TR(double, 64, 3)
        RK_TR(double, 128, 3)
        RK_TR(double, 256, 3)
        RK_TR(double, 512, 3)
        RK_TR(double, 1024, 3)
        RK_TR(double, 2048, 3)
        RK_TR(double, 4096, 3)
        RK_TR(double, 64, 4)
        RK_TR(double, 128, 4)
        RK_TR(double, 256, 4)
        RK_TR(double, 512, 4)
        RK_TR(double, 1024, 4)
        RK_TR(double, 2048, 4)
        RK_TR(double, 4096, 4)
    }
    return false;
}

}  // namespace rk
