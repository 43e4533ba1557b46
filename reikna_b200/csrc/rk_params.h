// Launch parameter blocks shared by the host planner and the device kernels.
#pragma once
#ifndef __CUDACC_RTC__
#include <stdint.h>
#endif

#include "../../include/reikna_b200.h"

namespace rk {

constexpr int MAXD = RK_MAXD;

// thread mapping of a line pass: position-fastest (lines contiguous along the FFT
// axis) or lane-fastest (adjacent lines are adjacent in memory, strided axis)
enum { MODE_POS = 0, MODE_LANE = 1 };

// value-op flags of one pass side
enum SideFlags : int32_t {
    SF_PRE_CONJ = 1,    // conjugate first
    SF_CHIRP = 2,       // multiply by chirp[a] (Bluestein)
    SF_TAB = 4,         // multiply by tab[a]
    SF_POST_CONJ = 8,   // conjugate after the tables
    SF_SCALE = 16,      // multiply by (scale_re + i scale_im)
    SF_WINDOW = 32,     // Hann window on the axis index (load side)
    SF_NORM = 64,       // |z|^post_param (store side, real output)
    SF_TW4 = 128,       // store side: multiply by W_tw4N^(c * k) (four-step twiddle)
    SF_FAST = 256,      // pass-dtype side, a = j, no axis padding, power-of-two axis
    SF_FAST2 = 512,     // pass-dtype side, a = c cA + j jB, no remap, 32-bit offsets
    SF_FASTR = 1024,    // real side of the pass precision, a = j, no remap, 32-bit offsets
    SF_RPAIR = 2048,    // real load side read as sample pairs: element u = x[2u] + i x[2u+1]
    SF_ADD = 4096,      // add (add_re + i add_im) after the scale (user elements only)
};

// Addressing of one buffer in a pass.  A line l in [0, O*C*I) decomposes as
// o = l / (C*I), c = (l / I) % C, i = l % I; o and i further decompose over the
// outer / inner dims (row-major).  Element j of the line sits on the logical axis
// index a = c*cA + j*jB; it is valid when a < ax_len and the user index
// u = (a + ax_shift) mod ax_len is < ax_bound (likewise for every other dim).
struct Side {
    void* ptr;
    void* ptr2;
    int32_t fmt;
    int32_t nd_o, nd_i;
    int32_t flags;
    int64_t o_shape[MAXD], o_stride[MAXD], o_bound[MAXD];
    int64_t i_shape[MAXD], i_stride[MAXD], i_bound[MAXD];
    int32_t o_shift[MAXD], i_shift[MAXD];
    int64_t ax_len, ax_bound, ax_stride;
    int64_t cA, jB;
    int64_t offset, offset2;
    int32_t ax_shift;
    int32_t win_len;
    double scale_re, scale_im;
    double add_re, add_im;
    double post_param;
    const void* chirp;
    const void* tab;
    const void* win;      // Hann window table (win_len entries, pass precision), or null
    uint64_t user[8];     // words for run-time compiled edge code (RK_FMT_USER)
};

// opaque 128-byte CUtensorMap (encoded on the host with cuTensorMapEncodeTiled)
struct alignas(64) TensorMapBytes {
    uint64_t w[16];
};

enum TmaMode : int32_t { TMA_NONE = 0, TMA_BULK = 1, TMA_TENSOR = 2 };

struct PassParams {
    TensorMapBytes tmap;  // load-side tensor map (TMA_TENSOR)
    int32_t tma_mode;     // TmaMode of the persistent pipelined kernel
    int32_t tma_boxes;    // tensor copies per tile (L split in boxes of <= 256 rows)
    int64_t ntiles;       // tiles of NL lines
    int64_t tile_stride;  // TMA_BULK: elements between consecutive tiles' first lines
    int64_t O, C, I;      // line decomposition
    int64_t nlines;       // O*C*I
    Side ld, st;
    const void* tw;       // stage twiddle tables of the pass length L (TwLayout)
    const void* tw2;      // same for the column length of a plane pass
    const void* tw4_hi;   // W_2^24^(4096 k)
    const void* tw4_lo;   // W_2^24^k
    int64_t tw4_N;        // four-step twiddle modulus (power of two <= 2^24)
    const void* blue_k;   // Bluestein kernel spectrum (fused single-pass kernel)
    int32_t* status;
    // real-signal step of a one-pass real transform, after the FFT of a last pass
    // (var 3) or before the FFT of a first pass (var 4): y[k] A_k + conj(y[mirror k])
    // B_k with A_k = rh (1 - i w_k), B_k = rh (1 + i w_k), w_k = rmix[k], and
    // mirror k = (L - k - rodd) mod L; rnyq: the bin L is also stored (var 3) or
    // read as the mirror of bin 0 (var 4)
    const void* rmix;
    const void* rtwid;  // antiperiodic inverse (variant 4): W_2L^m applied after the FFT
    double rh;
    int32_t rodd, rnyq;
};

// Clustered two-axis pass: axis r (rows, length L1) and the contiguous axis q
// (columns, length L2) of a plane; the plane index o decomposes over outer dims.
struct PlaneSide {
    void* ptr;
    void* ptr2;
    int32_t fmt;
    int32_t nd_o;
    int32_t flags;
    int32_t win_len;
    int64_t o_shape[MAXD], o_stride[MAXD], o_bound[MAXD];
    int32_t o_shift[MAXD];
    int64_t r_len, r_bound, r_stride;
    int64_t q_len, q_bound, q_stride;
    int32_t r_shift, q_shift;
    int64_t offset, offset2;
    double scale_re, scale_im;
    double post_param;
};

struct PlaneParams {
    int64_t nplanes;
    PlaneSide ld, st;
    const void* tw;
    int32_t* status;
};

constexpr int TWN_LOG = 14;           // base twiddle table: W_16384^k
constexpr int TWN = 1 << TWN_LOG;
constexpr int TW4_LOG = 24;           // two-level table for four-step twiddles
constexpr int TW4_HALF = 4096;

}  // namespace rk
