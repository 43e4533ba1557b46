// Host planner, device tables and C ABI of the FFT library.
//
// The planner follows the structure of reikna's get_fft_kernels
// (reikna/fft/fft.py:532-584): axes are processed innermost first, a power-of-two
// axis becomes a chain of passes, any other length goes through Bluestein's
// algorithm at M = 2 * bounding_power_of_2(N) (reikna/fft/fft.py:551-561).  The pass
// shapes are chosen for sm_100a instead of reikna's local/global split:
//   * one pass per axis when the whole line (or a 128-byte-wide tile of strided
//     lines) fits in one CTA's shared memory,
//   * a two-pass four-step split (N = N1 * N2, twiddle W_N^(n2 k1) fused into the
//     first pass' store) for longer axes (reikna uses radix-128 passes, fft.py:89),
//   * Bluestein fused into a single pass (chirp, forward FFT, kernel spectrum,
//     inverse FFT, chirp) when M fits one CTA, else four passes,
//   * two adjacent axes of a plane fused into one clustered pass that exchanges
//     rows and columns through distributed shared memory (rk_plane.cu).
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "rk_async.cuh"
#include "rk_internal.h"
#include "rk_kernels.cuh"

namespace rk {

constexpr int ilog2_c(int n) { return n <= 1 ? 0 : 1 + ilog2_c(n / 2); }

bool line_info_f32(int L, int mode, int var, LineInfo* out);
bool line_info_f64(int L, int mode, int var, LineInfo* out);

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }

bool line_info(int dbl, int L, int mode, int var, LineInfo* out) {
    if (var == 7) return mode == MODE_POS && blue2_info(dbl, L, out);
    return dbl ? line_info_f64(L, mode, var, out) : line_info_f32(L, mode, var, out);
}

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));               \
            return e_ == cudaErrorMemoryAllocation ? RK_ERR_NOMEM : RK_ERR_CUDA;         \
        }                                                                                \
    } while (0)

// ------------------------------------------------------------------------------
// device tables (FP64 generation)
// ------------------------------------------------------------------------------
// stage table segment: entries [m - 1][j1] = W_Lp^(j1 m), m in [1, R), j1 < J
__global__ void k_gen_stage(float2* f, double2* d, int Lp, int R, int J) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (R - 1) * J) return;
    const int m = e / J + 1, j1 = e % J;
    const int64_t k = ((int64_t)j1 * m) % Lp;
    double s, c;
    sincospi(2.0 * (double)k / (double)Lp, &s, &c);
    if (d) d[e] = make_double2(c, -s);
    if (f) f[e] = make_float2((float)c, (float)-s);
}

struct StageSeg {
    int64_t off;
    int Lp, R, J;
};

template <typename T, int L, int PL = 0> static void stage_segs(std::vector<StageSeg>& segs, int64_t base) {
    using RC = RadixP<T, L, PL>;
    int P = 1;
    for (int s = 0; s + 1 < RC::NS; ++s) {
        const int R = RC::R[s];
        segs.push_back(StageSeg{base + TwLayout<T, L, PL>::offset(s), L / P, R, L / (P * R)});
        P *= R;
    }
}

template <typename T, int L, int LMAX> static void stage_layout(std::vector<StageSeg>& segs, int64_t* offs, int64_t& total) {
    offs[ilog2_c(L)] = total;
    stage_segs<T, L>(segs, total);
    total += TwLayout<T, L>::total();
    if constexpr (L < LMAX) stage_layout<T, 2 * L, LMAX>(segs, offs, total);
}

__global__ void k_gen_tables(float2* hif, float2* lof, double2* hid, double2* lod) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < TW4_HALF) {
        double s, c;
        sincospi(2.0 * (double)k / (double)(1 << TW4_LOG), &s, &c);
        lod[k] = make_double2(c, -s);
        lof[k] = make_float2((float)c, (float)-s);
        sincospi(2.0 * (double)k * TW4_HALF / (double)(1 << TW4_LOG), &s, &c);
        hid[k] = make_double2(c, -s);
        hif[k] = make_float2((float)c, (float)-s);
    }
}

static std::mutex g_tab_mu;
static std::map<int, DeviceTables*> g_tabs;

int device_tables(int device, DeviceTables** out) {
    std::lock_guard<std::mutex> lk(g_tab_mu);
    auto it = g_tabs.find(device);
    if (it != g_tabs.end()) {
        *out = it->second;
        return RK_OK;
    }
    DeviceTables* t = new DeviceTables();
    std::vector<StageSeg> sf, sd;
    int64_t nf = 0, ndd = 0;
    stage_layout<float, 1, 16384>(sf, t->off_f, nf);
    stage_layout<double, 1, 8192>(sd, t->off_d, ndd);
    // the 16-element plan of 8192-point float32 lines, after the others
    t->off_f_r16 = nf;
    stage_segs<float, 8192, 1>(sf, nf);
    nf += TwLayout<float, 8192, 1>::total();
    CK(cudaMalloc(&t->stw_f, std::max<int64_t>(nf, 1) * sizeof(float2)));
    CK(cudaMalloc(&t->stw_d, std::max<int64_t>(ndd, 1) * sizeof(double2)));
    CK(cudaMalloc(&t->tw4hi_f, TW4_HALF * sizeof(float2)));
    CK(cudaMalloc(&t->tw4lo_f, TW4_HALF * sizeof(float2)));
    CK(cudaMalloc(&t->tw4hi_d, TW4_HALF * sizeof(double2)));
    CK(cudaMalloc(&t->tw4lo_d, TW4_HALF * sizeof(double2)));
    // status block: [0] status bits, [1] unused, [2..3] wait limit (SM clock cycles)
    CK(cudaMalloc(&t->status, 4 * sizeof(int32_t)));
    {
        int32_t init[4] = {0, 0, 0, 0};
        const long long lim = RK_WAIT_CYCLES;
        memcpy(init + 2, &lim, sizeof(lim));
        CK(cudaMemcpy(t->status, init, sizeof(init), cudaMemcpyHostToDevice));
    }
    t->bytes = nf * 8 + ndd * 16 + TW4_HALF * 48;
    for (const StageSeg& s : sf) {
        const int n = (s.R - 1) * s.J;
        k_gen_stage<<<(n + 255) / 256, 256>>>((float2*)t->stw_f + s.off, nullptr, s.Lp, s.R, s.J);
    }
    for (const StageSeg& s : sd) {
        const int n = (s.R - 1) * s.J;
        k_gen_stage<<<(n + 255) / 256, 256>>>(nullptr, (double2*)t->stw_d + s.off, s.Lp, s.R, s.J);
    }
    k_gen_tables<<<TW4_HALF / 256, 256>>>((float2*)t->tw4hi_f, (float2*)t->tw4lo_f, (double2*)t->tw4hi_d,
                                           (double2*)t->tw4lo_d);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    g_tabs[device] = t;
    *out = t;
    return RK_OK;
}

// Bluestein tables.  chirp[k] = exp(-i pi (k^2 mod 2N) / N), k < N, with k^2 mod 2N
// in exact 64-bit integers and the exponential in FP64.  b is the even sequence
// conj(chirp) laid out on the padded length M exactly as reikna's get_kweights
// (reikna/fft/fft.py:216-236): b[m] for m in [0, M-N], b[M-m] for m in [1, N-1].
__global__ void k_gen_chirp(int64_t N, int64_t M, float2* cf, double2* cd, double2* b) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M) return;
    const int64_t twoN = 2 * N;
    auto chirp = [&](int64_t m) {
        const int64_t r = (int64_t)(((unsigned __int128)m * (unsigned __int128)m) % (unsigned __int128)twoN);
        double s, c;
        sincospi((double)r / (double)N, &s, &c);
        return make_double2(c, -s);
    };
    if (k < N) {
        double2 c = chirp(k);
        if (cd) cd[k] = c;
        if (cf) cf[k] = make_float2((float)c.x, (float)c.y);
    }
    int64_t m;
    if (k <= M - N)
        m = k;
    else
        m = M - k;
    double2 c = chirp(m);
    b[k] = make_double2(c.x, -c.y);
}

// W^k = exp(-2 pi i k / 2L), k = 0 .. L, for the real-spectrum store (RK_FLAG_REAL_POST)
__global__ void k_gen_rpost(int64_t L, float2* f, double2* d) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k > L) return;
    double s, c;
    sincospi(-(double)k / (double)L, &s, &c);
    if (f) f[k] = make_float2((float)c, (float)s);
    if (d) d[k] = make_double2(c, s);
}

// exp(-i pi (2k + 1) / 2L), k = 0 .. L - 1, for the odd-harmonic step of the
// antiperiodic real transforms (RK_FLAG_ANTIPERIODIC)
__global__ void k_gen_rodd(int64_t L, float2* f, double2* d) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= L) return;
    double s, c;
    sincospi(-(double)(2 * k + 1) / (double)(2 * L), &s, &c);
    if (f) f[k] = make_float2((float)c, (float)s);
    if (d) d[k] = make_double2(c, s);
}

// von Hann window 0.5 (1 - cos(2 pi u / (w - 1))) for u < w and 1 beyond, u < n, in
// FP64, rounded once
__global__ void k_gen_window(int64_t n, int32_t w, float* f, double* d) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const double v = u >= w ? 1.0 : (w > 1 ? 0.5 * (1.0 - cospi(2.0 * (double)u / (double)(w - 1))) : 1.0);
    if (f) f[u] = (float)v;
    if (d) d[u] = v;
}

__global__ void k_scale_convert(const double2* src, int64_t n, double s, float2* df, double2* dd) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double2 v = src[k];
    v.x *= s;
    v.y *= s;
    if (dd) dd[k] = v;
    if (df) df[k] = make_float2((float)v.x, (float)v.y);
}

// ------------------------------------------------------------------------------
// planning
// ------------------------------------------------------------------------------
static bool is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }
static int64_t bpow2(int64_t n) {
    int64_t p = 1;
    while (p < n) p <<= 1;
    return p;
}
static int ilog2(int64_t n) {
    int l = 0;
    while ((int64_t(1) << l) < n) ++l;
    return l;
}
static int lane_max(int dbl) { return dbl ? 512 : 1024; }
static int pos_max(int dbl) { return dbl ? 8192 : 16384; }
static int fmt_is_complex(int f) { return f == RK_FMT_C64 || f == RK_FMT_C128; }
static int fmt_is_pair(int f) { return f == RK_FMT_F32_PAIR || f == RK_FMT_F64_PAIR; }
static int fmt_is_real(int f) { return f == RK_FMT_F32 || f == RK_FMT_F64; }
// arrays a side of this format reads or writes (RK_FMT_CONST / RK_FMT_IGNORE: none)
static int fmt_arrays(int f) {
    return fmt_is_pair(f) ? 2 : (f == RK_FMT_CONST || f == RK_FMT_IGNORE || f == RK_FMT_USER) ? 0 : 1;
}
static bool desc_has_user(const rk_fft_desc& d) {
    return d.input.format == RK_FMT_USER || d.output.format == RK_FMT_USER;
}
// an additive term (or a constant input) that only the general element path applies
static bool edge_has_add(const rk_edge& e) {
    return e.format == RK_FMT_CONST || e.add_slot >= 0 || e.add_re != 0.0 || e.add_im != 0.0;
}

// symbolic buffers while planning
enum SymBuf { SB_IN = 0, SB_OUT = 1, SB_T0 = 2, SB_T1 = 3, SB_M0 = 4, SB_M1 = 5 };

struct SideSpec {
    int buf = SB_IN;
    int64_t ax_len = 0;     // logical axis length seen through this buffer (N or M)
    int64_t cA = 0, jB = 1;
    int32_t flags = 0;
    int chirp_axis = -1;    // Bluestein table owner (axis) for chirp
    bool tab_k = false;     // kernel spectrum table
};

struct PassSpec {
    int kind = PK_LINE;
    int L = 0, mode = MODE_POS, var = 0;  // var: 0 plain, 1 Bluestein, 2 transposed store
    int axis = -1, axis2 = -1;
    int L1 = 0, L2 = 0;
    int64_t O = 1, C = 1, I = 1;
    bool inplace_safe = true;
    int64_t tw4_N = 0;
    int blue_axis = -1;     // fused Bluestein kernel spectrum owner
    bool pair = false;      // with the next pass: one plane-ordered pair launch
    SideSpec ld, st;
    std::string note;
};

struct BlueAxis {
    int axis;
    int64_t N, M;
};

struct Planned {
    std::vector<PassSpec> passes;
    std::vector<BlueAxis> blue;
    bool need_T0 = false, need_T1 = false, need_M = false;
    int64_t m_elems = 0;   // elements of an M-shaped temp
};

static int64_t prod_range(const int64_t* s, int a, int b) {
    int64_t p = 1;
    for (int i = a; i < b; ++i) p *= s[i];
    return p;
}

// A transform of the last axis only, of a real input of the plan's precision, whose
// output keeps at most the bins 0 .. N/2 contiguously (a spectrogram, or
// real_to_complex + crop_frequencies), N/2 a power of two one pass covers: the
// half-length route applies.  Any conjugation or scale of the input is folded into
// the output per call (the input is real, the transform linear).
// Returns the line-pass variant: 6 (bins stored along the line), 5 (a transposed
// output whose lines are adjacent in memory: bins stored lane-fastest), 0 = no.
static int half_eligible(const rk_fft_desc& d, int dbl) {
    if (d.flags & (RK_FLAG_NO_HALF | RK_FLAG_REAL_POST | RK_FLAG_REAL_PRE)) return 0;
    const int nd = d.ndim, ax = nd - 1;
    if (d.naxes != 1 || d.axes[0] != ax) return 0;
    const int64_t n = d.shape[ax];
    if (n % 2) return 0;
    const int64_t L = n / 2;
    if (!is_pow2(L) || L < 8 || L > (dbl ? 4096 : 8192)) return 0;
    const rk_edge& in = d.input;
    const rk_edge& out = d.output;
    const int rfmt = dbl ? RK_FMT_F64 : RK_FMT_F32, cfmt = dbl ? RK_FMT_C128 : RK_FMT_C64;
    if (edge_has_add(in) || edge_has_add(out)) return 0;
    if (in.format != rfmt || in.shape[ax] != n || in.shift[ax] != 0) return 0;
    if (in.window != RK_WIN_NONE && in.window_axis != ax) return 0;
    if (out.shift[ax] != 0 || out.shape[ax] > L + 1) return 0;
    if (!(out.format == cfmt || (out.format == rfmt && out.post == RK_POST_NORM))) return 0;
    if (out.strides[ax] == 1) return 6;
    if (ax > 0 && out.strides[ax - 1] == 1 && d.shape[ax - 1] > 1 && L <= lane_max(dbl)) return 5;
    return 0;
}

static int plan_passes(const rk_fft_desc& d, Planned& P) {
    const int dbl = d.dtype == RK_FMT_C128;
    std::vector<int> axes(d.axes, d.axes + d.naxes);
    std::sort(axes.begin(), axes.end(), std::greater<int>());
    axes.erase(std::remove_if(axes.begin(), axes.end(), [&](int a) { return d.shape[a] == 1; }), axes.end());

    const int nd = d.ndim;
    const int32_t real_flags = d.flags & (RK_FLAG_REAL_POST | RK_FLAG_REAL_PRE);
    if (real_flags == (RK_FLAG_REAL_POST | RK_FLAG_REAL_PRE)) {
        set_error("RK_FLAG_REAL_POST and RK_FLAG_REAL_PRE exclude each other");
        return RK_ERR_INVALID;
    }
    if ((d.flags & RK_FLAG_ANTIPERIODIC) && !real_flags) {
        set_error("RK_FLAG_ANTIPERIODIC needs RK_FLAG_REAL_POST or RK_FLAG_REAL_PRE");
        return RK_ERR_INVALID;
    }
    if (real_flags && (d.naxes != 1 || d.axes[0] != nd - 1 || d.shape[nd - 1] < 8)) {
        set_error("a one-pass real transform needs a transform of the last axis only, of at least 8 points");
        return RK_ERR_UNSUPPORTED;
    }
    if (real_flags && (edge_has_add(d.input) || edge_has_add(d.output) || d.output.format == RK_FMT_IGNORE ||
                       desc_has_user(d))) {
        set_error("a one-pass real transform takes no additive term, constant input or ignored output");
        return RK_ERR_UNSUPPORTED;
    }
    int cur = SB_IN;
    auto array_out = [&](bool inplace_ok) -> int {
        if (inplace_ok && (cur == SB_T0 || cur == SB_T1)) return cur;
        return cur == SB_T0 ? SB_T1 : SB_T0;
    };

    if (axes.empty()) {
        // trivial problem: transformations still run (reikna/fft/fft.py:647-662).  One
        // element per line: the last dim is the co-index c (a = c), L = 1.
        PassSpec p;
        p.L = 1;
        p.axis = nd - 1;
        p.O = prod_range(d.shape, 0, nd - 1);
        p.C = d.shape[nd - 1];
        p.I = 1;
        p.ld.buf = SB_IN;
        p.st.buf = SB_OUT;
        p.ld.ax_len = p.st.ax_len = d.shape[nd - 1];
        p.ld.cA = p.st.cA = 1;
        p.ld.jB = p.st.jB = 0;
        p.note = "copy";
        P.passes.push_back(p);
        return RK_OK;
    }

    if (const int hv = half_eligible(d, dbl)) {
        // a real signal along the last axis whose output keeps at most the bins
        // 0 .. N/2: one pass of the half-length FFT over the sample pairs
        // x[2u] + i x[2u+1], with the real-spectrum step in its store (the RFFT of
        // examples/demo_specialized_fft.py:175-241, chosen by the planner)
        const int ax = nd - 1;
        PassSpec p;
        p.L = (int)(d.shape[ax] / 2);
        p.mode = MODE_POS;
        p.var = hv;
        p.axis = ax;
        p.O = prod_range(d.shape, 0, ax);
        p.ld.buf = SB_IN; p.ld.ax_len = p.L; p.ld.cA = 0; p.ld.jB = 1; p.ld.flags = SF_RPAIR;
        p.st.buf = SB_OUT; p.st.ax_len = p.L; p.st.cA = 0; p.st.jB = 1;
        p.note = "half";
        P.passes.push_back(p);
        return RK_OK;
    }

    const int LM = lane_max(dbl), PM = pos_max(dbl);
    // the two innermost dims, both transformed powers of two: one clustered pass, or
    // (RK_FLAG_PAIR) a row pass and a column pass run as one plane-ordered launch
    PairInfo pair_probe;
    // (an edge read or written by run-time compiled code takes line passes only)
    const bool want_pair = !desc_has_user(d) && (d.flags & RK_FLAG_PAIR) && nd >= 2 && axes.size() >= 2 &&
                           axes[0] == nd - 1 &&
                           axes[1] == nd - 2 && is_pow2(d.shape[nd - 1]) && is_pow2(d.shape[nd - 2]) &&
                           pair_info(dbl, (int)d.shape[nd - 1], (int)d.shape[nd - 2], &pair_probe);
    const size_t pair_at = P.passes.size();
    if (!want_pair && !(d.flags & (RK_FLAG_NO_PLANE | RK_FLAG_BATCHABLE)) && !desc_has_user(d) && nd >= 2 &&
        axes.size() >= 2 &&
        axes[0] == nd - 1 && axes[1] == nd - 2 &&
        is_pow2(d.shape[nd - 1]) && is_pow2(d.shape[nd - 2])) {
        PlaneInfo pi;
        if (plane_info(dbl, (int)d.shape[nd - 2], (int)d.shape[nd - 1], (d.flags & RK_FLAG_PLANE_WIDE) ? 1 : 0, &pi)) {
            PassSpec p;
            p.kind = PK_PLANE;
            p.L1 = (int)d.shape[nd - 2];
            p.L2 = (int)d.shape[nd - 1];
            p.L = p.L2;
            p.axis = nd - 1;
            p.axis2 = nd - 2;
            p.O = prod_range(d.shape, 0, nd - 2);
            p.ld.buf = cur; p.ld.ax_len = p.L2; p.ld.cA = 0; p.ld.jB = 1;
            const bool last = axes.size() == 2;
            const int out = last ? SB_OUT : array_out(true);
            p.st.buf = out; p.st.ax_len = p.L1; p.st.cA = 0; p.st.jB = 1;
            p.note = "plane";
            P.passes.push_back(p);
            cur = out;
            axes.erase(axes.begin(), axes.begin() + 2);
        }
    }
    for (size_t ai = 0; ai < axes.size(); ++ai) {
        const int ax = axes[ai];
        const int64_t n = d.shape[ax];
        const int64_t O = prod_range(d.shape, 0, ax);
        const int64_t I = prod_range(d.shape, ax + 1, nd);
        const bool last_axis = ai + 1 == axes.size();
        if (n > (int64_t(1) << 30)) {
            set_error("axis length too large");
            return RK_ERR_UNSUPPORTED;
        }
        if (is_pow2(n)) {
            if ((I == 1 && n <= PM) || (I > 1 && n <= LM)) {
                PassSpec p;
                p.L = (int)n;
                p.mode = I == 1 ? MODE_POS : MODE_LANE;
                // a last pass whose output lines are adjacent in memory while the
                // axis is strided (a transposed output edge) stores lane-fastest
                // through shared memory
                if (I == 1 && last_axis && ax > 0 && n <= LM && d.output.strides[ax] != 1 &&
                    d.output.strides[ax - 1] == 1 && d.shape[ax - 1] > 1)
                    p.var = 2;
                // the real-signal spectrum step fused into the store (RK_FLAG_REAL_POST)
                // or into the load (RK_FLAG_REAL_PRE)
                if (real_flags && I == 1 && last_axis && n >= 8 && n <= (dbl ? 4096 : 8192))
                    p.var = (d.flags & RK_FLAG_REAL_POST) ? 3 : 4;
                p.axis = ax;
                p.O = O; p.C = 1; p.I = I;
                p.ld.buf = cur; p.ld.ax_len = n; p.ld.cA = 0; p.ld.jB = 1;
                const int out = last_axis ? SB_OUT : array_out(true);
                p.st.buf = out; p.st.ax_len = n; p.st.cA = 0; p.st.jB = 1;
                p.note = "single";
                P.passes.push_back(p);
                cur = out;
            } else {
                // four-step n = N1 * N2: pass A over n1 (stride N2*I), pass B over n2
                int64_t N1, N2;
                if (I == 1) {
                    N2 = std::min<int64_t>(256, n / 2);
                    N1 = n / N2;
                    if (N1 > LM) { N1 = LM; N2 = n / N1; }
                    if (N2 > PM) {
                        set_error("1-D length beyond two-pass range");
                        return RK_ERR_UNSUPPORTED;
                    }
                } else {
                    const int l = ilog2(n);
                    N1 = int64_t(1) << (l / 2);
                    N2 = n / N1;
                    if (N1 > LM || N2 > LM) {
                        set_error("strided axis length beyond two-pass range");
                        return RK_ERR_UNSUPPORTED;
                    }
                }
                PassSpec a;
                a.L = (int)N1; a.mode = MODE_LANE; a.axis = ax;
                a.O = O; a.C = N2; a.I = I;
                a.ld.buf = cur; a.ld.ax_len = n; a.ld.cA = 1; a.ld.jB = N2;
                const int mid = array_out(true);
                a.st.buf = mid; a.st.ax_len = n; a.st.cA = 1; a.st.jB = N2;
                a.st.flags |= SF_TW4; a.tw4_N = n;
                a.note = "fourstep-A";
                P.passes.push_back(a);
                cur = mid;
                PassSpec b;
                b.L = (int)N2; b.axis = ax;
                b.O = O; b.C = N1; b.I = I;
                b.mode = I == 1 ? MODE_POS : MODE_LANE;
                b.var = (I == 1 && N2 <= LM) ? 2 : 0;
                b.inplace_safe = false;
                b.ld.buf = cur; b.ld.ax_len = n; b.ld.cA = N2; b.ld.jB = 1;
                const int out = last_axis ? SB_OUT : array_out(false);
                b.st.buf = out; b.st.ax_len = n; b.st.cA = 1; b.st.jB = N1;
                b.note = "fourstep-B";
                P.passes.push_back(b);
                cur = out;
            }
        } else {
            const int64_t M = 2 * bpow2(n);
            P.blue.push_back(BlueAxis{ax, n, M});
            // a strided (lane-mode) fused Bluestein line holds up to 2048 complex64
            // points (four adjacent lines a CTA): one pass instead of four
            const int64_t blue_lane_max = (dbl || (d.flags & RK_FLAG_BATCHABLE)) ? LM : 2048;
            if ((I == 1 && M <= PM) || (I > 1 && M <= blue_lane_max)) {
                PassSpec p;
                p.L = (int)M; p.var = 1; p.blue_axis = ax;
                p.mode = I == 1 ? MODE_POS : MODE_LANE;
                // RK_FLAG_R16: 8192-point float32 lines on the 16-element plan with 512
                // threads (variant bit 16) instead of 32 elements on 256 threads
                if (!dbl && M == 8192 && I == 1 && (d.flags & RK_FLAG_R16)) p.var = 1 + 16;
                // RK_FLAG_BLUE_PAIR: 8192-point float32 lines on a two-CTA cluster
                // (variant 7, L = M/2 a CTA); not for the persistent batch kernel or
                // user edge code
                const bool pair2 = !dbl && M == 8192 && I == 1 && p.var == 1 && (d.flags & RK_FLAG_BLUE_PAIR) &&
                                   !(d.flags & RK_FLAG_BATCHABLE) && !desc_has_user(d);
                if (pair2) {
                    p.L = (int)(M / 2);
                    p.var = 7;
                }
                p.axis = ax;
                p.O = O; p.C = 1; p.I = I;
                p.ld.buf = cur; p.ld.ax_len = n; p.ld.cA = 0; p.ld.jB = 1;
                p.ld.flags = SF_CHIRP; p.ld.chirp_axis = ax;
                const int out = last_axis ? SB_OUT : array_out(true);
                p.st.buf = out; p.st.ax_len = n; p.st.cA = 0; p.st.jB = 1;
                p.st.flags = SF_PRE_CONJ | SF_CHIRP; p.st.chirp_axis = ax;
                p.note = pair2 ? "bluestein-pair" : "bluestein-fused";
                P.passes.push_back(p);
                cur = out;
            } else {
                int64_t N1, N2;
                if (I == 1) {
                    N2 = std::min<int64_t>(256, M / 2);
                    N1 = M / N2;
                    if (N1 > LM) { N1 = LM; N2 = M / N1; }
                    if (N2 > PM) {
                        set_error("Bluestein length beyond two-pass range");
                        return RK_ERR_UNSUPPORTED;
                    }
                } else {
                    const int l = ilog2(M);
                    N1 = int64_t(1) << (l / 2);
                    N2 = M / N1;
                    if (N1 > LM || N2 > LM) {
                        set_error("strided Bluestein length beyond two-pass range");
                        return RK_ERR_UNSUPPORTED;
                    }
                }
                P.need_M = true;
                P.m_elems = std::max<int64_t>(P.m_elems, O * M * I);
                // forward FFT_M of chirp * x
                PassSpec p1;
                p1.L = (int)N1; p1.mode = MODE_LANE; p1.axis = ax; p1.O = O; p1.C = N2; p1.I = I;
                p1.ld.buf = cur; p1.ld.ax_len = n; p1.ld.cA = 1; p1.ld.jB = N2;
                p1.ld.flags = SF_CHIRP; p1.ld.chirp_axis = ax;
                p1.st.buf = SB_M0; p1.st.ax_len = M; p1.st.cA = 1; p1.st.jB = N2;
                p1.st.flags = SF_TW4; p1.tw4_N = M;
                p1.note = "bluestein-A1";
                PassSpec p2;
                p2.L = (int)N2; p2.axis = ax; p2.O = O; p2.C = N1; p2.I = I;
                p2.mode = I == 1 ? MODE_POS : MODE_LANE;
                p2.var = (I == 1 && N2 <= LM) ? 2 : 0;
                p2.inplace_safe = false;
                p2.ld.buf = SB_M0; p2.ld.ax_len = M; p2.ld.cA = N2; p2.ld.jB = 1;
                p2.st.buf = SB_M1; p2.st.ax_len = M; p2.st.cA = 1; p2.st.jB = N1;
                p2.note = "bluestein-B1";
                // inverse FFT_M of (spectrum * K) via conjugation
                PassSpec p3 = p1;
                p3.ld = SideSpec();
                p3.ld.buf = SB_M1; p3.ld.ax_len = M; p3.ld.cA = 1; p3.ld.jB = N2;
                p3.ld.flags = SF_TAB | SF_POST_CONJ; p3.ld.tab_k = true; p3.ld.chirp_axis = ax;
                p3.st.buf = SB_M0;
                p3.note = "bluestein-A2";
                PassSpec p4 = p2;
                p4.ld.buf = SB_M0;
                const int out = last_axis ? SB_OUT : array_out(true);
                p4.st = SideSpec();
                p4.st.buf = out; p4.st.ax_len = n; p4.st.cA = 1; p4.st.jB = N1;
                p4.st.flags = SF_PRE_CONJ | SF_CHIRP; p4.st.chirp_axis = ax;
                p4.note = "bluestein-B2";
                P.passes.push_back(p1);
                P.passes.push_back(p2);
                P.passes.push_back(p3);
                P.passes.push_back(p4);
                cur = out;
            }
        }
    }
    if (real_flags) {
        const int ax = nd - 1;
        const bool ap = d.flags & RK_FLAG_ANTIPERIODIC;
        const bool post = d.flags & RK_FLAG_REAL_POST;
        const rk_edge& spec = post ? d.output : d.input;  // the edge holding the real signal's bins
        const int64_t L = d.shape[ax];
        const bool bins_ok = ap ? spec.shape[ax] == L
                                : (post ? (spec.shape[ax] == L || spec.shape[ax] == L + 1) : spec.shape[ax] == L + 1);
        if (P.passes.size() != 1 || P.passes[0].var != (post ? 3 : 4) || spec.strides[ax] != 1 || !bins_ok ||
            spec.shift[ax] != 0 || (!post && d.output.shape[ax] != L)) {
            set_error(post ? "RK_FLAG_REAL_POST needs a one-pass transform of the last axis (a power of two of 8 to "
                             "8192 points, 4096 for complex128) with a contiguous output of L or L + 1 bins (L with "
                             "RK_FLAG_ANTIPERIODIC)"
                           : "RK_FLAG_REAL_PRE needs a one-pass transform of the last axis (a power of two of 8 to "
                             "8192 points, 4096 for complex128) with a contiguous input of L + 1 bins (L with "
                             "RK_FLAG_ANTIPERIODIC) and an output of L pairs");
            return RK_ERR_UNSUPPORTED;
        }
    }
    if (want_pair && P.passes.size() >= pair_at + 2) {
        PassSpec& pa = P.passes[pair_at];
        const PassSpec& pb = P.passes[pair_at + 1];
        if (pa.note == "single" && pb.note == "single" && pa.mode == MODE_POS && pb.mode == MODE_LANE &&
            pa.axis == nd - 1 && pb.axis == nd - 2 && pb.I == d.shape[nd - 1]) {
            pa.pair = true;
            pa.note = "pair-rows";
            P.passes[pair_at + 1].note = "pair-cols";
        }
    }
    for (auto& p : P.passes) {
        for (int b : {p.ld.buf, p.st.buf}) {
            if (b == SB_T0) P.need_T0 = true;
            if (b == SB_T1) P.need_T1 = true;
        }
    }
    return RK_OK;
}

// ------------------------------------------------------------------------------
// side construction
// ------------------------------------------------------------------------------
struct DimList {
    int n = 0;
    int64_t shape[MAXD], stride[MAXD], bound[MAXD];
    int32_t shift[MAXD];
    void push(int64_t sh, int64_t st, int64_t bd, int32_t sf) {
        if (sh == 1) return;  // index is always 0
        shape[n] = sh; stride[n] = st; bound[n] = bd; shift[n] = sf;
        ++n;
    }
    void merge() {
        // merge adjacent dims (row-major, last fastest) that form one contiguous range
        int w = 0;
        for (int i = 0; i < n; ++i) {
            if (w > 0) {
                int j = w - 1;
                if (shift[j] == 0 && shift[i] == 0 && bound[j] == shape[j] && bound[i] == shape[i] &&
                    stride[j] == stride[i] * shape[i]) {
                    shape[j] *= shape[i];
                    bound[j] = shape[j];
                    stride[j] = stride[i];
                    continue;
                }
            }
            shape[w] = shape[i]; stride[w] = stride[i]; bound[w] = bound[i]; shift[w] = shift[i];
            ++w;
        }
        n = w;
    }
};

// Build the Side for buffer `buf` of a pass over axis `ax` of the FFT array.
static void build_side(const rk_fft_desc& d, const SideSpec& ss, int ax, int dbl, bool is_load, Side& s) {
    memset(&s, 0, sizeof(s));
    const int nd = d.ndim;
    const rk_edge* e = nullptr;
    if (ss.buf == SB_IN) e = &d.input;
    if (ss.buf == SB_OUT) e = &d.output;
    int64_t shape[MAXD], stride[MAXD], bound[MAXD];
    int32_t shift[MAXD];
    for (int i = 0; i < nd; ++i) shape[i] = d.shape[i];
    if (e) {
        for (int i = 0; i < nd; ++i) {
            stride[i] = e->strides[i];
            bound[i] = std::min<int64_t>(e->shape[i], d.shape[i]);
            shift[i] = e->shift[i];
        }
        s.fmt = e->format;
        s.offset = e->offset;
        s.offset2 = e->offset2;
    } else {
        // contiguous complex temp; the transformed axis may have the padded length
        int64_t st = 1;
        for (int i = nd - 1; i >= 0; --i) {
            const int64_t len = (i == ax) ? ss.ax_len : shape[i];
            stride[i] = st;
            st *= len;
            bound[i] = len;
            shift[i] = 0;
        }
        s.fmt = dbl ? RK_FMT_C128 : RK_FMT_C64;
    }
    DimList o, in;
    for (int i = 0; i < ax; ++i) o.push(shape[i], stride[i], bound[i], shift[i]);
    for (int i = ax + 1; i < nd; ++i) in.push(shape[i], stride[i], bound[i], shift[i]);
    o.merge();
    in.merge();
    s.nd_o = o.n;
    s.nd_i = in.n;
    for (int i = 0; i < o.n; ++i) {
        s.o_shape[i] = o.shape[i]; s.o_stride[i] = o.stride[i]; s.o_bound[i] = o.bound[i]; s.o_shift[i] = o.shift[i];
    }
    for (int i = 0; i < in.n; ++i) {
        s.i_shape[i] = in.shape[i]; s.i_stride[i] = in.stride[i]; s.i_bound[i] = in.bound[i]; s.i_shift[i] = in.shift[i];
    }
    s.ax_len = ss.ax_len;
    s.ax_bound = e ? std::min<int64_t>(bound[ax], ss.ax_len) : ss.ax_len;
    s.ax_stride = stride[ax];
    s.ax_shift = e ? shift[ax] : 0;
    s.cA = ss.cA;
    s.jB = ss.jB;
    s.flags = ss.flags;
    s.scale_re = 1.0;
    s.scale_im = 0.0;
    if (e) {
        if (edge_has_add(*e)) s.flags |= SF_ADD;  // value set per call
        if (is_load && e->window != RK_WIN_NONE && e->window_axis == ax) {
            s.flags |= SF_WINDOW;
            s.win_len = (int32_t)e->window_len;
        }
        if (!is_load && e->post == RK_POST_NORM) {
            s.flags |= SF_NORM;
            s.post_param = e->post_param;
        }
    }
}

// Mark a side for the lean block load/store path (load_block / store_block).
static void mark_fast(Side& s, int dbl, int L) {
    const int fmt = dbl ? RK_FMT_C128 : RK_FMT_C64;
    const int32_t bad = SF_CHIRP | SF_TAB | SF_WINDOW | SF_NORM | SF_TW4 | SF_ADD;
    if (s.fmt == fmt && s.cA == 0 && s.jB == 1 && s.ax_len == L && s.ax_bound == s.ax_len && is_pow2(L) &&
        !(s.flags & bad) && s.ax_stride >= 0 && s.ax_stride * (int64_t)L < (int64_t(1) << 31))
        s.flags |= SF_FAST;
}

// Switch a plain line pass to the persistent TMA-fed kernel when its load side is a
// whole-tile, 16-byte aligned layout (see rk_tma.cu).  Tensor maps over plan
// temporaries are encoded here; over the user's input they are encoded per call.
static void setup_tma(PassRec& r, int dbl, int nsm) {
    PassParams& p = r.prm;
    const Side& ld = p.ld;
    const Side& st = p.st;
    const int esz = dbl ? 16 : 8;
    if (!(ld.flags & SF_FAST) || !(st.flags & SF_FAST) || ld.ax_shift != 0 || p.C != 1) return;
    TmaInfo ti;
    if (!tma_info(dbl, r.L, r.mode, &ti)) return;
    const int64_t L = r.L, NL = ti.nl;
    for (int i = 0; i < ld.nd_o; ++i)
        if (ld.o_shift[i] != 0 || ld.o_bound[i] != ld.o_shape[i]) return;
    if (r.mode == MODE_POS) {
        if (p.I != 1 || ld.nd_i != 0 || ld.ax_stride != 1 || ld.nd_o > 1) return;
        if (ld.nd_o == 1 && ld.o_stride[0] != L) return;
        if ((ld.offset * esz) % 16 != 0 || (L * esz) % 16 != 0) return;
        p.tma_mode = TMA_BULK;
        p.tile_stride = NL * L;
    } else {
        if (p.I % NL != 0 || ld.nd_i != 1 || ld.i_stride[0] != 1 || ld.i_shape[0] != p.I || ld.i_shift[0] != 0 ||
            ld.i_bound[0] != p.I || ld.nd_o > 1)
            return;
        // (a broadcast input has zero strides: plain loads read it)
        if (ld.ax_stride <= 0 || (ld.ax_stride * esz) % 16 != 0) return;
        if (ld.nd_o == 1 && (ld.o_stride[0] <= 0 || (ld.o_stride[0] * esz) % 16 != 0)) return;
        if (ld.offset != 0) return;
        p.tma_mode = TMA_TENSOR;
        p.tma_boxes = (int)std::max<int64_t>(1, L / 256);
        r.tma_rows = (int)(L / p.tma_boxes);
        if (ld.ptr) {
            const int64_t so = ld.nd_o == 1 ? ld.o_stride[0] : L * p.I;
            if (!encode_lane_map(ld.ptr, dbl, p.I, L, p.O, ld.ax_stride, so, (int)NL, r.tma_rows, &p.tmap)) {
                p.tma_mode = TMA_NONE;
                return;
            }
            r.tma_ptr = ld.ptr;
        } else {
            r.tma_reencode = true;
        }
    }
    p.ntiles = (p.nlines + NL - 1) / NL;
    const int per = std::max(1, ti.per_sm());
    r.nblocks = std::min<int64_t>(p.ntiles, (int64_t)nsm * per);
    r.ti = ti;
    r.use_tma = true;
}

// Sides that cannot take SF_FAST but are still the pass dtype without an index remap
// (four-step index maps, Bluestein padding, chirp / table ops) take SF_FAST2.
static void mark_fast2(Side& s, int dbl, int64_t L, int64_t C) {
    if (s.flags & SF_FAST) return;
    const int fmt = dbl ? RK_FMT_C128 : RK_FMT_C64;
    if (s.fmt != fmt || s.ax_shift != 0 || (s.flags & (SF_WINDOW | SF_NORM | SF_ADD))) return;
    if (s.cA < 0 || s.jB < 0 || s.ax_stride < 0) return;
    const int64_t amax = (C - 1) * s.cA + (L - 1) * s.jB;
    const int64_t lim = int64_t(1) << 31;
    if (amax >= lim || s.ax_len >= lim || amax * std::max<int64_t>(s.ax_stride, 1) >= lim) return;
    s.flags |= SF_FAST2;
}

// Real sides of the pass precision with the plain index map a = j (signal frames in,
// magnitudes or real parts out) take SF_FASTR; a windowed load needs the plan's
// window table.
static void mark_fastr(Side& s, int dbl, int64_t L, bool load) {
    if (s.flags & (SF_FAST | SF_FAST2)) return;
    const int fmt = dbl ? RK_FMT_F64 : RK_FMT_F32;
    if (s.fmt != fmt || s.cA != 0 || s.jB != 1 || s.ax_shift != 0 || s.ax_stride < 0 || s.ax_len != L) return;
    const int64_t span = (s.flags & SF_RPAIR) ? 2 * L : L;  // samples along the axis
    if ((span - 1) * std::max<int64_t>(s.ax_stride, 1) >= (int64_t(1) << 31)) return;
    const int32_t conj = SF_PRE_CONJ | SF_POST_CONJ | SF_SCALE;
    if (load) {
        if (s.ax_bound != s.ax_len || (s.flags & ~(conj | SF_WINDOW | SF_RPAIR))) return;
        // the window table covers every position (pair-read sides: padded to 2L)
        if ((s.flags & SF_WINDOW) && (!s.win || (!(s.flags & SF_RPAIR) && s.win_len < L))) return;
    } else {
        if (s.ax_bound > s.ax_len || (s.flags & ~(conj | SF_NORM))) return;
    }
    s.flags |= SF_FASTR;
}

static int validate(const rk_fft_desc* d) {
    if (!d) { set_error("null descriptor"); return RK_ERR_INVALID; }
    if (d->dtype != RK_FMT_C64 && d->dtype != RK_FMT_C128) {
        set_error("FFT computation requires array of a complex dtype");
        return RK_ERR_INVALID;
    }
    if (d->ndim < 1 || d->ndim > RK_MAXD) { set_error("ndim out of range"); return RK_ERR_INVALID; }
    for (int i = 0; i < d->ndim; ++i)
        if (d->shape[i] < 1) { set_error("shape entries must be positive"); return RK_ERR_INVALID; }
    if (d->naxes < 0 || d->naxes > d->ndim) { set_error("bad number of axes"); return RK_ERR_INVALID; }
    bool seen[RK_MAXD] = {false};
    for (int i = 0; i < d->naxes; ++i) {
        int a = d->axes[i];
        if (a < 0 || a >= d->ndim) { set_error("axis out of range"); return RK_ERR_INVALID; }
        if (seen[a]) { set_error("repeated axis"); return RK_ERR_INVALID; }
        seen[a] = true;
    }
    for (const rk_edge* e : {&d->input, &d->output}) {
        if (e->ndim != d->ndim) { set_error("edge ndim must equal FFT ndim"); return RK_ERR_INVALID; }
        for (int i = 0; i < d->ndim; ++i) {
            if (e->shape[i] < 1) { set_error("edge shape entries must be positive"); return RK_ERR_INVALID; }
            if (e->shift[i] < 0 || e->shift[i] >= d->shape[i]) {
                set_error("edge shift out of range");
                return RK_ERR_INVALID;
            }
        }
        const bool special = (e == &d->input && e->format == RK_FMT_CONST) ||
                             (e == &d->output && e->format == RK_FMT_IGNORE) || e->format == RK_FMT_USER;
        if (!(fmt_is_complex(e->format) || fmt_is_real(e->format) || fmt_is_pair(e->format) || special)) {
            set_error("unsupported edge format");
            return RK_ERR_INVALID;
        }
        if (e->add_slot < -1 || e->post_slot < -1 || e->scale_slot < -1 || e->scale_div_slot < -1) {
            set_error("scalar slots are -1 (none) or a slot index");
            return RK_ERR_INVALID;
        }
    }
    if (d->input.post_slot >= 0) {
        set_error("a norm order slot belongs to the output edge");
        return RK_ERR_INVALID;
    }
    if (fmt_is_real(d->output.format) && d->output.post != RK_POST_NORM) {
        set_error("real output requires a norm post-operation");
        return RK_ERR_INVALID;
    }
    if (d->output.post == RK_POST_NORM && !fmt_is_real(d->output.format)) {
        set_error("norm post-operation requires a real output format");
        return RK_ERR_INVALID;
    }
    return RK_OK;
}

static const char* mode_name(int m) { return m == MODE_POS ? "pos" : "lane"; }
static const char* buf_name(int b) {
    switch (b) {
        case SB_IN: return "input";
        case SB_OUT: return "output";
        case SB_T0: return "temp0";
        case SB_T1: return "temp1";
        case SB_M0: return "tempM0";
        case SB_M1: return "tempM1";
    }
    return "?";
}

static std::string describe_json(const rk_fft_desc& d, const Planned& P) {
    std::ostringstream os;
    os << "{\"passes\": [";
    for (size_t i = 0; i < P.passes.size(); ++i) {
        const PassSpec& p = P.passes[i];
        if (i) os << ", ";
        os << "{\"kind\": \"" << (p.kind == PK_PLANE ? "plane" : "line") << "\", \"note\": \"" << p.note
           << "\", \"axis\": " << p.axis << ", \"axis2\": " << p.axis2 << ", \"L\": " << p.L << ", \"L1\": " << p.L1
           << ", \"L2\": " << p.L2 << ", \"mode\": \"" << mode_name(p.mode) << "\", \"var\": " << p.var
           << ", \"O\": " << p.O << ", \"C\": " << p.C << ", \"I\": " << p.I << ", \"in\": \"" << buf_name(p.ld.buf)
           << "\", \"out\": \"" << buf_name(p.st.buf) << "\"}";
    }
    os << "], \"bluestein\": [";
    for (size_t i = 0; i < P.blue.size(); ++i) {
        if (i) os << ", ";
        os << "{\"axis\": " << P.blue[i].axis << ", \"N\": " << P.blue[i].N << ", \"M\": " << P.blue[i].M << "}";
    }
    os << "], \"temps\": {\"T0\": " << (P.need_T0 ? 1 : 0) << ", \"T1\": " << (P.need_T1 ? 1 : 0)
       << ", \"M_elems\": " << P.m_elems << "}, \"dtype\": \"" << (d.dtype == RK_FMT_C128 ? "complex128" : "complex64")
       << "\"}";
    return os.str();
}

static int64_t edge_extent_bytes(const rk_edge& e, int second) {
    if (!fmt_arrays(e.format)) return 0;
    int esz = 8;
    switch (e.format) {
        case RK_FMT_C64: esz = 8; break;
        case RK_FMT_C128: esz = 16; break;
        case RK_FMT_F32: case RK_FMT_F32_PAIR: esz = 4; break;
        case RK_FMT_F64: case RK_FMT_F64_PAIR: esz = 8; break;
    }
    const int64_t* st = second ? e.strides2 : e.strides;
    int64_t hi = second ? e.offset2 : e.offset, lo = hi;
    for (int i = 0; i < e.ndim; ++i) {
        const int64_t span = (e.shape[i] - 1) * st[i];
        if (span > 0) hi += span; else lo += span;
    }
    return (hi + 1) * esz;
}

}  // namespace rk

using namespace rk;

// ------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------
extern "C" {

const char* rk_last_error(void) { return g_err.c_str(); }
const char* rk_version(void) { return "reikna_b200 0.1.0 (sm_100a)"; }

int rk_device_status(int32_t* status, int32_t clear) {
    if (!status) {
        set_error("null argument");
        return RK_ERR_INVALID;
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    DeviceTables* t = nullptr;
    int rc = device_tables(dev, &t);
    if (rc) return rc;
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(status, t->status, sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (clear) CK(cudaMemset(t->status, 0, sizeof(int32_t)));
    return RK_OK;
}

int rk_set_wait_limit(int64_t cycles) {
    if (cycles < 1000) {
        set_error("rk_set_wait_limit: the limit must be at least 1000 SM clock cycles");
        return RK_ERR_INVALID;
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    DeviceTables* t = nullptr;
    int rc = device_tables(dev, &t);
    if (rc) return rc;
    const long long lim = cycles;
    CK(cudaMemcpy(t->status + 2, &lim, sizeof(lim), cudaMemcpyHostToDevice));
    return RK_OK;
}

int rk_get_wait_limit(int64_t* cycles) {
    if (!cycles) {
        set_error("null argument");
        return RK_ERR_INVALID;
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    DeviceTables* t = nullptr;
    int rc = device_tables(dev, &t);
    if (rc) return rc;
    long long lim = 0;
    CK(cudaMemcpy(&lim, t->status + 2, sizeof(lim), cudaMemcpyDeviceToHost));
    *cycles = lim;
    return RK_OK;
}

int rk_stream_check(void* stream) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    DeviceTables* t = nullptr;
    int rc = device_tables(dev, &t);
    if (rc) return rc;
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    int32_t v = 0;
    CK(cudaMemcpy(&v, t->status, sizeof(v), cudaMemcpyDeviceToHost));
    if (v) {
        set_error("device status word " + std::to_string(v) +
                  ((v & RK_STATUS_TIMEOUT) ? " (a bounded wait ran out)" : "") +
                  ((v & RK_STATUS_BAD_VARIANT) ? " (a batched task had no tile body)" : ""));
        return RK_ERR_DEVICE;
    }
    return RK_OK;
}

int rk_abi_sizes(int64_t* edge_bytes, int64_t* desc_bytes) {
    if (!edge_bytes || !desc_bytes) {
        set_error("null argument");
        return RK_ERR_INVALID;
    }
    *edge_bytes = (int64_t)sizeof(rk_edge);
    *desc_bytes = (int64_t)sizeof(rk_fft_desc);
    return RK_OK;
}

int rk_edge_init(rk_edge* e, int32_t format, int32_t ndim, const int64_t* shape) {
    if (!e || ndim < 1 || ndim > RK_MAXD || !shape) {
        set_error("rk_edge_init: bad arguments");
        return RK_ERR_INVALID;
    }
    memset(e, 0, sizeof(*e));
    e->format = format;
    e->ndim = ndim;
    int64_t st = 1;
    for (int i = ndim - 1; i >= 0; --i) {
        e->shape[i] = shape[i];
        e->strides[i] = st;
        e->strides2[i] = st;
        st *= shape[i];
    }
    e->scale_re = 1.0;
    e->scale_im = 0.0;
    e->scale_slot = -1;
    e->scale_div_slot = -1;
    e->post = RK_POST_NONE;
    e->post_param = 2.0;
    e->window = RK_WIN_NONE;
    e->add_slot = -1;
    e->add_re = 0.0;
    e->add_im = 0.0;
    e->post_slot = -1;
    return RK_OK;
}

int rk_fft_plan_describe(const rk_fft_desc* desc, char* buf, int64_t cap, int64_t* needed) {
    int rc = validate(desc);
    if (rc) return rc;
    Planned P;
    rc = plan_passes(*desc, P);
    if (rc) return rc;
    std::string js = describe_json(*desc, P);
    if (needed) *needed = (int64_t)js.size() + 1;
    if (buf && cap > 0) {
        const int64_t n = std::min<int64_t>(cap - 1, (int64_t)js.size());
        memcpy(buf, js.data(), n);
        buf[n] = 0;
    }
    return RK_OK;
}

int rk_fft_plan_create(const rk_fft_desc* desc, rk_fft_plan** out) {
    if (!out) { set_error("null plan pointer"); return RK_ERR_INVALID; }
    *out = nullptr;
    int rc = validate(desc);
    if (rc) return rc;
    Planned P;
    rc = plan_passes(*desc, P);
    if (rc) return rc;
    const int dbl = desc->dtype == RK_FMT_C128;
    const int esz = dbl ? 16 : 8;

    // window must sit on the first processed axis
    if (desc->input.window != RK_WIN_NONE && (P.passes.empty() || P.passes[0].axis != desc->input.window_axis)) {
        set_error("window transformation must act along the first transformed axis");
        return RK_ERR_UNSUPPORTED;
    }

    int dev = 0;
    CK(cudaGetDevice(&dev));
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    DeviceTables* tabs = nullptr;
    rc = device_tables(dev, &tabs);
    if (rc) return rc;

    rk_fft_plan* plan = new rk_fft_plan();
    plan->device = dev;
    plan->desc = *desc;
    auto fail = [&](int code) {
        rk_fft_plan_destroy(plan);
        return code;
    };

    // temporaries
    int64_t arr_elems = 1;
    for (int i = 0; i < desc->ndim; ++i) arr_elems *= desc->shape[i];
    void* bufs[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    auto alloc = [&](int64_t bytes, void** p) -> int {
        cudaError_t e = cudaMalloc(p, (size_t)std::max<int64_t>(bytes, 16));
        if (e != cudaSuccess) {
            set_error(std::string("temporary allocation failed: ") + cudaGetErrorString(e));
            return RK_ERR_NOMEM;
        }
        plan->temps.push_back(*p);
        plan->temp_bytes.push_back(bytes);
        plan->device_bytes += bytes;
        return RK_OK;
    };
    if (P.need_T0 && (rc = alloc(arr_elems * esz, &bufs[SB_T0]))) return fail(rc);
    if (P.need_T1 && (rc = alloc(arr_elems * esz, &bufs[SB_T1]))) return fail(rc);
    if (P.need_M) {
        if ((rc = alloc(P.m_elems * esz, &bufs[SB_M0]))) return fail(rc);
        if ((rc = alloc(P.m_elems * esz, &bufs[SB_M1]))) return fail(rc);
    }

    // Bluestein tables: chirp (N) and kernel spectrum K = FFT_M(b) / M (M)
    std::map<int, std::pair<void*, void*>> blue_tabs;
    for (const BlueAxis& ba : P.blue) {
        void *chirp = nullptr, *K = nullptr, *b = nullptr, *Kd = nullptr;
        if ((rc = alloc(ba.N * esz, &chirp))) return fail(rc);
        if ((rc = alloc(ba.M * esz, &K))) return fail(rc);
        cudaError_t e1 = cudaMalloc(&b, ba.M * sizeof(double2));
        cudaError_t e2 = cudaMalloc(&Kd, ba.M * sizeof(double2));
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            cudaFree(b); cudaFree(Kd);
            set_error("Bluestein scratch allocation failed");
            return fail(RK_ERR_NOMEM);
        }
        const int64_t nb = (ba.M + 255) / 256;
        k_gen_chirp<<<(unsigned)nb, 256>>>(ba.N, ba.M, dbl ? nullptr : (float2*)chirp, dbl ? (double2*)chirp : nullptr,
                                            (double2*)b);
        cudaError_t ek = cudaGetLastError();
        if (ek != cudaSuccess) {
            cudaFree(b); cudaFree(Kd);
            set_error(std::string("chirp generation failed: ") + cudaGetErrorString(ek));
            return fail(RK_ERR_CUDA);
        }
        // forward FFT_M of b in complex128 with this library
        rk_fft_desc kd;
        memset(&kd, 0, sizeof(kd));
        kd.dtype = RK_FMT_C128;
        kd.ndim = 1;
        kd.shape[0] = ba.M;
        kd.naxes = 1;
        kd.axes[0] = 0;
        rk_edge_init(&kd.input, RK_FMT_C128, 1, kd.shape);
        rk_edge_init(&kd.output, RK_FMT_C128, 1, kd.shape);
        rk_fft_plan* kp = nullptr;
        int krc = rk_fft_plan_create(&kd, &kp);
        if (krc == RK_OK) {
            void* o[1] = {Kd};
            const void* in[1] = {b};
            krc = rk_fft_execute(kp, o, 1, in, 1, 0, nullptr, 0, nullptr);
        }
        if (krc == RK_OK) {
            k_scale_convert<<<(unsigned)nb, 256>>>((const double2*)Kd, ba.M, 1.0 / (double)ba.M,
                                                   dbl ? nullptr : (float2*)K, dbl ? (double2*)K : nullptr);
            cudaError_t e3 = cudaDeviceSynchronize();
            if (e3 != cudaSuccess) {
                set_error(std::string("Bluestein table generation failed: ") + cudaGetErrorString(e3));
                krc = RK_ERR_CUDA;
            }
        }
        if (kp) rk_fft_plan_destroy(kp);
        cudaFree(b);
        cudaFree(Kd);
        if (krc != RK_OK) return fail(krc);
        blue_tabs[ba.axis] = {chirp, K};
    }

    // materialise passes
    int64_t ntot = 1;
    for (int i = 0; i < desc->naxes; ++i) ntot *= desc->shape[desc->axes[i]];
    plan->n_total = (double)ntot;
    for (const PassSpec& ps : P.passes) {
        PassRec r;
        r.kind = ps.kind;
        r.dbl = dbl;
        r.L = ps.L;
        r.mode = ps.mode;
        r.blue = (ps.var & 15) == 1 || ps.var == 7;
        r.var = ps.var;
        r.axis = ps.axis;
        r.ld_buf = ps.ld.buf == SB_IN ? BUF_IN : ps.ld.buf == SB_OUT ? BUF_OUT : ps.ld.buf;
        r.st_buf = ps.st.buf == SB_IN ? BUF_IN : ps.st.buf == SB_OUT ? BUF_OUT : ps.st.buf;
        r.ld_edge = ps.ld.buf == SB_IN;
        r.st_edge = ps.st.buf == SB_OUT;
        r.user_bits = (r.ld_edge && desc->input.format == RK_FMT_USER ? 1 : 0) |
                      (r.st_edge && desc->output.format == RK_FMT_USER ? 2 : 0);
        r.inplace_safe = ps.inplace_safe;
        r.note = ps.note;
        PassParams& pp = r.prm;
        memset(&pp, 0, sizeof(pp));
        pp.O = ps.O; pp.C = ps.C; pp.I = ps.I;
        pp.nlines = ps.O * ps.C * ps.I;
        build_side(*desc, ps.ld, ps.axis, dbl, true, pp.ld);
        build_side(*desc, ps.st, ps.kind == PK_PLANE ? ps.axis2 : ps.axis, dbl, false, pp.st);
        // antiperiodic transforms: W_2L^m on the first load (forward, a load-side
        // table) or after the FFT of the inverse (variant 4's rtwid), which the last
        // store's conjugation turns into W_2L^-m
        const bool ap_tab = (ps.var == 3 || ps.var == 4) && (desc->flags & RK_FLAG_ANTIPERIODIC);
        if (ap_tab && ps.var == 3) pp.ld.flags |= SF_TAB;
        mark_fast(pp.ld, dbl, ps.kind == PK_PLANE ? ps.L2 : ps.L);
        mark_fast(pp.st, dbl, ps.kind == PK_PLANE ? ps.L1 : ps.L);
        mark_fast2(pp.ld, dbl, ps.kind == PK_PLANE ? ps.L2 : ps.L, ps.C);
        mark_fast2(pp.st, dbl, ps.kind == PK_PLANE ? ps.L1 : ps.L, ps.C);
        if (!r.ld_edge) pp.ld.ptr = bufs[ps.ld.buf];
        if (!r.st_edge) pp.st.ptr = bufs[ps.st.buf];
        if ((pp.ld.flags & SF_WINDOW) && pp.ld.win_len > 0) {
            // a pair-read side indexes the samples 2u and 2u + 1 of every position u < L
            const int64_t n = (pp.ld.flags & SF_RPAIR) ? std::max<int64_t>(pp.ld.win_len, 2 * (int64_t)ps.L)
                                                       : (int64_t)pp.ld.win_len;
            void* wt = nullptr;
            const int wrc = alloc(n * (dbl ? 8 : 4), &wt);
            if (wrc) return fail(wrc);
            k_gen_window<<<(unsigned)((n + 255) / 256), 256>>>(n, pp.ld.win_len, dbl ? nullptr : (float*)wt,
                                                              dbl ? (double*)wt : nullptr);
            CK(cudaGetLastError());
            pp.ld.win = wt;
        }
        if (ps.kind == PK_LINE) {
            mark_fastr(pp.ld, dbl, ps.L, true);
            mark_fastr(pp.st, dbl, ps.L, false);
        }
        if (ps.var >= 3 && ps.var <= 6) {
            const int cfmt = dbl ? RK_FMT_C128 : RK_FMT_C64, rfmt = dbl ? RK_FMT_F64 : RK_FMT_F32;
            const bool edges_ok = (pp.ld.flags & SF_RPAIR)
                                      ? (pp.ld.fmt == rfmt &&
                                         (pp.st.fmt == cfmt || (pp.st.fmt == rfmt && (pp.st.flags & SF_NORM))))
                                      : (pp.st.fmt == cfmt && pp.ld.fmt == cfmt);
            if (!edges_ok) {
                set_error("a one-pass real transform needs complex edges of the transform's precision");
                return fail(RK_ERR_UNSUPPORTED);
            }
            const bool ap = desc->flags & RK_FLAG_ANTIPERIODIC;
            const int64_t L = ps.L;
            const int esz = dbl ? 16 : 8;
            void* wt = nullptr;
            const int trc = alloc((L + 1) * esz, &wt);
            if (trc) return fail(trc);
            if (ap)
                k_gen_rodd<<<(unsigned)((L + 255) / 256), 256>>>(L, dbl ? nullptr : (float2*)wt,
                                                                 dbl ? (double2*)wt : nullptr);
            else
                k_gen_rpost<<<(unsigned)((L + 256) / 256), 256>>>(L, dbl ? nullptr : (float2*)wt,
                                                                  dbl ? (double2*)wt : nullptr);
            CK(cudaGetLastError());
            pp.rmix = wt;
            pp.rodd = ap ? 1 : 0;
            // forward: 2 (Z A + conj(Z') B) for the odd harmonics (the doubled half
            // period); inverse: one half of the forward's A, B (a quarter for them)
            pp.rh = ps.var != 4 ? (ap ? 1.0 : 0.5) : (ap ? 0.25 : 0.5);
            pp.rnyq = ap ? 0 : (ps.var == 4 ? 1 : (desc->output.shape[ps.axis] > L ? 1 : 0));
            if (ap_tab) {
                void* tt = nullptr;
                const int rc2 = alloc((L + 1) * esz, &tt);
                if (rc2) return fail(rc2);
                k_gen_rpost<<<(unsigned)((L + 256) / 256), 256>>>(L, dbl ? nullptr : (float2*)tt,
                                                                  dbl ? (double2*)tt : nullptr);
                CK(cudaGetLastError());
                if (ps.var == 3)
                    pp.ld.tab = tt;
                else
                    pp.rtwid = tt;
            }
        }
        if (ps.ld.chirp_axis >= 0) {
            auto& bt = blue_tabs[ps.ld.chirp_axis];
            pp.ld.chirp = bt.first;
            if (ps.ld.tab_k) pp.ld.tab = bt.second;
        }
        if (ps.st.chirp_axis >= 0) pp.st.chirp = blue_tabs[ps.st.chirp_axis].first;
        if (ps.blue_axis >= 0) pp.blue_k = blue_tabs[ps.blue_axis].second;
        if (ps.var == 7) {
            // W_M^n, n = 0 .. L, for the odd-bin CTA of the two-CTA Bluestein pass
            void* wt = nullptr;
            const int rc7 = alloc((int64_t)(ps.L + 1) * 8, &wt);
            if (rc7) return fail(rc7);
            k_gen_rpost<<<(unsigned)((ps.L + 256) / 256), 256>>>(ps.L, (float2*)wt, nullptr);
            CK(cudaGetLastError());
            pp.rtwid = wt;
        }
        {
            const int lg = ilog2(std::max(ps.L, 1));
            const int lg2 = ilog2(std::max(ps.kind == PK_PLANE ? ps.L1 : ps.L, 1));
            if (dbl) {
                pp.tw = (const double2*)tabs->stw_d + tabs->off_d[lg];
                pp.tw2 = (const double2*)tabs->stw_d + tabs->off_d[lg2];
            } else {
                pp.tw = (const float2*)tabs->stw_f + ((ps.var >> 4) ? tabs->off_f_r16 : tabs->off_f[lg]);
                pp.tw2 = (const float2*)tabs->stw_f + tabs->off_f[lg2];
            }
        }
        pp.tw4_hi = tabs->tw4hi_d;  // FP64 for both precisions (tw4() rounds once)
        pp.tw4_lo = tabs->tw4lo_d;
        pp.tw4_N = ps.tw4_N;
        pp.status = tabs->status;
        r.L1 = ps.L1;
        r.L2 = ps.L2;
        r.axis2 = ps.axis2;
        if (ps.kind == PK_PLANE) {
            PlaneInfo pi;
            if (!plane_info(dbl, ps.L1, ps.L2, (desc->flags & RK_FLAG_PLANE_WIDE) ? 1 : 0, &pi)) {
                set_error("no plane kernel instantiation");
                return fail(RK_ERR_UNSUPPORTED);
            }
            r.pi = pi;
            r.nblocks = ps.O;  // planes
            PlaneTmaInfo pti;
            const Side& ld = pp.ld;
            const int esz = dbl ? 16 : 8;
            bool ok_tma = !(desc->flags & (RK_FLAG_NO_TMA | RK_FLAG_PLANE_WIDE)) &&
                          plane_tma_info(dbl, ps.L1, ps.L2, &pti) && (ld.flags & SF_FAST) && ld.ax_shift == 0 &&
                          ld.ax_stride == 1 && ld.nd_i == 0 && ld.nd_o == 1 && ld.o_stride[0] == ps.L2 &&
                          ld.o_shift[0] == 0 && ld.o_bound[0] == ld.o_shape[0] && (ld.offset * esz) % 16 == 0;
            if (ok_tma) {
                const int ncl = pti.clusters();
                if (ncl > 0) {
                    pp.tile_stride = (int64_t)ps.L1 * ps.L2;
                    r.pti = pti;
                    r.use_plane_tma = true;
                    r.plane_tma_blocks = std::min<int64_t>(ps.O, ncl) * pti.q;
                }
            }
        } else {
            LineInfo li;
            bool ok = line_info(dbl, ps.L, ps.mode, ps.var, &li);
            if (!ok) {
                set_error("no kernel instantiation for pass " + ps.note + " L=" + std::to_string(ps.L));
                return fail(RK_ERR_UNSUPPORTED);
            }
            r.nblocks = (pp.nlines + li.nl - 1) / li.nl;
            r.li = li;
            if (!(desc->flags & RK_FLAG_NO_TMA) && ps.var == 0) setup_tma(r, dbl, nsm);
            if ((desc->flags & RK_FLAG_SPLIT_TC) && tc_eligible(r)) {
                const cudaError_t te = tc_prepare();
                if (te != cudaSuccess) {
                    set_error(std::string("tensor-core tables: ") + cudaGetErrorString(te));
                    return fail(RK_ERR_CUDA);
                }
                r.use_tc = true;
                r.use_tma = false;
            }
        }
        plan->passes.push_back(r);
    }
    for (size_t i = 0; i + 1 < plan->passes.size(); ++i) {
        if (!P.passes[i].pair) continue;
        PairInfo pi;
        if (!pair_info(dbl, plan->passes[i].L, plan->passes[i + 1].L, &pi)) continue;
        const int rc = pair_setup(plan->passes[i], plan->passes[i + 1], pi);
        if (rc == RK_ERR_NOMEM || rc == RK_ERR_CUDA) {
            set_error("pair launch set-up failed");
            return fail(rc);
        }
        if (rc == RK_OK) plan->device_bytes += plan->passes[i].pair_ntasks * 4 + (plan->passes[i].pair_planes + 1) * 4;
    }
    if (plan->passes.size() == 1) {
        // a single pass rewrites only the elements its CTA (or cluster) read, unless the
        // two edges place the same logical element at different addresses
        const rk_edge& a = desc->input;
        const rk_edge& b = desc->output;
        bool same = a.format == b.format && a.offset == b.offset && a.offset2 == b.offset2;
        for (int i = 0; same && i < desc->ndim; ++i)
            same = a.strides[i] == b.strides[i] && a.shift[i] == b.shift[i] && a.shape[i] == b.shape[i] &&
                   (!fmt_is_pair(a.format) || a.strides2[i] == b.strides2[i]);
        plan->alias_hazard = !same || !plan->passes[0].inplace_safe;
        plan->in_extent_bytes = edge_extent_bytes(desc->input, 0);
        if (fmt_is_pair(desc->input.format)) plan->in2_extent_bytes = edge_extent_bytes(desc->input, 1);
    }
    // set launch attributes now (cudaFuncSetAttribute is not allowed during capture)
    for (const PassRec& r : plan->passes) {
        if (r.kind == PK_PLANE)
            CK(r.pi.fn(r.prm, 0, nullptr));
        else
            CK(r.li.fn(r.prm, 0, nullptr));
        if (r.use_tma) CK(r.ti.fn(r.prm, 0, nullptr));
        if (r.use_plane_tma) CK(r.pti.fn(r.prm, 0, nullptr));
    }
    CK(cudaDeviceSynchronize());
    *out = plan;
    return RK_OK;
}

int rk_fft_profile(rk_fft_plan* plan, int32_t max_calls) {
    if (!plan || max_calls < 0) { set_error("bad arguments"); return RK_ERR_INVALID; }
    for (cudaEvent_t e : plan->prof_ev) cudaEventDestroy(e);
    plan->prof_ev.clear();
    plan->prof_max = plan->prof_used = 0;
    if (max_calls == 0) return RK_OK;
    const size_t n = 2 * plan->passes.size() * (size_t)max_calls;
    plan->prof_ev.resize(n);
    for (size_t i = 0; i < n; ++i) CK(cudaEventCreate(&plan->prof_ev[i]));
    plan->prof_max = max_calls;
    return RK_OK;
}

int rk_fft_profile_read(rk_fft_plan* plan, double* ms, int32_t n_passes, int32_t* calls) {
    if (!plan || !ms || !calls || n_passes < (int32_t)plan->passes.size()) {
        set_error("bad arguments");
        return RK_ERR_INVALID;
    }
    const size_t np = plan->passes.size();
    for (size_t p = 0; p < np; ++p) ms[p] = 0.0;
    for (int32_t c = 0; c < plan->prof_used; ++c)
        for (size_t p = 0; p < np; ++p) {
            cudaEvent_t a = plan->prof_ev[2 * (c * np + p)], b = plan->prof_ev[2 * (c * np + p) + 1];
            CK(cudaEventSynchronize(b));
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, a, b));
            ms[p] += t;
        }
    *calls = plan->prof_used;
    return RK_OK;
}

int rk_fft_plan_destroy(rk_fft_plan* plan) {
    if (!plan) return RK_OK;
    for (cudaEvent_t e : plan->prof_ev) cudaEventDestroy(e);
    for (void* p : plan->temps) cudaFree(p);
    if (plan->alias_tmp) cudaFree(plan->alias_tmp);
    for (rk::PassRec& r : plan->passes) {
        if (r.pair_tasks) cudaFree(r.pair_tasks);
        if (r.pair_counters) cudaFree(r.pair_counters);
        if (r.user_lib) cudaLibraryUnload((cudaLibrary_t)r.user_lib);
    }
    delete plan;
    return RK_OK;
}

int rk_fft_plan_device_bytes(const rk_fft_plan* plan, int64_t* bytes) {
    if (!plan || !bytes) { set_error("null argument"); return RK_ERR_INVALID; }
    *bytes = plan->device_bytes;
    return RK_OK;
}

int rk_fft_plan_launches(const rk_fft_plan* plan, int32_t* n) {
    if (!plan || !n) { set_error("null argument"); return RK_ERR_INVALID; }
    *n = (int32_t)plan->passes.size();
    return RK_OK;
}

int rk_fft_plan_tc_passes(const rk_fft_plan* plan, int32_t* n) {
    if (!plan || !n) { set_error("null argument"); return RK_ERR_INVALID; }
    int32_t k = 0;
    for (const PassRec& r : plan->passes) k += r.use_tc ? 1 : 0;
    *n = k;
    return RK_OK;
}

static void apply_edge_scale(const rk_edge& e, const double* scalars, int32_t n_scalars, double& re, double& im,
                             int* bad) {
    re = e.scale_re;
    im = e.scale_im;
    if (e.scale_slot >= 0) {
        if (e.scale_slot >= n_scalars) { *bad = 1; return; }
        const double sr = scalars[2 * e.scale_slot], si = scalars[2 * e.scale_slot + 1];
        const double r = re * sr - im * si, i = re * si + im * sr;
        re = r; im = i;
    }
    if (e.scale_div_slot >= 0) {
        if (e.scale_div_slot >= n_scalars) { *bad = 1; return; }
        const double sr = scalars[2 * e.scale_div_slot], si = scalars[2 * e.scale_div_slot + 1];
        const double den = sr * sr + si * si;
        const double r = (re * sr + im * si) / den, i = (im * sr - re * si) / den;
        re = r; im = i;
    }
}

}  // extern "C"

namespace rk {

// Per-call launch parameters of every pass of a plan: user pointers, runtime scale,
// inverse conjugations; `tma` says whether the pass may take its TMA kernel for this
// call.  Stages a private copy of the input when an in-place call meets a remapping
// single-pass plan.  Shared by rk_fft_execute and the batched launch.
int build_call_params(rk_fft_plan* plan, void* const* outputs, int32_t n_outputs, const void* const* inputs,
                      int32_t n_inputs, int32_t inverse, const double* scalars, int32_t n_scalars, cudaStream_t st,
                      std::vector<PassParams>& out, std::vector<char>* tma_ok, const uint64_t* user_in,
                      int32_t n_user_in, const uint64_t* user_out, int32_t n_user_out) {
    if (n_user_in < 0 || n_user_in > 8 || n_user_out < 0 || n_user_out > 8 || (n_user_in && !user_in) ||
        (n_user_out && !user_out)) {
        set_error("user code takes at most 8 words per edge");
        return RK_ERR_INVALID;
    }
    if (!plan) { set_error("null plan"); return RK_ERR_INVALID; }
    const rk_fft_desc& d = plan->desc;
    const int need_in = fmt_arrays(d.input.format);
    const int need_out = fmt_arrays(d.output.format);
    if ((need_in && !inputs) || (need_out && !outputs) || n_inputs < need_in || n_outputs < need_out) {
        set_error("wrong number of input/output arrays");
        return RK_ERR_INVALID;
    }
    for (int i = 0; i < need_in; ++i)
        if (!inputs[i]) { set_error("null input pointer"); return RK_ERR_INVALID; }
    for (int i = 0; i < need_out; ++i)
        if (!outputs[i]) { set_error("null output pointer"); return RK_ERR_INVALID; }
    const void* in0 = need_in ? inputs[0] : nullptr;
    const void* in1 = need_in > 1 ? inputs[1] : nullptr;
    void* out0 = need_out ? outputs[0] : nullptr;
    void* out1 = need_out > 1 ? outputs[1] : nullptr;

    // in-place call of a single remapping pass: read from a private copy
    if (plan->alias_hazard && in0 && out0 &&
        (in0 == out0 || (in1 && (in1 == out0 || (out1 && in1 == out1))) || (out1 && in0 == out1))) {
        const int64_t need = plan->in_extent_bytes + plan->in2_extent_bytes + 256;
        if (!plan->alias_tmp) {
            cudaError_t e = cudaMalloc(&plan->alias_tmp, (size_t)need);
            if (e != cudaSuccess) {
                set_error("in-place staging allocation failed");
                return RK_ERR_NOMEM;
            }
            plan->device_bytes += need;
        }
        char* t = (char*)plan->alias_tmp;
        CK(cudaMemcpyAsync(t, in0, (size_t)plan->in_extent_bytes, cudaMemcpyDeviceToDevice, st));
        in0 = t;
        if (in1) {
            char* t2 = t + ((plan->in_extent_bytes + 255) / 256) * 256;
            CK(cudaMemcpyAsync(t2, in1, (size_t)plan->in2_extent_bytes, cudaMemcpyDeviceToDevice, st));
            in1 = t2;
        }
    }

    int bad = 0;
    double in_re, in_im, out_re, out_im;
    apply_edge_scale(d.input, scalars, n_scalars, in_re, in_im, &bad);
    apply_edge_scale(d.output, scalars, n_scalars, out_re, out_im, &bad);
    // additive terms: the constant plus the slot's value; applied after the scale,
    // so the inverse's 1/N (a factor of the output scale) does not touch them
    double add_in[2] = {d.input.add_re, d.input.add_im}, add_out[2] = {d.output.add_re, d.output.add_im};
    for (int k = 0; k < 2; ++k) {
        const rk_edge& e = k ? d.output : d.input;
        double* a = k ? add_out : add_in;
        if (e.add_slot >= 0) {
            if (e.add_slot >= n_scalars) { bad = 1; continue; }
            a[0] += scalars[2 * e.add_slot];
            a[1] += scalars[2 * e.add_slot + 1];
        }
    }
    double order = d.output.post_param;
    if (d.output.post_slot >= 0) {
        if (d.output.post_slot >= n_scalars) bad = 1; else order = scalars[2 * d.output.post_slot];
    }
    if (bad) { set_error("scalar slot out of range"); return RK_ERR_INVALID; }
    if (inverse) {
        out_re /= plan->n_total;
        out_im /= plan->n_total;
    }
    const size_t np = plan->passes.size();
    for (size_t i = 0; i < np; ++i) {
        PassRec& r = plan->passes[i];
        bool tma = r.use_tma || r.use_plane_tma;
        if (tma && r.ld_edge) {
            // a view of the user's array may start off the 16-byte grid the bulk
            // copies need: such calls take the plain kernel
            const int esz = r.dbl ? 16 : 8;
            if ((((uintptr_t)in0) + (uintptr_t)(r.prm.ld.offset * esz)) % 16 != 0) tma = false;
        }
        if (tma && r.tma_reencode && r.tma_ptr != in0) {
            const Side& ld = r.prm.ld;
            const int64_t so = ld.nd_o == 1 ? ld.o_stride[0] : (int64_t)r.L * r.prm.I;
            if (encode_lane_map(const_cast<void*>(in0), r.dbl, r.prm.I, r.L, r.prm.O, ld.ax_stride, so, r.ti.nl,
                                r.tma_rows, &r.prm.tmap))
                r.tma_ptr = in0;
            else
                tma = false;
        }
        PassParams p = r.prm;
        if (r.ld_edge) {
            p.ld.ptr = const_cast<void*>(in0);
            p.ld.ptr2 = const_cast<void*>(in1);
            if (in_re != 1.0 || in_im != 0.0) {
                p.ld.flags |= SF_SCALE;
                p.ld.scale_re = in_re;
                p.ld.scale_im = in_im;
            }
            p.ld.add_re = add_in[0];
            p.ld.add_im = add_in[1];
            for (int k = 0; k < n_user_in; ++k) p.ld.user[k] = user_in[k];
            if (d.input.conj) p.ld.flags ^= SF_PRE_CONJ;
        }
        if (r.st_edge) {
            p.st.ptr = out0;
            p.st.ptr2 = out1;
            if (out_re != 1.0 || out_im != 0.0) {
                p.st.flags |= SF_SCALE;
                p.st.scale_re = out_re;
                p.st.scale_im = out_im;
            }
            p.st.add_re = add_out[0];
            p.st.add_im = add_out[1];
            for (int k = 0; k < n_user_out; ++k) p.st.user[k] = user_out[k];
            if (p.st.flags & SF_NORM) p.st.post_param = order;
        }
        if (inverse) {
            // IFFT(x) = conj(FFT(conj(x))) / N: conjugate on the first load and last store
            if (i == 0) p.ld.flags ^= SF_PRE_CONJ;
            if (i == np - 1) p.st.flags ^= SF_POST_CONJ;
        }
        if (r.st_edge && d.output.conj) p.st.flags ^= SF_POST_CONJ;
        if (p.ld.flags & SF_RPAIR) {
            // the half-length route reads a real signal as sample pairs: a multiplier c
            // of the input (conjugated by the input's conjugations) multiplies the
            // transform, so it moves to the store, conjugated once more by the store's
            // conjugation (the store conjugates X before scaling)
            double cr = 1.0, ci = 0.0;
            if (p.ld.flags & SF_SCALE) { cr = p.ld.scale_re; ci = p.ld.scale_im; }
            const bool ld_conj = ((p.ld.flags & SF_PRE_CONJ) != 0) != ((p.ld.flags & SF_POST_CONJ) != 0);
            const bool st_conj = ((p.st.flags & SF_PRE_CONJ) != 0) != ((p.st.flags & SF_POST_CONJ) != 0);
            if (ld_conj != st_conj) ci = -ci;
            p.ld.flags &= ~(SF_SCALE | SF_PRE_CONJ | SF_POST_CONJ);
            double sr = 1.0, si = 0.0;
            if (p.st.flags & SF_SCALE) { sr = p.st.scale_re; si = p.st.scale_im; }
            const double nr = sr * cr - si * ci, ni = sr * ci + si * cr;
            if (nr != 1.0 || ni != 0.0) {
                p.st.flags |= SF_SCALE;
                p.st.scale_re = nr;
                p.st.scale_im = ni;
            } else {
                p.st.flags &= ~SF_SCALE;
            }
        }
        out.push_back(p);
        if (tma_ok) tma_ok->push_back(tma ? 1 : 0);
    }
    return RK_OK;
}

}  // namespace rk

extern "C" {

int rk_fft_plan_pass_info(const rk_fft_plan* plan, int32_t index, int32_t* info, int64_t* smem) {
    if (!plan || !info || !smem || index < 0 || index >= (int32_t)plan->passes.size()) {
        set_error("rk_fft_plan_pass_info: bad arguments");
        return RK_ERR_INVALID;
    }
    const PassRec& r = plan->passes[index];
    info[0] = r.kind;
    info[1] = r.L;
    info[2] = r.mode;
    info[3] = r.var;
    info[4] = r.dbl;
    info[5] = r.kind == PK_LINE ? r.li.nt : r.pi.nt;
    info[6] = r.user_bits;
    info[7] = r.kind == PK_LINE ? r.li.nl : 0;
    *smem = (int64_t)(r.kind == PK_LINE ? r.li.smem : r.pi.smem);
    return RK_OK;
}

int rk_fft_plan_set_pass_kernel(rk_fft_plan* plan, int32_t index, const void* image, int64_t size, const char* name) {
    if (!plan || !image || size <= 0 || !name || index < 0 || index >= (int32_t)plan->passes.size()) {
        set_error("rk_fft_plan_set_pass_kernel: bad arguments");
        return RK_ERR_INVALID;
    }
    PassRec& r = plan->passes[index];
    if (r.kind != PK_LINE || r.use_tc || r.use_tma || r.pair_first) {
        set_error("rk_fft_plan_set_pass_kernel: only plain line passes take an installed kernel");
        return RK_ERR_UNSUPPORTED;
    }
    int cur = 0;
    CK(cudaGetDevice(&cur));
    if (cur != plan->device) CK(cudaSetDevice(plan->device));
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kern = nullptr;
    cudaError_t e = cudaLibraryLoadData(&lib, image, nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&kern, lib, name);
    if (e == cudaSuccess && r.li.smem > 48 * 1024)
        e = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r.li.smem);
    if (cur != plan->device) cudaSetDevice(cur);
    if (e != cudaSuccess) {
        if (lib) cudaLibraryUnload(lib);
        set_error(std::string("rk_fft_plan_set_pass_kernel: ") + cudaGetErrorString(e));
        return RK_ERR_CUDA;
    }
    if (r.user_lib) cudaLibraryUnload((cudaLibrary_t)r.user_lib);
    r.user_lib = lib;
    r.user_kern = (const void*)kern;
    return RK_OK;
}

int rk_fft_execute(rk_fft_plan* plan, void* const* outputs, int32_t n_outputs, const void* const* inputs,
                   int32_t n_inputs, int32_t inverse, const double* scalars, int32_t n_scalars, void* stream) {
    return rk_fft_execute_user(plan, outputs, n_outputs, inputs, n_inputs, inverse, scalars, n_scalars, nullptr, 0,
                               nullptr, 0, stream);
}

int rk_fft_execute_user(rk_fft_plan* plan, void* const* outputs, int32_t n_outputs, const void* const* inputs,
                        int32_t n_inputs, int32_t inverse, const double* scalars, int32_t n_scalars,
                        const uint64_t* user_in, int32_t n_user_in, const uint64_t* user_out, int32_t n_user_out,
                        void* stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (plan && inverse && (plan->desc.flags & RK_FLAG_REAL_POST)) {
        set_error("a plan with RK_FLAG_REAL_POST runs forward only");
        return RK_ERR_INVALID;
    }
    if (plan && !inverse && (plan->desc.flags & RK_FLAG_REAL_PRE)) {
        set_error("a plan with RK_FLAG_REAL_PRE runs inverse only");
        return RK_ERR_INVALID;
    }
    std::vector<PassParams> prm;
    std::vector<char> tma;
    prm.reserve(4);
    if (plan)
        for (const PassRec& r : plan->passes)
            if (r.user_bits && !r.user_kern) {
                set_error("a pass of this plan runs transformation code compiled at run time: install its kernel "
                          "with rk_fft_plan_set_pass_kernel first");
                return RK_ERR_INVALID;
            }
    int rc = build_call_params(plan, outputs, n_outputs, inputs, n_inputs, inverse, scalars, n_scalars, st, prm, &tma,
                               user_in, n_user_in, user_out, n_user_out);
    if (rc) return rc;
    const size_t np = plan->passes.size();
    for (size_t i = 0; i < np; ++i) {
        const PassRec& r = plan->passes[i];
        const PassParams& p = prm[i];
        const bool prof = plan->prof_used < plan->prof_max;
        const size_t ev = 2 * ((size_t)plan->prof_used * np + i);
        if (prof) CK(cudaEventRecord(plan->prof_ev[ev], st));
        cudaError_t e;
        if (r.pair_first && i + 1 < np) {
            // rows and columns in one launch: the second pass records an empty interval
            e = pair_launch(r, p, prm[i + 1], p.status, st);
            if (e != cudaSuccess) {
                set_error(std::string("kernel launch failed (pair): ") + cudaGetErrorString(e));
                return RK_ERR_CUDA;
            }
            if (prof) {
                CK(cudaEventRecord(plan->prof_ev[ev + 1], st));
                CK(cudaEventRecord(plan->prof_ev[ev + 2], st));
                CK(cudaEventRecord(plan->prof_ev[ev + 3], st));
            }
            ++i;
            continue;
        }
        if (r.user_kern) {
            void* args[1] = {const_cast<PassParams*>(&p)};
            const unsigned grid = (unsigned)((p.nlines + r.li.nl - 1) / r.li.nl);
            e = grid ? cudaLaunchKernel(r.user_kern, dim3(grid), dim3(r.li.nt), args, r.li.smem, st) : cudaSuccess;
        } else if (r.kind == PK_PLANE)
            e = tma[i] ? r.pti.fn(p, r.plane_tma_blocks, st) : r.pi.fn(p, r.nblocks, st);
        else if (r.use_tc)
            e = tc_launch(p, r.L, st);
        else
            e = tma[i] ? r.ti.fn(p, r.nblocks, st) : r.li.fn(p, (p.nlines + r.li.nl - 1) / r.li.nl, st);
        if (e != cudaSuccess) {
            set_error(std::string("kernel launch failed (") + r.note + "): " + cudaGetErrorString(e));
            return RK_ERR_CUDA;
        }
        if (prof) CK(cudaEventRecord(plan->prof_ev[ev + 1], st));
    }
    if (plan->prof_used < plan->prof_max) ++plan->prof_used;
    return RK_OK;
}

}  // extern "C"
