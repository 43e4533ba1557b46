// Allocation-free batched 1-D complex64 FFT (rk_fft1d_c64_noalloc).
//
// Some callers cannot allocate device memory at the point where they need a
// transform: code running inside a memory pool or arena that owns every byte of
// the device, real-time loops that must not call into the allocator (cudaMalloc
// can synchronise the device and take unbounded time), and plug-in hosts that
// hand out only the buffers they own.  For them this entry point runs the same
// two-pass four-step transform as a planned FFT (pass A: lane-mode FFT over n1 with
// the W_n^(n2 k1) twiddle on its store; pass B: position-mode FFT over n2 with a
// transposed store), but its intermediate buffer and its twiddle tables are
// file-scope __device__ arrays of fixed size that exist for as long as the library
// is loaded.  It calls no cudaMalloc, cudaFree or any other allocating routine.
//
// Limits and sharing: batch * n <= RK_NOALLOC_MAX_ELEMS complex64 elements (the
// scratch is 32 MiB per device that loads the library).  Every call on a device uses
// the same scratch, so calls that can overlap on the GPU (different streams, no
// ordering between them) race; calls on one stream are ordered and safe.  The
// current device must own the stream and both arrays (checked).  The first
// call on each device resolves the arrays' device addresses with
// cudaGetSymbolAddress and fills the twiddle tables with a few kernel launches and a
// device synchronisation; make that first call before any stream capture.  Pass A
// overwrites every scratch element before pass B reads it, so nothing in the
// scratch has to start at zero and the previous call's contents never leak into a
// result.
#include <cuda_runtime.h>
#include <string.h>

#include <mutex>
#include <string>

#include "rk_internal.h"
#include "rk_kernels.cuh"

namespace rk {

__global__ void k_gen_stage(float2* f, double2* d, int Lp, int R, int J);

constexpr int ilog2_l(int n) { return n <= 1 ? 0 : 1 + ilog2_l(n / 2); }

constexpr int64_t NOALLOC_MAX_ELEMS = int64_t(1) << 22;  // 4 Mi complex64 = 32 MiB
constexpr int NOALLOC_MIN_LOG = 12, NOALLOC_MAX_LOG = 20;

// stage twiddle tables of every line length the four-step split can use here
template <int L> struct NaTw {
    static constexpr int64_t size() { return TwLayout<float, L>::total(); }
};
constexpr int64_t na_tw_total() {
    return NaTw<2>::size() + NaTw<4>::size() + NaTw<8>::size() + NaTw<16>::size() + NaTw<32>::size() +
           NaTw<64>::size() + NaTw<128>::size() + NaTw<256>::size() + NaTw<512>::size() + NaTw<1024>::size() +
           NaTw<2048>::size();
}

static __device__ __align__(256) float2 g_na_scratch[NOALLOC_MAX_ELEMS];
static __device__ __align__(256) float2 g_na_stage_tw[na_tw_total() > 0 ? na_tw_total() : 1];
static __device__ __align__(256) double2 g_na_tw4[2 * TW4_HALF];  // [hi | lo]

__global__ void k_na_tw4(double2* hi, double2* lo) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= TW4_HALF) return;
    double s, c;
    sincospi(2.0 * (double)k / (double)(1 << TW4_LOG), &s, &c);
    lo[k] = make_double2(c, -s);
    sincospi(2.0 * (double)k * TW4_HALF / (double)(1 << TW4_LOG), &s, &c);
    hi[k] = make_double2(c, -s);
}

struct NaDevice {
    bool ready = false;
    float2* scratch = nullptr;
    float2* stage_tw = nullptr;
    double2* tw4 = nullptr;
    int64_t off[12] = {0};  // stage table offset of L = 2^i
};

static std::mutex g_na_mu;
static NaDevice g_na[64];

template <int L> static void na_layout(NaDevice& d, int64_t& total, bool gen) {
    using RC = Radix<float, L>;
    d.off[ilog2_l(L)] = total;
    if (gen) {
        int P = 1;
        for (int s = 0; s + 1 < RC::NS; ++s) {
            const int R = RC::R[s];
            const int J = L / (P * R);
            const int n = (R - 1) * J;
            k_gen_stage<<<(n + 255) / 256, 256>>>(d.stage_tw + total + TwLayout<float, L>::offset(s), nullptr, L / P, R,
                                                  J);
            P *= R;
        }
    }
    total += TwLayout<float, L>::total();
    if constexpr (L < 2048) na_layout<2 * L>(d, total, gen);
}

static int na_setup(int dev, NaDevice** out) {
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (dev < 0 || dev >= 64) {
        set_error("rk_fft1d_c64_noalloc: device index out of range");
        return RK_ERR_INVALID;
    }
    NaDevice& d = g_na[dev];
    if (!d.ready) {
        // host code sees only stand-ins for the __device__ arrays: resolve their
        // addresses on this device before handing them to kernels
        cudaError_t e = cudaGetSymbolAddress((void**)&d.scratch, g_na_scratch);
        if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&d.stage_tw, g_na_stage_tw);
        if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&d.tw4, g_na_tw4);
        if (e != cudaSuccess) {
            set_error(std::string("rk_fft1d_c64_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            return RK_ERR_CUDA;
        }
        int64_t total = 0;
        na_layout<2>(d, total, true);
        k_na_tw4<<<TW4_HALF / 256, 256>>>(d.tw4, d.tw4 + TW4_HALF);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            set_error(std::string("rk_fft1d_c64_noalloc: table set-up failed: ") + cudaGetErrorString(e));
            return RK_ERR_CUDA;
        }
        d.ready = true;
    }
    *out = &d;
    return RK_OK;
}

// contiguous (batch, n) complex64 side of a four-step pass over the flat index
static void na_side(Side& s, void* ptr, int64_t batch, int64_t n, int64_t cA, int64_t jB) {
    memset(&s, 0, sizeof(s));
    s.ptr = ptr;
    s.fmt = RK_FMT_C64;
    s.nd_o = batch > 1 ? 1 : 0;
    s.o_shape[0] = batch;
    s.o_stride[0] = n;
    s.o_bound[0] = batch;
    s.nd_i = 0;
    s.ax_len = n;
    s.ax_bound = n;
    s.ax_stride = 1;
    s.cA = cA;
    s.jB = jB;
    s.scale_re = 1.0;
}

}  // namespace rk

using namespace rk;

extern "C" int rk_fft1d_c64_noalloc(void* out, const void* in, int64_t n, int64_t batch, int32_t inverse,
                                    void* stream) {
    if (!out || !in) {
        set_error("rk_fft1d_c64_noalloc: null array pointer");
        return RK_ERR_INVALID;
    }
    if (n < (int64_t(1) << NOALLOC_MIN_LOG) || n > (int64_t(1) << NOALLOC_MAX_LOG) || (n & (n - 1))) {
        set_error("rk_fft1d_c64_noalloc: n must be a power of two in [4096, 1048576]");
        return RK_ERR_INVALID;
    }
    if (batch < 1 || batch > NOALLOC_MAX_ELEMS / n) {
        set_error("rk_fft1d_c64_noalloc: batch * n exceeds the static scratch of " +
                  std::to_string(NOALLOC_MAX_ELEMS) + " complex64 elements (32 MiB)");
        return RK_ERR_INVALID;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error(std::string("rk_fft1d_c64_noalloc: ") + cudaGetErrorString(e));
        return RK_ERR_CUDA;
    }
    // the static arrays used below are the current device's: the stream and both
    // arrays must belong to that device too
    if (stream) {
        int sdev = -1;
        e = cudaStreamGetDevice((cudaStream_t)stream, &sdev);
        if (e != cudaSuccess) {
            set_error(std::string("rk_fft1d_c64_noalloc: stream: ") + cudaGetErrorString(e));
            return RK_ERR_INVALID;
        }
        if (sdev != dev) {
            set_error("rk_fft1d_c64_noalloc: the stream belongs to device " + std::to_string(sdev) +
                      ", not to the current device " + std::to_string(dev));
            return RK_ERR_INVALID;
        }
    }
    const void* arrays[2] = {out, in};
    for (int i = 0; i < 2; ++i) {
        cudaPointerAttributes pa;
        e = cudaPointerGetAttributes(&pa, arrays[i]);
        if (e != cudaSuccess || (pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged) ||
            pa.device != dev) {
            cudaGetLastError();
            set_error(std::string("rk_fft1d_c64_noalloc: ") + (i ? "in" : "out") +
                      " must be device memory of the current device " + std::to_string(dev));
            return RK_ERR_INVALID;
        }
    }
    NaDevice* d = nullptr;
    int rc = na_setup(dev, &d);
    if (rc) return rc;

    // the same split as the planner's contiguous-axis four-step
    int64_t N2 = n / 2 < 256 ? n / 2 : 256, N1 = n / N2;
    if (N1 > 1024) {
        N1 = 1024;
        N2 = n / N1;
    }
    LineInfo la, lb;
    if (!line_info(0, (int)N1, MODE_LANE, 0, &la) || !line_info(0, (int)N2, MODE_POS, 2, &lb)) {
        set_error("rk_fft1d_c64_noalloc: no kernel for this split");
        return RK_ERR_UNSUPPORTED;
    }
    cudaStream_t st = (cudaStream_t)stream;

    PassParams a;
    memset(&a, 0, sizeof(a));
    a.O = batch;
    a.C = N2;
    a.I = 1;
    a.nlines = batch * N2;
    na_side(a.ld, const_cast<void*>(in), batch, n, 1, N2);
    na_side(a.st, d->scratch, batch, n, 1, N2);
    a.st.flags = SF_TW4;
    if (inverse) a.ld.flags |= SF_PRE_CONJ;
    a.tw = d->stage_tw + d->off[ilog2_l((int)N1)];
    a.tw2 = a.tw;
    a.tw4_hi = d->tw4;
    a.tw4_lo = d->tw4 + TW4_HALF;
    a.tw4_N = n;

    PassParams b;
    memset(&b, 0, sizeof(b));
    b.O = batch;
    b.C = N1;
    b.I = 1;
    b.nlines = batch * N1;
    na_side(b.ld, d->scratch, batch, n, N2, 1);
    na_side(b.st, out, batch, n, 1, N1);
    if (inverse) {
        b.st.flags = SF_POST_CONJ | SF_SCALE;
        b.st.scale_re = 1.0 / (double)n;
    }
    b.tw = d->stage_tw + d->off[ilog2_l((int)N2)];
    b.tw2 = b.tw;

    e = la.fn(a, (a.nlines + la.nl - 1) / la.nl, st);
    if (e == cudaSuccess) e = lb.fn(b, (b.nlines + lb.nl - 1) / lb.nl, st);
    if (e != cudaSuccess) {
        set_error(std::string("rk_fft1d_c64_noalloc: launch failed: ") + cudaGetErrorString(e));
        return RK_ERR_CUDA;
    }
    return RK_OK;
}
