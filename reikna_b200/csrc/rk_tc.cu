// Tensor-core split-precision line passes for 256- and 1024-point complex64 transforms
// along a contiguous axis (the precision mode, RK_FLAG_SPLIT_TC).
//
// L = R^2 with R = 16 or 32, n = R n1 + n2, k = k1 + R k2:
//   X[k] = sum_n2 W_R^(n2 k2) W_L^(n2 k1) sum_n1 W_R^(n1 k1) x[n]
// Both radix-R stages are real matrix products on the 5th-generation tensor cores
// (tcgen05.mma, kind::tf32, FP32 accumulator in tensor memory).  A tile is 128 vectors
// (128 / R lines); the vectors are the M = 128 rows of the A operand, whose K = 2R
// columns are the R real parts then the R imaginary parts; B is the real form of the
// R-point DFT matrix (N = 2R output reals).
//
// Stage 1: row m = (line l, n2) is the vector over n1.  Two or four threads share a row
// (one tensor-memory lane, parts of its columns): they load its elements (a warp reads 32
// consecutive n2 of one n1), write them as 16-byte K-major operand rows, read the
// accumulator back (tcgen05.ld), multiply by W_L^(n2 k1) and write the values as column
// n2 of the stage-2 rows (l, k1); the operand's padded strides keep those column stores
// free of bank conflicts.  Stage 2: row (l, k1) comes back as X[k1 + R k2] and goes
// straight to global memory, consecutive lanes on consecutive k1.
//
// Precision: tf32 keeps 11 significant bits.  Every operand is split as hi = tf32(v)
// rounded to nearest and lo = v - hi (exact in FP32), which the tensor core reads
// rounded to nearest as well (half an ulp added, the low 13 bits ignored): about 22
// significant bits.  The product is hi*hi + lo*hi + hi*lo accumulated in FP32; lo*lo
// is 2^-22 of it.  tf32 has FP32's exponent range, so no vector needs scaling.  The
// DFT matrices (split the same way) and the twiddles are FP64-generated once a device
// and rounded once; the twiddle multiply runs in FP32 on the CUDA cores.  The inverse
// transform uses the conjugate tables instead of conjugating data.
//
// The grid is persistent: two CTAs of 512 threads an SM (R = 32, four threads a row)
// or four of 256 (R = 16, two a row); a thread prefetches the next tile's input into
// registers while the current tile is on the tensor cores.  Tensor memory (2R columns)
// is allocated once a CTA and freed before exit, also after a timed-out wait (after a
// second bounded wait for the products in flight); every wait is clock-bounded.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "rk_async.cuh"
#include "rk_internal.h"

namespace rk {

namespace {

template <int R, int TPR = 2>
struct TcCfg {
    static constexpr int L = R * R;
    static constexpr int ROWS = 128;         // rows of a product = tensor-memory lanes
    static constexpr int NT = 32 * 4 * TPR;  // TPR threads a row (parts of its columns)
    static constexpr int LINES = ROWS / R;   // lines a tile
    static constexpr int K = 2 * R;          // reals a vector (and output reals)
    static constexpr int H = R / TPR;        // complex values a thread holds of a row
    // A operand, K-major, no swizzle: core matrices of 8 rows x 4 K (16 bytes),
    // K-adjacent core matrices A_LBO apart, 8-row groups A_SBO apart.  A_LBO = 144
    // (not 128) spreads the eight 16-byte chunks of one row over all 32 banks (the
    // stage-2 column stores of a warp hit one row); for R = 16 a warp stores into two
    // rows 16 apart, which the extra 32 bytes of A_SBO put on the other 16 banks.
    static constexpr int A_LBO = 144;
    static constexpr int A_SBO = (K / 4) * A_LBO + (R == 16 ? 32 : 0);
    static constexpr int A_BYTES = (ROWS / 8) * A_SBO;
    // B operand, K-major, no swizzle: K-adjacent core matrices 128 bytes apart (LBO),
    // 8-row groups B_SBO apart
    static constexpr int B_SBO = (K / 4) * 128;
    static constexpr int B_BYTES = (K / 8) * B_SBO;
    static constexpr int TWLD = R + 1;       // padded twiddle row (conflict-free column reads)
    static constexpr int TW_BYTES = R * TWLD * 8;
    static constexpr int TAB_BYTES = 2 * B_BYTES + TW_BYTES;  // B hi | B lo | twiddles
    static constexpr int OFF_TAB = 2 * A_BYTES;               // A hi | A lo | tables | barrier
    static constexpr int OFF_TW = OFF_TAB + 2 * B_BYTES;
    static constexpr int OFF_BAR = OFF_TAB + TAB_BYTES;
    static constexpr int SMEM = OFF_BAR + 16;
    static constexpr int MINB = TPR == 4 ? 2 : (R == 32 ? 2 : 4);
    static_assert(H % 4 == 0, "a thread's part of a row is whole 16-byte operand chunks");
    // instruction descriptor: D f32, A and B tf32, both K-major, N = 2R, M = 128
    static constexpr uint32_t IDESC =
        (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(K >> 3) << 17) | ((128u >> 4) << 24);
    static_assert(TAB_BYTES % 16 == 0 && A_BYTES % 16 == 0 && OFF_BAR % 16 == 0, "16-byte operand grid");
    static_assert(ROWS % R == 0 && R % 8 == 0, "tile shape");
};

// FP64-generated tables a direction (0 forward, 1 inverse), in the shared-memory image
// the kernel copies: B hi, B lo (operand layout), twiddles W_L^(n2 k1) at [n2][k1]
__device__ __align__(16) unsigned char g_tc16[2][TcCfg<16>::TAB_BYTES];
__device__ __align__(16) unsigned char g_tc32[2][TcCfg<32>::TAB_BYTES];

template <int R>
__device__ __forceinline__ const unsigned char* tc_tab(int dir) {
    if constexpr (R == 16)
        return g_tc16[dir];
    else
        return g_tc32[dir];
}

// byte offset of element (row m, column k) of the K-major A operand
template <int R>
__host__ __device__ constexpr uint32_t a_off(int m, int k) {
    return (uint32_t)((m >> 3) * TcCfg<R>::A_SBO + (k >> 2) * TcCfg<R>::A_LBO + (m & 7) * 16 + (k & 3) * 4);
}

// byte offset of element (row j, column k) of the K-major B operand
template <int R>
__host__ __device__ constexpr uint32_t b_off(int j, int k) {
    return (uint32_t)((j >> 3) * TcCfg<R>::B_SBO + (k >> 2) * 128 + (j & 7) * 16 + (k & 3) * 4);
}

// tf32 rounded to nearest (ties away from zero), low 13 bits cleared: the value the
// tensor core reads
__device__ __forceinline__ uint32_t tf32_hi(float v) { return (__float_as_uint(v) + 0x1000u) & 0xFFFFE000u; }

// split four values into hi / lo and store them as one 16-byte chunk of each operand
template <int R>
__device__ __forceinline__ void put_split(unsigned char* a, uint32_t off, float v0, float v1, float v2, float v3) {
    const uint32_t h0 = tf32_hi(v0), h1 = tf32_hi(v1), h2 = tf32_hi(v2), h3 = tf32_hi(v3);
    // the tensor core ignores the low 13 bits: half an ulp added rounds lo to nearest
    const uint32_t l0 = __float_as_uint(v0 - __uint_as_float(h0)) + 0x1000u;
    const uint32_t l1 = __float_as_uint(v1 - __uint_as_float(h1)) + 0x1000u;
    const uint32_t l2 = __float_as_uint(v2 - __uint_as_float(h2)) + 0x1000u;
    const uint32_t l3 = __float_as_uint(v3 - __uint_as_float(h3)) + 0x1000u;
    *reinterpret_cast<uint4*>(a + off) = make_uint4(h0, h1, h2, h3);
    *reinterpret_cast<uint4*>(a + TcCfg<R>::A_BYTES + off) = make_uint4(l0, l1, l2, l3);
}

// one value split into hi / lo, stored as single elements of each operand
template <int R>
__device__ __forceinline__ void put_split1(unsigned char* a, uint32_t off, float v) {
    const uint32_t h = tf32_hi(v);
    *reinterpret_cast<uint32_t*>(a + off) = h;
    *reinterpret_cast<uint32_t*>(a + TcCfg<R>::A_BYTES + off) = __float_as_uint(v - __uint_as_float(h)) + 0x1000u;
}

// shared-memory matrix descriptor, no swizzle (sm_100 descriptor version 1)
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46);
}

template <uint32_t IDESC>
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(IDESC), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// N consecutive accumulator columns of this thread's lane into r (N = 4, 8 or 16);
// the registers hold the values only after tcgen05.wait::ld
template <int N>
__device__ __forceinline__ void tc_ldn(uint32_t taddr, uint32_t* r) {
    if constexpr (N == 16) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
            "%14, %15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr)
            : "memory");
    } else if constexpr (N == 8) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                       "=r"(r[7])
                     : "r"(taddr)
                     : "memory");
    } else {
        static_assert(N == 4, "4, 8 or 16 columns");
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                     : "r"(taddr)
                     : "memory");
    }
}

// this thread's part of its accumulator row: columns [c0, c0 + H) (real parts) and
// [R + c0, R + c0 + H) (imaginary parts), read only after the wait
template <int R, int H>
__device__ __forceinline__ void tc_ld_part(uint32_t taddr, int c0, float* re, float* im) {
    uint32_t a[H], b[H];
    tc_ldn<H>(taddr + c0, a);
    tc_ldn<H>(taddr + R + c0, b);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < H; ++i) {
        re[i] = __uint_as_float(a[i]);
        im[i] = __uint_as_float(b[i]);
    }
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// xconj bit 0: conjugate the input, bit 1: the output (only when exactly one side
// conjugates; both together run the inverse tables)
template <int R, int TPR>
__global__ void __launch_bounds__(TcCfg<R, TPR>::NT, TcCfg<R, TPR>::MINB)
    k_tc(const __grid_constant__ PassParams p, int dir, int xconj) {
    using C = TcCfg<R, TPR>;
    constexpr int L = C::L, H = C::H;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int t = threadIdx.x, warp = t >> 5;
    // this thread's row (= tensor-memory lane: warp w reaches lanes 32 (w mod 4) ..)
    // and its part of the row's columns
    const int row = (warp & 3) * 32 + (t & 31), c0 = (warp >> 2) * H;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + C::OFF_BAR);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + C::OFF_BAR + 8);
    const uint32_t sbase = smem_u32(sm);

    {
        const uint4* g = reinterpret_cast<const uint4*>(tc_tab<R>(dir));
        uint4* s = reinterpret_cast<uint4*>(sm + C::OFF_TAB);
        for (int i = t; i < C::TAB_BYTES / 16; i += C::NT) s[i] = g[i];
    }
    if (t == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(C::K)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);

    const Side& ld = p.ld;
    const Side& st = p.st;
    const bool ld_scale = ld.flags & SF_SCALE, st_scale = st.flags & SF_SCALE;
    const float2 lsc = make_float2((float)ld.scale_re, (float)ld.scale_im);
    const float2 ssc = make_float2((float)st.scale_re, (float)st.scale_im);
    const float2* src = reinterpret_cast<const float2*>(ld.ptr) + ld.offset;
    float2* dst = reinterpret_cast<float2*>(st.ptr) + st.offset;
    const int64_t nlines = p.nlines;
    const int64_t ntiles = (nlines + C::LINES - 1) / C::LINES;
    const int l = row / R, rr = row % R;   // stage 1: rr = n2; stage 2: rr = k1

    // operand offsets as a thread base plus compile-time steps (l R + c0 is a multiple
    // of 8, or of 4 with H = 4, so row l R + c0 + i stays in the base's 8-row group
    // for i < 8 and H = 4 alike; c0 is a multiple of 4): stage 1 writes row `row`, columns c0 + 4c (real) and
    // R + c0 + 4c (imaginary); stage 2 writes rows l R + c0 + i, columns rr and R + rr
    constexpr uint32_t IM = (uint32_t)(R / 4) * C::A_LBO;  // column k -> k + R
    const uint32_t base1 = a_off<R>(row, c0);
    const uint32_t base2 = a_off<R>(l * R + c0, rr);
    auto step2 = [](int i) -> uint32_t { return (uint32_t)((i >> 3) * C::A_SBO + (i & 7) * 16); };

    // stage-1 input of this thread: x[l][R n1 + n2], n1 = c0 .. c0 + H - 1
    float2 x[H];
    auto load = [&](int64_t tile) {
        const int64_t line = tile * C::LINES + l;
        const bool in = line < nlines;
        const float2* s = src + line * L + rr + R * c0;
#pragma unroll
        for (int i = 0; i < H; ++i) x[i] = in ? s[R * i] : make_float2(0.f, 0.f);
    };

    // MMA of one stage: every thread's operand stores are visible to the tensor core,
    // then thread 0 issues the K / 8 steps of lo*hi + hi*lo, then those of hi*hi (the
    // small terms summed first, so the large ones take the fewest accumulation steps),
    // and commits them
    auto issue = [&]() {
        if (t == 0) {
            tc_fence_after();
            auto ad = [&](int part, int s) {
                return tc_desc(sbase + part * C::A_BYTES + 2 * s * C::A_LBO, C::A_LBO, C::A_SBO);
            };
            auto bd = [&](int part, int s) {
                return tc_desc(sbase + C::OFF_TAB + part * C::B_BYTES + s * 256, 128, C::B_SBO);
            };
#pragma unroll
            for (int s = 0; s < C::K / 8; ++s) {
                tc_mma<C::IDESC>(tmem, ad(1, s), bd(0, s), s > 0);
                tc_mma<C::IDESC>(tmem, ad(0, s), bd(1, s), 1);
            }
#pragma unroll
            for (int s = 0; s < C::K / 8; ++s) tc_mma<C::IDESC>(tmem, ad(0, s), bd(0, s), 1);
            tc_commit(bar);
        }
    };

    uint32_t phase = 0;
    bool ok = true;
    if (blockIdx.x < ntiles) load(blockIdx.x);
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        // ---- stage 1: A row (l, n2), column n1 (real) / R + n1 (imaginary) ----
#pragma unroll
        for (int c = 0; c < H / 4; ++c) {
            float re[4], im[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                float2 u = x[4 * c + i];
                if (ld_scale) u = cmulf(u, lsc);
                if (xconj & 1) u.y = -u.y;
                re[i] = u.x;
                im[i] = u.y;
            }
            put_split<R>(sm, base1 + c * C::A_LBO, re[0], re[1], re[2], re[3]);
            put_split<R>(sm, base1 + c * C::A_LBO + IM, im[0], im[1], im[2], im[3]);
        }
        fence_proxy_async_smem();
        tc_fence_before();
        // every thread leaves together when any wait ran out
        if (!__syncthreads_and(ok)) break;
        issue();
        ok = mbar_wait(bar, phase, p.status);
        phase ^= 1;
        tc_fence_after();
        {
            // row (l, n2): Y[k1] at columns k1 (real) and R + k1 (imaginary)
            float re[H], im[H];
            tc_ld_part<R, H>(trow, c0, re, im);
            const float2* tw = reinterpret_cast<const float2*>(sm + C::OFF_TW) + rr * C::TWLD + c0;
            // ---- stage 2: A row (l, k1), column n2 (real) / R + n2 (imaginary) ----
#pragma unroll
            for (int i = 0; i < H; ++i) {
                const float2 u = cmulf(make_float2(re[i], im[i]), tw[i]);
                put_split1<R>(sm, base2 + step2(i), u.x);
                put_split1<R>(sm, base2 + step2(i) + IM, u.y);
            }
        }
        fence_proxy_async_smem();
        tc_fence_before();
        if (!__syncthreads_and(ok)) break;
        issue();
        // the next tile's input: issued here, after the last proxy fence of this tile
        // (the fence would wait for loads in flight), used by the next stage 1
        if (tile + gridDim.x < ntiles) load(tile + gridDim.x);
        ok = mbar_wait(bar, phase, p.status);
        phase ^= 1;
        tc_fence_after();
        {
            // row (l, k1): X[k1 + R k2] at columns k2 and R + k2
            float re[H], im[H];
            tc_ld_part<R, H>(trow, c0, re, im);
            const int64_t line = tile * C::LINES + l;
            if (ok && line < nlines) {
                float2* o = dst + line * L + rr + R * c0;
#pragma unroll
                for (int i = 0; i < H; ++i) {
                    float2 y = make_float2(re[i], im[i]);
                    if (xconj & 2) y.y = -y.y;
                    if (st_scale) y = cmulf(y, ssc);
                    o[R * i] = y;
                }
            }
        }
        tc_fence_before();
    }
    // after a timed-out wait the last committed products may still be running: wait for
    // their commit once more (bounded) before the tensor memory they write is freed
    if (!ok) mbar_wait(bar, phase ^ 1, p.status);
    // all tensor-memory reads are done (or abandoned after a timed-out wait)
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::K) : "memory");
}

// tf32 rounded to nearest, as a float (host and device)
__host__ __device__ inline float tf32_round(float v) {
    uint32_t b;
    memcpy(&b, &v, 4);
    b = (b + 0x1000u) & 0xFFFFE000u;
    float r;
    memcpy(&r, &b, 4);
    return r;
}

template <int R>
__global__ void k_tc_tables(unsigned char* tab, int inv) {
    using C = TcCfg<R>;
    constexpr int K = C::K, L = C::L;
    float* bhi = reinterpret_cast<float*>(tab);
    float* blo = reinterpret_cast<float*>(tab + C::B_BYTES);
    float2* tw = reinterpret_cast<float2*>(tab + 2 * C::B_BYTES);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < K * K) {
        // B[j][k]: output real j (k1 = j mod R, imaginary if j >= R) from input real k
        // (n1 = k mod R); forward Y = X (c - i s): Yr = Xr c + Xi s, Yi = Xi c - Xr s
        const int j = i / K, k = i % K;
        const int m = ((j % R) * (k % R)) % R;
        double s, c;
        sincospi(2.0 * m / R, &s, &c);
        if (inv) s = -s;
        const bool jim = j >= R, kim = k >= R;
        const double v = jim == kim ? c : (kim ? s : -s);
        const float hi = tf32_round((float)v);
        const float lo = tf32_round((float)(v - (double)hi));
        bhi[b_off<R>(j, k) / 4] = hi;
        blo[b_off<R>(j, k) / 4] = lo;
    }
    if (i < R * C::TWLD) {
        const int n2 = i / C::TWLD, k1 = i % C::TWLD;
        float2 w = make_float2(0.f, 0.f);
        if (k1 < R) {
            double s, c;
            sincospi(2.0 * (double)(n2 * k1) / L, &s, &c);
            w = make_float2((float)c, (float)(inv ? s : -s));
        }
        tw[i] = w;
    }
}

template <int R>
cudaError_t gen_tables(unsigned char (*tab)[TcCfg<R>::TAB_BYTES]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, *tab);
    if (e != cudaSuccess) return e;
    constexpr int n = std::max(TcCfg<R>::K * TcCfg<R>::K, R * TcCfg<R>::TWLD);
    for (int dir = 0; dir < 2; ++dir)
        k_tc_tables<R><<<(n + 255) / 256, 256>>>(static_cast<unsigned char*>(p) + dir * TcCfg<R>::TAB_BYTES, dir);
    return cudaGetLastError();
}

template <int R, int TPR>
cudaError_t launch_tc(const PassParams& p, int dir, int xconj, cudaStream_t st) {
    using C = TcCfg<R, TPR>;
    static std::mutex mu;
    static int grid_by_dev[64] = {0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    int grid;
    {
        std::lock_guard<std::mutex> lk(mu);
        grid = grid_by_dev[dev];
        if (grid == 0) {
            e = cudaFuncSetAttribute(k_tc<R, TPR>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
            if (e != cudaSuccess) return e;
            // the whole unified L1 as shared memory: two (R = 32) CTAs an SM need it
            e = cudaFuncSetAttribute(k_tc<R, TPR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared);
            if (e != cudaSuccess) return e;
            // resident CTAs an SM: shared memory (1 KB reserved a CTA), registers (a
            // warp's allocation rounded to 256), threads, and the SM's 512 tensor-memory
            // columns (2R a CTA); the occupancy query reports one CTA where two fit
            cudaFuncAttributes fa;
            e = cudaFuncGetAttributes(&fa, k_tc<R, TPR>);
            if (e != cudaSuccess) return e;
            int nsm = 0, smem_sm = 0;
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
            const int warp_regs = ((fa.numRegs * 32 + 255) / 256) * 256;
            const int per_sm = std::max(1, std::min({smem_sm / (C::SMEM + 1024), 65536 / (warp_regs * (C::NT / 32)),
                                                     2048 / C::NT, 512 / C::K}));
            grid = grid_by_dev[dev] = per_sm * nsm;
        }
    }
    const int64_t ntiles = (p.nlines + C::LINES - 1) / C::LINES;
    if (ntiles <= 0) return cudaSuccess;
    const int g = (int)std::min<int64_t>(grid, ntiles);
    k_tc<R, TPR><<<g, C::NT, C::SMEM, st>>>(p, dir, xconj);
    return cudaGetLastError();
}

}  // namespace

bool tc_eligible(const PassRec& r) {
    const PassParams& p = r.prm;
    if (r.dbl || r.kind != PK_LINE || (r.L != 256 && r.L != 1024) || r.mode != MODE_POS || r.var != 0) return false;
    if (p.C != 1 || p.I != 1) return false;
    for (const Side* s : {&p.ld, &p.st}) {
        if (!(s->flags & SF_FAST) || s->ax_stride != 1 || s->ax_shift != 0 || s->nd_i != 0) return false;
        if (s->flags & ~(SF_FAST | SF_FAST2 | SF_SCALE | SF_PRE_CONJ | SF_POST_CONJ)) return false;
        if (s->nd_o > 1) return false;
        if (s->nd_o == 1 && (s->o_stride[0] != r.L || s->o_shift[0] != 0 || s->o_bound[0] != s->o_shape[0]))
            return false;
    }
    return true;
}

cudaError_t tc_prepare() {
    static std::mutex mu;
    static bool ready[64] = {false};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    if (ready[dev]) return cudaSuccess;
    if ((e = gen_tables<16>(&g_tc16[0])) != cudaSuccess) return e;
    if ((e = gen_tables<32>(&g_tc32[0])) != cudaSuccess) return e;
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return e;
    ready[dev] = true;
    return cudaSuccess;
}

cudaError_t tc_launch(const PassParams& p, int L, cudaStream_t st) {
    const bool lc = ((p.ld.flags & SF_PRE_CONJ) != 0) != ((p.ld.flags & SF_POST_CONJ) != 0);
    const bool sc = ((p.st.flags & SF_PRE_CONJ) != 0) != ((p.st.flags & SF_POST_CONJ) != 0);
    // conj(F(conj(a x))) = a F^-1 x: both sides conjugating is the inverse transform
    const int dir = lc && sc ? 1 : 0;
    const int xconj = dir ? 0 : (lc ? 1 : 0) | (sc ? 2 : 0);
    // threads a row: 4 for 1024-point lines (32 warps an SM: 83.8 us against 87.6 with
    // 2 on 16384 lines), 2 for 256-point ones (70.8 us against 76.6 with 4 on 65536)
    if (L == 1024) return launch_tc<32, 4>(p, dir, xconj, st);
    if (L == 256) return launch_tc<16, 2>(p, dir, xconj, st);
    return cudaErrorInvalidValue;
}

}  // namespace rk
