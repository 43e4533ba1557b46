// Tensor-core split-precision line pass for 1024-point complex64 transforms along a
// contiguous axis (the precision mode, RK_FLAG_SPLIT_TC).
//
// A 1024-point DFT is taken as 16 x 16 x 4: two radix-16 stages on the tensor cores
// and a radix-4 stage on the CUDA cores.  A radix-16 DFT of 128 vectors is one
// 128 x 32 x 32 real matrix product: the rows are the vectors (real parts then
// imaginary parts, K = 32), the 32 x 32 matrix is the real form of the 16-point DFT
// matrix, and the 32 output columns are the real and imaginary parts of the result.
//
// Precision: every operand is split as hi + lo with hi = fp16(v) and lo = fp16(v -
// hi), which keeps about 22 significant bits; the product is hi*hi + lo*hi + hi*lo
// accumulated in FP32 in tensor memory (lo*lo is below FP32 rounding of the sum).
// Each vector is first scaled by a power of two that brings its largest component to
// [2^14, 2^15), so fp16's range holds it, and the result is scaled back exactly.
// Twiddles are FP64-generated and rounded once to FP32; they and the radix-4 stage
// run in FP32 on the CUDA cores.
//
// Per tile of two lines (2048 points) the CTA's 128 threads each own one row of the
// matrix product: they convert their vector into the hi / lo operand tiles (the
// no-swizzle K-major canonical layout of the UMMA shared-memory descriptor), one
// elected thread issues the six tcgen05.mma of a stage and commits them to an
// mbarrier, and every thread reads its row of the FP32 accumulator back from tensor
// memory with tcgen05.ld.  The grid is persistent; tensor memory (32 columns) is
// allocated once per CTA and freed before exit, also after a timed-out wait.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "rk_async.cuh"
#include "rk_internal.h"
#include "rk_kernels.cuh"

namespace rk {

namespace {

constexpr int TC_NT = 128;     // threads = rows of one matrix product
constexpr int TC_L = 1024;
constexpr int TC_LINES = 2;    // lines per tile (2 x 64 vectors of 16 per stage)

struct __align__(128) TcSmem {
    __half a_hi[TC_NT * 32];   // 8 KB each, canonical K-major layout
    __half a_lo[TC_NT * 32];
    __half b_hi[32 * 32];
    __half b_lo[32 * 32];
    float2 in[TC_LINES * TC_L];  // next tile's input, fetched by a bulk copy
    float2 tw[TC_L];           // stage twiddles of the 1024-point plan (TwLayout order)
    uint64_t bar;              // matrix products done
    uint64_t inbar;            // input tile landed
    uint32_t tmem;
};

// Between the two stages the 2 x 16 x 64 intermediate X1[line][k1][n2] is exchanged
// through the operand tiles (a_hi and a_lo, 16 KB together), which are free once the
// first stage's products are done; column n2 of row (line, k1) sits at n2 ^ 4 (k1 & 7)
// so that both the stage-1 writes and the stage-2 reads spread over the banks.
__device__ __forceinline__ float2* xbuf(TcSmem& S) { return reinterpret_cast<float2*>(S.a_hi); }
__device__ __forceinline__ int x_idx(int row, int col) { return row * 64 + (col ^ ((row & 7) << 2)); }

// element (row r, column k) of a 32-column operand in the no-swizzle K-major layout:
// 8 x 8 core matrices of 128 contiguous bytes, K-adjacent ones 128 bytes apart (LBO),
// row-adjacent ones 512 bytes apart (SBO)
__device__ __forceinline__ int op_idx(int r, int k) { return (r >> 3) * 256 + (k >> 3) * 64 + (r & 7) * 8 + (k & 7); }

__device__ __forceinline__ uint64_t smem_desc(const void* p) {
    const uint64_t addr = smem_u32(p);
    return ((addr >> 4) & 0x3FFF) | (uint64_t(128 >> 4) << 16) | (uint64_t(512 >> 4) << 32) | (uint64_t(1) << 46);
}

// kind::f16 instruction descriptor: D f32, A and B f16, both K-major, N = 32, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (0u << 7) | (0u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(TC_IDESC), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// this thread's 32 accumulator columns (its row = its tensor-memory lane)
__device__ __forceinline__ void tc_ld_row(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// scale the 16-point vector u to [2^14, 2^15) at its largest component, split it into
// hi / lo fp16 rows of the operand tiles; returns the exponent to undo
__device__ __forceinline__ int tc_put_row(TcSmem& S, int row, const float2* u) {
    float m = 0.f;
#pragma unroll
    for (int j = 0; j < 16; ++j) m = fmaxf(m, fmaxf(fabsf(u[j].x), fabsf(u[j].y)));
    // exponent field of m (zero and subnormals read as -127); the clamp keeps both
    // 2^e and 2^-e normal floats, so scaling by them is exact
    const int e = m > 0.f ? min(125, max(-125, 14 - ((__float_as_int(m) >> 23) - 127))) : 0;
    const float f = __int_as_float((127 + e) << 23);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        // column chunk c holds k = 8c .. 8c+7: real parts (c < 2) or imaginary parts;
        // pairs convert with one f16x2 rounding each
        __align__(16) __half2 hi[4], lo[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int j = (c & 1) * 8 + 2 * i;
            const float2 v = c < 2 ? make_float2(u[j].x * f, u[j + 1].x * f) : make_float2(u[j].y * f, u[j + 1].y * f);
            hi[i] = __float22half2_rn(v);
            const float2 h = __half22float2(hi[i]);
            lo[i] = __float22half2_rn(make_float2(v.x - h.x, v.y - h.y));
        }
        *reinterpret_cast<uint4*>(&S.a_hi[op_idx(row, 8 * c)]) = *reinterpret_cast<const uint4*>(hi);
        *reinterpret_cast<uint4*>(&S.a_lo[op_idx(row, 8 * c)]) = *reinterpret_cast<const uint4*>(lo);
    }
    return e;
}

// one radix-16 stage of the 128 rows: split products into tensor memory, then this
// thread's row back, scaled by 2^-e; false if the wait ran out
__device__ __forceinline__ bool tc_stage(TcSmem& S, uint32_t tmem, uint32_t& phase, int e, float2* y,
                                         int32_t* status, const float2* next = nullptr, uint32_t next_bytes = 0) {
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0 && next_bytes) {
        // every thread has read the input buffer: fetch the next tile into it
        mbar_arrive_expect_tx(&S.inbar, next_bytes);
        bulk_g2s(S.in, next, next_bytes, &S.inbar);
    }
    if (threadIdx.x == 0) {
        tc_fence_after();
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            // K step s covers operand columns 16 s .. 16 s + 15 (two 128-byte chunks)
            const uint64_t ah = smem_desc(&S.a_hi[s * 128]), al = smem_desc(&S.a_lo[s * 128]);
            const uint64_t bh = smem_desc(&S.b_hi[s * 128]), bl = smem_desc(&S.b_lo[s * 128]);
            tc_mma(tmem, ah, bh, s > 0);
            tc_mma(tmem, al, bh, 1);
            tc_mma(tmem, ah, bl, 1);
        }
        tc_commit(&S.bar);
    }
    bool ok = mbar_wait(&S.bar, phase, status);
    phase ^= 1;
    // every thread leaves together when any wait ran out
    ok = __syncthreads_and(ok);
    if (!ok) return false;
    tc_fence_after();
    float v[32];
    const uint32_t warp = threadIdx.x >> 5;
    tc_ld_row(tmem + ((warp * 32) << 16), v);
    const float g = __int_as_float((127 - e) << 23);
#pragma unroll
    for (int q = 0; q < 16; ++q) y[q] = make_float2(v[q] * g, v[16 + q] * g);
    return true;
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void __launch_bounds__(TC_NT) k_tc1024(const __grid_constant__ PassParams p) {
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>(tc_smem_raw);
    const int t = threadIdx.x;
    const int warp = t >> 5;

    // the FP64-generated stage twiddles of the pass (stage 0: W_1024^(n2 k1) at
    // [k1 - 1][n2]; stage 1: W_64^(m2 q1) at 960 + [q1 - 1][m2]) and the real 32 x 32
    // DFT-16 matrix B[n][k] (K-major) as hi / lo
    static_assert(Radix<float, TC_L>::NS == 3 && Radix<float, TC_L>::R[0] == 16 && Radix<float, TC_L>::R[1] == 16 &&
                      Radix<float, TC_L>::R[2] == 4 && TwLayout<float, TC_L>::total() == 1020,
                  "the tensor-core pass follows the 16 x 16 x 4 plan of 1024-point lines");
    const float2* stw = reinterpret_cast<const float2*>(p.tw);
    for (int e = t; e < TC_L; e += TC_NT) {
        if (e < 1020) S.tw[e] = stw[e];
        const int n = e >> 5, k = e & 31;
        const int m = ((k & 15) * (n & 15)) & 15;
        double sv, cv;
        sincospi(m / 8.0, &sv, &cv);
        // Y = X W_16^(jq):  Yr = Xr c + Xi s,  Yi = Xi c - Xr s
        const double v = ((k < 16) == (n < 16)) ? cv : (k < 16 ? -sv : sv);
        const __half hi = __double2half(v);
        S.b_hi[op_idx(n, k)] = hi;
        S.b_lo[op_idx(n, k)] = __double2half(v - (double)__half2float(hi));
    }
    if (t == 0) {
        mbar_init(&S.bar, 1);
        mbar_init(&S.inbar, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(smem_u32(&S.tmem))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = S.tmem;

    const Side& ld = p.ld;
    const Side& st = p.st;
    const bool ld_scale = ld.flags & SF_SCALE, st_scale = st.flags & SF_SCALE;
    const bool ld_conj = ((ld.flags & SF_PRE_CONJ) != 0) != ((ld.flags & SF_POST_CONJ) != 0);
    const bool st_conj = ((st.flags & SF_PRE_CONJ) != 0) != ((st.flags & SF_POST_CONJ) != 0);
    const float2 lsc = make_float2((float)ld.scale_re, (float)ld.scale_im);
    const float2 ssc = make_float2((float)st.scale_re, (float)st.scale_im);
    const float2* src = reinterpret_cast<const float2*>(ld.ptr) + ld.offset;
    float2* dst = reinterpret_cast<float2*>(st.ptr) + st.offset;
    const int64_t ntiles = (p.nlines + TC_LINES - 1) / TC_LINES;
    uint32_t phase = 0, iphase = 0;
    // input tiles come by bulk copy when the array sits on the 16-byte grid the copy
    // needs, else by plain loads
    const bool bulk = (reinterpret_cast<uintptr_t>(src) & 15) == 0;
    auto tile_bytes = [&](int64_t tile) -> uint32_t {
        if (tile >= ntiles) return 0;
        const int64_t lines = std::min<int64_t>(TC_LINES, p.nlines - tile * TC_LINES);
        return (uint32_t)(lines * TC_L * sizeof(float2));
    };
    bool pending = false;  // thread 0: a bulk copy is in flight
    if (bulk && t == 0 && blockIdx.x < ntiles) {
        pending = true;
        mbar_arrive_expect_tx(&S.inbar, tile_bytes(blockIdx.x));
        bulk_g2s(S.in, src + (int64_t)blockIdx.x * TC_LINES * TC_L, tile_bytes(blockIdx.x), &S.inbar);
    }

    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        // ---- stage 1: radix 16 over n1 of n = 64 n1 + n2; row t = (line, n2) ----
        {
            const int ll = t >> 6, n2 = t & 63;
            const int64_t line = tile * TC_LINES + ll;
            const bool ok = line < p.nlines;
            float2 u[16];
            if (bulk) {
                bool landed = mbar_wait(&S.inbar, iphase, p.status);
                if (landed) {
                    iphase ^= 1;
                    pending = false;
                }
                if (!__syncthreads_and(landed)) break;
#pragma unroll
                for (int j = 0; j < 16; ++j) u[j] = ok ? S.in[ll * TC_L + 64 * j + n2] : make_float2(0.f, 0.f);
            } else {
#pragma unroll
                for (int j = 0; j < 16; ++j) u[j] = ok ? src[line * TC_L + 64 * j + n2] : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                if (ld_scale) u[j] = cmulf(u[j], lsc);
                if (ld_conj) u[j].y = -u[j].y;
            }
            const int e = tc_put_row(S, t, u);
            float2 y[16];
            const int64_t nxt = tile + gridDim.x;
            if (t == 0) pending = bulk && tile_bytes(nxt) > 0;
            if (!tc_stage(S, tmem, phase, e, y, p.status, src + nxt * TC_LINES * TC_L, bulk ? tile_bytes(nxt) : 0))
                break;
            // twiddle W_1024^(n2 k1), then X1[line][k1][n2] to the exchange buffer
#pragma unroll
            for (int k1 = 0; k1 < 16; ++k1)
                xbuf(S)[x_idx(ll * 16 + k1, n2)] = k1 ? cmulf(y[k1], S.tw[(k1 - 1) * 64 + n2]) : y[0];
        }
        tc_fence_before();
        __syncthreads();
        // ---- stage 2: radix 16 over m1 of n2 = 4 m1 + m2; row t = (line, k1, m2) ----
        {
            const int ll = t >> 6, k1 = (t >> 2) & 15, m2 = t & 3;
            float2 u[16];
#pragma unroll
            for (int m1 = 0; m1 < 16; ++m1) u[m1] = xbuf(S)[x_idx(ll * 16 + k1, 4 * m1 + m2)];
            __syncthreads();  // the exchange buffer becomes the operand tiles again
            const int e = tc_put_row(S, t, u);
            float2 y[16];
            if (!tc_stage(S, tmem, phase, e, y, p.status)) break;
            // twiddle W_64^(m2 q1), then radix 4 over m2 through the (now free)
            // operand tiles: row (line, k1) holds V_m2[q1] at column 4 q1 + m2; this
            // thread then takes q1 = 4 m2 + i (i < 4) for all m2' and computes
            //   Z[q1 + 16 q2] = sum_m2' V_m2'[q1] (-i)^(m2' q2),  q2 = 0 .. 3
            const int row = ll * 16 + k1;
#pragma unroll
            for (int q1 = 0; q1 < 16; ++q1)
                xbuf(S)[x_idx(row, 4 * q1 + m2)] = q1 ? cmulf(y[q1], S.tw[960 + (q1 - 1) * 4 + m2]) : y[0];
            __syncthreads();
            const int64_t line = tile * TC_LINES + ll;
            const bool ok = line < p.nlines;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int q1 = 4 * m2 + i;
                float2 v[4];
#pragma unroll
                for (int mm = 0; mm < 4; ++mm) v[mm] = xbuf(S)[x_idx(row, 4 * q1 + mm)];
                // radix 4 with W_4 = -i
                const float2 a = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
                const float2 b = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
                const float2 c = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
                const float2 d = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
                float2 z[4];
                z[0] = make_float2(a.x + c.x, a.y + c.y);
                z[1] = make_float2(b.x + d.y, b.y - d.x);  // b - i d
                z[2] = make_float2(a.x - c.x, a.y - c.y);
                z[3] = make_float2(b.x - d.y, b.y + d.x);  // b + i d
#pragma unroll
                for (int q2 = 0; q2 < 4; ++q2) {
                    float2 o = z[q2];
                    if (st_conj) o.y = -o.y;
                    if (st_scale) o = cmulf(o, ssc);
                    if (ok) dst[line * TC_L + k1 + 16 * q1 + 256 * q2] = o;
                }
            }
        }
        tc_fence_before();
        __syncthreads();
    }
    // a copy still in flight after a timed-out wait lands before the CTA leaves
    if (pending) mbar_wait(&S.inbar, iphase, p.status);
    // all tensor-memory reads are done (or abandoned after a timed-out wait)
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
}

}  // namespace

bool tc_eligible(const PassRec& r) {
    const PassParams& p = r.prm;
    if (r.dbl || r.kind != PK_LINE || r.L != TC_L || r.mode != MODE_POS || r.var != 0) return false;
    if (p.C != 1 || p.I != 1) return false;
    for (const Side* s : {&p.ld, &p.st}) {
        if (!(s->flags & SF_FAST) || s->ax_stride != 1 || s->ax_shift != 0 || s->nd_i != 0) return false;
        if (s->flags & ~(SF_FAST | SF_FAST2 | SF_SCALE | SF_PRE_CONJ | SF_POST_CONJ)) return false;
        if (s->nd_o > 1) return false;
        if (s->nd_o == 1 && (s->o_stride[0] != TC_L || s->o_shift[0] != 0 || s->o_bound[0] != s->o_shape[0]))
            return false;
    }
    return true;
}

size_t tc_smem_bytes() { return sizeof(TcSmem) + 128; }

cudaError_t tc_launch(const PassParams& p, int64_t /*nblocks*/, cudaStream_t st) {
    static int grid = 0;
    const size_t smem = tc_smem_bytes();
    if (grid == 0) {
        cudaError_t e = cudaFuncSetAttribute(k_tc1024, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int nsm = 0, dev = 0, smem_sm = 0;
        cudaFuncAttributes fa;
        e = cudaFuncGetAttributes(&fa, k_tc1024);
        if (e != cudaSuccess) return e;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        // resident CTAs by shared memory (1 KB reserved a CTA) and registers; 32
        // tensor-memory columns a CTA: at most 16 CTAs of an SM can hold them
        const int by_smem = smem_sm / (int)(smem + 1024);
        const int by_regs = 65536 / std::max(1, fa.numRegs * TC_NT);
        grid = std::max(1, std::min({by_smem, by_regs, 16})) * nsm;
    }
    const int64_t ntiles = (p.nlines + TC_LINES - 1) / TC_LINES;
    if (ntiles <= 0) return cudaSuccess;
    const int g = (int)std::min<int64_t>(grid, ntiles);
    k_tc1024<<<g, TC_NT, smem, st>>>(p);
    return cudaGetLastError();
}

}  // namespace rk
