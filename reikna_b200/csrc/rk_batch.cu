// Persistent batched launch: many FFT plans of different lengths, axes and
// transformations in one kernel launch.
//
// The batch is a list of tasks (one task = one CTA tile of one pass) ordered by
// level: the first passes of every member, then the second passes, and so on.  A
// grid of at most one wave of resident CTAs pulls task indices from a global
// counter.  A task of pass k of a member first waits until every tile of pass k-1
// of the same member is done (per-pass completion counters, release/acquire at GPU
// scope).  Because tasks are handed out in order and every claimed task is running
// on a resident CTA, a waiting task only waits on tasks that are already executing:
// no deadlock.  Waits are clock-bounded and record a status bit instead of spinning
// forever.  The tile bodies are the same device code as the per-pass kernels
// (line_body), dispatched by a variant id; all batchable variants use 256 threads.
#include <cuda_runtime.h>
#include <string.h>

#include <string>
#include <vector>

#include "rk_async.cuh"
#include "rk_internal.h"
#include "rk_kernels.cuh"

namespace rk {

struct BatchPass {
    PassParams prm;
    int64_t nblocks;
    int32_t variant;
    int32_t dep;      // pass index that must be complete first, -1 = none
};

struct BatchTask {
    int32_t pass;
    int32_t pad;
    int64_t block;
};

struct BatchArgs {
    const BatchPass* passes;
    const BatchTask* tasks;
    int64_t ntasks;
    unsigned long long* next;
    unsigned long long* done;
    int32_t* status;
};

constexpr int BATCH_NT = 256;

__host__ __device__ constexpr int vid(int dbl, int var, int mode, int lg) {
    return (dbl << 12) | (var << 10) | (mode << 8) | lg;
}

template <typename T, int L, int MODE, int VAR>
__device__ __noinline__ void batch_body(const PassParams* p, int64_t block, unsigned char* smem) {
    static_assert(LineCfg<T, L, MODE>::NT == BATCH_NT, "batched variants run with 256 threads");
    line_body<T, L, MODE, VAR>(*p, block, smem, threadIdx.x);
}

#define RK_BV(TY, LL, MODE, VAR) \
    case vid(sizeof(TY) == 8, VAR, MODE, ilog2_b(LL)): batch_body<TY, LL, MODE, VAR>(p, block, smem); return true;

__host__ __device__ constexpr int ilog2_b(int n) { return n <= 1 ? 0 : 1 + ilog2_b(n / 2); }

__device__ bool batch_dispatch(int v, const PassParams* p, int64_t block, unsigned char* smem) {
    switch (v) {
        RK_BV(float, 1, MODE_POS, 0)
        RK_BV(float, 2, MODE_POS, 0)
        RK_BV(float, 4, MODE_POS, 0)
        RK_BV(float, 8, MODE_POS, 0)
        RK_BV(float, 16, MODE_POS, 0)
        RK_BV(float, 32, MODE_POS, 0)
        RK_BV(float, 64, MODE_POS, 0)
        RK_BV(float, 128, MODE_POS, 0)
        RK_BV(float, 256, MODE_POS, 0)
        RK_BV(float, 512, MODE_POS, 0)
        RK_BV(float, 1024, MODE_POS, 0)
        RK_BV(float, 2048, MODE_POS, 0)
        RK_BV(float, 4096, MODE_POS, 0)
        RK_BV(float, 8192, MODE_POS, 0)
        RK_BV(float, 16, MODE_LANE, 0)
        RK_BV(float, 32, MODE_LANE, 0)
        RK_BV(float, 64, MODE_LANE, 0)
        RK_BV(float, 128, MODE_LANE, 0)
        RK_BV(float, 256, MODE_LANE, 0)
        RK_BV(float, 64, MODE_POS, 1)
        RK_BV(float, 128, MODE_POS, 1)
        RK_BV(float, 256, MODE_POS, 1)
        RK_BV(float, 512, MODE_POS, 1)
        RK_BV(float, 1024, MODE_POS, 1)
        RK_BV(float, 2048, MODE_POS, 1)
        RK_BV(float, 4096, MODE_POS, 1)
        RK_BV(float, 8192, MODE_POS, 1)
        RK_BV(float, 64, MODE_LANE, 1)
        RK_BV(float, 128, MODE_LANE, 1)
        RK_BV(float, 256, MODE_LANE, 1)
        RK_BV(float, 16, MODE_POS, 2)
        RK_BV(float, 32, MODE_POS, 2)
        RK_BV(float, 64, MODE_POS, 2)
        RK_BV(float, 128, MODE_POS, 2)
        RK_BV(float, 256, MODE_POS, 2)
        RK_BV(float, 512, MODE_POS, 2)
        RK_BV(float, 1024, MODE_POS, 2)
        default:
            return false;
    }
}
#undef RK_BV

bool batch_variant(int dbl, int L, int mode, int var, int* out) {
    if (dbl || L < 1 || (L & (L - 1))) return false;
    const int lg = ilog2_b(L);
    bool ok = false;
    if (var == 0 && mode == MODE_POS) ok = L <= 8192;
    if (var == 0 && mode == MODE_LANE) ok = L >= 16 && L <= 256;
    if (var == 1 && mode == MODE_POS) ok = L >= 64 && L <= 8192;
    if (var == 1 && mode == MODE_LANE) ok = L >= 64 && L <= 256;
    if (var == 2) ok = mode == MODE_POS && L >= 16 && L <= 1024;
    if (ok) *out = vid(0, var, mode, lg);
    return ok;
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Each CTA holds at most two claimed tasks: the one it runs and the next one, claimed
// early so that the claim's latency hides behind the tile.  The lowest-index claimed
// task that is not done is always running (every task it depends on has a lower
// index, so it is done), hence the CTAs never wait on each other in a cycle.
// Registers are held to 128 (two CTAs an SM) for every tile body.
__global__ void __launch_bounds__(BATCH_NT, 2) k_batch(const BatchArgs a) {
    extern __shared__ __align__(16) unsigned char rk_smem[];
    __shared__ __align__(16) PassParams s_prm;
    __shared__ long long s_task[2];
    __shared__ int s_healthy;
    static_assert(sizeof(PassParams) % 16 == 0, "parameter copy moves 16-byte words");
    if (threadIdx.x == 0) {
        s_task[0] = (long long)atomicAdd(a.next, 1ull);
        s_healthy = 1;
    }
    __syncthreads();
    for (int cur = 0;; cur ^= 1) {
        const long long t = s_task[cur];
        if (t >= a.ntasks) break;
        if (threadIdx.x == 0) s_task[cur ^ 1] = (long long)atomicAdd(a.next, 1ull);
        const BatchTask tk = a.tasks[t];
        const BatchPass* bp = a.passes + tk.pass;
        // the pass parameters go to shared memory: the tile body reads them often
        const uint4* src = reinterpret_cast<const uint4*>(&bp->prm);
        uint4* dst = reinterpret_cast<uint4*>(&s_prm);
        for (int i = threadIdx.x; i < (int)(sizeof(PassParams) / 16); i += BATCH_NT) dst[i] = src[i];
        const int dep = bp->dep;
        if (dep >= 0 && threadIdx.x == 0) {
            const unsigned long long need = (unsigned long long)a.passes[dep].nblocks;
            bool ok = ld_acquire(a.done + dep) >= need;
            if (!ok && s_healthy) {
                const long long t0 = clock64(), lim = wait_limit(a.status);
                while (!(ok = ld_acquire(a.done + dep) >= need))
                    if (clock64() - t0 > lim) break;
            }
            if (!ok) {
                s_healthy = 0;
                atomicOr(a.status, RK_STATUS_TIMEOUT);
            }
        }
        __syncthreads();
        if (dep >= 0) __threadfence();
        // after a wait ran out the CTA's results are void (the status word says so):
        // it only marks its remaining tasks done, so nothing else waits on them
        if (s_healthy && !batch_dispatch(bp->variant, &s_prm, tk.block, rk_smem) && threadIdx.x == 0)
            atomicOr(a.status, RK_STATUS_BAD_VARIANT);
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(a.done + tk.pass, 1ull);
        }
    }
}

int build_call_params(rk_fft_plan* plan, void* const* outputs, int32_t n_outputs, const void* const* inputs,
                      int32_t n_inputs, int32_t inverse, const double* scalars, int32_t n_scalars, cudaStream_t st,
                      std::vector<PassParams>& out, std::vector<char>* tma_ok, const uint64_t* user_in = nullptr,
                      int32_t n_user_in = 0, const uint64_t* user_out = nullptr, int32_t n_user_out = 0);

}  // namespace rk

struct rk_batch {
    static constexpr int RING = 4;
    std::vector<rk_fft_plan*> plans;
    std::vector<int> first;                    // first batch pass of each member
    std::vector<rk::BatchPass> passes;         // host copy, pointers patched per call
    std::vector<rk::BatchTask> tasks;
    rk::BatchPass* d_passes = nullptr;
    rk::BatchTask* d_tasks = nullptr;
    unsigned long long* d_counters = nullptr;  // next + done[npasses]
    std::vector<rk::BatchPass> uploaded;       // what d_passes holds (empty: nothing yet)
    rk::BatchPass* h_pinned = nullptr;         // RING staging slots
    cudaEvent_t slot_ev[RING] = {};
    bool slot_used[RING] = {};
    int slot = 0;
    int grid = 0;
    size_t smem = 0;
    int device = 0;
};

using namespace rk;

extern "C" int rk_batch_create(rk_fft_plan* const* plans, int32_t nplans, rk_batch** out) {
    if (!plans || nplans < 1 || !out) {
        set_error("rk_batch_create: bad arguments");
        return RK_ERR_INVALID;
    }
    *out = nullptr;
    rk_batch* b = new rk_batch();
    auto fail = [&](int code, const std::string& msg) {
        set_error(msg);
        rk_batch_destroy(b);
        return code;
    };
    size_t smem = 0;
    int maxlevel = 0;
    for (int i = 0; i < nplans; ++i) {
        rk_fft_plan* p = plans[i];
        if (!p) return fail(RK_ERR_INVALID, "rk_batch_create: null plan");
        for (int j = 0; j < i; ++j)
            if (plans[j] == p)
                return fail(RK_ERR_INVALID, "rk_batch_create: a plan appears twice (its temporaries would be shared)");
        b->plans.push_back(p);
        maxlevel = std::max<int>(maxlevel, (int)p->passes.size());
        for (const PassRec& r : p->passes) {
            int v = 0;
            if (r.kind != PK_LINE || r.use_tc || r.user_bits || !batch_variant(r.dbl, r.L, r.mode, r.var, &v))
                return fail(RK_ERR_UNSUPPORTED, "rk_batch_create: pass '" + r.note + "' (L=" + std::to_string(r.L) +
                                                     ") has no batched variant");
            smem = std::max(smem, r.li.smem);
        }
    }
    // batch passes grouped by member; tasks ordered by level
    b->first.resize(nplans);
    for (int i = 0; i < nplans; ++i) {
        b->first[i] = (int)b->passes.size();
        const rk_fft_plan* p = plans[i];
        for (size_t k = 0; k < p->passes.size(); ++k) {
            const PassRec& r = p->passes[k];
            BatchPass bp;
            memset(&bp, 0, sizeof(bp));
            bp.prm = r.prm;
            bp.nblocks = (r.prm.nlines + r.li.nl - 1) / r.li.nl;
            int v = 0;
            batch_variant(r.dbl, r.L, r.mode, r.var, &v);
            bp.variant = v;
            bp.dep = k == 0 ? -1 : (int)b->passes.size() - 1;
            b->passes.push_back(bp);
        }
    }
    for (int lvl = 0; lvl < maxlevel; ++lvl)
        for (int i = 0; i < nplans; ++i)
            if (lvl < (int)plans[i]->passes.size()) {
                const int bpi = b->first[i] + lvl;
                for (int64_t blk = 0; blk < b->passes[bpi].nblocks; ++blk) b->tasks.push_back(BatchTask{bpi, 0, blk});
            }
    const size_t np = b->passes.size();
    if (cudaGetDevice(&b->device) != cudaSuccess) return fail(RK_ERR_CUDA, "rk_batch_create: no device");
    if (cudaMalloc(&b->d_passes, np * sizeof(BatchPass)) != cudaSuccess ||
        cudaMalloc(&b->d_tasks, b->tasks.size() * sizeof(BatchTask)) != cudaSuccess ||
        cudaMalloc(&b->d_counters, (np + 1) * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMallocHost(&b->h_pinned, rk_batch::RING * np * sizeof(BatchPass)) != cudaSuccess)
        return fail(RK_ERR_NOMEM, "rk_batch_create: allocation failed");
    for (int k = 0; k < rk_batch::RING; ++k)
        if (cudaEventCreateWithFlags(&b->slot_ev[k], cudaEventDisableTiming) != cudaSuccess)
            return fail(RK_ERR_CUDA, "rk_batch_create: event creation failed");
    if (cudaMemcpy(b->d_tasks, b->tasks.data(), b->tasks.size() * sizeof(BatchTask), cudaMemcpyHostToDevice) !=
        cudaSuccess)
        return fail(RK_ERR_CUDA, "rk_batch_create: task upload failed");
    b->smem = smem;
    if (cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return fail(RK_ERR_CUDA, "rk_batch_create: shared memory attribute failed");
    int per = 0, nsm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch, BATCH_NT, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess)
        return fail(RK_ERR_CUDA, "rk_batch_create: occupancy query failed");
    b->grid = std::max(1, std::min<int>((int)b->tasks.size(), std::max(1, per) * nsm));
    *out = b;
    return RK_OK;
}

extern "C" int rk_batch_execute(rk_batch* b, void* const* const* outputs, const void* const* const* inputs,
                                const int32_t* inverse, const double* const* scalars, const int32_t* n_scalars,
                                void* stream) {
    if (!b || !outputs || !inputs) {
        set_error("rk_batch_execute: bad arguments");
        return RK_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const size_t np = b->passes.size();
    std::vector<PassParams> prm;
    for (size_t i = 0; i < b->plans.size(); ++i) {
        rk_fft_plan* p = b->plans[i];
        const int nin = (p->desc.input.format == RK_FMT_F32_PAIR || p->desc.input.format == RK_FMT_F64_PAIR) ? 2 : 1;
        const int nout = (p->desc.output.format == RK_FMT_F32_PAIR || p->desc.output.format == RK_FMT_F64_PAIR) ? 2 : 1;
        prm.clear();
        const int rc = build_call_params(p, outputs[i], nout, inputs[i], nin, inverse ? inverse[i] : 0,
                                         scalars ? scalars[i] : nullptr, n_scalars ? n_scalars[i] : 0, st, prm,
                                         nullptr);
        if (rc) return rc;
        for (size_t k = 0; k < prm.size(); ++k) b->passes[b->first[i] + k].prm = prm[k];
    }
    // calls with the same pointers and scalars as the last upload skip it; a staging
    // slot is rewritten only after the upload that last read it is done
    cudaError_t e = cudaSuccess;
    if (b->uploaded.size() != np || memcmp(b->uploaded.data(), b->passes.data(), np * sizeof(BatchPass)) != 0) {
        const int k = b->slot;
        b->slot = (b->slot + 1) % rk_batch::RING;
        if (b->slot_used[k]) e = cudaEventSynchronize(b->slot_ev[k]);
        BatchPass* h = b->h_pinned + (size_t)k * np;
        if (e == cudaSuccess) {
            memcpy(h, b->passes.data(), np * sizeof(BatchPass));
            e = cudaMemcpyAsync(b->d_passes, h, np * sizeof(BatchPass), cudaMemcpyHostToDevice, st);
        }
        if (e == cudaSuccess) e = cudaEventRecord(b->slot_ev[k], st);
        if (e == cudaSuccess) {
            b->slot_used[k] = true;
            b->uploaded = b->passes;
        } else {
            b->uploaded.clear();
        }
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(b->d_counters, 0, (np + 1) * sizeof(unsigned long long), st);
    if (e != cudaSuccess) {
        set_error(std::string("rk_batch_execute: ") + cudaGetErrorString(e));
        return RK_ERR_CUDA;
    }
    DeviceTables* tabs = nullptr;
    int rc = device_tables(b->device, &tabs);
    if (rc) return rc;
    BatchArgs a;
    a.passes = b->d_passes;
    a.tasks = b->d_tasks;
    a.ntasks = (int64_t)b->tasks.size();
    a.next = b->d_counters;
    a.done = b->d_counters + 1;
    a.status = tabs->status;
    k_batch<<<b->grid, BATCH_NT, b->smem, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("rk_batch_execute: launch failed: ") + cudaGetErrorString(e));
        return RK_ERR_CUDA;
    }
    return RK_OK;
}

extern "C" int rk_batch_destroy(rk_batch* b) {
    if (!b) return RK_OK;
    for (int k = 0; k < rk_batch::RING; ++k)
        if (b->slot_ev[k]) {
            cudaEventSynchronize(b->slot_ev[k]);
            cudaEventDestroy(b->slot_ev[k]);
        }
    cudaFree(b->d_passes);
    cudaFree(b->d_tasks);
    cudaFree(b->d_counters);
    if (b->h_pinned) cudaFreeHost(b->h_pinned);
    delete b;
    return RK_OK;
}

extern "C" int rk_batch_info(const rk_batch* b, int64_t* ntasks, int32_t* npasses, int32_t* grid) {
    if (!b) {
        set_error("null batch");
        return RK_ERR_INVALID;
    }
    if (ntasks) *ntasks = (int64_t)b->tasks.size();
    if (npasses) *npasses = (int32_t)b->passes.size();
    if (grid) *grid = b->grid;
    return RK_OK;
}

extern "C" int rk_selftest_stalled_wait(void* stream) {
    using namespace rk;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    DeviceTables* tabs = nullptr;
    int rc = e == cudaSuccess ? device_tables(dev, &tabs) : RK_ERR_CUDA;
    if (rc) {
        set_error(std::string("rk_selftest_stalled_wait: ") + cudaGetErrorString(e));
        return rc;
    }
    // pass 0: one tile and no task, so it never completes; pass 1: one task that
    // depends on it (no tile body: the variant id matches none)
    BatchPass hp[2];
    memset(hp, 0, sizeof(hp));
    hp[0].nblocks = 1;
    hp[0].variant = -1;
    hp[0].dep = -1;
    hp[1].nblocks = 1;
    hp[1].variant = -1;
    hp[1].dep = 0;
    BatchTask ht = {1, 0, 0};
    void* mem = nullptr;
    const size_t pbytes = sizeof(hp), tbytes = sizeof(ht), cbytes = 3 * sizeof(unsigned long long);
    const size_t toff = (pbytes + 255) / 256 * 256, coff = toff + 256;
    cudaStream_t st = (cudaStream_t)stream;
    e = cudaMalloc(&mem, coff + cbytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(mem, hp, pbytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync((char*)mem + toff, &ht, tbytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync((char*)mem + coff, 0, cbytes, st);
    if (e == cudaSuccess) {
        BatchArgs a;
        a.passes = reinterpret_cast<const BatchPass*>(mem);
        a.tasks = reinterpret_cast<const BatchTask*>((char*)mem + toff);
        a.ntasks = 1;
        a.next = reinterpret_cast<unsigned long long*>((char*)mem + coff);
        a.done = a.next + 1;
        a.status = tabs->status;
        k_batch<<<1, BATCH_NT, 0, st>>>(a);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (mem) cudaFree(mem);
    if (e != cudaSuccess) {
        set_error(std::string("rk_selftest_stalled_wait: ") + cudaGetErrorString(e));
        return RK_ERR_CUDA;
    }
    return rk_stream_check(stream);
}
