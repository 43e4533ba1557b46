// Asynchronous bulk copies (TMA) and mbarriers for sm_100a, in inline PTX.
//
// Waits are bounded: a wait that does not complete within RK_WAIT_LIMIT polls, or
// within the wait limit in SM clock cycles (about one second unless the host sets
// another with rk_set_wait_limit), sets bit RK_STATUS_TIMEOUT in the device status
// word and returns false, so a kernel never spins forever (the host reads the word
// with rk_device_status()).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "rk_params.h"

namespace rk {

constexpr uint32_t RK_WAIT_LIMIT = 1u << 26;
// status bits RK_STATUS_TIMEOUT / RK_STATUS_BAD_VARIANT: include/reikna_b200.h

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make mbarrier initialisation visible to the async proxy
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order earlier generic-proxy shared memory accesses before later async-proxy ones
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// about one second of SM clock: no legitimate wait in these kernels comes near it
constexpr long long RK_WAIT_CYCLES = 2000000000LL;

// The device status block is four 32-bit words: [0] status bits, [1] unused,
// [2..3] the wait limit in SM clock cycles (int64, set by rk_set_wait_limit).
// Without a status block the default limit applies.
__device__ __forceinline__ long long wait_limit(const int32_t* status) {
    return status ? *reinterpret_cast<const volatile long long*>(status + 2) : RK_WAIT_CYCLES;
}

// bounded wait on phase `parity`; false (and the status bit set) on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int32_t* status) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64(), lim = wait_limit(status);
    for (uint32_t i = 0; i < RK_WAIT_LIMIT; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (clock64() - t0 > lim) break;
    }
    if (status) atomicOr(status, RK_STATUS_TIMEOUT);
    return false;
}

// same, acquiring at cluster scope (data and arrivals from other CTAs of the cluster)
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity, int32_t* status) {
    if (mbar_try_wait_cluster(bar, parity)) return true;
    const long long t0 = clock64(), lim = wait_limit(status);
    for (uint32_t i = 0; i < RK_WAIT_LIMIT; ++i) {
        if (mbar_try_wait_cluster(bar, parity)) return true;
        if (clock64() - t0 > lim) break;
    }
    if (status) atomicOr(status, RK_STATUS_TIMEOUT);
    return false;
}

// shared::cluster address of the same shared variable in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t mapa(uint32_t local_addr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local_addr), "r"(rank));
    return r;
}

// arrive on an mbarrier of another CTA of the cluster (release at cluster scope)
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}

// asynchronous store into another CTA's shared memory whose bytes complete the
// transaction count of that CTA's mbarrier
__device__ __forceinline__ void st_async(uint32_t cluster_addr, float2 v, uint32_t cluster_bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];" ::"r"(
                     cluster_addr),
                 "f"(v.x), "f"(v.y), "r"(cluster_bar)
                 : "memory");
}
__device__ __forceinline__ void st_async(uint32_t cluster_addr, double2 v, uint32_t cluster_bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(
                     cluster_addr),
                 "d"(v.x), "d"(v.y), "r"(cluster_bar)
                 : "memory");
}

// 1-D bulk copy global -> shared, completion counted on `bar` (bytes % 16 == 0,
// both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// 3-D tiled tensor copy global -> shared (box given by the tensor map)
__device__ __forceinline__ void tma_g2s_3d(void* dst, const void* tmap, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace rk
