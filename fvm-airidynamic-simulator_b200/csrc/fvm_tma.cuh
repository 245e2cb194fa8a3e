// fvm_tma.cuh -- TMA tensor loads and mbarrier helpers (sm_100a inline PTX).
//
// Loads are local-GPU only and never use cluster multicast.  Every wait on an
// mbarrier is bounded: after kWaitCycles SM cycles the caller gets `false`,
// records an error word and leaves the kernel at a uniform point.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace fvm {

constexpr long long kWaitCycles = 4000000000LL;  // ~2 s of SM clock per bounded wait
constexpr uint32_t kErrTimeout = 1u;       // device error word bits
constexpr uint32_t kErrSmemAlign = 4u;     // staging area not 128-byte aligned (kernel did nothing)

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-window address of p through an instruction the compiler does not
// look into: no alignment it assumes for p (say, from an __align__ on an
// extern __shared__ array) is folded into the result.
__device__ __forceinline__ uint32_t smem_addr_opaque(const void *p) {
    uint32_t a;
    asm volatile(
        "{\n\t.reg .u64 t;\n\tcvta.to.shared.u64 t, %1;\n\tcvt.u32.u64 %0, t;\n\t}"
        : "=r"(a)
        : "l"(p));
    return a;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this thread's generic-proxy shared-memory accesses before later
// async-proxy (TMA) writes to the same locations.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of `bar`; false once `limit` SM cycles
// have passed without completion.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, long long limit = kWaitCycles) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (true) {
#pragma unroll 1
        for (int k = 0; k < 64; k++)
            if (mbar_try_wait(bar, parity)) return true;
        if (clock64() - t0 > limit) return false;
    }
}

// 3-D tiled TMA load (x, y, field) into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// Programmatic dependent launch: a step kernel launched with programmatic
// stream serialization may start while its predecessor's last CTAs finish.
// pdl_wait blocks until the predecessor grid has completed and its memory
// operations are visible (a no-op without a programmatic dependency); code
// before it must not read what the predecessor writes.  pdl_trigger lets
// the successor launch once every CTA of this grid has issued it or exited;
// the successor still waits for this grid's completion before reading.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" :::); }

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap *map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Warp max of a non-negative float (NaN-free inputs assumed by the callers).
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Max of non-negative floats via their order-preserving bit patterns.
__device__ __forceinline__ void atomic_max_nonneg(float *addr, float v) {
    if (!(v >= 0.0f)) return;  // drops NaN and negatives
    atomicMax(reinterpret_cast<unsigned int *>(addr), __float_as_uint(v));
}

}  // namespace fvm
