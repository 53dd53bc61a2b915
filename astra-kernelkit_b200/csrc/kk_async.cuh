// Shared-memory barriers and tensor copies (TMA) for sm_100a, as inline
// PTX: the staging used by the forward projector's shared-memory path.
//
// Every wait is bounded: a wait that has not completed after
// WAIT_BUDGET_CYCLES SM clocks gives up and returns false, the caller
// records the timeout (kk_wait_timeouts() reports it to the host) and
// stops, and later blocks of the launch see the record and return at
// once, so a broken pipeline ends the kernel instead of hanging the GPU.
// No load here uses cluster multicast; the tensor maps cover this GPU's
// own memory only.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace kk {

// about 0.14 s at the B200's clocks: far above any legitimate wait (a
// tile copy from L2 takes microseconds)
constexpr long long WAIT_BUDGET_CYCLES = 1LL << 28;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// make the initialised barriers visible to the other threads and to the
// async (TMA) proxy; followed by a block barrier at the call site
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// arrive and announce `bytes` of asynchronous copies completing on bar
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

// one test of the phase; a warp whose phase is not complete yet sleeps up
// to WAIT_SUSPEND_NS (woken early when the phase completes) instead of
// spinning on the issue slots the working warps need
constexpr uint32_t WAIT_SUSPEND_NS = 2000;

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity), "n"(WAIT_SUSPEND_NS)
        : "memory");
    return done != 0;
}

// Wait until the barrier's phase with this parity has completed; false
// if the budget ran out first.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > WAIT_BUDGET_CYCLES) return false;
    return true;
}

// 3D tiled tensor copy global -> shared, completing on bar. Coordinates
// are element indices, fastest dimension first; the fastest one must be a
// multiple of 16 bytes. Out-of-range elements are filled with zeros.
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)map) : "memory");
}

}  // namespace kk

// host: cuTensorMapEncodeTiled through the runtime's driver entry point
// (no link-time dependency on libcuda); kk_capi.cu
int kk_encode_tile_map(CUtensorMap* map, CUtensorMapDataType type, int rank, void* base, const uint64_t* dims,
                       const uint64_t* strides_bytes, const uint32_t* box, const char* who);
