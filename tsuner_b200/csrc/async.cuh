// async.cuh -- shared-memory mbarriers (with time-bounded waits) and TMA
// tensor loads, used by the stage kernels and the corrector.  Every wait is
// bounded by the global timer: a caller that sees `false` records an error
// for the host, waits once more for its own copies in flight and returns.
#pragma once
#include <cuda.h>  // CUtensorMap (type only; the encoder is fetched from the driver at run time)
#include <cuda_runtime.h>

#include <cstdint>

namespace tsu {

constexpr unsigned long long kWaitNs = 500000000ull;  // 0.5 s per bounded wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// p advanced to the next multiple of ALIGN bytes of the shared window.  The
// pad is added to the pointer (not computed through an integer round trip),
// so the compiler still knows it addresses shared memory and keeps its
// accesses shared-memory instructions.
template <int ALIGN, typename T>
__device__ __forceinline__ T *smem_align(T *p) {
    const uint32_t pad = (ALIGN - (smem_u32(p) & (ALIGN - 1))) & (ALIGN - 1);
    return reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(p) + pad);
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// waits for the phase of parity `parity` to complete; false after `limit_ns`
__device__ __forceinline__ bool mbar_wait_for(uint64_t *bar, unsigned parity, unsigned long long limit_ns) {
    const unsigned long long t0 = gtimer();
    while (!mbar_try(bar, parity))
        if (gtimer() - t0 > limit_ns) return false;
    return true;
}
// the wait that drains a CTA's own copies / MMAs on the error path: always
// the full kWaitNs
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
    return mbar_wait_for(bar, parity, kWaitNs);
}

// Limit of a CTA's ordinary waits, whose expiry is reported as an error.  It
// is kWaitNs unless a test lowers it (tsu_set_wait_limit_ns) to make those
// waits run out while the copies are still in flight; the drain waits above
// keep the full limit, so a CTA never leaves with its own copies or MMAs
// still running.  One copy per compilation unit (set through that unit's
// set_wait_limit_* host function on the current device).
static __device__ unsigned long long g_wait_limit_ns = kWaitNs;
// non-blocking probe of the phase (try_wait may suspend the thread until the
// phase completes, for a hardware-chosen time)
__device__ __forceinline__ bool mbar_test(uint64_t *bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_first(uint64_t *bar, unsigned parity) {
    const unsigned long long lim = *static_cast<volatile unsigned long long *>(&g_wait_limit_ns);
    if (lim >= kWaitNs) return mbar_wait_for(bar, parity, lim);
    // a lowered limit (tests of the error path): poll without suspending, so
    // that the limit, not try_wait's own suspension, decides
    const unsigned long long t0 = gtimer();
    for (;;) {
        if (mbar_test(bar, parity)) return true;
        if (gtimer() - t0 >= lim) return false;
    }
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Tiled TMA loads (no multicast) into this CTA's shared memory; the box's
// bytes complete on `bar`.  The innermost coordinate times the element size
// must be a multiple of 16 bytes (callers guarantee it); outer coordinates
// may lie outside the tensor (zero fill).
// request a line into L2 (no register is written)
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

// host: cuTensorMapEncodeTiled from the driver (no link against libcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn tensor_map_encoder();

}  // namespace tsu
