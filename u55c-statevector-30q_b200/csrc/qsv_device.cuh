// qsv_device.cuh -- sm_100a device helpers: mbarriers, bulk-async (TMA engine) copies, proxy fences,
// bounded waits, and the MUX2 pair arithmetic.
#pragma once
#include "qsv_plan.h"
#ifdef __CUDACC_RTC__
// the tensor-map parameter of a sweep kernel: 128 opaque bytes, 64-byte aligned (cuda.h's CUtensorMap)
struct alignas(64) CUtensorMap {
    unsigned long long opaque[16];
};
#else
#include <cuda.h>
#include <cuda_runtime.h>
#endif

namespace qsv {
namespace dev {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait on an mbarrier phase. Gives up after limit_ns (2 s by default; a sweep tile takes
// microseconds), records the failure in the device status word and in the CTA's abort flag, and returns
// false so the caller can leave its loop; a wait that sees another thread's abort returns false as well.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag, int *status,
                                          uint64_t limit_ns = QSV_WAIT_US_DEFAULT * 1000ull) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*abort_flag) return false;
        if (globaltimer_ns() - t0 > limit_ns) {
            *abort_flag = 1;
            atomicOr(status, 1);
            return false;
        }
    }
}
// Bounded wait that ignores the abort flag: after an abort, the thread that issued bulk-async loads waits
// (at most limit_ns) for the ones still in flight before the CTA exits. Returns whether the phase completed.
__device__ __forceinline__ bool mbar_wait_drain(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
    const uint64_t t0 = globaltimer_ns();
    while (!mbar_try_wait(bar, parity))
        if (globaltimer_ns() - t0 > limit_ns) return false;
    return true;
}
// the wait limit a sweep's parameters ask for, in nanoseconds
__device__ __forceinline__ uint64_t wait_limit_ns(uint32_t wait_us) {
    return (uint64_t)(wait_us ? wait_us : QSV_WAIT_US_DEFAULT) * 1000ull;
}

// bulk-async copy global -> shared, completion counted on an mbarrier (bytes)
__device__ __forceinline__ void bulk_g2s(void *sdst, const void *gsrc, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(sdst)),
        "l"(__cvta_generic_to_global(gsrc)), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// bulk-async copy shared -> global, tracked by the issuing thread's bulk groups
__device__ __forceinline__ void bulk_s2g(void *gdst, const void *ssrc, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(__cvta_generic_to_global(gdst)),
                 "r"(smem_u32(ssrc)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// make this thread's generic-proxy shared-memory writes visible to the async proxy (bulk stores)
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// ------------------------------------------------------------------ MUX2 pair arithmetic
// Canonical fused-multiply-add order (the CPU oracle uses the same chains):
//   y0.re = fma(m00.re, x0.re, fma(-m00.im, x0.im, fma(m01.re, x1.re, -(m01.im * x1.im))))
//   y0.im = fma(m00.re, x0.im, fma( m00.im, x0.re, fma(m01.re, x1.im,   m01.im * x1.re)))
//   y1 likewise with (m11, m10) and the roles of x0 / x1 exchanged.
// For an output amplitude "own" with partner "oth": y = a*own + b*oth with (a, b) = (m00, m01) for
// the bit-0 amplitude and (m11, m10) for the bit-1 amplitude.
__device__ __forceinline__ void lin_own(float &yr, float &yi, float ar, float ai, float br, float bi, float owr,
                                        float owi, float otr, float oti) {
    yr = fmaf(ar, owr, fmaf(-ai, owi, fmaf(br, otr, -__fmul_rn(bi, oti))));
    yi = fmaf(ar, owi, fmaf(ai, owr, fmaf(br, oti, __fmul_rn(bi, otr))));
}
// diagonal form: y = a*own (the off-diagonal terms are exact zeros in the dense chain)
__device__ __forceinline__ void diag_own(float &yr, float &yi, float ar, float ai, float owr, float owi) {
    yr = fmaf(ar, owr, -__fmul_rn(ai, owi));
    yi = fmaf(ar, owi, __fmul_rn(ai, owr));
}

// apply matrix m of class cls to the pair (x0, x1) held by one thread
__device__ __forceinline__ void pair_apply(float &x0r, float &x0i, float &x1r, float &x1i, const float *m, int cls) {
    if (cls == QSV_M_DENSE) {
        float y0r, y0i, y1r, y1i;
        lin_own(y0r, y0i, m[0], m[1], m[2], m[3], x0r, x0i, x1r, x1i);
        lin_own(y1r, y1i, m[6], m[7], m[4], m[5], x1r, x1i, x0r, x0i);
        x0r = y0r; x0i = y0i; x1r = y1r; x1i = y1i;
    } else if (cls == QSV_M_DIAG) {
        float y0r, y0i, y1r, y1i;
        diag_own(y0r, y0i, m[0], m[1], x0r, x0i);
        diag_own(y1r, y1i, m[6], m[7], x1r, x1i);
        x0r = y0r; x0i = y0i; x1r = y1r; x1i = y1i;
    } else if (cls == QSV_M_DIAG1) {
        float y1r, y1i;
        diag_own(y1r, y1i, m[6], m[7], x1r, x1i);
        x1r = y1r; x1i = y1i;
    } else if (cls == QSV_M_XSWAP) {
        float t = x0r; x0r = x1r; x1r = t;
        t = x0i; x0i = x1i; x1i = t;
    }
    // QSV_M_IDENT: unchanged
}

}  // namespace dev
}  // namespace qsv
