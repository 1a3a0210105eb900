// qsv_sweep.cu -- the pass engine's interpreter kernel: one persistent, warp-specialised launch per sweep.
//
// Replaces the reference's HLS engine kernels/sv/sv_engine.cpp (reader :86-118 / compute :164-279 /
// writer :120-152 DATAFLOW per pass). The staging pipeline (persistent CTA per SM, producer warp with
// TMA / bulk-async copies, mbarrier hand-offs) is qsv_sweep_body.cuh; this file supplies the interpreter
// body and the host launchers:
//   * consumer warps apply the sweep's ops in registers. A thread keeps 2^RB float4 (the two halves of
//     each float4 = tile bit 0) repacked as float2 (re, re) / (im, im) pairs so that every register-bit op
//     runs on two amplitude pairs per packed FP32x2 FMA; ops on lane bits exchange with warp shuffles; an op
//     whose target is on a warp bit starts a new phase (shared-memory round trip in another layout);
//   * the interpreter reads each op's slot and variant at run time; qsv_jit.cpp compiles kernels with the
//     same body specialised to one sweep structure and launches those when they are ready.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>

#include "qsv_device.cuh"
#include "qsv_ops.cuh"
#include "qsv_planner.h"
#include "qsv_sweep_body.cuh"

namespace qsv {
namespace dev {

// Device status word: kernels OR a bit in when a bounded wait gives up (1 = mbarrier wait timeout).
__device__ int g_status = 0;

// The interpreter: the sweep's phases and ops are read at run time (op table in shared memory), one code
// path per op variant selected by a switch.
struct InterpBody {
    using Amp = float2;
    static constexpr int kHalfBits = 1;
    static constexpr bool kSmemOps = true;
    template <int NV, int RB, int WB>
    static __device__ __forceinline__ void tile(float2 *tile, const QsvSweep &P, const QsvOp *sops, int lane, int warp,
                                                int bar) {
        constexpr int NC = 1 << (5 + WB);
        for (int ph = 0; ph < P.nphases; ph++) {
            if (ph > 0) named_bar_sync(bar, NC);
            const QsvPhase &Q = P.phases[ph];
            run_phase<NV, RB, WB>(tile, Q, sops, Q.op_begin, Q.op_end, lane, warp, P.swz != 0, ph > 0,
                                  ph + 1 < P.nphases);
        }
    }
};

template <int KW, int RB, int WB, int S>
__global__ void __launch_bounds__((1 << (5 + WB)) + 32, (KW >= 13 ? 1 : 2))
    sweep_kernel(float2 *__restrict__ state, const __grid_constant__ QsvSweep P, const __grid_constant__ CUtensorMap tmap) {
    sweep_pipeline<KW, RB, WB, S, 1, InterpBody>(state, P, &tmap, &g_status);
}

// ---------------------------------------------------------------- host launchers
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// tensor map of the state for a sweep staged with one box per tile (see qsv_plan.h)
cudaError_t make_tmap(CUtensorMap *map, float2 *state, const QsvSweep &sw) {
    std::memset(map, 0, sizeof(*map));
    if (!sw.tma_rank) return cudaSuccess;
    auto fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    cuuint64_t dims[QSV_TMA_MAX_RANK], strides[QSV_TMA_MAX_RANK];
    cuuint32_t box[QSV_TMA_MAX_RANK], estr[QSV_TMA_MAX_RANK];
    // dim d starts at the window bit following the previous dim's box + free bits
    int start = 0;
    for (int d = 0; d < sw.tma_rank; d++) {
        if (d > 0) strides[d - 1] = (cuuint64_t)8 << start;
        dims[d] = (cuuint64_t)1 << (sw.tdim_box[d] + sw.tdim_free[d]);
        box[d] = 1u << sw.tdim_box[d];
        estr[d] = 1;
        start += sw.tdim_box[d] + sw.tdim_free[d];
    }
    // a swizzled sweep's first dim is tile bits 0-3: 16 amplitudes = 128-byte rows, the 128-byte swizzle's span
    if (sw.swz && (sw.tdim_box[0] != 4 || sw.tma_rank < 2)) return cudaErrorInvalidValue;
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_INT64, sw.tma_rank, state, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, sw.swz ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int KW, int RB, int WB, int S>
static cudaError_t launch_sweep_t(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream) {
    constexpr int NT = (1 << (5 + WB)) + 32;
    const size_t smem = sweep_smem_bytes<KW, S, InterpBody>();
    static int configured_dev = -1;     // attribute set once per device (under the engine's launch lock)
    static int per_sm = 1;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (configured_dev != dev) {
        e = cudaFuncSetAttribute(sweep_kernel<KW, RB, WB, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_kernel<KW, RB, WB, S>, NT, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        configured_dev = dev;
    }
    alignas(64) CUtensorMap map;
    e = make_tmap(&map, state, sw);
    if (e != cudaSuccess) return e;
    int64_t grid = (int64_t)nsm * per_sm;
    if (grid > sw.ntiles) grid = sw.ntiles;
    sweep_kernel<KW, RB, WB, S><<<(unsigned)grid, NT, smem, stream>>>(state, sw, map);
    return cudaGetLastError();
}

}  // namespace dev

// device address of the status word, for kernels in other translation units
cudaError_t status_word_ptr(int **out) {
    static int *ptr[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, dev::g_status);
        if (e != cudaSuccess) return e;
        ptr[dev] = static_cast<int *>(p);
    }
    *out = ptr[dev];
    return cudaSuccess;
}

cudaError_t take_device_status(int *out) {
    int zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(out, dev::g_status, sizeof(int));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(dev::g_status, &zero, sizeof(int));
}

cudaError_t launch_sweep(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream) {
    int rb = 4, wb = 3;
    layout_for_kw(sw.kw, &rb, &wb);
    switch (sw.kw) {
        case 13:
            if (rb == 3) return dev::launch_sweep_t<13, 3, 4, 3>(state, sw, nsm, stream);
            return dev::launch_sweep_t<13, 4, 3, 3>(state, sw, nsm, stream);
        case 12: return dev::launch_sweep_t<12, 4, 2, 3>(state, sw, nsm, stream);
        case 11: return dev::launch_sweep_t<11, 3, 2, 3>(state, sw, nsm, stream);
        case 10: return dev::launch_sweep_t<10, 2, 2, 3>(state, sw, nsm, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace qsv
