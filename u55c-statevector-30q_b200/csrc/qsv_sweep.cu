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

#include <atomic>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <string>

#include "qsv_device.cuh"
#include "qsv_ops.cuh"
#include "qsv_planner.h"
#include "qsv_stream.cuh"
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

// ---------------------------------------------------------------- streaming interpreter
// The tile stays in shared memory and each group of ops (plan_stream) is one round trip of it: a thread
// takes items of 8 float4 = 16 amplitudes on tile bits {0, q[0], q[1], q[2]} (float4 r holds item base |
// r.0 * 2^q[0] | r.1 * 2^q[1] | r.2 * 2^q[2]), applies the group's ops to them in registers and stores them
// back. Only one item's 32 floats are live across the run-time dispatch of an op (the phase interpreter
// keeps 64), any target bit can be an item bit, so a sweep needs no phase layouts, and ops on tile bit 0
// and diagonal ops on any bit ride along with the group. The ops run through the phase interpreter's code
// paths (reg_op with the item bits as register bits 0-2, comp_op_fast), so every value is the same.

static_assert(sizeof(QsvOp) == 96 && offsetof(QsvOp, cm_thr) == 64 && offsetof(QsvOp, cm_reg) == 68 &&
                  offsetof(QsvOp, cls0) == 72 && offsetof(QsvOp, variant) == 76 && offsetof(QsvOp, m1) == 32,
              "op_hdr reads the op record's fields as one 16-byte vector at offset 64");

template <bool IP>
struct StreamBody {
    using Amp = float2;
    static constexpr int kHalfBits = 1;
    static constexpr bool kSmemOps = true;
    template <int NV, int RB, int WB>
    static __device__ __forceinline__ void tile(float2 *tile, const QsvSweep &P, const QsvOp *sops, int lane, int warp,
                                                int bar) {
        constexpr int NCG = 1 << (5 + WB);
        constexpr int KW = 1 + 3 + 2 + RB + WB;
        const int ctid = warp * 32 + lane;
        const bool swz = P.swz != 0;
        const int ng = P.ngroups;
        for (int gi = 0; gi < ng; gi++) {
            if (gi > 0) named_bar_sync(bar, NCG);
            const QsvGroup g = P.groups[gi];
            const bool sin = gi > 0, sout = gi + 1 < ng;
            const int ob = g.op_begin, oe = g.op_end;
            auto ops = [&](float2 (&R)[8], float2 (&I)[8], uint32_t x) {
                for (int o = ob; o < oe; o++) stream_op<IP>(sops + o, R, I, x);
            };
            if (sin && sout) stream_items<KW, NCG, true, true>(tile, g, ctid, swz, ops);
            else if (sin) stream_items<KW, NCG, true, false>(tile, g, ctid, swz, ops);
            else if (sout) stream_items<KW, NCG, false, true>(tile, g, ctid, swz, ops);
            else stream_items<KW, NCG, false, false>(tile, g, ctid, swz, ops);
        }
    }
};

template <int KW, int RB, int WB, int S, int G, bool IP>
__global__ void __launch_bounds__(G * (1 << (5 + WB)) + 32, (KW >= 13 ? 1 : 2))
    sweep_stream_kernel(float2 *__restrict__ state, const __grid_constant__ QsvSweep P,
                        const __grid_constant__ CUtensorMap tmap) {
    sweep_pipeline<KW, RB, WB, S, G, StreamBody<IP>>(state, P, &tmap, &g_status);
}

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

template <int KW, int RB, int WB, int S, int G, bool IP>
static cudaError_t launch_stream_t(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream) {
    constexpr int NT = G * (1 << (5 + WB)) + 32;
    const size_t smem = sweep_smem_bytes<KW, S, StreamBody<IP>>();
    static int configured_dev = -1;     // attribute set once per device (under the engine's launch lock)
    static int per_sm = 1;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (configured_dev != dev) {
        e = cudaFuncSetAttribute(sweep_stream_kernel<KW, RB, WB, S, G, IP>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_stream_kernel<KW, RB, WB, S, G, IP>, NT, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        configured_dev = dev;
    }
    alignas(64) CUtensorMap map;
    e = make_tmap(&map, state, sw);
    if (e != cudaSuccess) return e;
    int64_t grid = (int64_t)nsm * per_sm;
    if (grid > sw.ntiles) grid = sw.ntiles;
    sweep_stream_kernel<KW, RB, WB, S, G, IP><<<(unsigned)grid, NT, smem, stream>>>(state, sw, map);
    return cudaGetLastError();
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

// Interpreter choice (process-wide): 0 = phase layouts, 1 = streaming.
static std::atomic<int> g_interp{0};
int set_interp(int mode) {
    if (mode < 0 || mode > 1) return -1;
    return g_interp.exchange(mode);
}

// The streaming interpreter runs the sweep's own op records re-planned for its items (plan_stream).
static cudaError_t launch_stream(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream) {
    thread_local QsvSweep s2;
    std::memcpy(&s2, &sw, sizeof(QsvSweep));
    std::string err;
    if (plan_stream(s2, err) != QSV_OK) return cudaErrorInvalidValue;
    // QSV_STREAM_IP=0 (tuning): the chains in their usual issue order instead of the in-place one
    static const bool ip = [] {
        const char *e = std::getenv("QSV_STREAM_IP");
        return !(e && std::atoi(e) == 0);
    }();
    if (ip) {
        switch (sw.kw) {
            case 13: return dev::launch_stream_t<13, 4, 3, 3, 1, true>(state, s2, nsm, stream);
            case 12: return dev::launch_stream_t<12, 4, 2, 3, 1, true>(state, s2, nsm, stream);
            case 11: return dev::launch_stream_t<11, 3, 2, 3, 1, true>(state, s2, nsm, stream);
            case 10: return dev::launch_stream_t<10, 2, 2, 3, 1, true>(state, s2, nsm, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (sw.kw) {
        case 13: return dev::launch_stream_t<13, 4, 3, 3, 1, false>(state, s2, nsm, stream);
        case 12: return dev::launch_stream_t<12, 4, 2, 3, 1, false>(state, s2, nsm, stream);
        case 11: return dev::launch_stream_t<11, 3, 2, 3, 1, false>(state, s2, nsm, stream);
        case 10: return dev::launch_stream_t<10, 2, 2, 3, 1, false>(state, s2, nsm, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_sweep(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream) {
    if (g_interp.load(std::memory_order_relaxed) == 1) return launch_stream(state, sw, nsm, stream);
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
