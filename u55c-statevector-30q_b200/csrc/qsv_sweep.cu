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

// The fields of an op record a kernel reads, from one 16-byte shared-memory load.
struct OpHdr {
    uint32_t cm_thr, cm_reg, cm_c, kind, cls0, cls1, slot, tbit, variant, r00;
};
__device__ __forceinline__ OpHdr op_hdr(const QsvOp *op) {
    const uint4 h = *reinterpret_cast<const uint4 *>(reinterpret_cast<const unsigned char *>(op) + 64);
    OpHdr o;
    o.cm_thr = h.x;
    o.cm_reg = h.y & 0xffu; o.cm_c = (h.y >> 8) & 0xffu; o.kind = (h.y >> 16) & 0xffu;
    o.cls0 = h.z & 0xffu; o.cls1 = (h.z >> 8) & 0xffu; o.slot = (h.z >> 16) & 0xffu; o.tbit = h.z >> 24;
    o.variant = h.w & 0xffu; o.r00 = (h.w >> 8) & 0xffu;
    return o;
}

// diagonal op whose target is a tile bit of the item base: every amplitude of the item has the same
// target-bit value `one`
template <int NV, bool IP>
__device__ __forceinline__ void base_diag(float2 (&R)[NV], float2 (&I)[NV], const OpHdr &op, const float *m0,
                                          const float *m1, bool tok, bool one) {
    if (op.variant == QSV_V_UNI_DIAG) {
        const float ar = one ? m0[6] : m0[0], ai = one ? m0[7] : m0[1];
#pragma unroll
        for (int r = 0; r < NV; r++) cmul2_t<IP>(R[r], I[r], ar, ai);
        return;
    }
    // QSV_V_CTRL_DIAG1(_SEL): amplitudes with the target bit and every control set get m11
    if (!(one && tok)) return;
    const int cm_reg = (int)op.cm_reg;
#pragma unroll
    for (int r = 0; r < NV; r++)
        if ((r & cm_reg) == cm_reg) cmul2_t<IP>(R[r], I[r], m1[6], m1[7]);
}

template <bool IP>
__device__ __forceinline__ void stream_op(const QsvOp *op, float2 (&R)[8], float2 (&I)[8], uint32_t base) {
    const OpHdr h = op_hdr(op);
    if (h.variant == QSV_V_SKIP) return;
    float m0[8], m1[8];
    const float4 *mv = reinterpret_cast<const float4 *>(op);
#pragma unroll
    for (int v = 0; v < 2; v++) {
        const float4 a = mv[v], c = mv[2 + v];
        m0[4 * v] = a.x; m0[4 * v + 1] = a.y; m0[4 * v + 2] = a.z; m0[4 * v + 3] = a.w;
        m1[4 * v] = c.x; m1[4 * v + 1] = c.y; m1[4 * v + 2] = c.z; m1[4 * v + 3] = c.w;
    }
    const bool tok = (base & h.cm_thr) == h.cm_thr;
    switch (h.slot) {
        case QSV_SLOT_COMP: comp_op_fast<8>(R, I, h, m0, m1, tok); break;
        case QSV_SLOT_REG0: reg_op<8, 0, IP>(R, I, h, m0, m1, tok); break;
        case QSV_SLOT_REG0 + 1: reg_op<8, 1, IP>(R, I, h, m0, m1, tok); break;
        case QSV_SLOT_REG0 + 2: reg_op<8, 2, IP>(R, I, h, m0, m1, tok); break;
        case QSV_SLOT_BASE: base_diag<8, IP>(R, I, h, m0, m1, tok, (base >> h.tbit) & 1u); break;
        default: break;
    }
}

// insert a zero bit at position q (bits q and above move up by one)
__device__ __forceinline__ uint32_t insert0(uint32_t x, uint32_t q) {
    return ((x >> q) << (q + 1)) | (x & ((1u << q) - 1u));
}

// One group over the whole tile. SIN / SOUT: the tile holds the in-tile order (re0, re1, im0, im1) per
// float4 on entry / exit, instead of the state's interleaved order (first group in, last group out).
template <int KW, int NCG, bool SIN, bool SOUT, bool IP>
__device__ __forceinline__ void stream_group(float2 *tile, const QsvOp *sops, const QsvGroup &g, int ctid, bool swz) {
    const uint32_t q[3] = {g.q[0], g.q[1], g.q[2]};
    uint32_t soff[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const uint32_t o = ((r & 1) ? 1u << q[0] : 0u) | ((r & 2) ? 1u << q[1] : 0u) | ((r & 4) ? 1u << q[2] : 0u);
        soff[r] = swz ? swz128(o) : o;
    }
    // the item bits in ascending order, for the zero insertions
    uint32_t s0 = q[0], s1 = q[1], s2 = q[2], t;
    if (s0 > s1) { t = s0; s0 = s1; s1 = t; }
    if (s1 > s2) { t = s1; s1 = s2; s2 = t; }
    if (s0 > s1) { t = s0; s0 = s1; s1 = t; }
    const int ob = g.op_begin, oe = g.op_end;
    for (int it = ctid; it < (1 << (KW - 4)); it += NCG) {
        const uint32_t x = insert0(insert0(insert0((uint32_t)it << 1, s0), s1), s2);
        const uint32_t sx = swz ? swz128(x) : x;                          // swz128 is linear over XOR
        float2 R[8], I[8];
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const float4 v = *reinterpret_cast<const float4 *>(tile + (sx ^ soff[r]));
            R[r] = SIN ? make_float2(v.x, v.y) : make_float2(v.x, v.z);
            I[r] = SIN ? make_float2(v.z, v.w) : make_float2(v.y, v.w);
        }
        for (int o = ob; o < oe; o++) stream_op<IP>(sops + o, R, I, x);
#pragma unroll
        for (int r = 0; r < 8; r++)
            *reinterpret_cast<float4 *>(tile + (sx ^ soff[r])) =
                SOUT ? make_float4(R[r].x, R[r].y, I[r].x, I[r].y) : make_float4(R[r].x, I[r].x, R[r].y, I[r].y);
    }
}

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
            if (sin && sout) stream_group<KW, NCG, true, true, IP>(tile, sops, g, ctid, swz);
            else if (sin) stream_group<KW, NCG, true, false, IP>(tile, sops, g, ctid, swz);
            else if (sout) stream_group<KW, NCG, false, true, IP>(tile, sops, g, ctid, swz);
            else stream_group<KW, NCG, false, false, IP>(tile, sops, g, ctid, swz);
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
