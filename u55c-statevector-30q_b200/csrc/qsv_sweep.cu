// qsv_sweep.cu -- the pass engine: one persistent, warp-specialised launch per sweep (sm_100a).
//
// Replaces the reference's HLS engine kernels/sv/sv_engine.cpp (reader :86-118 / compute :164-279 /
// writer :120-152 DATAFLOW per pass). B200 design:
//   * one CTA per SM (KW = 13: three 64 KiB tile buffers), grid-strided over the 2^(n-13) tiles;
//   * a producer warp streams tiles HBM -> shared memory and back with the TMA engine: one tensor-map
//     box per tile when the window's contiguous runs are short, one bulk-async copy per sub-block when
//     they are long; completion is counted on mbarriers, up to three tiles are in flight;
//   * consumer warps apply the sweep's ops in registers. A thread keeps 2^RB float4 (the two halves of
//     each float4 = tile bit 0) repacked as float2 (re, re) / (im, im) pairs so that every register-bit op
//     runs on two amplitude pairs per packed FP32x2 FMA; ops on lane bits exchange with warp shuffles; an op
//     whose target is on a warp bit starts a new phase (shared-memory round trip in another layout).
// The tile addressing is the reference's (model.py:25-40 / sv_engine.cpp:61-84,116): tile T's base is
// pdep(T, free bits) and sub-block s sits at base | pdep(s, H).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>

#include "qsv_device.cuh"
#include "qsv_planner.h"

namespace qsv {
namespace dev {

// Device status word: kernels OR a bit in when a bounded wait gives up (1 = mbarrier wait timeout).
__device__ int g_status = 0;

__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// ---------------------------------------------------------------- packed (two pairs per instruction) math
// x0 = (R0, I0), x1 = (R1, I1), each float2 holding the same component of two independent pairs.
// Canonical chain per output (see qsv_device.cuh), on both pairs at once.
__device__ __forceinline__ void dense2(float2 &R0, float2 &I0, float2 &R1, float2 &I1, const float *m) {
    float2 t, u;
    t = __fmul2_rn(f2(-m[3]), I1); t = __ffma2_rn(f2(m[2]), R1, t); t = __ffma2_rn(f2(-m[1]), I0, t);
    const float2 y0r = __ffma2_rn(f2(m[0]), R0, t);
    u = __fmul2_rn(f2(m[3]), R1);  u = __ffma2_rn(f2(m[2]), I1, u); u = __ffma2_rn(f2(m[1]), R0, u);
    const float2 y0i = __ffma2_rn(f2(m[0]), I0, u);
    t = __fmul2_rn(f2(-m[5]), I0); t = __ffma2_rn(f2(m[4]), R0, t); t = __ffma2_rn(f2(-m[7]), I1, t);
    const float2 y1r = __ffma2_rn(f2(m[6]), R1, t);
    u = __fmul2_rn(f2(m[5]), R0);  u = __ffma2_rn(f2(m[4]), I0, u); u = __ffma2_rn(f2(m[7]), R1, u);
    const float2 y1i = __ffma2_rn(f2(m[6]), I1, u);
    R0 = y0r; I0 = y0i; R1 = y1r; I1 = y1i;
}
// dense with per-lane coefficients (c[e] = (coefficient for pair .x, coefficient for pair .y))
__device__ __forceinline__ void dense2v(float2 &R0, float2 &I0, float2 &R1, float2 &I1, const float2 *c) {
    const float2 n1 = make_float2(-c[1].x, -c[1].y), n3 = make_float2(-c[3].x, -c[3].y);
    const float2 n5 = make_float2(-c[5].x, -c[5].y), n7 = make_float2(-c[7].x, -c[7].y);
    float2 t, u;
    t = __fmul2_rn(n3, I1); t = __ffma2_rn(c[2], R1, t); t = __ffma2_rn(n1, I0, t);
    const float2 y0r = __ffma2_rn(c[0], R0, t);
    u = __fmul2_rn(c[3], R1); u = __ffma2_rn(c[2], I1, u); u = __ffma2_rn(c[1], R0, u);
    const float2 y0i = __ffma2_rn(c[0], I0, u);
    t = __fmul2_rn(n5, I0); t = __ffma2_rn(c[4], R0, t); t = __ffma2_rn(n7, I1, t);
    const float2 y1r = __ffma2_rn(c[6], R1, t);
    u = __fmul2_rn(c[5], R0); u = __ffma2_rn(c[4], I0, u); u = __ffma2_rn(c[7], R1, u);
    const float2 y1i = __ffma2_rn(c[6], I1, u);
    R0 = y0r; I0 = y0i; R1 = y1r; I1 = y1i;
}
// y = a * x for a packed amplitude pair (a splat)
__device__ __forceinline__ void cmul2(float2 &R, float2 &I, float ar, float ai) {
    const float2 yr = __ffma2_rn(f2(ar), R, __fmul2_rn(f2(-ai), I));
    const float2 yi = __ffma2_rn(f2(ar), I, __fmul2_rn(f2(ai), R));
    R = yr; I = yi;
}
__device__ __forceinline__ void swap2(float2 &a, float2 &b) {
    const float2 t = a; a = b; b = t;
}

// ---------------------------------------------------------------- ops by target slot
// Register-bit target RBIT: pairs (slot r, slot r | 2^RBIT); each float2 carries two pairs (tile bit 0 =
// 0 in .x, 1 in .y). One tight unrolled loop per code variant (selected on the host).
template <int NV, int RBIT>
__device__ __forceinline__ void reg_op(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op, const float *m0,
                                       const float *m1, bool thread_ok) {
    const int cm_reg = op.cm_reg;
#define QSV_FOR_PAIRS for (int r = 0; r < NV; r++) if (!(r & (1 << RBIT)))
#define QSV_P1 (r | (1 << RBIT))
    switch (op.variant) {
        case QSV_V_UNI_DENSE:
#pragma unroll
            QSV_FOR_PAIRS dense2(R[r], I[r], R[QSV_P1], I[QSV_P1], m0);
            break;
        case QSV_V_UNI_DIAG:
#pragma unroll
            QSV_FOR_PAIRS { cmul2(R[r], I[r], m0[0], m0[1]); cmul2(R[QSV_P1], I[QSV_P1], m0[6], m0[7]); }
            break;
        case QSV_V_UNI_SWAP:
#pragma unroll
            QSV_FOR_PAIRS { swap2(R[r], R[QSV_P1]); swap2(I[r], I[QSV_P1]); }
            break;
        case QSV_V_CTRL_DENSE:
#pragma unroll
            QSV_FOR_PAIRS if (thread_ok && (r & cm_reg) == cm_reg) dense2(R[r], I[r], R[QSV_P1], I[QSV_P1], m1);
            break;
        case QSV_V_CTRL_DIAG1:
#pragma unroll
            QSV_FOR_PAIRS if (thread_ok && (r & cm_reg) == cm_reg) cmul2(R[QSV_P1], I[QSV_P1], m1[6], m1[7]);
            break;
        case QSV_V_CTRL_SWAP:
#pragma unroll
            QSV_FOR_PAIRS if (thread_ok && (r & cm_reg) == cm_reg) { swap2(R[r], R[QSV_P1]); swap2(I[r], I[QSV_P1]); }
            break;
        case QSV_V_CTRL_DENSE_SEL: {
            const float id[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f};
#pragma unroll
            QSV_FOR_PAIRS {
                const bool s = thread_ok && (r & cm_reg) == cm_reg;
                float c[8];
#pragma unroll
                for (int e = 0; e < 8; e++) c[e] = s ? m1[e] : id[e];
                dense2(R[r], I[r], R[QSV_P1], I[QSV_P1], c);
            }
            break;
        }
        case QSV_V_CTRL_DIAG1_SEL:
#pragma unroll
            QSV_FOR_PAIRS {
                const bool s = thread_ok && (r & cm_reg) == cm_reg;
                cmul2(R[QSV_P1], I[QSV_P1], s ? m1[6] : 1.f, s ? m1[7] : 0.f);
            }
            break;
        case QSV_V_CTRL_SWAP_SEL:
#pragma unroll
            QSV_FOR_PAIRS {
                const bool s = thread_ok && (r & cm_reg) == cm_reg;
                const float2 a = R[r], b = R[QSV_P1], c = I[r], d = I[QSV_P1];
                R[r] = s ? b : a; R[QSV_P1] = s ? a : b;
                I[r] = s ? d : c; I[QSV_P1] = s ? c : d;
            }
            break;
        case QSV_V_MUX: {
            const bool cc = op.cm_c;
#pragma unroll
            QSV_FOR_PAIRS {
                const bool sy = thread_ok && (r & cm_reg) == cm_reg, sx = sy && !cc;
                float2 c[8];
#pragma unroll
                for (int e = 0; e < 8; e++) c[e] = make_float2(sx ? m1[e] : m0[e], sy ? m1[e] : m0[e]);
                dense2v(R[r], I[r], R[QSV_P1], I[QSV_P1], c);
            }
            break;
        }
        default: break;
    }
#undef QSV_FOR_PAIRS
#undef QSV_P1
}

// tile-bit-0 target: the pair is the two halves of one slot (scalar arithmetic, any variant)
template <int NV>
__device__ __forceinline__ void comp_op(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op, const float *m0,
                                     const float *m1, bool thread_ok) {
    const int cm_reg = op.cm_reg;
    const bool uni = op.kind == QSV_K_UNI, ctrl = op.kind == QSV_K_CTRL;
#pragma unroll
    for (int r = 0; r < NV; r++) {
        const bool s = !uni && thread_ok && (r & cm_reg) == cm_reg;
        if (ctrl && !s) continue;
        float x0r = R[r].x, x0i = I[r].x, x1r = R[r].y, x1i = I[r].y;
        if (s) pair_apply(x0r, x0i, x1r, x1i, m1, op.cls1);
        else pair_apply(x0r, x0i, x1r, x1i, m0, op.cls0);
        R[r] = make_float2(x0r, x1r);
        I[r] = make_float2(x0i, x1i);
    }
}

// lane-bit target: exchange with the partner lane; each thread computes its own amplitude as
// a * own + b * other with (a, b) = (m00, m01) on the bit-0 side and (m11, m10) on the bit-1 side
template <int NV>
__device__ __forceinline__ void lane_op(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op, const float *m0,
                                        const float *m1, bool thread_ok, int lanebit, int lane) {
    const int mine = (lane >> lanebit) & 1;
    const int xm = 1 << lanebit;
    const int cm_reg = op.cm_reg;
    const bool uni = op.kind == QSV_K_UNI, ctrl = op.kind == QSV_K_CTRL, cc = op.cm_c;
    const float a0r = mine ? m0[6] : m0[0], a0i = mine ? m0[7] : m0[1];
    const float b0r = mine ? m0[4] : m0[2], b0i = mine ? m0[5] : m0[3];
    const float a1r = mine ? m1[6] : m1[0], a1i = mine ? m1[7] : m1[1];
    const float b1r = mine ? m1[4] : m1[2], b1i = mine ? m1[5] : m1[3];
#pragma unroll
    for (int r = 0; r < NV; r++) {
        float2 oR, oI;
        oR.x = __shfl_xor_sync(0xffffffffu, R[r].x, xm);
        oR.y = __shfl_xor_sync(0xffffffffu, R[r].y, xm);
        oI.x = __shfl_xor_sync(0xffffffffu, I[r].x, xm);
        oI.y = __shfl_xor_sync(0xffffffffu, I[r].y, xm);
        const bool sy = !uni && thread_ok && (r & cm_reg) == cm_reg, sx = sy && !cc;
        // unselected pairs of a controlled op use M0 = identity: (a, b) = (1, 0) leaves the amplitude's
        // value unchanged, so the arithmetic runs branch-free on every lane
        const float u0r = ctrl ? 1.f : a0r, u0i = ctrl ? 0.f : a0i, v0r = ctrl ? 0.f : b0r, v0i = ctrl ? 0.f : b0i;
        const float2 ar = make_float2(sx ? a1r : u0r, sy ? a1r : u0r);
        const float2 ai = make_float2(sx ? a1i : u0i, sy ? a1i : u0i);
        const float2 br = make_float2(sx ? b1r : v0r, sy ? b1r : v0r);
        const float2 bi = make_float2(sx ? b1i : v0i, sy ? b1i : v0i);
        float2 t = __fmul2_rn(make_float2(-bi.x, -bi.y), oI);
        t = __ffma2_rn(br, oR, t);
        t = __ffma2_rn(make_float2(-ai.x, -ai.y), I[r], t);
        const float2 yr = __ffma2_rn(ar, R[r], t);
        float2 u = __fmul2_rn(bi, oR);
        u = __ffma2_rn(br, oI, u);
        u = __ffma2_rn(ai, R[r], u);
        const float2 yi = __ffma2_rn(ar, I[r], u);
        R[r] = yr;
        I[r] = yi;
    }
}

template <int NV, int RB>
__device__ __forceinline__ void apply_op(const QsvOp &op, float2 (&R)[NV], float2 (&I)[NV], uint32_t tb, int lane) {
    if (op.variant == QSV_V_SKIP) return;
    float m0[8], m1[8];
#pragma unroll
    for (int e = 0; e < 8; e++) { m0[e] = op.m0[e]; m1[e] = op.m1[e]; }
    const uint32_t cm_thr = op.cm_thr;
    const bool thread_ok = (tb & cm_thr) == cm_thr;
    const int slot = op.slot;
    if (slot >= QSV_SLOT_LANE0) {
        lane_op<NV>(R, I, op, m0, m1, thread_ok, slot - QSV_SLOT_LANE0, lane);
        return;
    }
    switch (slot) {
        case QSV_SLOT_COMP: comp_op<NV>(R, I, op, m0, m1, thread_ok); break;
        case QSV_SLOT_REG0 + 0: reg_op<NV, 0>(R, I, op, m0, m1, thread_ok); break;
        case QSV_SLOT_REG0 + 1: if constexpr (RB > 1) reg_op<NV, (RB > 1 ? 1 : 0)>(R, I, op, m0, m1, thread_ok); break;
        case QSV_SLOT_REG0 + 2: if constexpr (RB > 2) reg_op<NV, (RB > 2 ? 2 : 0)>(R, I, op, m0, m1, thread_ok); break;
        case QSV_SLOT_REG0 + 3: if constexpr (RB > 3) reg_op<NV, (RB > 3 ? 3 : 0)>(R, I, op, m0, m1, thread_ok); break;
        default: break;
    }
}

// ---------------------------------------------------------------- tensor-map TMA
__device__ __forceinline__ void tma_load(void *sdst, const CUtensorMap *map, const int32_t *c, int rank, uint64_t *bar) {
    const uint64_t m = reinterpret_cast<uint64_t>(map);
    const uint32_t d = smem_u32(sdst), b = smem_u32(bar);
    switch (rank) {
        case 2:
            asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                         ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(b) : "memory");
            break;
        case 3:
            asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                         ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(b) : "memory");
            break;
        case 4:
            asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
                         ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(b) : "memory");
            break;
        default:
            asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
                         ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(b) : "memory");
            break;
    }
}
__device__ __forceinline__ void tma_store(const CUtensorMap *map, const int32_t *c, int rank, const void *ssrc) {
    const uint64_t m = reinterpret_cast<uint64_t>(map);
    const uint32_t s = smem_u32(ssrc);
    switch (rank) {
        case 2:
            asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
                         ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(s) : "memory");
            break;
        case 3:
            asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];"
                         ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(s) : "memory");
            break;
        case 4:
            asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];"
                         ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(s) : "memory");
            break;
        default:
            asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];"
                         ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(s) : "memory");
            break;
    }
}

// ---------------------------------------------------------------- the sweep kernel
template <int KW, int RB, int WB, int S>
__global__ void __launch_bounds__((1 << (5 + WB)) + 32, (KW >= 13 ? 1 : 2))
    sweep_kernel(float2 *__restrict__ state, const __grid_constant__ QsvSweep P, const __grid_constant__ CUtensorMap tmap) {
    constexpr int NC = 1 << (5 + WB);        // consumer threads
    constexpr int NV = 1 << RB;              // float4 per consumer thread
    constexpr int TILE = 1 << KW;            // amplitudes per tile
    static_assert(1 + 3 + 2 + RB + WB == KW, "layout must cover the window");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    float2 *bufs = reinterpret_cast<float2 *>(smem_raw);
    // the sweep's op table, copied once from the parameter block: shared-memory reads of an op's fields
    // are independent short-latency loads (the constant-bank path serialises them per op)
    QsvOp *sops = reinterpret_cast<QsvOp *>(smem_raw + ((size_t)S << KW) * sizeof(float2));
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t done[S];
    __shared__ volatile int abort_flag;

    const int tid = threadIdx.x;
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(P.ops);
        uint32_t *dst = reinterpret_cast<uint32_t *>(sops);
        const int words = P.nops * (int)(sizeof(QsvOp) / 4);
        for (int i = tid; i < words; i += blockDim.x) dst[i] = src[i];
    }
    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&done[s], NC);
        }
        abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();

    const int64_t ntiles = P.ntiles;
    const int64_t first = blockIdx.x, stride = gridDim.x;
    const int64_t nmine = first < ntiles ? (ntiles - 1 - first) / stride + 1 : 0;

    if (tid >= NC) {
        // ------------------------------------------------------------ producer warp
        const int lane = tid & 31;
        const int lo = P.lo;
        const int rank = P.tma_rank;
        auto coords = [&](int64_t T, int32_t *c) {
            int pos = 0;
            for (int d = 0; d < rank; d++) {
                const int f = P.tdim_free[d];
                c[d] = (int32_t)(((T >> pos) & ((1ll << f) - 1)) << P.tdim_box[d]);
                pos += f;
            }
        };
        const int nsub = 1 << (KW - lo);
        const uint32_t subbytes = 8u << lo;
        const int nh = P.nh;
        auto tile_base = [&](int64_t T) -> int64_t {
            int64_t x = T << lo;                      // free bits are the bits outside [0, lo) U H
            for (int i = 0; i < nh; i++) {
                const int h = P.H[i];
                x = ((x >> h) << (h + 1)) | (x & ((1ll << h) - 1));
            }
            return x;
        };
        auto sub_off = [&](int s) -> int64_t {
            int64_t o = 0;
            for (int i = 0; i < KW - lo; i++)
                if ((s >> i) & 1) o |= 1ll << P.H[i];
            return o;
        };
        auto issue_load = [&](int64_t j, int b) {
            const int64_t T = first + j * stride;
            float2 *dst = bufs + (size_t)b * TILE;
            if (rank) {
                if (lane == 0) {
                    int32_t c[QSV_TMA_MAX_RANK];
                    coords(T, c);
                    mbar_arrive_expect_tx(&full[b], (uint32_t)TILE * 8u);
                    tma_load(dst, &tmap, c, rank, &full[b]);
                }
                return;
            }
            const int64_t base = tile_base(T);
            if (lane == 0) mbar_arrive_expect_tx(&full[b], (uint32_t)TILE * 8u);
            __syncwarp();
            for (int s = lane; s < nsub; s += 32) bulk_g2s(dst + (s << lo), state + (base | sub_off(s)), subbytes, &full[b]);
        };
        auto issue_store = [&](int64_t j, int b) {
            const int64_t T = first + j * stride;
            const float2 *src = bufs + (size_t)b * TILE;
            if (rank) {
                if (lane == 0) {
                    int32_t c[QSV_TMA_MAX_RANK];
                    coords(T, c);
                    tma_store(&tmap, c, rank, src);
                    bulk_commit();
                }
                return;
            }
            const int64_t base = tile_base(T);
            for (int s = lane; s < nsub; s += 32) bulk_s2g(state + (base | sub_off(s)), src + (s << lo), subbytes);
            bulk_commit();
        };
        for (int64_t j = 0; j < S && j < nmine; j++) issue_load(j, (int)j);
        for (int64_t j = 0; j < nmine; j++) {
            const int b = (int)(j % S);
            const uint32_t par = (uint32_t)((j / S) & 1);
            if (!mbar_wait(&done[b], par, &abort_flag, &g_status)) break;
            issue_store(j, b);
            if (j + S < nmine) {
                bulk_wait_read_all();                 // this lane's stores have read the buffer
                __syncwarp();
                issue_load(j + S, b);
            }
        }
        bulk_wait_all();
        return;
    }

    // ---------------------------------------------------------------- consumer warps
    const int lane = tid & 31, warp = tid >> 5;
    for (int64_t j = 0; j < nmine; j++) {
        const int b = (int)(j % S);
        const uint32_t par = (uint32_t)((j / S) & 1);
        if (!mbar_wait(&full[b], par, &abort_flag, &g_status)) break;
        float2 *tile = bufs + (size_t)b * TILE;
        for (int ph = 0; ph < P.nphases; ph++) {
            if (ph > 0) named_bar_sync(1, NC);
            const QsvPhase &Q = P.phases[ph];
            uint32_t tb = ((uint32_t)(lane & 7) << 1) | ((uint32_t)((lane >> 3) & 1) << Q.lane_bits[0]) |
                          ((uint32_t)((lane >> 4) & 1) << Q.lane_bits[1]);
#pragma unroll
            for (int w = 0; w < WB; w++) tb |= (uint32_t)((warp >> w) & 1) << Q.warp_bits[w];
            uint32_t rbit[RB];
#pragma unroll
            for (int r = 0; r < RB; r++) rbit[r] = 1u << Q.reg_bits[r];
            auto pos = [&](int r) -> uint32_t {
                uint32_t o = tb;
#pragma unroll
                for (int q = 0; q < RB; q++)
                    if ((r >> q) & 1) o |= rbit[q];
                return o;
            };
            float2 R[NV], I[NV];
#pragma unroll
            for (int r = 0; r < NV; r++) {
                const float4 v = *reinterpret_cast<const float4 *>(tile + pos(r));
                R[r] = make_float2(v.x, v.z);
                I[r] = make_float2(v.y, v.w);
            }
            for (int o = Q.op_begin; o < Q.op_end; o++) apply_op<NV, RB>(sops[o], R, I, tb, lane);
#pragma unroll
            for (int r = 0; r < NV; r++)
                *reinterpret_cast<float4 *>(tile + pos(r)) = make_float4(R[r].x, I[r].x, R[r].y, I[r].y);
        }
        fence_proxy_async_smem();
        mbar_arrive(&done[b]);
    }
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
static cudaError_t make_tmap(CUtensorMap *map, float2 *state, const QsvSweep &sw) {
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
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_INT64, sw.tma_rank, state, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int KW, int RB, int WB, int S>
static cudaError_t launch_sweep_t(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream) {
    constexpr int NT = (1 << (5 + WB)) + 32;
    const size_t smem = ((size_t)S << KW) * sizeof(float2) + sizeof(QsvOp) * QSV_MAX_SWEEP_OPS;
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
