// qsv_sweep_d.cu -- complex128 sweeps: the pass engine on FP64 states with FP64 matrices (sm_100a).
//
// No reference counterpart (the FPGA engine is complex64 only); this is the on-GPU FP64 path of the
// precision study (a 32-qubit complex128 state is 64 GiB). Same sweep plans, addressing and staging
// pipeline as the complex64 engine (qsv_sweep_body.cuh, bulk-async copies only), with one 16-byte
// amplitude per thread slot: tile bits 0-2 are lane bits 0-2, two chosen tile bits are lane bits 3-4,
// four are register bits and the rest warp bits (windows of at most 12 qubits: 3 x 64 KiB buffers).
// Every pair update is the canonical fused-multiply-add chain in double precision
//   y0.re = fma(m00.re, x0.re, fma(-m00.im, x0.im, fma(m01.re, x1.re, -(m01.im * x1.im))))  (etc.)
// which the CPU oracle's complex128 engine writes identically, so results agree value for value; the
// diagonal / swap / identity forms skip exact-zero terms only.
#include <cuda_runtime.h>

#include "qsv_device.cuh"
#include "qsv_planner.h"
#include "qsv_sweep_body.cuh"

namespace qsv {
namespace dev {

__device__ __forceinline__ void lin_own_d(double &yr, double &yi, double ar, double ai, double br, double bi,
                                          double owr, double owi, double otr, double oti) {
    yr = fma(ar, owr, fma(-ai, owi, fma(br, otr, -__dmul_rn(bi, oti))));
    yi = fma(ar, owi, fma(ai, owr, fma(br, oti, __dmul_rn(bi, otr))));
}
__device__ __forceinline__ void diag_own_d(double &yr, double &yi, double ar, double ai, double owr, double owi) {
    yr = fma(ar, owr, -__dmul_rn(ai, owi));
    yi = fma(ar, owi, __dmul_rn(ai, owr));
}

// pair (x0, x1) held by one thread, matrix m of class cls
__device__ __forceinline__ void pair_apply_d(double2 &x0, double2 &x1, const double *m, int cls) {
    if (cls == QSV_M_DENSE) {
        double2 y0, y1;
        lin_own_d(y0.x, y0.y, m[0], m[1], m[2], m[3], x0.x, x0.y, x1.x, x1.y);
        lin_own_d(y1.x, y1.y, m[6], m[7], m[4], m[5], x1.x, x1.y, x0.x, x0.y);
        x0 = y0;
        x1 = y1;
    } else if (cls == QSV_M_DIAG) {
        double2 y0, y1;
        diag_own_d(y0.x, y0.y, m[0], m[1], x0.x, x0.y);
        diag_own_d(y1.x, y1.y, m[6], m[7], x1.x, x1.y);
        x0 = y0;
        x1 = y1;
    } else if (cls == QSV_M_DIAG1) {
        double2 y1;
        diag_own_d(y1.x, y1.y, m[6], m[7], x1.x, x1.y);
        x1 = y1;
    } else if (cls == QSV_M_XSWAP) {
        const double2 t = x0;
        x0 = x1;
        x1 = t;
    }
}

// own amplitude with its partner oth from the other lane; mine = 1 on the bit-1 side
__device__ __forceinline__ void own_apply_d(double2 &own, const double2 oth, const double *m, int cls, bool mine) {
    if (cls == QSV_M_DENSE) {
        double2 y;
        lin_own_d(y.x, y.y, mine ? m[6] : m[0], mine ? m[7] : m[1], mine ? m[4] : m[2], mine ? m[5] : m[3], own.x,
                  own.y, oth.x, oth.y);
        own = y;
    } else if (cls == QSV_M_DIAG || (cls == QSV_M_DIAG1 && mine)) {
        double2 y;
        diag_own_d(y.x, y.y, mine ? m[6] : m[0], mine ? m[7] : m[1], own.x, own.y);
        own = y;
    } else if (cls == QSV_M_XSWAP) {
        own = oth;
    }
}

template <int NV, int RBIT>
__device__ __forceinline__ void reg_op_d(double2 (&A)[NV], const QsvOpD &op, const double *m0, const double *m1,
                                         bool tok) {
    constexpr int B = 1 << RBIT;
    const int cm_reg = op.cm_reg, kind = op.kind, cls0 = op.cls0, cls1 = op.cls1;
#pragma unroll
    for (int r = 0; r < NV; r++) {
        if (r & B) continue;
        if (kind == QSV_K_UNI) {
            pair_apply_d(A[r], A[r | B], m0, cls0);
            continue;
        }
        const bool s = tok && (r & cm_reg) == cm_reg;
        if (s) pair_apply_d(A[r], A[r | B], m1, cls1);
        else if (kind == QSV_K_MUX) pair_apply_d(A[r], A[r | B], m0, cls0);
    }
}

template <int NV>
__device__ __forceinline__ void lane_op_d(double2 (&A)[NV], const QsvOpD &op, const double *m0, const double *m1,
                                          bool tok, int lanebit, int lane) {
    const int xm = 1 << lanebit;
    const bool mine = (lane >> lanebit) & 1;
    const int cm_reg = op.cm_reg, kind = op.kind, cls0 = op.cls0, cls1 = op.cls1;
#pragma unroll
    for (int r = 0; r < NV; r++) {
        double2 oth;
        oth.x = __shfl_xor_sync(0xffffffffu, A[r].x, xm);
        oth.y = __shfl_xor_sync(0xffffffffu, A[r].y, xm);
        const bool use1 = kind != QSV_K_UNI && tok && (r & cm_reg) == cm_reg;
        if (kind == QSV_K_CTRL && !use1) continue;
        // separate calls: a pointer select between the coefficient arrays would put them in local memory
        if (use1) own_apply_d(A[r], oth, m1, cls1, mine);
        else own_apply_d(A[r], oth, m0, cls0, mine);
    }
}

template <int NV, int RB>
__device__ __forceinline__ void apply_op_d(const QsvOpD &op, double2 (&A)[NV], uint32_t tb, int lane) {
    if (op.variant == QSV_V_SKIP) return;
    double m0[8], m1[8];
#pragma unroll
    for (int e = 0; e < 8; e++) { m0[e] = op.m0[e]; m1[e] = op.m1[e]; }
    const bool tok = (tb & op.cm_thr) == op.cm_thr;
    const int slot = op.slot;
    if (slot >= QSV_SLOT_LANE0) {
        lane_op_d<NV>(A, op, m0, m1, tok, slot - QSV_SLOT_LANE0, lane);
        return;
    }
    switch (slot) {
        case QSV_SLOT_REG0 + 0: reg_op_d<NV, 0>(A, op, m0, m1, tok); break;
        case QSV_SLOT_REG0 + 1: if constexpr (RB > 1) reg_op_d<NV, (RB > 1 ? 1 : 0)>(A, op, m0, m1, tok); break;
        case QSV_SLOT_REG0 + 2: if constexpr (RB > 2) reg_op_d<NV, (RB > 2 ? 2 : 0)>(A, op, m0, m1, tok); break;
        case QSV_SLOT_REG0 + 3: if constexpr (RB > 3) reg_op_d<NV, (RB > 3 ? 3 : 0)>(A, op, m0, m1, tok); break;
        default: break;
    }
}

// the complex128 interpreter body: per phase, each thread loads its 2^RB amplitudes (tile bits 0-2 from
// lane bits 0-2), applies the phase's ops and stores them back
struct InterpBodyD {
    using Amp = double2;
    static constexpr int kHalfBits = 0;
    static constexpr bool kSmemOps = true;
    template <int NV, int RB, int WB>
    static __device__ __forceinline__ void tile(double2 *tile, const QsvSweepD &P, const QsvOpD *sops, int lane,
                                                int warp, int bar) {
        constexpr int NC = 1 << (5 + WB);
        for (int ph = 0; ph < P.nphases; ph++) {
            if (ph > 0) named_bar_sync(bar, NC);
            const QsvPhase &Q = P.phases[ph];
            uint32_t tb = (uint32_t)(lane & 7) | ((uint32_t)((lane >> 3) & 1) << Q.lane_bits[0]) |
                          ((uint32_t)((lane >> 4) & 1) << Q.lane_bits[1]);
#pragma unroll
            for (int w = 0; w < WB; w++) tb |= (uint32_t)((warp >> w) & 1) << Q.warp_bits[w];
            uint32_t rbit[RB];
#pragma unroll
            for (int q = 0; q < RB; q++) rbit[q] = 1u << Q.reg_bits[q];
            auto pos = [&](int r) -> uint32_t {
                uint32_t o = tb;
#pragma unroll
                for (int q = 0; q < RB; q++)
                    if ((r >> q) & 1) o |= rbit[q];
                return o;
            };
            double2 A[NV];
#pragma unroll
            for (int r = 0; r < NV; r++) A[r] = tile[pos(r)];
            for (int o = Q.op_begin; o < Q.op_end; o++) apply_op_d<NV, RB>(sops[o], A, tb, lane);
#pragma unroll
            for (int r = 0; r < NV; r++) tile[pos(r)] = A[r];
        }
    }
};

template <int KW, int RB, int WB, int S>
__global__ void __launch_bounds__((1 << (5 + WB)) + 32, 1)
    sweep_kernel_c128(double2 *__restrict__ state, const __grid_constant__ QsvSweepD P, int *status) {
    sweep_pipeline<KW, RB, WB, S, 1, InterpBodyD, QsvSweepD>(state, P, nullptr, status);
}

template <int KW, int RB, int WB, int S>
static cudaError_t launch_c128_t(double2 *state, const QsvSweepD &sw, int nsm, int *status, cudaStream_t stream) {
    constexpr int NT = (1 << (5 + WB)) + 32;
    const size_t smem = sweep_smem_bytes<KW, S, InterpBodyD, QsvSweepD>();
    static int configured_dev = -1;     // attribute set once per device (under the engine's launch lock)
    static int per_sm = 1;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (configured_dev != dev) {
        e = cudaFuncSetAttribute(sweep_kernel_c128<KW, RB, WB, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_kernel_c128<KW, RB, WB, S>, NT, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        configured_dev = dev;
    }
    int64_t grid = (int64_t)nsm * per_sm;
    if (grid > sw.ntiles) grid = sw.ntiles;
    sweep_kernel_c128<KW, RB, WB, S><<<(unsigned)grid, NT, smem, stream>>>(state, sw, status);
    return cudaGetLastError();
}

}  // namespace dev

cudaError_t status_word_ptr(int **out);

cudaError_t launch_sweep_c128(double2 *state, const QsvSweepD &sw, int nsm, cudaStream_t stream) {
    if (sw.tma_rank != 0) return cudaErrorInvalidValue;        // complex128 plans stage with bulk copies
    int *status = nullptr;
    cudaError_t e = status_word_ptr(&status);
    if (e != cudaSuccess) return e;
    switch (sw.kw) {
        case 12: return dev::launch_c128_t<12, 4, 3, 3>(state, sw, nsm, status, stream);
        case 11: return dev::launch_c128_t<11, 4, 2, 3>(state, sw, nsm, status, stream);
        case 10: return dev::launch_c128_t<10, 4, 1, 3>(state, sw, nsm, status, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace qsv
