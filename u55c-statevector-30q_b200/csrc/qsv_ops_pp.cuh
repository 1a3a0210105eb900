// qsv_ops_pp.cuh -- the interpreter's ping-pong form: ops that rewrite every amplitude a thread holds read
// one register set and write the other.
//
// The interpreter (qsv_sweep.cu) dispatches each op at run time. When every op updates the thread's 2^RB
// packed slots in place, the values of each dispatch branch must end up in the same registers at the join
// after the switch, and the compiler reconciles them with register moves (the profile of the in-place
// interpreter shows about two moves per FMA). Here the ops whose code path writes every slot (uniform
// dense / diagonal / swap, general MUX, and the branch-free controlled dense form) are applied out of place:
// A -> B, then the next one B -> A, so each branch computes its results straight into the other set and the
// join has nothing to reconcile. Ops that update only some slots (controlled ops with a branch per slot)
// stay in place on the current set (qsv_ops.cuh). The host marks each op's form (QsvOp::oop, set by
// the planner). Same arithmetic as qsv_ops.cuh, chain for chain, so values are identical.
#pragma once
#include "qsv_ops.cuh"

namespace qsv {
namespace dev {

// ---------------------------------------------------------------- packed math, results to new registers
// dense2 (qsv_ops.cuh) with outputs separate from inputs: the same chains, term for term
__device__ __forceinline__ void dense2o(const float2 R0, const float2 I0, const float2 R1, const float2 I1, float2 &oR0,
                                        float2 &oI0, float2 &oR1, float2 &oI1, const float *m) {
    float2 t, u;
    t = __fmul2_rn(f2(-m[3]), I1); t = __ffma2_rn(f2(m[2]), R1, t); t = __ffma2_rn(f2(-m[1]), I0, t);
    oR0 = __ffma2_rn(f2(m[0]), R0, t);
    u = __fmul2_rn(f2(m[3]), R1);  u = __ffma2_rn(f2(m[2]), I1, u); u = __ffma2_rn(f2(m[1]), R0, u);
    oI0 = __ffma2_rn(f2(m[0]), I0, u);
    t = __fmul2_rn(f2(-m[5]), I0); t = __ffma2_rn(f2(m[4]), R0, t); t = __ffma2_rn(f2(-m[7]), I1, t);
    oR1 = __ffma2_rn(f2(m[6]), R1, t);
    u = __fmul2_rn(f2(m[5]), R0);  u = __ffma2_rn(f2(m[4]), I0, u); u = __ffma2_rn(f2(m[7]), R1, u);
    oI1 = __ffma2_rn(f2(m[6]), I1, u);
}
// dense2_r0 with separate outputs (m00 real: its two imaginary terms, exact zeros, are skipped)
__device__ __forceinline__ void dense2o_r0(const float2 R0, const float2 I0, const float2 R1, const float2 I1,
                                           float2 &oR0, float2 &oI0, float2 &oR1, float2 &oI1, const float *m) {
    float2 t, u;
    t = __fmul2_rn(f2(-m[3]), I1); t = __ffma2_rn(f2(m[2]), R1, t);
    oR0 = __ffma2_rn(f2(m[0]), R0, t);
    u = __fmul2_rn(f2(m[3]), R1);  u = __ffma2_rn(f2(m[2]), I1, u);
    oI0 = __ffma2_rn(f2(m[0]), I0, u);
    t = __fmul2_rn(f2(-m[5]), I0); t = __ffma2_rn(f2(m[4]), R0, t); t = __ffma2_rn(f2(-m[7]), I1, t);
    oR1 = __ffma2_rn(f2(m[6]), R1, t);
    u = __fmul2_rn(f2(m[5]), R0);  u = __ffma2_rn(f2(m[4]), I0, u); u = __ffma2_rn(f2(m[7]), R1, u);
    oI1 = __ffma2_rn(f2(m[6]), I1, u);
}
// dense2v with separate outputs (per-lane coefficients c[e] = (pair .x, pair .y))
__device__ __forceinline__ void dense2vo(const float2 R0, const float2 I0, const float2 R1, const float2 I1,
                                         float2 &oR0, float2 &oI0, float2 &oR1, float2 &oI1, const float2 *c) {
    const float2 n1 = make_float2(-c[1].x, -c[1].y), n3 = make_float2(-c[3].x, -c[3].y);
    const float2 n5 = make_float2(-c[5].x, -c[5].y), n7 = make_float2(-c[7].x, -c[7].y);
    float2 t, u;
    t = __fmul2_rn(n3, I1); t = __ffma2_rn(c[2], R1, t); t = __ffma2_rn(n1, I0, t);
    oR0 = __ffma2_rn(c[0], R0, t);
    u = __fmul2_rn(c[3], R1); u = __ffma2_rn(c[2], I1, u); u = __ffma2_rn(c[1], R0, u);
    oI0 = __ffma2_rn(c[0], I0, u);
    t = __fmul2_rn(n5, I0); t = __ffma2_rn(c[4], R0, t); t = __ffma2_rn(n7, I1, t);
    oR1 = __ffma2_rn(c[6], R1, t);
    u = __fmul2_rn(c[5], R0); u = __ffma2_rn(c[4], I0, u); u = __ffma2_rn(c[7], R1, u);
    oI1 = __ffma2_rn(c[6], I1, u);
}
// cmul2 with separate outputs: y = a * x
__device__ __forceinline__ void cmul2o(const float2 R, const float2 I, float2 &oR, float2 &oI, float ar, float ai) {
    oR = __ffma2_rn(f2(ar), R, __fmul2_rn(f2(-ai), I));
    oI = __ffma2_rn(f2(ar), I, __fmul2_rn(f2(ai), R));
}
// lane_lin with separate outputs: y = a*own + b*oth
__device__ __forceinline__ void lane_lin_o(const float2 R, const float2 I, const float2 oR, const float2 oI, float2 &yR,
                                           float2 &yI, const float2 ar, const float2 ai, const float2 nai,
                                           const float2 br, const float2 bi, const float2 nbi) {
    float2 t = __fmul2_rn(nbi, oI);
    t = __ffma2_rn(br, oR, t);
    t = __ffma2_rn(nai, I, t);
    yR = __ffma2_rn(ar, R, t);
    float2 u = __fmul2_rn(bi, oR);
    u = __ffma2_rn(br, oI, u);
    u = __ffma2_rn(ai, R, u);
    yI = __ffma2_rn(ar, I, u);
}

// ---------------------------------------------------------------- out-of-place ops by slot
template <int NV, int RBIT>
__device__ __forceinline__ void reg_op_oop(const float2 (&Ri)[NV], const float2 (&Ii)[NV], float2 (&Ro)[NV],
                                           float2 (&Io)[NV], const QsvOp &op, const float *m0, const float *m1,
                                           bool tok) {
    constexpr int B = 1 << RBIT;
    const int cm_reg = op.cm_reg;
    switch (op.variant) {
        case QSV_V_UNI_DENSE:
            if (op.r00) {
#pragma unroll
                for (int r = 0; r < NV; r++)
                    if (!(r & B)) dense2o_r0(Ri[r], Ii[r], Ri[r | B], Ii[r | B], Ro[r], Io[r], Ro[r | B], Io[r | B], m0);
            } else {
#pragma unroll
                for (int r = 0; r < NV; r++)
                    if (!(r & B)) dense2o(Ri[r], Ii[r], Ri[r | B], Ii[r | B], Ro[r], Io[r], Ro[r | B], Io[r | B], m0);
            }
            break;
        case QSV_V_UNI_DIAG:
#pragma unroll
            for (int r = 0; r < NV; r++) {
                if (r & B) continue;
                cmul2o(Ri[r], Ii[r], Ro[r], Io[r], m0[0], m0[1]);
                cmul2o(Ri[r | B], Ii[r | B], Ro[r | B], Io[r | B], m0[6], m0[7]);
            }
            break;
        case QSV_V_UNI_SWAP:
#pragma unroll
            for (int r = 0; r < NV; r++) { Ro[r] = Ri[r ^ B]; Io[r] = Ii[r ^ B]; }
            break;
        case QSV_V_CTRL_DENSE_SEL: {
            const float id[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f};
#pragma unroll
            for (int r = 0; r < NV; r++) {
                if (r & B) continue;
                const bool s = tok && (r & cm_reg) == cm_reg;
                float c[8];
#pragma unroll
                for (int e = 0; e < 8; e++) c[e] = s ? m1[e] : id[e];
                dense2o(Ri[r], Ii[r], Ri[r | B], Ii[r | B], Ro[r], Io[r], Ro[r | B], Io[r | B], c);
            }
            break;
        }
        default: {    // QSV_V_MUX
            const bool cc = op.cm_c;
#pragma unroll
            for (int r = 0; r < NV; r++) {
                if (r & B) continue;
                const bool sy = tok && (r & cm_reg) == cm_reg, sx = sy && !cc;
                float2 c[8];
#pragma unroll
                for (int e = 0; e < 8; e++) c[e] = make_float2(sx ? m1[e] : m0[e], sy ? m1[e] : m0[e]);
                dense2vo(Ri[r], Ii[r], Ri[r | B], Ii[r | B], Ro[r], Io[r], Ro[r | B], Io[r | B], c);
            }
            break;
        }
    }
}

// tile-bit-0 target, uniform dense or diagonal matrix: scalar arithmetic on the two halves of each slot
template <int NV>
__device__ __forceinline__ void comp_op_oop(const float2 (&Ri)[NV], const float2 (&Ii)[NV], float2 (&Ro)[NV],
                                            float2 (&Io)[NV], const QsvOp &op, const float *m0) {
    const int mode = op.cls0 == QSV_M_DIAG ? 2 : op.r00 ? 1 : 0;
#pragma unroll
    for (int r = 0; r < NV; r++) {
        float x0r = Ri[r].x, x0i = Ii[r].x, x1r = Ri[r].y, x1i = Ii[r].y;
        if (mode == 0) pair_t<QSV_M_DENSE>(x0r, x0i, x1r, x1i, m0);
        else if (mode == 1) pair_t<QSV_M_DENSE_R0>(x0r, x0i, x1r, x1i, m0);
        else pair_t<QSV_M_DIAG>(x0r, x0i, x1r, x1i, m0);
        Ro[r] = make_float2(x0r, x1r);
        Io[r] = make_float2(x0i, x1i);
    }
}

// lane-bit target: uniform dense / diagonal / swap, or the general MUX
template <int NV>
__device__ __forceinline__ void lane_op_oop(const float2 (&Ri)[NV], const float2 (&Ii)[NV], float2 (&Ro)[NV],
                                            float2 (&Io)[NV], const QsvOp &op, const float *m0, const float *m1,
                                            bool tok, int lanebit, int lane) {
    const int xm = 1 << lanebit;
    const bool mine = (lane >> lanebit) & 1;
    const int var = op.variant;
    if (var == QSV_V_UNI_DENSE) {
        const float a_r = mine ? m0[6] : m0[0], a_i = mine ? m0[7] : m0[1];
        const float b_r = mine ? m0[4] : m0[2], b_i = mine ? m0[5] : m0[3];
        const float2 ar = f2(a_r), ai = f2(a_i), nai = f2(-a_i), br = f2(b_r), bi = f2(b_i), nbi = f2(-b_i);
#pragma unroll
        for (int r = 0; r < NV; r++) {
            float2 oR, oI;
            shfl4(Ri[r], Ii[r], oR, oI, xm);
            lane_lin_o(Ri[r], Ii[r], oR, oI, Ro[r], Io[r], ar, ai, nai, br, bi, nbi);
        }
        return;
    }
    if (var == QSV_V_UNI_DIAG) {
        const float a_r = mine ? m0[6] : m0[0], a_i = mine ? m0[7] : m0[1];
#pragma unroll
        for (int r = 0; r < NV; r++) cmul2o(Ri[r], Ii[r], Ro[r], Io[r], a_r, a_i);
        return;
    }
    if (var == QSV_V_UNI_SWAP) {
#pragma unroll
        for (int r = 0; r < NV; r++) shfl4(Ri[r], Ii[r], Ro[r], Io[r], xm);
        return;
    }
    // general MUX (lane_op of qsv_ops.cuh with separate outputs)
    const int cm_reg = op.cm_reg;
    const bool ctrl = op.kind == QSV_K_CTRL, cc = op.cm_c;
    const float a0r = mine ? m0[6] : m0[0], a0i = mine ? m0[7] : m0[1];
    const float b0r = mine ? m0[4] : m0[2], b0i = mine ? m0[5] : m0[3];
    const float a1r = mine ? m1[6] : m1[0], a1i = mine ? m1[7] : m1[1];
    const float b1r = mine ? m1[4] : m1[2], b1i = mine ? m1[5] : m1[3];
#pragma unroll
    for (int r = 0; r < NV; r++) {
        float2 oR, oI;
        shfl4(Ri[r], Ii[r], oR, oI, xm);
        const bool sy = tok && (r & cm_reg) == cm_reg, sx = sy && !cc;
        const float u0r = ctrl ? 1.f : a0r, u0i = ctrl ? 0.f : a0i, v0r = ctrl ? 0.f : b0r, v0i = ctrl ? 0.f : b0i;
        const float2 ar = make_float2(sx ? a1r : u0r, sy ? a1r : u0r);
        const float2 ai = make_float2(sx ? a1i : u0i, sy ? a1i : u0i);
        const float2 br = make_float2(sx ? b1r : v0r, sy ? b1r : v0r);
        const float2 bi = make_float2(sx ? b1i : v0i, sy ? b1i : v0i);
        lane_lin_o(Ri[r], Ii[r], oR, oI, Ro[r], Io[r], ar, ai, make_float2(-ai.x, -ai.y), br, bi,
                   make_float2(-bi.x, -bi.y));
    }
}

template <int NV, int RB>
__device__ __forceinline__ void apply_op_oop(const QsvOp &op, const float2 (&Ri)[NV], const float2 (&Ii)[NV],
                                             float2 (&Ro)[NV], float2 (&Io)[NV], uint32_t tb, int lane) {
    float m0[8], m1[8];
#pragma unroll
    for (int e = 0; e < 8; e++) { m0[e] = op.m0[e]; m1[e] = op.m1[e]; }
    const uint32_t cm_thr = op.cm_thr;
    const bool tok = (tb & cm_thr) == cm_thr;
    const int slot = op.slot;
    if (slot >= QSV_SLOT_LANE0) {
        lane_op_oop<NV>(Ri, Ii, Ro, Io, op, m0, m1, tok, slot - QSV_SLOT_LANE0, lane);
        return;
    }
    switch (slot) {
        case QSV_SLOT_COMP: comp_op_oop<NV>(Ri, Ii, Ro, Io, op, m0); break;
        case QSV_SLOT_REG0 + 0: reg_op_oop<NV, 0>(Ri, Ii, Ro, Io, op, m0, m1, tok); break;
        case QSV_SLOT_REG0 + 1: if constexpr (RB > 1) reg_op_oop<NV, (RB > 1 ? 1 : 0)>(Ri, Ii, Ro, Io, op, m0, m1, tok); break;
        case QSV_SLOT_REG0 + 2: if constexpr (RB > 2) reg_op_oop<NV, (RB > 2 ? 2 : 0)>(Ri, Ii, Ro, Io, op, m0, m1, tok); break;
        default: if constexpr (RB > 3) reg_op_oop<NV, (RB > 3 ? 3 : 0)>(Ri, Ii, Ro, Io, op, m0, m1, tok); break;
    }
}

// One phase of a tile with the ping-pong interpreter: the thread's slots in register set A; each op marked
// oop moves them to the other set, the others update the current set in place (apply_op, qsv_ops.cuh).
template <int NV, int RB, int WB, class PH>
__device__ __forceinline__ void run_phase_pp(float2 *tile, const PH &Q, const QsvOp *ops, int op_begin, int op_end,
                                             int lane, int warp, bool swz = false) {
    uint32_t tb = ((uint32_t)(lane & 1) << Q.lane_lo[0]) | ((uint32_t)((lane >> 1) & 1) << Q.lane_lo[1]) |
                  ((uint32_t)((lane >> 2) & 1) << Q.lane_lo[2]) | ((uint32_t)((lane >> 3) & 1) << Q.lane_bits[0]) |
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
    auto addr = [&](int r) -> uint32_t { return swz ? swz128(pos(r)) : pos(r); };
    float2 RA[NV], IA[NV], RB_[NV], IB_[NV];
#pragma unroll
    for (int r = 0; r < NV; r++) {
        const float4 v = *reinterpret_cast<const float4 *>(tile + addr(r));
        RA[r] = make_float2(v.x, v.z);
        IA[r] = make_float2(v.y, v.w);
    }
    bool inB = false;
    for (int o = op_begin; o < op_end; o++) {
        const QsvOp &op = ops[o];
        if (op.oop) {
            if (inB) apply_op_oop<NV, RB>(op, RB_, IB_, RA, IA, tb, lane);
            else apply_op_oop<NV, RB>(op, RA, IA, RB_, IB_, tb, lane);
            inB = !inB;
        } else {
            if (inB) apply_op<NV, RB>(op, RB_, IB_, tb, lane);
            else apply_op<NV, RB>(op, RA, IA, tb, lane);
        }
    }
    if (inB) {
#pragma unroll
        for (int r = 0; r < NV; r++)
            *reinterpret_cast<float4 *>(tile + addr(r)) = make_float4(RB_[r].x, IB_[r].x, RB_[r].y, IB_[r].y);
    } else {
#pragma unroll
        for (int r = 0; r < NV; r++)
            *reinterpret_cast<float4 *>(tile + addr(r)) = make_float4(RA[r].x, IA[r].x, RA[r].y, IA[r].y);
    }
}

}  // namespace dev
}  // namespace qsv
