// qsv_ops.cuh -- in-register application of MUX2 ops for the tile kernels (sweep and batch).
//
// A consumer thread keeps 2^RB float4 of its tile (the two halves of each float4 = tile bit 0) repacked
// as float2 (re, re) / (im, im) pairs, so one packed FP32x2 FMA updates two amplitude pairs. Ops on tile
// bit 0 pair the halves of a float4 (scalar arithmetic), ops on register bits pair two float4, ops on lane
// bits exchange with the partner lane by warp shuffles. The arithmetic is the canonical fused-multiply-add
// chain of qsv_device.cuh for every variant (the specialised variants only skip exact-zero terms).
#pragma once
#include "qsv_device.cuh"

namespace qsv {
namespace dev {

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
// dense with m00 real: the two m00.im terms (exact zeros) are skipped; same values as dense2
__device__ __forceinline__ void dense2_r0(float2 &R0, float2 &I0, float2 &R1, float2 &I1, const float *m) {
    float2 t, u;
    t = __fmul2_rn(f2(-m[3]), I1); t = __ffma2_rn(f2(m[2]), R1, t);
    const float2 y0r = __ffma2_rn(f2(m[0]), R0, t);
    u = __fmul2_rn(f2(m[3]), R1);  u = __ffma2_rn(f2(m[2]), I1, u);
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

// The same chains as dense2 / dense2_r0 / cmul2, issued with every partial sum first and the final
// multiply-adds last: each final is the last use of the input it replaces, so it can be written over that
// input's register (code that dispatches ops at run time then keeps the amplitudes in place).
__device__ __forceinline__ void dense2_ip(float2 &R0, float2 &I0, float2 &R1, float2 &I1, const float *m) {
    float2 t0 = __fmul2_rn(f2(-m[3]), I1), u0 = __fmul2_rn(f2(m[3]), R1);
    float2 t1 = __fmul2_rn(f2(-m[5]), I0), u1 = __fmul2_rn(f2(m[5]), R0);
    t0 = __ffma2_rn(f2(m[2]), R1, t0); u0 = __ffma2_rn(f2(m[2]), I1, u0);
    t1 = __ffma2_rn(f2(m[4]), R0, t1); u1 = __ffma2_rn(f2(m[4]), I0, u1);
    t0 = __ffma2_rn(f2(-m[1]), I0, t0); u0 = __ffma2_rn(f2(m[1]), R0, u0);
    t1 = __ffma2_rn(f2(-m[7]), I1, t1); u1 = __ffma2_rn(f2(m[7]), R1, u1);
    R0 = __ffma2_rn(f2(m[0]), R0, t0); I0 = __ffma2_rn(f2(m[0]), I0, u0);
    R1 = __ffma2_rn(f2(m[6]), R1, t1); I1 = __ffma2_rn(f2(m[6]), I1, u1);
}
__device__ __forceinline__ void dense2_r0_ip(float2 &R0, float2 &I0, float2 &R1, float2 &I1, const float *m) {
    float2 t0 = __fmul2_rn(f2(-m[3]), I1), u0 = __fmul2_rn(f2(m[3]), R1);
    float2 t1 = __fmul2_rn(f2(-m[5]), I0), u1 = __fmul2_rn(f2(m[5]), R0);
    t0 = __ffma2_rn(f2(m[2]), R1, t0); u0 = __ffma2_rn(f2(m[2]), I1, u0);
    t1 = __ffma2_rn(f2(m[4]), R0, t1); u1 = __ffma2_rn(f2(m[4]), I0, u1);
    t1 = __ffma2_rn(f2(-m[7]), I1, t1); u1 = __ffma2_rn(f2(m[7]), R1, u1);
    R0 = __ffma2_rn(f2(m[0]), R0, t0); I0 = __ffma2_rn(f2(m[0]), I0, u0);
    R1 = __ffma2_rn(f2(m[6]), R1, t1); I1 = __ffma2_rn(f2(m[6]), I1, u1);
}
__device__ __forceinline__ void cmul2_ip(float2 &R, float2 &I, float ar, float ai) {
    const float2 p = __fmul2_rn(f2(-ai), I), q = __fmul2_rn(f2(ai), R);
    R = __ffma2_rn(f2(ar), R, p);
    I = __ffma2_rn(f2(ar), I, q);
}
template <bool IP>
__device__ __forceinline__ void dense2_t(float2 &R0, float2 &I0, float2 &R1, float2 &I1, const float *m) {
    if constexpr (IP) dense2_ip(R0, I0, R1, I1, m);
    else dense2(R0, I0, R1, I1, m);
}
template <bool IP>
__device__ __forceinline__ void dense2_r0_t(float2 &R0, float2 &I0, float2 &R1, float2 &I1, const float *m) {
    if constexpr (IP) dense2_r0_ip(R0, I0, R1, I1, m);
    else dense2_r0(R0, I0, R1, I1, m);
}
template <bool IP>
__device__ __forceinline__ void cmul2_t(float2 &R, float2 &I, float ar, float ai) {
    if constexpr (IP) cmul2_ip(R, I, ar, ai);
    else cmul2(R, I, ar, ai);
}
__device__ __forceinline__ void swap2(float2 &a, float2 &b) {
    const float2 t = a; a = b; b = t;
}

// ---------------------------------------------------------------- ops by target slot
// Register-bit target RBIT: pairs (slot r, slot r | 2^RBIT); each float2 carries two pairs (tile bit 0 =
// 0 in .x, 1 in .y). One tight unrolled loop per code variant (selected on the host).
template <int NV, int RBIT, bool IP, int V, class O>
__device__ __forceinline__ void reg_case(float2 (&R)[NV], float2 (&I)[NV], const O &op, const float *m0,
                                         const float *m1, bool thread_ok) {
    const int cm_reg = op.cm_reg;
#define QSV_FOR_PAIRS for (int r = 0; r < NV; r++) if (!(r & (1 << RBIT)))
#define QSV_P1 (r | (1 << RBIT))
    if constexpr (V == QSV_V_UNI_DENSE) {
        if (op.r00) {
#pragma unroll
            QSV_FOR_PAIRS dense2_r0_t<IP>(R[r], I[r], R[QSV_P1], I[QSV_P1], m0);
        } else {
#pragma unroll
            QSV_FOR_PAIRS dense2_t<IP>(R[r], I[r], R[QSV_P1], I[QSV_P1], m0);
        }
    } else if constexpr (V == QSV_V_UNI_DIAG) {
#pragma unroll
        QSV_FOR_PAIRS { cmul2_t<IP>(R[r], I[r], m0[0], m0[1]); cmul2_t<IP>(R[QSV_P1], I[QSV_P1], m0[6], m0[7]); }
    } else if constexpr (V == QSV_V_UNI_SWAP) {
#pragma unroll
        QSV_FOR_PAIRS { swap2(R[r], R[QSV_P1]); swap2(I[r], I[QSV_P1]); }
    } else if constexpr (V == QSV_V_CTRL_DENSE) {
#pragma unroll
        QSV_FOR_PAIRS if (thread_ok && (r & cm_reg) == cm_reg) dense2_t<IP>(R[r], I[r], R[QSV_P1], I[QSV_P1], m1);
    } else if constexpr (V == QSV_V_CTRL_DIAG1) {
#pragma unroll
        QSV_FOR_PAIRS if (thread_ok && (r & cm_reg) == cm_reg) cmul2_t<IP>(R[QSV_P1], I[QSV_P1], m1[6], m1[7]);
    } else if constexpr (V == QSV_V_CTRL_SWAP) {
#pragma unroll
        QSV_FOR_PAIRS if (thread_ok && (r & cm_reg) == cm_reg) { swap2(R[r], R[QSV_P1]); swap2(I[r], I[QSV_P1]); }
    } else if constexpr (V == QSV_V_CTRL_DENSE_SEL) {
        const float id[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f};
#pragma unroll
        QSV_FOR_PAIRS {
            const bool s = thread_ok && (r & cm_reg) == cm_reg;
            float c[8];
#pragma unroll
            for (int e = 0; e < 8; e++) c[e] = s ? m1[e] : id[e];
            dense2_t<IP>(R[r], I[r], R[QSV_P1], I[QSV_P1], c);
        }
    } else if constexpr (V == QSV_V_CTRL_DIAG1_SEL) {
#pragma unroll
        QSV_FOR_PAIRS {
            const bool s = thread_ok && (r & cm_reg) == cm_reg;
            cmul2_t<IP>(R[QSV_P1], I[QSV_P1], s ? m1[6] : 1.f, s ? m1[7] : 0.f);
        }
    } else if constexpr (V == QSV_V_CTRL_SWAP_SEL) {
#pragma unroll
        QSV_FOR_PAIRS {
            const bool s = thread_ok && (r & cm_reg) == cm_reg;
            const float2 a = R[r], b = R[QSV_P1], c = I[r], d = I[QSV_P1];
            R[r] = s ? b : a; R[QSV_P1] = s ? a : b;
            I[r] = s ? d : c; I[QSV_P1] = s ? c : d;
        }
    } else if constexpr (V == QSV_V_MUX) {
        const bool cc = op.cm_c;
#pragma unroll
        QSV_FOR_PAIRS {
            const bool sy = thread_ok && (r & cm_reg) == cm_reg, sx = sy && !cc;
            float2 c[8];
#pragma unroll
            for (int e = 0; e < 8; e++) c[e] = make_float2(sx ? m1[e] : m0[e], sy ? m1[e] : m0[e]);
            dense2v(R[r], I[r], R[QSV_P1], I[QSV_P1], c);
        }
    }
#undef QSV_FOR_PAIRS
#undef QSV_P1
}

// the code path of op.variant, chosen at run time
template <int NV, int RBIT, bool IP = false, class O = QsvOp>
__device__ __forceinline__ void reg_op(float2 (&R)[NV], float2 (&I)[NV], const O &op, const float *m0,
                                       const float *m1, bool thread_ok) {
    switch (op.variant) {
        case QSV_V_UNI_DENSE: reg_case<NV, RBIT, IP, QSV_V_UNI_DENSE>(R, I, op, m0, m1, thread_ok); break;
        case QSV_V_UNI_DIAG: reg_case<NV, RBIT, IP, QSV_V_UNI_DIAG>(R, I, op, m0, m1, thread_ok); break;
        case QSV_V_UNI_SWAP: reg_case<NV, RBIT, IP, QSV_V_UNI_SWAP>(R, I, op, m0, m1, thread_ok); break;
        case QSV_V_CTRL_DENSE: reg_case<NV, RBIT, IP, QSV_V_CTRL_DENSE>(R, I, op, m0, m1, thread_ok); break;
        case QSV_V_CTRL_DIAG1: reg_case<NV, RBIT, IP, QSV_V_CTRL_DIAG1>(R, I, op, m0, m1, thread_ok); break;
        case QSV_V_CTRL_SWAP: reg_case<NV, RBIT, IP, QSV_V_CTRL_SWAP>(R, I, op, m0, m1, thread_ok); break;
        case QSV_V_CTRL_DENSE_SEL: reg_case<NV, RBIT, IP, QSV_V_CTRL_DENSE_SEL>(R, I, op, m0, m1, thread_ok); break;
        case QSV_V_CTRL_DIAG1_SEL: reg_case<NV, RBIT, IP, QSV_V_CTRL_DIAG1_SEL>(R, I, op, m0, m1, thread_ok); break;
        case QSV_V_CTRL_SWAP_SEL: reg_case<NV, RBIT, IP, QSV_V_CTRL_SWAP_SEL>(R, I, op, m0, m1, thread_ok); break;
        case QSV_V_MUX: reg_case<NV, RBIT, IP, QSV_V_MUX>(R, I, op, m0, m1, thread_ok); break;
        default: break;
    }
}

// tile-bit-0 target: the pair is the two halves of one slot (scalar arithmetic, any variant)
template <int NV, class O = QsvOp>
__device__ __forceinline__ void comp_op(float2 (&R)[NV], float2 (&I)[NV], const O &op, const float *m0,
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

// ---------------------------------------------------------------- shared building blocks
// lane update y = a*own + b*oth on two packed pairs (the lane_op arithmetic with hoisted coefficients)
__device__ __forceinline__ void lane_lin(float2 &R, float2 &I, const float2 oR, const float2 oI, const float2 ar,
                                         const float2 ai, const float2 nai, const float2 br, const float2 bi,
                                         const float2 nbi) {
    float2 t = __fmul2_rn(nbi, oI);
    t = __ffma2_rn(br, oR, t);
    t = __ffma2_rn(nai, I, t);
    const float2 yr = __ffma2_rn(ar, R, t);
    float2 u = __fmul2_rn(bi, oR);
    u = __ffma2_rn(br, oI, u);
    u = __ffma2_rn(ai, R, u);
    const float2 yi = __ffma2_rn(ar, I, u);
    R = yr;
    I = yi;
}
__device__ __forceinline__ void shfl4(const float2 &R, const float2 &I, float2 &oR, float2 &oI, int xm) {
    oR.x = __shfl_xor_sync(0xffffffffu, R.x, xm);
    oR.y = __shfl_xor_sync(0xffffffffu, R.y, xm);
    oI.x = __shfl_xor_sync(0xffffffffu, I.x, xm);
    oI.y = __shfl_xor_sync(0xffffffffu, I.y, xm);
}
// pair_apply with the matrix class fixed at compile time
template <int CLS>
__device__ __forceinline__ void pair_t(float &x0r, float &x0i, float &x1r, float &x1i, const float *m) {
    if constexpr (CLS == QSV_M_DENSE) {
        float y0r, y0i, y1r, y1i;
        lin_own(y0r, y0i, m[0], m[1], m[2], m[3], x0r, x0i, x1r, x1i);
        lin_own(y1r, y1i, m[6], m[7], m[4], m[5], x1r, x1i, x0r, x0i);
        x0r = y0r; x0i = y0i; x1r = y1r; x1i = y1i;
    } else if constexpr (CLS == QSV_M_DENSE_R0) {
        // m00.im is an exact zero: its two terms are skipped
        const float t = fmaf(m[2], x1r, -__fmul_rn(m[3], x1i));
        const float u = fmaf(m[2], x1i, __fmul_rn(m[3], x1r));
        float y1r, y1i;
        lin_own(y1r, y1i, m[6], m[7], m[4], m[5], x1r, x1i, x0r, x0i);
        x0r = fmaf(m[0], x0r, t); x0i = fmaf(m[0], x0i, u); x1r = y1r; x1i = y1i;
    } else if constexpr (CLS == QSV_M_DIAG) {
        float y0r, y0i, y1r, y1i;
        diag_own(y0r, y0i, m[0], m[1], x0r, x0i);
        diag_own(y1r, y1i, m[6], m[7], x1r, x1i);
        x0r = y0r; x0i = y0i; x1r = y1r; x1i = y1i;
    } else if constexpr (CLS == QSV_M_DIAG1) {
        float y1r, y1i;
        diag_own(y1r, y1i, m[6], m[7], x1r, x1i);
        x1r = y1r; x1i = y1i;
    } else if constexpr (CLS == QSV_M_XSWAP) {
        float t = x0r; x0r = x1r; x1r = t;
        t = x0i; x0i = x1i; x1i = t;
    }
}

// ---------------------------------------------------------------- one dispatch per op
// The interpreter's fast paths: a uniform switch per op selects a tight loop (coefficients hoisted, no
// per-pair selects). Same values as comp_op / lane_op (forms that skip work skip exact-zero terms or
// unselected pairs only).
template <int NV, int CLS, bool CTRL>
__device__ __forceinline__ void comp_loop(float2 (&R)[NV], float2 (&I)[NV], const float *m, int cm_reg, bool tok) {
#pragma unroll
    for (int r = 0; r < NV; r++) {
        if (CTRL && !(tok && (r & cm_reg) == cm_reg)) continue;
        float x0r = R[r].x, x0i = I[r].x, x1r = R[r].y, x1i = I[r].y;
        pair_t<CLS>(x0r, x0i, x1r, x1i, m);
        R[r] = make_float2(x0r, x1r);
        I[r] = make_float2(x0i, x1i);
    }
}

template <int NV, class O = QsvOp>
__device__ __forceinline__ void comp_op_fast(float2 (&R)[NV], float2 (&I)[NV], const O &op, const float *m0,
                                             const float *m1, bool tok) {
    const int cm_reg = op.cm_reg;
    if (op.kind == QSV_K_UNI) {
        switch (op.cls0) {
            case QSV_M_DENSE:
                if (op.r00) comp_loop<NV, QSV_M_DENSE_R0, false>(R, I, m0, 0, true);
                else comp_loop<NV, QSV_M_DENSE, false>(R, I, m0, 0, true);
                return;
            case QSV_M_DIAG: comp_loop<NV, QSV_M_DIAG, false>(R, I, m0, 0, true); return;
            case QSV_M_DIAG1: comp_loop<NV, QSV_M_DIAG1, false>(R, I, m0, 0, true); return;
            case QSV_M_XSWAP: comp_loop<NV, QSV_M_XSWAP, false>(R, I, m0, 0, true); return;
            case QSV_M_IDENT: return;
            default: break;
        }
    } else if (op.kind == QSV_K_CTRL) {
        switch (op.cls1) {
            case QSV_M_DENSE: comp_loop<NV, QSV_M_DENSE, true>(R, I, m1, cm_reg, tok); return;
            case QSV_M_DIAG: comp_loop<NV, QSV_M_DIAG, true>(R, I, m1, cm_reg, tok); return;
            case QSV_M_DIAG1: comp_loop<NV, QSV_M_DIAG1, true>(R, I, m1, cm_reg, tok); return;
            case QSV_M_XSWAP: comp_loop<NV, QSV_M_XSWAP, true>(R, I, m1, cm_reg, tok); return;
            case QSV_M_IDENT: return;
            default: break;
        }
    }
    comp_op<NV, O>(R, I, op, m0, m1, tok);
}

// comp_op_fast with the kind and matrix classes fixed at compile time (the same code paths)
template <int NV, int KIND, int CLS0, int CLS1, class O>
__device__ __forceinline__ void comp_fixed(float2 (&R)[NV], float2 (&I)[NV], const O &op, const float *m0,
                                           const float *m1, bool tok) {
    constexpr bool fast = CLS0 == QSV_M_DENSE || CLS0 == QSV_M_DIAG || CLS0 == QSV_M_DIAG1 ||
                          CLS0 == QSV_M_XSWAP || CLS0 == QSV_M_IDENT;
    constexpr bool fast1 = CLS1 == QSV_M_DENSE || CLS1 == QSV_M_DIAG || CLS1 == QSV_M_DIAG1 ||
                           CLS1 == QSV_M_XSWAP || CLS1 == QSV_M_IDENT;
    if constexpr (KIND == QSV_K_UNI && fast) {
        if constexpr (CLS0 == QSV_M_DENSE) {
            if (op.r00) comp_loop<NV, QSV_M_DENSE_R0, false>(R, I, m0, 0, true);
            else comp_loop<NV, QSV_M_DENSE, false>(R, I, m0, 0, true);
        } else if constexpr (CLS0 != QSV_M_IDENT) {
            comp_loop<NV, CLS0, false>(R, I, m0, 0, true);
        }
    } else if constexpr (KIND == QSV_K_CTRL && fast1) {
        if constexpr (CLS1 != QSV_M_IDENT) comp_loop<NV, CLS1, true>(R, I, m1, (int)op.cm_reg, tok);
    } else {
        comp_op<NV, O>(R, I, op, m0, m1, tok);
    }
}

template <int NV>
__device__ __forceinline__ void lane_op_fast(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op, const float *m0,
                                             const float *m1, bool tok, int lanebit, int lane) {
    const int xm = 1 << lanebit;
    const bool mine = (lane >> lanebit) & 1;
    const int cm_reg = op.cm_reg;
    const int var = op.variant;
    if (var == QSV_V_UNI_DENSE || var == QSV_V_CTRL_DENSE || var == QSV_V_CTRL_DENSE_SEL) {
        const bool uni = var == QSV_V_UNI_DENSE;
        // value selects (a pointer select between the two coefficient arrays would put them in local memory)
        const float a_r = uni ? (mine ? m0[6] : m0[0]) : (mine ? m1[6] : m1[0]);
        const float a_i = uni ? (mine ? m0[7] : m0[1]) : (mine ? m1[7] : m1[1]);
        const float b_r = uni ? (mine ? m0[4] : m0[2]) : (mine ? m1[4] : m1[2]);
        const float b_i = uni ? (mine ? m0[5] : m0[3]) : (mine ? m1[5] : m1[3]);
        const float2 ar = f2(a_r), ai = f2(a_i), nai = f2(-a_i), br = f2(b_r), bi = f2(b_i), nbi = f2(-b_i);
        if (uni) {
#pragma unroll
            for (int r = 0; r < NV; r++) {
                float2 oR, oI;
                shfl4(R[r], I[r], oR, oI, xm);
                lane_lin(R[r], I[r], oR, oI, ar, ai, nai, br, bi, nbi);
            }
        } else {
#pragma unroll
            for (int r = 0; r < NV; r++) {
                if ((r & cm_reg) != cm_reg) continue;
                float2 oR, oI;
                shfl4(R[r], I[r], oR, oI, xm);
                float2 yR = R[r], yI = I[r];
                lane_lin(yR, yI, oR, oI, ar, ai, nai, br, bi, nbi);
                R[r] = tok ? yR : R[r];
                I[r] = tok ? yI : I[r];
            }
        }
        return;
    }
    if (var == QSV_V_UNI_DIAG) {
        const float a_r = mine ? m0[6] : m0[0], a_i = mine ? m0[7] : m0[1];
#pragma unroll
        for (int r = 0; r < NV; r++) cmul2(R[r], I[r], a_r, a_i);
        return;
    }
    if (var == QSV_V_CTRL_DIAG1 || var == QSV_V_CTRL_DIAG1_SEL) {
        const bool s = mine && tok;
        const float d_r = m1[6], d_i = m1[7];
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if ((r & cm_reg) != cm_reg) continue;
            float2 yR = R[r], yI = I[r];
            cmul2(yR, yI, d_r, d_i);
            R[r] = s ? yR : R[r];
            I[r] = s ? yI : I[r];
        }
        return;
    }
    if (var == QSV_V_UNI_SWAP || var == QSV_V_CTRL_SWAP || var == QSV_V_CTRL_SWAP_SEL) {
        const bool uni = var == QSV_V_UNI_SWAP;
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if (!uni && (r & cm_reg) != cm_reg) continue;
            float2 oR, oI;
            shfl4(R[r], I[r], oR, oI, xm);
            R[r] = (uni || tok) ? oR : R[r];
            I[r] = (uni || tok) ? oI : I[r];
        }
        return;
    }
    if (var == QSV_V_SKIP) return;
    if (var == QSV_V_MUX && op.kind == QSV_K_CTRL && op.cm_c) {
        // M0 = identity, tile bit 0 among the controls: only the .y halves can be selected
        if (op.cls1 == QSV_M_XSWAP) {
#pragma unroll
            for (int r = 0; r < NV; r++) {
                if ((r & cm_reg) != cm_reg) continue;
                const float oR = __shfl_xor_sync(0xffffffffu, R[r].y, xm);
                const float oI = __shfl_xor_sync(0xffffffffu, I[r].y, xm);
                R[r].y = tok ? oR : R[r].y;
                I[r].y = tok ? oI : I[r].y;
            }
            return;
        }
        if (op.cls1 == QSV_M_DIAG1) {
            const bool s = mine && tok;
#pragma unroll
            for (int r = 0; r < NV; r++) {
                if ((r & cm_reg) != cm_reg) continue;
                float yr, yi;
                diag_own(yr, yi, m1[6], m1[7], R[r].y, I[r].y);
                R[r].y = s ? yr : R[r].y;
                I[r].y = s ? yi : I[r].y;
            }
            return;
        }
        if (op.cls1 == QSV_M_DENSE || op.cls1 == QSV_M_DIAG) {
            const float a_r = mine ? m1[6] : m1[0], a_i = mine ? m1[7] : m1[1];
            const float b_r = mine ? m1[4] : m1[2], b_i = mine ? m1[5] : m1[3];
#pragma unroll
            for (int r = 0; r < NV; r++) {
                if ((r & cm_reg) != cm_reg) continue;
                const float oR = __shfl_xor_sync(0xffffffffu, R[r].y, xm);
                const float oI = __shfl_xor_sync(0xffffffffu, I[r].y, xm);
                float yr, yi;
                lin_own(yr, yi, a_r, a_i, b_r, b_i, R[r].y, I[r].y, oR, oI);
                R[r].y = tok ? yr : R[r].y;
                I[r].y = tok ? yi : I[r].y;
            }
            return;
        }
    }
    lane_op<NV>(R, I, op, m0, m1, tok, lanebit, lane);
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
        lane_op_fast<NV>(R, I, op, m0, m1, thread_ok, slot - QSV_SLOT_LANE0, lane);
        return;
    }
    switch (slot) {
        case QSV_SLOT_COMP: comp_op_fast<NV>(R, I, op, m0, m1, thread_ok); break;
        case QSV_SLOT_REG0 + 0: reg_op<NV, 0>(R, I, op, m0, m1, thread_ok); break;
        case QSV_SLOT_REG0 + 1: if constexpr (RB > 1) reg_op<NV, (RB > 1 ? 1 : 0)>(R, I, op, m0, m1, thread_ok); break;
        case QSV_SLOT_REG0 + 2: if constexpr (RB > 2) reg_op<NV, (RB > 2 ? 2 : 0)>(R, I, op, m0, m1, thread_ok); break;
        case QSV_SLOT_REG0 + 3: if constexpr (RB > 3) reg_op<NV, (RB > 3 ? 3 : 0)>(R, I, op, m0, m1, thread_ok); break;
        default: break;
    }
}

// Shared-memory position of tile index x in a swizzled tile (the tensor map's 128-byte swizzle: the 16-byte
// chunk index, tile bits 1-3, is XORed with tile bits 4-6). Linear over XOR, so a thread's base and a
// register offset (disjoint bits) can be swizzled separately.
__device__ __forceinline__ uint32_t swz128(uint32_t x) { return x ^ ((x >> 3) & 0xEu); }

// One phase of a tile in shared memory: read the thread's 2^RB float4 in the phase's layout, apply ops
// [op_begin, op_end), write them back. PH is any phase record with reg_bits / lane_lo / lane_bits /
// warp_bits; swz: the tile is stored swizzled. split_in / split_out: the slots hold (re0, re1, im0, im1),
// the in-tile order between two phases (no repacking into the register pairs), instead of the state's
// interleaved order (first phase in, last phase out).
template <int NV, int RB, int WB, class PH>
__device__ __forceinline__ void run_phase(float2 *tile, const PH &Q, const QsvOp *ops, int op_begin, int op_end,
                                          int lane, int warp, bool swz = false, bool split_in = false,
                                          bool split_out = false) {
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
    float2 R[NV], I[NV];
    if (split_in) {
#pragma unroll
        for (int r = 0; r < NV; r++) {
            const float4 v = *reinterpret_cast<const float4 *>(tile + addr(r));
            R[r] = make_float2(v.x, v.y);
            I[r] = make_float2(v.z, v.w);
        }
    } else {
#pragma unroll
        for (int r = 0; r < NV; r++) {
            const float4 v = *reinterpret_cast<const float4 *>(tile + addr(r));
            R[r] = make_float2(v.x, v.z);
            I[r] = make_float2(v.y, v.w);
        }
    }
    for (int o = op_begin; o < op_end; o++) apply_op<NV, RB>(ops[o], R, I, tb, lane);
    if (split_out) {
#pragma unroll
        for (int r = 0; r < NV; r++)
            *reinterpret_cast<float4 *>(tile + addr(r)) = make_float4(R[r].x, R[r].y, I[r].x, I[r].y);
    } else {
#pragma unroll
        for (int r = 0; r < NV; r++)
            *reinterpret_cast<float4 *>(tile + addr(r)) = make_float4(R[r].x, I[r].x, R[r].y, I[r].y);
    }
}

}  // namespace dev
}  // namespace qsv
