// qsv_jit_ops.cuh -- MUX2 op application with the op's structure fixed at compile time.
//
// Used by sweep kernels specialised to one sweep structure (generated and compiled at run time by
// qsv_jit.cpp). Target slot, code variant, register-control mask and thread-control mask are template
// arguments, so per-op dispatch disappears, controls on register bits resolve at compile time (a
// controlled swap on register bits becomes a register renaming), and the phase layout's shared-memory
// offsets become immediates. The matrices stay data: they are read from the kernel's parameter block at
// fixed offsets. Every update uses the interpreter's arithmetic (qsv_ops.cuh / qsv_device.cuh); forms
// that skip work only skip exact-zero terms or unselected pairs, so values equal the interpreter's and the
// CPU oracle's (up to the sign of a zero).
#pragma once
#include "qsv_ops.cuh"

namespace qsv {
namespace dev {

// thread base of a phase: lane bits 0-2 on tile bits L0-L2, lane bits 3-4 on tile bits LB0 / LB1
template <int L0, int L1, int L2, int LB0, int LB1>
__device__ __forceinline__ uint32_t jit_lane_base(int lane) {
    return ((uint32_t)(lane & 1) << L0) | ((uint32_t)((lane >> 1) & 1) << L1) | ((uint32_t)((lane >> 2) & 1) << L2) |
           ((uint32_t)((lane >> 3) & 1) << LB0) | ((uint32_t)((lane >> 4) & 1) << LB1);
}
template <int WBIT>
__device__ __forceinline__ uint32_t jit_warp_bit(int warp, int w) {
    return (uint32_t)((warp >> w) & 1) << WBIT;
}

// offset of register slot r in a phase whose register bits are the tile bits RBITS...
template <int... RBITS>
__device__ __forceinline__ constexpr uint32_t jit_reg_off(int r) {
    constexpr int bits[] = {RBITS...};
    uint32_t o = 0;
    for (int q = 0; q < (int)sizeof...(RBITS); q++)
        if ((r >> q) & 1) o += 1u << bits[q];
    return o;
}

// SWZ: the tile is stored with the 128-byte swizzle (swz128); the thread base and the register offsets
// (disjoint bits) are swizzled separately and combined with XOR, the offsets at compile time.
// SPLIT: the 16-byte slot holds (re0, re1, im0, im1) -- the in-tile order between two phases of a tile,
// which loads and stores straight into the (re, re) / (im, im) register pairs -- instead of the state's
// interleaved (re0, im0, re1, im1), which the first phase reads and the last phase writes.
template <int NV, int SWZ, int SPLIT, int... RBITS>
__device__ __forceinline__ void jit_load(const float2 *tile, uint32_t tb, float2 (&R)[NV], float2 (&I)[NV]) {
    const uint32_t base = SWZ ? swz128(tb) : tb;
#pragma unroll
    for (int r = 0; r < NV; r++) {
        const uint32_t off = jit_reg_off<RBITS...>(r);
        const float4 v = *reinterpret_cast<const float4 *>(tile + (base ^ (SWZ ? swz128(off) : off)));
        R[r] = SPLIT ? make_float2(v.x, v.y) : make_float2(v.x, v.z);
        I[r] = SPLIT ? make_float2(v.z, v.w) : make_float2(v.y, v.w);
    }
}
template <int NV, int SWZ, int SPLIT, int... RBITS>
__device__ __forceinline__ void jit_store(float2 *tile, uint32_t tb, const float2 (&R)[NV], const float2 (&I)[NV]) {
    const uint32_t base = SWZ ? swz128(tb) : tb;
#pragma unroll
    for (int r = 0; r < NV; r++) {
        const uint32_t off = jit_reg_off<RBITS...>(r);
        *reinterpret_cast<float4 *>(tile + (base ^ (SWZ ? swz128(off) : off))) =
            SPLIT ? make_float4(R[r].x, R[r].y, I[r].x, I[r].y) : make_float4(R[r].x, I[r].x, R[r].y, I[r].y);
    }
}

// Dense op on register bit RBIT, coefficient-major: every (c, c) pair is built once and applied to all 2^RB / 2
// register pairs before the next one, so at most one pair is live at a time; each output keeps dense2's chain
// (qsv_ops.cuh) term for term, so values are identical. Holds four partial sums per register pair (needs the
// register budget of one consumer group). R0: m00 is real (its two imaginary terms, exact zeros, skipped).
template <int NV, int RBIT, bool R0>
__device__ __forceinline__ void jit_dense_cm(float2 (&R)[NV], float2 (&I)[NV], const float *m) {
    constexpr int B = 1 << RBIT;
    constexpr int NP = NV / 2;
    float2 t0r[NP], t0i[NP], t1r[NP], t1i[NP];
    auto lo = [](int p) { return (p & (B - 1)) | ((p & ~(B - 1)) << 1); };   // p-th register with bit RBIT clear
    {
        const float2 c = f2(-m[3]);
#pragma unroll
        for (int p = 0; p < NP; p++) t0r[p] = __fmul2_rn(c, I[lo(p) | B]);
    }
    {
        const float2 c = f2(m[3]);
#pragma unroll
        for (int p = 0; p < NP; p++) t0i[p] = __fmul2_rn(c, R[lo(p) | B]);
    }
    {
        const float2 c = f2(-m[5]);
#pragma unroll
        for (int p = 0; p < NP; p++) t1r[p] = __fmul2_rn(c, I[lo(p)]);
    }
    {
        const float2 c = f2(m[5]);
#pragma unroll
        for (int p = 0; p < NP; p++) t1i[p] = __fmul2_rn(c, R[lo(p)]);
    }
    {
        const float2 c = f2(m[2]);
#pragma unroll
        for (int p = 0; p < NP; p++) {
            t0r[p] = __ffma2_rn(c, R[lo(p) | B], t0r[p]);
            t0i[p] = __ffma2_rn(c, I[lo(p) | B], t0i[p]);
        }
    }
    {
        const float2 c = f2(m[4]);
#pragma unroll
        for (int p = 0; p < NP; p++) {
            t1r[p] = __ffma2_rn(c, R[lo(p)], t1r[p]);
            t1i[p] = __ffma2_rn(c, I[lo(p)], t1i[p]);
        }
    }
    if constexpr (!R0) {
        {
            const float2 c = f2(-m[1]);
#pragma unroll
            for (int p = 0; p < NP; p++) t0r[p] = __ffma2_rn(c, I[lo(p)], t0r[p]);
        }
        {
            const float2 c = f2(m[1]);
#pragma unroll
            for (int p = 0; p < NP; p++) t0i[p] = __ffma2_rn(c, R[lo(p)], t0i[p]);
        }
    }
    {
        const float2 c = f2(-m[7]);
#pragma unroll
        for (int p = 0; p < NP; p++) t1r[p] = __ffma2_rn(c, I[lo(p) | B], t1r[p]);
    }
    {
        const float2 c = f2(m[7]);
#pragma unroll
        for (int p = 0; p < NP; p++) t1i[p] = __ffma2_rn(c, R[lo(p) | B], t1i[p]);
    }
    {
        const float2 c = f2(m[0]);
#pragma unroll
        for (int p = 0; p < NP; p++) {
            R[lo(p)] = __ffma2_rn(c, R[lo(p)], t0r[p]);
            I[lo(p)] = __ffma2_rn(c, I[lo(p)], t0i[p]);
        }
    }
    {
        const float2 c = f2(m[6]);
#pragma unroll
        for (int p = 0; p < NP; p++) {
            R[lo(p) | B] = __ffma2_rn(c, R[lo(p) | B], t1r[p]);
            I[lo(p) | B] = __ffma2_rn(c, I[lo(p) | B], t1i[p]);
        }
    }
}

template <int NV, int RBIT, int VAR>
__device__ __forceinline__ void jit_reg_cm(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op) {
    float m[8];
#pragma unroll
    for (int e = 0; e < 8; e++) m[e] = op.m0[e];
    jit_dense_cm<NV, RBIT, VAR == QSV_V_UNI_DENSE_R0>(R, I, m);
}

__device__ __forceinline__ void jit_mat(float (&m)[8], const float *src) {
#pragma unroll
    for (int e = 0; e < 8; e++) m[e] = src[e];
}

// ---------------------------------------------------------------- register-bit target
template <int NV, int RBIT, int VAR, int CMREG, uint32_t CMTHR>
__device__ __forceinline__ void jit_reg(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op, uint32_t tb) {
    constexpr int B = 1 << RBIT;
    const bool tok = (CMTHR == 0u) || ((tb & CMTHR) == CMTHR);
    if constexpr (VAR == QSV_V_SKIP) {
        return;
    } else if constexpr (VAR == QSV_V_UNI_DENSE) {
        float m[8];
        jit_mat(m, op.m0);
#pragma unroll
        for (int r = 0; r < NV; r++)
            if (!(r & B)) dense2(R[r], I[r], R[r | B], I[r | B], m);
    } else if constexpr (VAR == QSV_V_UNI_DENSE_R0) {
        float m[8];
        jit_mat(m, op.m0);
#pragma unroll
        for (int r = 0; r < NV; r++)
            if (!(r & B)) dense2_r0(R[r], I[r], R[r | B], I[r | B], m);
    } else if constexpr (VAR == QSV_V_UNI_DIAG) {
        const float a0 = op.m0[0], a1 = op.m0[1], d0 = op.m0[6], d1 = op.m0[7];
#pragma unroll
        for (int r = 0; r < NV; r++)
            if (!(r & B)) { cmul2(R[r], I[r], a0, a1); cmul2(R[r | B], I[r | B], d0, d1); }
    } else if constexpr (VAR == QSV_V_UNI_SWAP) {
#pragma unroll
        for (int r = 0; r < NV; r++)
            if (!(r & B)) { swap2(R[r], R[r | B]); swap2(I[r], I[r | B]); }
    } else if constexpr (VAR == QSV_V_CTRL_DENSE) {
        float m[8];
        jit_mat(m, op.m1);
        if (tok) {
#pragma unroll
            for (int r = 0; r < NV; r++)
                if (!(r & B) && (r & CMREG) == CMREG) dense2(R[r], I[r], R[r | B], I[r | B], m);
        }
    } else if constexpr (VAR == QSV_V_CTRL_DIAG1) {
        const float d0 = op.m1[6], d1 = op.m1[7];
        if (tok) {
#pragma unroll
            for (int r = 0; r < NV; r++)
                if (!(r & B) && (r & CMREG) == CMREG) cmul2(R[r | B], I[r | B], d0, d1);
        }
    } else if constexpr (VAR == QSV_V_CTRL_SWAP) {
        if (CMTHR == 0u) {
#pragma unroll
            for (int r = 0; r < NV; r++)
                if (!(r & B) && (r & CMREG) == CMREG) { swap2(R[r], R[r | B]); swap2(I[r], I[r | B]); }
        } else if (tok) {
#pragma unroll
            for (int r = 0; r < NV; r++)
                if (!(r & B) && (r & CMREG) == CMREG) { swap2(R[r], R[r | B]); swap2(I[r], I[r | B]); }
        }
    } else if constexpr (VAR == QSV_V_CTRL_DENSE_SEL) {
        const float id[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 1.f, 0.f};
        float m[8];
        jit_mat(m, op.m1);
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if ((r & B) || (r & CMREG) != CMREG) continue;
            float c[8];
#pragma unroll
            for (int e = 0; e < 8; e++) c[e] = tok ? m[e] : id[e];
            dense2(R[r], I[r], R[r | B], I[r | B], c);
        }
    } else if constexpr (VAR == QSV_V_CTRL_DIAG1_SEL) {
        const float d0 = tok ? op.m1[6] : 1.f, d1 = tok ? op.m1[7] : 0.f;
#pragma unroll
        for (int r = 0; r < NV; r++)
            if (!(r & B) && (r & CMREG) == CMREG) cmul2(R[r | B], I[r | B], d0, d1);
    } else if constexpr (VAR == QSV_V_CTRL_SWAP_SEL) {
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if ((r & B) || (r & CMREG) != CMREG) continue;
            const float2 a = R[r], b = R[r | B], c = I[r], d = I[r | B];
            R[r] = tok ? b : a; R[r | B] = tok ? a : b;
            I[r] = tok ? d : c; I[r | B] = tok ? c : d;
        }
    } else {
        float m0[8], m1[8];
        jit_mat(m0, op.m0);
        jit_mat(m1, op.m1);
        reg_op<NV, RBIT>(R, I, op, m0, m1, tok);
    }
}

// ---------------------------------------------------------------- lane-bit target (LB = lane bit 0..4)
// lane updates use lane_lin / shfl4 (qsv_ops.cuh): y = a*own + b*oth, (a, b) = (m00, m01) on the bit-0
// side and (m11, m10) on the bit-1 side -- the interpreter's lane update.
template <int NV, int LB, int VAR, int CMREG, uint32_t CMTHR>
__device__ __forceinline__ void jit_lane(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op, uint32_t tb, int lane) {
    constexpr int XM = 1 << LB;
    const bool mine = (lane >> LB) & 1;
    const bool tok = (CMTHR == 0u) || ((tb & CMTHR) == CMTHR);
    if constexpr (VAR == QSV_V_SKIP) {
        return;
    } else if constexpr (VAR == QSV_V_UNI_DENSE || VAR == QSV_V_CTRL_DENSE || VAR == QSV_V_CTRL_DENSE_SEL) {
        constexpr bool UNI = VAR == QSV_V_UNI_DENSE;
        const float *m = UNI ? op.m0 : op.m1;
        const float a_r = mine ? m[6] : m[0], a_i = mine ? m[7] : m[1];
        const float b_r = mine ? m[4] : m[2], b_i = mine ? m[5] : m[3];
        const float2 ar = f2(a_r), ai = f2(a_i), nai = f2(-a_i), br = f2(b_r), bi = f2(b_i), nbi = f2(-b_i);
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if (!UNI && (r & CMREG) != CMREG) continue;
            float2 oR, oI;
            shfl4(R[r], I[r], oR, oI, XM);
            float2 yR = R[r], yI = I[r];
            lane_lin(yR, yI, oR, oI, ar, ai, nai, br, bi, nbi);
            if (UNI || CMTHR == 0u) {
                R[r] = yR; I[r] = yI;
            } else {
                R[r] = tok ? yR : R[r];
                I[r] = tok ? yI : I[r];
            }
        }
    } else if constexpr (VAR == QSV_V_UNI_DIAG) {
        // diagonal: each amplitude is scaled by its own diagonal entry, no exchange
        const float a_r = mine ? op.m0[6] : op.m0[0], a_i = mine ? op.m0[7] : op.m0[1];
#pragma unroll
        for (int r = 0; r < NV; r++) cmul2(R[r], I[r], a_r, a_i);
    } else if constexpr (VAR == QSV_V_CTRL_DIAG1 || VAR == QSV_V_CTRL_DIAG1_SEL) {
        // diag(1, d) where selected: only the bit-1 side changes
        const bool s = mine && tok;
        const float d_r = op.m1[6], d_i = op.m1[7];
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if ((r & CMREG) != CMREG) continue;
            float2 yR = R[r], yI = I[r];
            cmul2(yR, yI, d_r, d_i);
            R[r] = s ? yR : R[r];
            I[r] = s ? yI : I[r];
        }
    } else if constexpr (VAR == QSV_V_UNI_SWAP || VAR == QSV_V_CTRL_SWAP || VAR == QSV_V_CTRL_SWAP_SEL) {
        constexpr bool UNI = VAR == QSV_V_UNI_SWAP;
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if (!UNI && (r & CMREG) != CMREG) continue;
            float2 oR, oI;
            shfl4(R[r], I[r], oR, oI, XM);
            if (UNI || CMTHR == 0u) {
                R[r] = oR; I[r] = oI;
            } else {
                R[r] = tok ? oR : R[r];
                I[r] = tok ? oI : I[r];
            }
        }
    } else {
        float m0[8], m1[8];
        jit_mat(m0, op.m0);
        jit_mat(m1, op.m1);
        lane_op<NV>(R, I, op, m0, m1, tok, LB, lane);
    }
}

// ---------------------------------------------------------------- tile-bit-0 target (halves of a float4)
// the interpreter's comp_op with kind, classes and register controls fixed at compile time (pair_t:
// pair_apply with the class fixed, qsv_ops.cuh)
template <int NV, int KIND, int CLS0, int CLS1, int CMREG, uint32_t CMTHR>
__device__ __forceinline__ void jit_comp(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op, uint32_t tb) {
    const bool tok = (CMTHR == 0u) || ((tb & CMTHR) == CMTHR);
    float m0[8], m1[8];
    jit_mat(m0, op.m0);
    jit_mat(m1, op.m1);
#pragma unroll
    for (int r = 0; r < NV; r++) {
        constexpr bool UNI = KIND == QSV_K_UNI, CTRL = KIND == QSV_K_CTRL;
        const bool regsel = !UNI && (r & CMREG) == CMREG;
        if (CTRL && !regsel) continue;
        float x0r = R[r].x, x0i = I[r].x, x1r = R[r].y, x1i = I[r].y;
        if (UNI) {
            pair_t<CLS0>(x0r, x0i, x1r, x1i, m0);
        } else if (CMTHR == 0u) {
            if (regsel) pair_t<CLS1>(x0r, x0i, x1r, x1i, m1);
            else pair_t<CLS0>(x0r, x0i, x1r, x1i, m0);
        } else {
            if (regsel && tok) pair_t<CLS1>(x0r, x0i, x1r, x1i, m1);
            else if (!CTRL) pair_t<CLS0>(x0r, x0i, x1r, x1i, m0);
        }
        R[r] = make_float2(x0r, x1r);
        I[r] = make_float2(x0i, x1i);
    }
}

// ---------------------------------------------------------------- controlled ops with a control on tile bit 0
// M0 = identity and tile bit 0 among the controls: only the bit-0 = 1 half of each float4 (the .y lanes of
// the packed pairs) can be selected. XSWAP / DIAG1 / DENSE M1 in scalar arithmetic on that half; other
// matrices take the interpreter's general path.
template <int NV, int RBIT, int CLS1, int CMREG, uint32_t CMTHR>
__device__ __forceinline__ bool jit_reg_ctrl_c(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op, uint32_t tb) {
    constexpr int B = 1 << RBIT;
    const bool tok = (CMTHR == 0u) || ((tb & CMTHR) == CMTHR);
    if constexpr (CLS1 == QSV_M_XSWAP) {
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if ((r & B) || (r & CMREG) != CMREG) continue;
            const float a = R[r].y, b = R[r | B].y, c = I[r].y, d = I[r | B].y;
            R[r].y = tok ? b : a; R[r | B].y = tok ? a : b;
            I[r].y = tok ? d : c; I[r | B].y = tok ? c : d;
        }
        return true;
    } else if constexpr (CLS1 == QSV_M_DIAG1 || CLS1 == QSV_M_DENSE || CLS1 == QSV_M_DIAG) {
        float m[8];
        jit_mat(m, op.m1);
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if ((r & B) || (r & CMREG) != CMREG) continue;
            float x0r = R[r].y, x0i = I[r].y, x1r = R[r | B].y, x1i = I[r | B].y;
            pair_t<CLS1>(x0r, x0i, x1r, x1i, m);
            R[r].y = tok ? x0r : R[r].y; I[r].y = tok ? x0i : I[r].y;
            R[r | B].y = tok ? x1r : R[r | B].y; I[r | B].y = tok ? x1i : I[r | B].y;
        }
        return true;
    }
    return false;
}

template <int NV, int LB, int CLS1, int CMREG, uint32_t CMTHR>
__device__ __forceinline__ bool jit_lane_ctrl_c(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op, uint32_t tb,
                                                int lane) {
    constexpr int XM = 1 << LB;
    const bool mine = (lane >> LB) & 1;
    const bool tok = (CMTHR == 0u) || ((tb & CMTHR) == CMTHR);
    if constexpr (CLS1 == QSV_M_XSWAP) {
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if ((r & CMREG) != CMREG) continue;
            const float oR = __shfl_xor_sync(0xffffffffu, R[r].y, XM);
            const float oI = __shfl_xor_sync(0xffffffffu, I[r].y, XM);
            R[r].y = tok ? oR : R[r].y;
            I[r].y = tok ? oI : I[r].y;
        }
        return true;
    } else if constexpr (CLS1 == QSV_M_DIAG1) {
        const bool s = mine && tok;
        const float d_r = op.m1[6], d_i = op.m1[7];
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if ((r & CMREG) != CMREG) continue;
            float yr, yi;
            diag_own(yr, yi, d_r, d_i, R[r].y, I[r].y);
            R[r].y = s ? yr : R[r].y;
            I[r].y = s ? yi : I[r].y;
        }
        return true;
    } else if constexpr (CLS1 == QSV_M_DENSE || CLS1 == QSV_M_DIAG) {
        const float *m = op.m1;
        const float a_r = mine ? m[6] : m[0], a_i = mine ? m[7] : m[1];
        const float b_r = mine ? m[4] : m[2], b_i = mine ? m[5] : m[3];
#pragma unroll
        for (int r = 0; r < NV; r++) {
            if ((r & CMREG) != CMREG) continue;
            const float oR = __shfl_xor_sync(0xffffffffu, R[r].y, XM);
            const float oI = __shfl_xor_sync(0xffffffffu, I[r].y, XM);
            float yr, yi;
            lin_own(yr, yi, a_r, a_i, b_r, b_i, R[r].y, I[r].y, oR, oI);
            R[r].y = tok ? yr : R[r].y;
            I[r].y = tok ? yi : I[r].y;
        }
        return true;
    }
    return false;
}

template <int NV, int RBIT, int KIND, int CLS1, int CMC, int CMREG, uint32_t CMTHR>
__device__ __forceinline__ void jit_reg_mux(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op, uint32_t tb) {
    if constexpr (KIND == QSV_K_CTRL && CMC)
        if (jit_reg_ctrl_c<NV, RBIT, CLS1, CMREG, CMTHR>(R, I, op, tb)) return;
    jit_reg<NV, RBIT, QSV_V_MUX, CMREG, CMTHR>(R, I, op, tb);
}

template <int NV, int LB, int KIND, int CLS1, int CMC, int CMREG, uint32_t CMTHR>
__device__ __forceinline__ void jit_lane_mux(float2 (&R)[NV], float2 (&I)[NV], const QsvOp &op, uint32_t tb, int lane) {
    if constexpr (KIND == QSV_K_CTRL && CMC)
        if (jit_lane_ctrl_c<NV, LB, CLS1, CMREG, CMTHR>(R, I, op, tb, lane)) return;
    jit_lane<NV, LB, QSV_V_MUX, CMREG, CMTHR>(R, I, op, tb, lane);
}

}  // namespace dev
}  // namespace qsv
