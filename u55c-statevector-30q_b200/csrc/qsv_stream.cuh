// qsv_stream.cuh -- the streaming form of a sweep's tile work (sm_100a), shared by the streaming interpreter
// (qsv_sweep.cu) and kernels generated at run time (qsv_jit.cpp).
//
// The tile stays in shared memory and each group of ops (plan_stream in qsv_planner.cpp) is one round trip
// of it: a thread takes items of 8 float4 = 16 amplitudes on tile bits {0, q[0], q[1], q[2]} (float4 r holds
// item base | r.0 * 2^q[0] | r.1 * 2^q[1] | r.2 * 2^q[2]), applies the group's ops to them in registers and
// stores them back. Any target bit can be an item bit, so a sweep needs no phase layouts, and ops on tile
// bit 0 and diagonal ops on any bit ride along with the group. The ops run through the phase interpreter's
// code paths (reg_op with the item bits as register bits 0-2, comp_op_fast), so every value is the same.
//
// Two ways to run a group's ops on an item: stream_op reads each op's slot and variant at run time (one
// dispatch per op and item); stream_op_fixed takes them as template arguments (straight-line code for a
// group's op sequence, with item bits, control masks and matrices still read at run time).
#pragma once
#include "qsv_device.cuh"
#include "qsv_ops.cuh"

namespace qsv {
namespace dev {

// The fields of an op record a kernel reads, from one 16-byte shared-memory load (QsvOp keeps them in the
// 16 bytes at offset 64).
struct OpHdr {
    uint32_t cm_thr, cm_reg, cm_c, kind, cls0, cls1, slot, tbit, variant, r00;
};
__device__ __forceinline__ uint4 op_hdr_words(const QsvOp *op) {
    return *reinterpret_cast<const uint4 *>(reinterpret_cast<const unsigned char *>(op) + 64);
}
__device__ __forceinline__ OpHdr op_hdr(const QsvOp *op) {
    const uint4 h = op_hdr_words(op);
    OpHdr o;
    o.cm_thr = h.x;
    o.cm_reg = h.y & 0xffu; o.cm_c = (h.y >> 8) & 0xffu; o.kind = (h.y >> 16) & 0xffu;
    o.cls0 = h.z & 0xffu; o.cls1 = (h.z >> 8) & 0xffu; o.slot = (h.z >> 16) & 0xffu; o.tbit = h.z >> 24;
    o.variant = h.w & 0xffu; o.r00 = (h.w >> 8) & 0xffu;
    return o;
}
// M0 and M1 of an op record: four 16-byte loads
__device__ __forceinline__ void op_mats(const QsvOp *op, float (&m0)[8], float (&m1)[8], bool need0, bool need1) {
    const float4 *mv = reinterpret_cast<const float4 *>(op);
#pragma unroll
    for (int v = 0; v < 2; v++) {
        if (need0) {
            const float4 a = mv[v];
            m0[4 * v] = a.x; m0[4 * v + 1] = a.y; m0[4 * v + 2] = a.z; m0[4 * v + 3] = a.w;
        }
        if (need1) {
            const float4 c = mv[2 + v];
            m1[4 * v] = c.x; m1[4 * v + 1] = c.y; m1[4 * v + 2] = c.z; m1[4 * v + 3] = c.w;
        }
    }
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

// one op on one item, its code path chosen from the record's slot and variant
template <bool IP>
__device__ __forceinline__ void stream_apply(const OpHdr &h, const float *m0, const float *m1, float2 (&R)[8],
                                             float2 (&I)[8], uint32_t base) {
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

// run-time dispatch: slot and variant read from the record
template <bool IP>
__device__ __forceinline__ void stream_op(const QsvOp *op, float2 (&R)[8], float2 (&I)[8], uint32_t base) {
    const OpHdr h = op_hdr(op);
    if (h.variant == QSV_V_SKIP) return;
    float m0[8], m1[8];
    op_mats(op, m0, m1, true, true);
    stream_apply<IP>(h, m0, m1, R, I, base);
}

// compile-time dispatch: slot, variant, kind, matrix classes and r00 fixed by the caller (they must equal the
// record's); control masks, target bit and matrices read from the record
template <bool IP, int SLOT, int VAR, int KIND, int CLS0, int CLS1, int R00>
__device__ __forceinline__ void stream_op_fixed(const QsvOp *op, float2 (&R)[8], float2 (&I)[8], uint32_t base) {
    if constexpr (VAR != QSV_V_SKIP) {
        const uint4 w = op_hdr_words(op);
        OpHdr h;
        h.cm_thr = w.x;
        h.cm_reg = w.y & 0xffu; h.cm_c = (w.y >> 8) & 0xffu; h.kind = KIND;
        h.cls0 = CLS0; h.cls1 = CLS1; h.slot = SLOT; h.tbit = w.z >> 24;
        h.variant = VAR; h.r00 = R00;
        constexpr bool need0 = KIND != QSV_K_CTRL || VAR == QSV_V_MUX;
        constexpr bool need1 = KIND != QSV_K_UNI;
        float m0[8], m1[8];
#pragma unroll
        for (int e = 0; e < 8; e++) { m0[e] = 0.f; m1[e] = 0.f; }
        op_mats(op, m0, m1, need0, need1);
        const bool tok = (base & h.cm_thr) == h.cm_thr;
        if constexpr (SLOT == QSV_SLOT_COMP) comp_fixed<8, KIND, CLS0, CLS1>(R, I, h, m0, m1, tok);
        else if constexpr (SLOT >= QSV_SLOT_REG0 && SLOT <= QSV_SLOT_REG0 + 2)
            reg_case<8, SLOT - QSV_SLOT_REG0, IP, VAR>(R, I, h, m0, m1, tok);
        else if constexpr (SLOT == QSV_SLOT_BASE) base_diag<8, IP>(R, I, h, m0, m1, tok, (base >> h.tbit) & 1u);
    }
}

// insert a zero bit at position q (bits q and above move up by one)
__device__ __forceinline__ uint32_t insert0(uint32_t x, uint32_t q) {
    return ((x >> q) << (q + 1)) | (x & ((1u << q) - 1u));
}

// One group over the whole tile: every item of this thread is loaded, handed to body(R, I, base) and stored.
// SIN / SOUT: the tile holds the in-tile order (re0, re1, im0, im1) per float4 on entry / exit, instead of the
// state's interleaved order (first group in, last group out). swz: the tile is stored swizzled (swz128).
template <int KW, int NCG, bool SIN, bool SOUT, class F>
__device__ __forceinline__ void stream_items(float2 *tile, const QsvGroup &g, int ctid, bool swz, F &&body) {
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
        body(R, I, x);
#pragma unroll
        for (int r = 0; r < 8; r++)
            *reinterpret_cast<float4 *>(tile + (sx ^ soff[r])) =
                SOUT ? make_float4(R[r].x, R[r].y, I[r].x, I[r].y) : make_float4(R[r].x, I[r].x, R[r].y, I[r].y);
    }
}

// stream_items with the entry / exit order chosen at run time (selects on the loaded and stored values; one
// copy of the loop serves every group position)
template <int KW, int NCG, class F>
__device__ __forceinline__ void stream_items_rt(float2 *tile, const QsvGroup &g, int ctid, bool swz, bool sin,
                                                bool sout, F &&body) {
    const uint32_t q[3] = {g.q[0], g.q[1], g.q[2]};
    uint32_t soff[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const uint32_t o = ((r & 1) ? 1u << q[0] : 0u) | ((r & 2) ? 1u << q[1] : 0u) | ((r & 4) ? 1u << q[2] : 0u);
        soff[r] = swz ? swz128(o) : o;
    }
    uint32_t s0 = q[0], s1 = q[1], s2 = q[2], t;
    if (s0 > s1) { t = s0; s0 = s1; s1 = t; }
    if (s1 > s2) { t = s1; s1 = s2; s2 = t; }
    if (s0 > s1) { t = s0; s0 = s1; s1 = t; }
#pragma unroll 1
    for (int it = ctid; it < (1 << (KW - 4)); it += NCG) {
        const uint32_t x = insert0(insert0(insert0((uint32_t)it << 1, s0), s1), s2);
        const uint32_t sx = swz ? swz128(x) : x;
        float2 R[8], I[8];
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const float4 v = *reinterpret_cast<const float4 *>(tile + (sx ^ soff[r]));
            R[r] = make_float2(v.x, sin ? v.y : v.z);
            I[r] = make_float2(sin ? v.z : v.y, v.w);
        }
        body(R, I, x);
#pragma unroll
        for (int r = 0; r < 8; r++)
            *reinterpret_cast<float4 *>(tile + (sx ^ soff[r])) =
                make_float4(R[r].x, sout ? R[r].y : I[r].x, sout ? I[r].x : R[r].y, I[r].y);
    }
}

}  // namespace dev
}  // namespace qsv
