// qsv_planner.cpp -- host decode of QSV2 segments and construction of the sweep plan.
//
// decode_segment follows the stream layout of host/sv/isa.py:1-32 and the reader in host/sv/model.py:7-22
// (validation mirrors what the reference engine assumes: magic, L, k <= L, m <= MAX_HIGH, <= 64 ops per
// pass, opcode MUX2, record bounds). Each op is converted from pass-tile coordinates to physical qubits
// (tile qubit q < k-m is physical q, tile qubit k-m+i is h_i; host/sv/isa.py:14-15).
#include "qsv_planner.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>

namespace qsv {

static inline float f_of(int32_t w) {
    float f;
    std::memcpy(&f, &w, 4);
    return f;
}

static inline double d_of(const int32_t *w) {
    double d;
    std::memcpy(&d, w, 8);
    return d;
}

int decode_segment(const int32_t *seg, size_t nwords, int n, std::vector<PhysPass> &out, std::string &err,
                   int dtype) {
    out.clear();
    if (!seg || nwords < QSV2_HDR_WORDS) { err = "segment shorter than its header"; return QSV_ERR_BAD_STREAM; }
    if ((uint32_t)seg[0] != QSV2_MAGIC) { err = "bad QSV2 magic"; return QSV_ERR_BAD_STREAM; }
    if (seg[4] != dtype) {
        err = seg[4] == 1 ? "segment carries FP64 matrices (complex128) but the state is complex64"
              : seg[4] == 0 ? "segment carries FP32 matrices (complex64) but the state is complex128"
                            : "unknown element type in header word 4";
        return QSV_ERR_BAD_STREAM;
    }
    const size_t opw = dtype ? QSV2_OP_WORDS_C128 : QSV2_OP_WORDS;
    const int L = seg[1], npass = seg[2], k = seg[3];
    if (L != n) { err = "segment L (" + std::to_string(L) + ") != state qubits (" + std::to_string(n) + ")"; return QSV_ERR_BAD_STREAM; }
    if (k < 1 || k > L || npass < 0) { err = "bad segment header (k, n_passes)"; return QSV_ERR_BAD_STREAM; }
    size_t pos = QSV2_HDR_WORDS;
    for (int p = 0; p < npass; p++) {
        if (pos + QSV2_PASS_WORDS > nwords) { err = "truncated pass header"; return QSV_ERR_BAD_STREAM; }
        const int m = seg[pos], nops = seg[pos + 3];
        const int h[4] = {seg[pos + 1], seg[pos + 2], seg[pos + 4], seg[pos + 5]};
        if (m < 0 || m > 4 || m > k || nops < 0 || nops > QSV2_MAX_OPS) { err = "bad pass header"; return QSV_ERR_BAD_STREAM; }
        for (int i = 0; i < m; i++) {
            if (h[i] < k - m || h[i] >= L) { err = "high qubit outside [k-m, L)"; return QSV_ERR_BAD_STREAM; }
            for (int j = 0; j < i; j++)
                if (h[j] == h[i]) { err = "repeated high qubit"; return QSV_ERR_BAD_STREAM; }
        }
        pos += QSV2_PASS_WORDS;
        PhysPass pp;
        for (int o = 0; o < nops; o++) {
            if (pos + opw > nwords) { err = "truncated op record"; return QSV_ERR_BAD_STREAM; }
            const int32_t *rec = seg + pos;
            if (rec[0] != QSV2_OP_MUX2) { err = "unknown opcode " + std::to_string(rec[0]); return QSV_ERR_BAD_STREAM; }
            const int t = rec[1];
            const uint32_t cm = (uint32_t)rec[2];
            if (t < 0 || t >= k || (k < 32 && (cm >> k))) { err = "op target/cmask outside the tile"; return QSV_ERR_BAD_STREAM; }
            auto phys = [&](int tq) { return tq < k - m ? tq : h[tq - (k - m)]; };
            PhysOp op;
            op.t = phys(t);
            op.cmask = 0;
            for (int b = 0; b < k; b++)
                if ((cm >> b) & 1) op.cmask |= 1ull << phys(b);
            // a control on the target bit can never be set in i0, so M1 is never selected: keep that
            // meaning by recording it (the engine tests i0, which has the target bit clear)
            if (dtype) {
                for (int e = 0; e < 8; e++) {
                    op.d0[e] = d_of(rec + 8 + 2 * e);
                    op.d1[e] = d_of(rec + 24 + 2 * e);
                    op.m0[e] = (float)op.d0[e];
                    op.m1[e] = (float)op.d1[e];
                }
            } else {
                for (int e = 0; e < 8; e++) {
                    op.m0[e] = f_of(rec[8 + e]);
                    op.m1[e] = f_of(rec[16 + e]);
                    op.d0[e] = op.m0[e];
                    op.d1[e] = op.m1[e];
                }
            }
            pp.ops.push_back(op);
            pos += opw;
        }
        out.push_back(std::move(pp));
    }
    if (pos != nwords) { err = "trailing words after the last pass"; return QSV_ERR_BAD_STREAM; }
    return QSV_OK;
}

static int g_rb13 = 4;      // register bits of the 13-qubit layout: 4 (256 consumer threads) or 3 (512)
// targets (tile bits >= 4) a phase may place on lane bits 3, 4 (0..2). 1 measured fastest on the 30-qubit
// random-layer program (interpreter and specialised kernels); 0 on the 30-qubit QFT
static int g_phase_lanes = 1;

int set_phase_lanes(int k) {
    if (k < 0 || k > 2) return -1;
    g_phase_lanes = k;
    return 0;
}

// swizzled layouts for complex64 tensor-map sweeps (QsvSweepT::swz): on unless QSV_SWIZZLE=0
static bool swizzle_enabled() {
    static const bool on = [] {
        const char *e = std::getenv("QSV_SWIZZLE");
        return !(e && std::atoi(e) == 0);
    }();
    return on;
}

int set_rb13(int rb) {
    if (rb != 3 && rb != 4) return -1;
    g_rb13 = rb;
    return 0;
}

int layout_for_kw(int kw, int *rb, int *wb) {
    switch (kw) {
        case 13: *rb = g_rb13; *wb = 13 - 6 - g_rb13; return 0;
        case 12: *rb = 4; *wb = 2; return 0;
        case 11: *rb = 3; *wb = 2; return 0;
        case 10: *rb = 2; *wb = 2; return 0;
        default: return -1;
    }
}

int layout_for_kw_c128(int kw, int *rb, int *wb) {
    if (kw < 10 || kw > 12) return -1;
    *rb = 4;
    *wb = kw - 9;
    return 0;
}

static uint64_t op_qubits(const PhysOp &op) { return op.cmask | (1ull << op.t); }

static int window_lo(uint64_t qset, int n, int kw) {
    // largest lo with lo + |{q in qset : q >= lo}| <= kw
    int best = -1;
    for (int lo = 0; lo <= std::min(n, kw); lo++) {
        int cnt = __builtin_popcountll(lo >= 64 ? 0 : (qset >> lo));
        if (lo + cnt <= kw) best = lo;
    }
    return best;
}

template <class T>
static uint8_t classify(const T *m) {
    auto z = [](T x) { return x == (T)0; };
    const bool offz = z(m[2]) && z(m[3]) && z(m[4]) && z(m[5]);
    if (offz && m[0] == (T)1 && z(m[1]) && m[6] == (T)1 && z(m[7])) return QSV_M_IDENT;
    if (offz && m[0] == (T)1 && z(m[1])) return QSV_M_DIAG1;
    if (offz) return QSV_M_DIAG;
    if (z(m[0]) && z(m[1]) && m[2] == (T)1 && z(m[3]) && m[4] == (T)1 && z(m[5]) && z(m[6]) && z(m[7]))
        return QSV_M_XSWAP;
    return QSV_M_DENSE;
}

static void set_mats(QsvOp &o, const PhysOp &p) {
    std::memcpy(o.m0, p.m0, sizeof(o.m0));
    std::memcpy(o.m1, p.m1, sizeof(o.m1));
}
static void set_mats(QsvOpD &o, const PhysOp &p) {
    std::memcpy(o.m0, p.d0, sizeof(o.m0));
    std::memcpy(o.m1, p.d1, sizeof(o.m1));
}

// Tensor-map staging for windows with short contiguous runs: one dim per chunk (<= 8 bits) of each run of
// window bits, each spanning the free bits up to the next window bit. Returns the rank, 0 if it does not fit.
// swz: the map of a swizzled sweep, whose first dim is exactly tile bits 0-3 (128-byte rows, the span of
// the 128-byte swizzle); needs lo >= 4, any lo.
template <class SW>
static int tma_dims(const SW &sw, uint8_t *tfree, uint8_t *tbox, uint8_t *tstart, bool swz = false) {
    if (swz ? sw.lo < 4 : sw.lo >= QSV_TMA_TENSOR_LO) return 0;
    int wb[QSV_KW_MAX], nw = 0;            // window bits ascending
    for (int q = 0; q < sw.lo; q++) wb[nw++] = q;
    for (int i = 0; i < sw.nh; i++) wb[nw++] = sw.H[i];
    int rank = 0, i = 0;
    while (i < nw) {
        const int maxlen = (swz && rank == 0) ? 4 : 8;
        int start = wb[i], len = 1;
        while (i + len < nw && wb[i + len] == start + len && len < maxlen) len++;
        const int next = (i + len < nw) ? wb[i + len] : sw.n;
        const int fr = next - (start + len);
        if (rank == QSV_TMA_MAX_RANK || len + fr > 31) return 0;
        tstart[rank] = (uint8_t)start;
        tbox[rank] = (uint8_t)len;
        tfree[rank] = (uint8_t)fr;
        rank++;
        i += len;
    }
    return rank;
}

// Ops [b, e) in tile coordinates of a window (tile_of[q] = tile bit of physical qubit q) with their matrix
// classes, kinds and code variants (independent of the thread layout).
template <class OpT>
static void classify_ops(const std::vector<PhysOp> &ops, size_t b, size_t e, const int *tile_of, int n,
                         std::vector<OpT> &out) {
    constexpr bool C128 = std::is_same<OpT, QsvOpD>::value;
    out.assign(e - b, OpT());
    for (size_t i = b; i < e; i++) {
        OpT &o = out[i - b];
        std::memset(&o, 0, sizeof(o));
        const PhysOp &p = ops[i];
        set_mats(o, p);
        o.tbit = (uint8_t)tile_of[p.t];
        o.cmask = 0;
        for (int q = 0; q < n; q++)
            if ((p.cmask >> q) & 1) o.cmask |= 1u << tile_of[q];
        o.cls0 = classify(o.m0);
        o.cls1 = classify(o.m1);
        // identical matrices, or a control on the target bit (i0 never has it set): M1 is never
        // selected / cannot change any value, so the op runs unconditioned with M0
        if (std::memcmp(o.m0, o.m1, sizeof(o.m0)) == 0 || ((o.cmask >> o.tbit) & 1)) {
            o.cmask = 0;
            std::memcpy(o.m1, o.m0, sizeof(o.m0));
            o.cls1 = o.cls0;
        }
        o.r00 = (uint8_t)(o.cls0 == QSV_M_DENSE && o.m0[1] == 0);
        if (o.cmask == 0) { o.kind = QSV_K_UNI; o.cls = o.cls0; }
        else if (o.cls0 == QSV_M_IDENT) { o.kind = QSV_K_CTRL; o.cls = o.cls1; }
        else { o.kind = QSV_K_MUX; o.cls = QSV_M_DENSE; }
        o.cm_c = C128 ? 0 : (uint8_t)(o.cmask & 1u);
        // code path; the dense arithmetic gives the same values on diagonal / permutation matrices
        if (o.kind == QSV_K_UNI) {
            o.variant = o.cls == QSV_M_IDENT ? QSV_V_SKIP
                        : o.cls == QSV_M_XSWAP ? QSV_V_UNI_SWAP
                        : (o.cls == QSV_M_DIAG || o.cls == QSV_M_DIAG1) ? QSV_V_UNI_DIAG : QSV_V_UNI_DENSE;
        } else if (o.kind == QSV_K_CTRL && !o.cm_c) {
            o.variant = o.cls == QSV_M_IDENT ? QSV_V_SKIP
                        : o.cls == QSV_M_XSWAP ? QSV_V_CTRL_SWAP
                        : o.cls == QSV_M_DIAG1 ? QSV_V_CTRL_DIAG1 : QSV_V_CTRL_DENSE;
        } else {
            o.variant = QSV_V_MUX;
        }
    }
}

// The phases of classified ops, greedy in op order, and each op's slot and layout-dependent fields. Plain
// layout: tile bits above the fixed lane bits (>= 4 for complex64, whose tile bit 0 is the packed half of a
// float4 and bits 1-3 are lanes; >= 3 for complex128, bits 0-2 lanes) that are targets need a register or
// lane slot. swz (complex64 only): the swizzled layout, in which lane bit l (0-2) sits on tile bit 1+l or
// 4+l, chosen per phase, so tile bits 1-3 need slots like the others and can be register bits; lane_cap
// bounds its lane-bit targets (warp-shuffle ops) per phase.
template <class OpT>
static int plan_phases(std::vector<OpT> &out, int kw, std::vector<QsvPhaseX> &phases, std::string &err,
                       bool swz, int lane_cap) {
    constexpr bool C128 = std::is_same<OpT, QsvOpD>::value;
    constexpr int FIXED_LO = C128 ? 0 : 1;       // first tile bit on lane bits 0-2
    constexpr int FREE_LO = FIXED_LO + 3;        // tile bits from here on need a slot when targeted
    int rb, wb;
    if (C128 ? layout_for_kw_c128(kw, &rb, &wb) : layout_for_kw(kw, &rb, &wb)) {
        err = "unsupported window size";
        return QSV_ERR_UNSUPPORTED;
    }
    phases.clear();
    if (C128) swz = false;
    const size_t nops = out.size();
    // swizzled layout: tile bits 1+l and 4+l pair up on lane bit l
    auto pair_of = [&](int t) { return (swz && t >= 1 && t <= 6) ? (t - 1) % 3 : -1; };
    auto partner_of = [](int t) { return t <= 3 ? t + 3 : t - 3; };
    struct Assign {
        int regs[QSV_RB_MAX], nr;   // register-bit targets, most used first
        int pl[3];                  // swizzled: target on lane bit l (a pair member), -1 if none
        int fl[2], nf;              // targets on lane bits 3-4
    };
    // slots for a phase's targets, most used first: a register bit (unless the target's pair partner holds
    // one: lane bit l must stay on one of the pair), else the pair's lane bit, else a free lane bit (at most
    // g_phase_lanes of them). False if they do not fit. Without swz this is the plain capacity rule
    // rb + g_phase_lanes over tile bits >= FREE_LO, whose lane bits 0-2 are fixed.
    auto assign = [&](const int *used, const int *cnt, int nu, Assign &A) -> bool {
        int order[QSV_KW_MAX];
        for (int u = 0; u < nu; u++) order[u] = u;
        std::stable_sort(order, order + nu, [&](int x, int y) { return cnt[x] > cnt[y]; });
        A.nr = 0;
        A.nf = 0;
        A.pl[0] = A.pl[1] = A.pl[2] = -1;
        for (int k = 0; k < nu; k++) {
            const int t = used[order[k]];
            const int l = pair_of(t);
            bool partner_reg = false;
            if (l >= 0)
                for (int r = 0; r < A.nr; r++) partner_reg |= A.regs[r] == partner_of(t);
            const int nlane = A.nf + (A.pl[0] >= 0) + (A.pl[1] >= 0) + (A.pl[2] >= 0);
            if (A.nr < rb && !partner_reg) A.regs[A.nr++] = t;
            else if (l >= 0 && A.pl[l] < 0 && nlane < lane_cap) A.pl[l] = t;
            else if (A.nf < g_phase_lanes && nlane < lane_cap) A.fl[A.nf++] = t;
            else return false;
        }
        return true;
    };
    const int need_lo = swz ? 1 : FREE_LO;      // targets from this tile bit on need a slot
    size_t i = 0;
    while (i < nops) {
        size_t j = i;
        int used[QSV_KW_MAX], cnt[QSV_KW_MAX], nu = 0;
        Assign A, B;
        assign(used, cnt, 0, A);
        while (j < nops) {
            const int tb = out[j].tbit;
            if (tb >= need_lo) {
                int f = -1;
                for (int u = 0; u < nu; u++)
                    if (used[u] == tb) f = u;
                if (f < 0) {
                    used[nu] = tb;
                    cnt[nu] = 0;
                    if (!assign(used, cnt, nu + 1, B)) break;
                    A = B;
                    f = nu++;
                }
                cnt[f]++;
            }
            j++;
        }
        // final slots with the phase's use counts (the fit does not depend on the order; keep the last
        // fitting assignment should it differ)
        if (assign(used, cnt, nu, B)) A = B;
        QsvPhaseX ph;
        std::memset(&ph, 0, sizeof(ph));
        bool taken[QSV_KW_MAX] = {false};
        for (int r = 0; r < A.nr; r++) taken[A.regs[r]] = true;
        for (int f = 0; f < A.nf; f++) taken[A.fl[f]] = true;
        for (int l = 0; l < 3; l++) {
            int t = FIXED_LO + l;
            if (swz) {
                if (A.pl[l] >= 0) t = A.pl[l];
                else t = taken[1 + l] ? 4 + l : 1 + l;
            }
            ph.lane_lo[l] = (uint8_t)t;
            taken[t] = true;
        }
        // unused register / lane slots and the warp slots take the remaining bits
        int regs[QSV_RB_MAX], nr = 0, lanes[2], nl = 0;
        for (int r = 0; r < A.nr; r++) regs[nr++] = A.regs[r];
        for (int f = 0; f < A.nf; f++) lanes[nl++] = A.fl[f];
        int rest[QSV_KW_MAX], nrest = 0;
        for (int t = need_lo; t < kw; t++)
            if (!taken[t]) rest[nrest++] = t;
        if (nrest != (rb - nr) + (2 - nl) + wb) { err = "internal: layout does not cover the window"; return QSV_ERR_UNSUPPORTED; }
        int ri = 0;
        while (nr < rb) regs[nr++] = rest[ri++];
        while (nl < 2) lanes[nl++] = rest[ri++];
        for (int w = 0; w < wb; w++) ph.warp_bits[w] = (uint8_t)rest[ri++];
        for (int r = 0; r < rb; r++) ph.reg_bits[r] = (uint8_t)regs[r];
        ph.lane_bits[0] = (uint8_t)lanes[0];
        ph.lane_bits[1] = (uint8_t)lanes[1];
        ph.op_begin = (int32_t)i;
        ph.op_end = (int32_t)j;
        uint32_t regmask = 0;
        for (int r = 0; r < rb; r++) regmask |= 1u << ph.reg_bits[r];
        uint32_t lanemask = (1u << ph.lane_bits[0]) | (1u << ph.lane_bits[1]);
        for (int l = 0; l < 3; l++) lanemask |= 1u << ph.lane_lo[l];
        for (size_t o = i; o < j; o++) {
            OpT &op = out[o];
            const int tb = op.tbit;
            if (!C128 && tb == 0) {
                op.slot = QSV_SLOT_COMP;
            } else {
                op.slot = 0xff;
                for (int r = 0; r < rb; r++)
                    if (ph.reg_bits[r] == tb) op.slot = (uint8_t)(QSV_SLOT_REG0 + r);
                for (int l = 0; l < 3; l++)
                    if (ph.lane_lo[l] == tb) op.slot = (uint8_t)(QSV_SLOT_LANE0 + l);
                for (int l = 0; l < 2; l++)
                    if (ph.lane_bits[l] == tb) op.slot = (uint8_t)(QSV_SLOT_LANE0 + 3 + l);
                if (op.slot == 0xff) { err = "internal: target not placed"; return QSV_ERR_UNSUPPORTED; }
            }
            // control split for this phase's layout: register-index part, tile-bit-0 part, thread part
            op.cm_reg = 0;
            for (int r = 0; r < rb; r++)
                if ((op.cmask >> ph.reg_bits[r]) & 1) op.cm_reg |= (uint8_t)(1u << r);
            op.cm_thr = op.cmask & ~regmask & (C128 ? ~0u : ~1u);
            // controls on lane bits make the selection differ between the lanes of a warp: take the
            // branch-free form of the controlled variants there
            if (op.cm_thr & lanemask) {
                if (op.variant == QSV_V_CTRL_DENSE) op.variant = QSV_V_CTRL_DENSE_SEL;
                else if (op.variant == QSV_V_CTRL_DIAG1) op.variant = QSV_V_CTRL_DIAG1_SEL;
                else if (op.variant == QSV_V_CTRL_SWAP) op.variant = QSV_V_CTRL_SWAP_SEL;
            }
        }
        phases.push_back(ph);
        i = j;
    }
    return QSV_OK;
}

template <class OpT>
static int plan_window(const std::vector<PhysOp> &ops, size_t b, size_t e, const int *tile_of, int n, int kw,
                       std::vector<OpT> &out, std::vector<QsvPhaseX> &phases, std::string &err, bool swz = false,
                       int lane_cap = 8) {
    classify_ops<OpT>(ops, b, e, tile_of, n, out);
    return plan_phases<OpT>(out, kw, phases, err, swz, lane_cap);
}

template <class OpT>
static int fill_sweep(const std::vector<PhysOp> &ops, size_t b, size_t e, uint64_t qset, int n, int kw,
                      QsvSweepT<OpT> &sw, std::string &err) {
    constexpr bool C128 = std::is_same<OpT, QsvOpD>::value;
    int rb, wb;
    if (C128 ? layout_for_kw_c128(kw, &rb, &wb) : layout_for_kw(kw, &rb, &wb)) {
        err = "unsupported window size";
        return QSV_ERR_UNSUPPORTED;
    }
    std::memset(&sw, 0, sizeof(sw));
    const int lo = window_lo(qset, n, kw);
    if (lo < QSV_LO_MIN) { err = "op qubits do not fit one 13-qubit window"; return QSV_ERR_UNSUPPORTED; }
    sw.n = n;
    sw.kw = kw;
    sw.lo = lo;
    int tile_of[64];
    for (int q = 0; q < 64; q++) tile_of[q] = -1;
    for (int q = 0; q < lo; q++) tile_of[q] = q;
    int nh = 0;
    for (int q = lo; q < n; q++)
        if ((qset >> q) & 1) { sw.H[nh] = (uint8_t)q; tile_of[q] = lo + nh; nh++; }
    sw.nh = nh;
    sw.ntiles = 1ll << (n - kw);
    if (!C128) {       // complex128 tiles are staged with bulk copies only
        uint8_t tfree[QSV_TMA_MAX_RANK], tbox[QSV_TMA_MAX_RANK], tstart[QSV_TMA_MAX_RANK];
        const int r = tma_dims(sw, tfree, tbox, tstart);
        sw.tma_rank = (uint8_t)r;
        for (int d = 0; d < r; d++) { sw.tdim_free[d] = tfree[d]; sw.tdim_box[d] = tbox[d]; }
    }
    std::vector<OpT> base, vops;
    std::vector<QsvPhaseX> vph;
    classify_ops<OpT>(ops, b, e, tile_of, n, base);
    vops = base;
    int rc = plan_phases<OpT>(vops, kw, vph, err, false, 8);
    if (rc) return rc;
    // the swizzled layout where it costs less: cost = lane ops + 2 per phase change (a shared-memory round
    // trip moves as many bytes through the shared-memory pipe as two shuffle ops); ties keep the plain one
    int plain_lane = 0;
    for (const OpT &x : vops) plain_lane += x.slot >= QSV_SLOT_LANE0 && x.variant != QSV_V_SKIP;
    if (!C128 && swizzle_enabled() && plain_lane > 0) {
        uint8_t tfree[QSV_TMA_MAX_RANK], tbox[QSV_TMA_MAX_RANK], tstart[QSV_TMA_MAX_RANK];
        const int r = tma_dims(sw, tfree, tbox, tstart, true);
        // QSV_PHASE_COST overrides the weight of a phase change (tuning studies)
        static const int phase_cost = [] {
            const char *e = std::getenv("QSV_PHASE_COST");
            return e ? std::atoi(e) : 2;
        }();
        auto cost = [](const std::vector<OpT> &o, const std::vector<QsvPhaseX> &p) {
            int lane = 0;
            for (const OpT &x : o) lane += x.slot >= QSV_SLOT_LANE0 && x.variant != QSV_V_SKIP;
            return lane + phase_cost * ((int)p.size() - 1);
        };
        // phases with fewer shuffle ops but more round trips, or the reverse: try lane-op budgets per phase
        for (int cap : {0, 1, 2, 8}) {
            if (!r) break;
            std::vector<OpT> sops = base;
            std::vector<QsvPhaseX> sph;
            std::string serr;
            if (plan_phases<OpT>(sops, kw, sph, serr, true, cap) == QSV_OK &&
                sph.size() <= QSV_MAX_PHASES && cost(sops, sph) < cost(vops, vph)) {
                vops.swap(sops);
                vph.swap(sph);
                sw.swz = 1;
                sw.tma_rank = (uint8_t)r;
                for (int d = 0; d < r; d++) { sw.tdim_free[d] = tfree[d]; sw.tdim_box[d] = tbox[d]; }
            }
        }
    }
    if (vops.size() > QSV_MAX_SWEEP_OPS || vph.size() > QSV_MAX_PHASES) { err = "sweep too large"; return QSV_ERR_UNSUPPORTED; }
    sw.nops = (int)vops.size();
    sw.nphases = (int)vph.size();
    std::memcpy(sw.ops, vops.data(), vops.size() * sizeof(OpT));
    for (size_t p = 0; p < vph.size(); p++) {
        QsvPhase &d = sw.phases[p];
        const QsvPhaseX &x = vph[p];
        std::memcpy(d.reg_bits, x.reg_bits, sizeof(d.reg_bits));
        std::memcpy(d.lane_bits, x.lane_bits, sizeof(d.lane_bits));
        std::memcpy(d.warp_bits, x.warp_bits, sizeof(d.warp_bits));
        std::memcpy(d.lane_lo, x.lane_lo, sizeof(d.lane_lo));
        d.op_begin = (uint8_t)x.op_begin;
        d.op_end = (uint8_t)x.op_end;
    }
    return QSV_OK;
}

int plan_whole_state(const std::vector<PhysPass> &passes, int n, std::vector<QsvOp> &ops_out,
                     std::vector<QsvPhaseX> &phases_out, std::string &err) {
    std::vector<PhysOp> ops;
    for (const PhysPass &p : passes) ops.insert(ops.end(), p.ops.begin(), p.ops.end());
    int tile_of[64];
    for (int q = 0; q < 64; q++) tile_of[q] = q < n ? q : -1;
    return plan_window<QsvOp>(ops, 0, ops.size(), tile_of, n, n, ops_out, phases_out, err);
}

template <class OpT>
int build_sweeps(const std::vector<PhysPass> &passes, int n, int kw, int lo_merge,
                 std::vector<QsvSweepT<OpT>> &out, std::string &err) {
    out.clear();
    std::vector<PhysOp> ops;
    uint64_t cur = 0;
    size_t begin = 0;
    auto flush = [&]() -> int {
        if (ops.size() > begin) {
            out.emplace_back();
            int rc = fill_sweep<OpT>(ops, begin, ops.size(), cur, n, kw, out.back(), err);
            if (rc) return rc;
        }
        begin = ops.size();
        cur = 0;
        return QSV_OK;
    };
    for (const PhysPass &p : passes) {
        if (p.ops.empty()) continue;
        uint64_t q = 0;
        for (const PhysOp &o : p.ops) q |= op_qubits(o);
        const uint64_t merged = cur | q;
        const size_t nmerged = ops.size() - begin + p.ops.size();
        const bool fits = window_lo(merged, n, kw) >= lo_merge && nmerged <= QSV_MAX_SWEEP_OPS;
        if (ops.size() > begin && !fits) {
            int rc = flush();
            if (rc) return rc;
        }
        ops.insert(ops.end(), p.ops.begin(), p.ops.end());   // a QSV2 pass has <= 64 ops < the sweep budget
        cur |= q;
    }
    return flush();
}
template int build_sweeps<QsvOp>(const std::vector<PhysPass> &, int, int, int, std::vector<QsvSweep> &,
                                 std::string &);
template int build_sweeps<QsvOpD>(const std::vector<PhysPass> &, int, int, int, std::vector<QsvSweepD> &,
                                  std::string &);

// Groups for the streaming interpreter, greedy in op order: a group takes ops while their targets (tile
// bits >= 1, except diagonal ops, which act element by element and so run on any tile bit of the item)
// span at most three distinct tile bits; the fourth distinct target starts the next group. A group with
// fewer than three such targets takes the highest free tile bits as item bits (their 16-byte chunks are
// spread over all shared-memory banks). Every group but the last holds three ops on distinct targets, so a
// sweep of at most QSV_MAX_SWEEP_OPS ops needs at most QSV_MAX_SWEEP_OPS / 3 + 1 groups.
int plan_stream(QsvSweep &sw, std::string &err) {
    static_assert(QSV_MAX_GROUPS >= QSV_MAX_SWEEP_OPS / 3 + 1, "group table too small");
    const int kw = sw.kw, nops = sw.nops;
    auto elementwise = [](const QsvOp &o) {
        return o.variant == QSV_V_SKIP || o.variant == QSV_V_UNI_DIAG || o.variant == QSV_V_CTRL_DIAG1 ||
               o.variant == QSV_V_CTRL_DIAG1_SEL;
    };
    int ng = 0;
    for (int i = 0; i < nops;) {
        int S[3] = {-1, -1, -1}, ns = 0, j = i;
        auto has = [&](int t) { return t == S[0] || t == S[1] || t == S[2]; };
        for (; j < nops; j++) {
            const QsvOp &o = sw.ops[j];
            if (o.tbit == 0 || elementwise(o) || has(o.tbit)) continue;
            if (ns == 3) break;
            S[ns++] = o.tbit;
        }
        for (int t = kw - 1; ns < 3 && t >= 1; t--)
            if (!has(t)) S[ns++] = t;
        if (ng == QSV_MAX_GROUPS || ns < 3) { err = "internal: streaming plan does not fit"; return QSV_ERR_UNSUPPORTED; }
        QsvGroup &g = sw.groups[ng++];
        std::memset(&g, 0, sizeof(g));
        uint32_t item = 1u;
        for (int k = 0; k < 3; k++) {
            g.q[k] = (uint8_t)S[k];
            item |= 1u << S[k];
        }
        g.op_begin = (uint8_t)i;
        g.op_end = (uint8_t)j;
        g.type = -1;
        for (int o = i; o < j; o++) {
            QsvOp &op = sw.ops[o];
            const int t = op.tbit;
            // the branch-free controlled forms (chosen for lane-bit controls of a phase layout) give the
            // same values as the plain ones, which skip unselected pairs: items have no lane bits
            if (op.variant == QSV_V_CTRL_DENSE_SEL) op.variant = QSV_V_CTRL_DENSE;
            else if (op.variant == QSV_V_CTRL_DIAG1_SEL) op.variant = QSV_V_CTRL_DIAG1;
            else if (op.variant == QSV_V_CTRL_SWAP_SEL) op.variant = QSV_V_CTRL_SWAP;
            op.slot = QSV_SLOT_BASE;
            if (t == 0) op.slot = QSV_SLOT_COMP;
            op.cm_reg = 0;
            for (int k = 0; k < 3; k++) {
                if (t == S[k]) op.slot = (uint8_t)(QSV_SLOT_REG0 + k);
                op.cm_reg |= (uint8_t)(((op.cmask >> S[k]) & 1u) << k);
            }
            op.cm_thr = op.cmask & ~item;
        }
        i = j;
    }
    sw.ngroups = ng;
    return QSV_OK;
}

int serialize_stream(const std::vector<QsvSweep> &sw, int32_t *out, size_t cap) {
    std::vector<int32_t> w;
    w.push_back((int32_t)sw.size());
    for (const QsvSweep &s : sw) {
        w.push_back(s.kw); w.push_back(s.ngroups); w.push_back(s.nops);
        for (int g = 0; g < s.ngroups; g++) {
            const QsvGroup &G = s.groups[g];
            for (int k = 0; k < 3; k++) w.push_back(G.q[k]);
            w.push_back(G.op_begin); w.push_back(G.op_end);
        }
        for (int o = 0; o < s.nops; o++) {
            const QsvOp &op = s.ops[o];
            w.push_back(op.tbit); w.push_back(op.slot); w.push_back(op.variant); w.push_back((int32_t)op.cmask);
            w.push_back(op.cm_reg); w.push_back((int32_t)op.cm_thr); w.push_back(op.kind);
        }
    }
    if (out) std::memcpy(out, w.data(), sizeof(int32_t) * std::min(cap, w.size()));
    return (int)w.size();
}

int serialize(const std::vector<QsvSweep> &sw, int32_t *out, size_t cap) {
    std::vector<int32_t> w;
    w.push_back((int32_t)sw.size());
    for (const QsvSweep &s : sw) {
        int rb = 0, wb = 0;
        layout_for_kw(s.kw, &rb, &wb);
        w.push_back(s.kw); w.push_back(s.lo); w.push_back(s.nh);
        for (int i = 0; i < QSV_KW_MAX; i++) w.push_back(i < s.nh ? s.H[i] : -1);
        w.push_back(s.tma_rank);
        for (int d = 0; d < QSV_TMA_MAX_RANK; d++) w.push_back(d < s.tma_rank ? s.tdim_free[d] : -1);
        for (int d = 0; d < QSV_TMA_MAX_RANK; d++) w.push_back(d < s.tma_rank ? s.tdim_box[d] : -1);
        w.push_back(s.swz);
        w.push_back(s.nphases); w.push_back(s.nops);
        for (int p = 0; p < s.nphases; p++) {
            const QsvPhase &ph = s.phases[p];
            for (int r = 0; r < QSV_RB_MAX; r++) w.push_back(r < rb ? ph.reg_bits[r] : -1);
            w.push_back(ph.lane_bits[0]); w.push_back(ph.lane_bits[1]);
            for (int r = 0; r < QSV_WB_MAX; r++) w.push_back(r < wb ? ph.warp_bits[r] : -1);
            w.push_back(ph.op_begin); w.push_back(ph.op_end);
            for (int l = 0; l < 3; l++) w.push_back(ph.lane_lo[l]);
        }
        for (int o = 0; o < s.nops; o++) {
            const QsvOp &op = s.ops[o];
            w.push_back(op.tbit); w.push_back(op.slot); w.push_back((int32_t)op.cmask);
            w.push_back(op.cls0); w.push_back(op.cls1);
            w.push_back(op.kind); w.push_back(op.cls); w.push_back(op.cm_reg); w.push_back(op.cm_c);
            w.push_back((int32_t)op.cm_thr); w.push_back(op.variant);
            int32_t b[8];
            std::memcpy(b, op.m0, 32);
            for (int e = 0; e < 8; e++) w.push_back(b[e]);
            std::memcpy(b, op.m1, 32);
            for (int e = 0; e < 8; e++) w.push_back(b[e]);
        }
    }
    if (out) std::memcpy(out, w.data(), sizeof(int32_t) * std::min(cap, w.size()));
    return (int)w.size();
}

}  // namespace qsv
