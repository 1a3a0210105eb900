// qsv_planner.h -- host-side decode of QSV2 segments into sweep plans (see qsv_plan.h).
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/qsv_b200.h"
#include "qsv_plan.h"

#define QSV2_MAGIC 0x51535632u
#define QSV2_HDR_WORDS 8
#define QSV2_PASS_WORDS 8
#define QSV2_OP_WORDS 24
#define QSV2_OP_WORDS_C128 40    // complex128 extension: FP64 matrices (header word 4 = 1)
#define QSV2_OP_MUX2 1
#define QSV2_MAX_OPS 64

namespace qsv {

// one MUX2 op in physical coordinates
struct PhysOp {
    int t;                 // target qubit
    uint64_t cmask;        // control qubits
    float m0[8], m1[8];    // complex64 segments
    double d0[8], d1[8];   // complex128 segments
};
struct PhysPass {
    std::vector<PhysOp> ops;
};

// Validate a segment for an n-qubit state and convert its ops to physical qubits. dtype 0: complex64
// (the reference's streams), 1: complex128 (FP64 matrices); header word 4 must equal dtype.
int decode_segment(const int32_t *seg, size_t nwords, int n, std::vector<PhysPass> &out, std::string &err,
                   int dtype = 0);
// Register/warp bit split of the consumer layout for a window of kw qubits (kw in 10..13).
int layout_for_kw(int kw, int *rb, int *wb);
// Choose the 13-qubit layout: 4 register bits x 8 consumer warps, or 3 x 16 (process-wide).
int set_rb13(int rb);
// How many of a phase's targets (tile bits >= 4) may sit on lane bits 3, 4 (0..2; default 1).
int set_phase_lanes(int k);
// Register/warp bit split of the complex128 layout for a window of kw qubits (kw in 10..12): tile bits
// 0-2 on lane bits 0-2, two chosen lane bits, 4 register bits, kw - 9 warp bits.
int layout_for_kw_c128(int kw, int *rb, int *wb);
// Merge consecutive passes into sweeps of window kw; merged windows keep >= 2^lo_merge contiguous amps.
// OpT = QsvOp (complex64) or QsvOpD (complex128).
template <class OpT>
int build_sweeps(const std::vector<PhysPass> &passes, int n, int kw, int lo_merge,
                 std::vector<QsvSweepT<OpT>> &out, std::string &err);
// Whole-state program of an n-qubit circuit (n in 10..13: the state is one tile): every op of every pass,
// in order, with its phases.
int plan_whole_state(const std::vector<PhysPass> &passes, int n, std::vector<QsvOp> &ops_out,
                     std::vector<QsvPhaseX> &phases_out, std::string &err);
// Re-plan a complex64 sweep for the streaming interpreter: groups of consecutive ops with at most three
// distinct target tile bits >= 1 (ops on tile bit 0 and diagonal ops on other bits join any group), and
// each op's slot / control split for its group's item layout. Replaces the phase fields of the ops.
int plan_stream(QsvSweep &sw, std::string &err);
// Flatten streaming plans (plan_stream) into int32 words: sweeps; per sweep kw, ngroups, nops, then per group
// q0 q1 q2 op_begin op_end, then per op tbit slot variant cmask cm_reg cm_thr kind.
int serialize_stream(const std::vector<QsvSweep> &sw, int32_t *out, size_t cap);
// Flatten a plan into int32 words (layout documented in qsv_b200.h / the planner tests).
int serialize(const std::vector<QsvSweep> &sw, int32_t *out, size_t cap);

}  // namespace qsv
