// qsv_plan.h -- the sweep plan: how the engine executes a QSV2 segment (shared by host and device).
//
// A QSV2 pass (host/sv/isa.py:13-21) applies its MUX2 ops to every 2^k-amplitude tile of one qubit
// window. Consecutive passes whose combined qubit set fits one engine window are executed as ONE sweep
// over HBM: applying pass A's ops and then pass B's ops tile by tile gives exactly the amplitudes that
// pass-by-pass execution gives, because every op only reads and writes amplitude pairs inside the tile
// and ops are applied in program order.
//
// Sweep window: W = {0, ..., lo-1} U H (H sorted, all >= lo), |W| = KW. Tile bit i <-> physical qubit
// W[i]. A tile is 2^(KW - lo) sub-blocks of 2^lo contiguous amplitudes (sub-block s at
// base | pdep(s, H)); tile T's base is pdep(T, free bits), the free bits being the qubits outside W.
//
// Tile staging: with long sub-blocks (lo >= QSV_TMA_TENSOR_LO) one bulk-async copy per sub-block; with
// short ones a single tensor-map TMA box per tile. The tensor map views the state as up to 5 dims, one per
// run of consecutive window bits (the low run [0, lo) and each run of H); every dim also spans the free
// bits directly above its run, so a tile's free bits become box coordinates: coordinate of dim d =
// (next tdim_free[d] bits of T) << tdim_box[d].
//
// In-tile execution: consumer thread layout per phase (KW = 1 + 3 + 2 + RB + WB tile bits):
//   tile bit 0          -> the two halves of one float4 (a thread keeps them packed as re/im float2 pairs)
//   tile bits 1, 2, 3   -> lane bits 0, 1, 2 (conflict-free 128-bit shared-memory accesses)
//   lane_bits[0..1]     -> lane bits 3, 4
//   reg_bits[0..RB-1]   -> register index bits (2^RB float4 per thread)
//   warp_bits[..]       -> warp index bits
// An op can run in a phase when its target is tile bit 0..3, a register bit or a lane bit of that phase;
// controls may sit anywhere in the window.
#pragma once
#ifdef __CUDACC_RTC__
// compiled at run time by NVRTC (sweep kernels specialised to one structure): no host headers there
typedef signed char int8_t;
typedef unsigned char uint8_t;
typedef short int16_t;
typedef unsigned short uint16_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
#else
#include <stdint.h>
#endif

#define QSV_KW_MAX 13
#define QSV_RB_MAX 4
#define QSV_WB_MAX 4
#define QSV_MAX_SWEEP_OPS 96
#define QSV_MAX_PHASES 24
#define QSV_LO_MIN 3            // smallest sub-block: 2^3 amplitudes = 64 bytes (QSV2 guarantees k-m >= 3)
#define QSV_TMA_TENSOR_LO 9     // sub-blocks shorter than 2^9 amplitudes are staged with a tensor-map box
#define QSV_SMEM_ALIGN 1024     // sweep kernels align their tile buffers to this in dynamic shared memory
#define QSV_TMA_MAX_RANK 5
#define QSV_WAIT_US_DEFAULT 2000000u   // bounded mbarrier waits: 2 s (a tile takes microseconds)

// matrix classes (host-detected, exact comparisons). The specialised forms give the same values as the
// dense fused-multiply-add chain (the skipped terms are exact zeros).
#define QSV_M_DENSE 0
#define QSV_M_DIAG 1            // off-diagonal entries are (+/-)0
#define QSV_M_IDENT 2           // identity: pair left unchanged
#define QSV_M_XSWAP 3           // [[0,1],[1,0]]: the two amplitudes are exchanged
#define QSV_M_DIAG1 4           // diag(1, d): only the bit-1 amplitude changes
// dense with m00 real (its imaginary part an exact zero, as in every U3): the two m00.im terms of the
// chain are skipped. Used as a code path only; op records keep QSV_M_DENSE and set r00.
#define QSV_M_DENSE_R0 5

// op kinds
#define QSV_K_UNI 0             // one matrix (M0) for every pair
#define QSV_K_CTRL 1            // M0 = identity: pairs whose controls are all set get M1
#define QSV_K_MUX 2             // general: M1 where the controls are set, M0 elsewhere (dense math)

// code path of an op (host-chosen from kind, class and controls): one tight loop per variant
#define QSV_V_SKIP 0            // identity everywhere
#define QSV_V_UNI_DENSE 1       // y = M0 x
#define QSV_V_UNI_DIAG 2        // y0 = m00 x0, y1 = m11 x1
#define QSV_V_UNI_SWAP 3        // exchange
#define QSV_V_CTRL_DENSE 4      // y = M1 x where selected (M0 = I)
#define QSV_V_CTRL_DIAG1 5      // y1 = m11 x1 where selected (M0 = I, M1 = diag(1, d))
#define QSV_V_CTRL_SWAP 6       // exchange where selected (M0 = I, M1 = X)
#define QSV_V_MUX 7             // general selection, per-pair coefficient select, dense arithmetic
// controlled ops whose controls vary across the lanes of a warp: selects instead of branches
#define QSV_V_CTRL_DENSE_SEL 8
#define QSV_V_CTRL_DIAG1_SEL 9
#define QSV_V_CTRL_SWAP_SEL 10
// code path only (op records keep QSV_V_UNI_DENSE and set r00): dense with m00 real, register-bit target
#define QSV_V_UNI_DENSE_R0 11

// where the target of an op lives in its phase
#define QSV_SLOT_COMP 0         // tile bit 0 (inside a float4)
#define QSV_SLOT_REG0 1         // 1 + r: register bit r
#define QSV_SLOT_LANE0 8        // 8 + l: lane bit l (warp shuffle)
#define QSV_SLOT_BASE 7         // streaming interpreter: diagonal op on a tile bit of the item base

// 96 bytes, 16-byte aligned: the matrices are four 16-byte vectors and every field a kernel reads is in
// the 16 bytes at offset 64 (one vector load per op in the streaming interpreter).
struct alignas(16) QsvOp {
    float m0[8];                // M0 = m00 m01 m10 m11 as (re, im)
    float m1[8];                // M1
    uint32_t cm_thr;            // the part of cmask on lane / warp tile bits (tested on the thread base)
    uint8_t cm_reg;             // the part of cmask on register bits, as a mask over the register index
    uint8_t cm_c;               // 1 if tile bit 0 is a control
    uint8_t kind;               // QSV_K_*
    uint8_t cls;                // QSV_M_* of the matrix the kind applies (M0 for UNI, M1 for CTRL)
    uint8_t cls0, cls1;         // QSV_M_* of M0, M1
    uint8_t slot;               // QSV_SLOT_*
    uint8_t tbit;               // target tile bit
    uint8_t variant;            // QSV_V_*
    uint8_t r00;                // 1: M0 is dense with m00 real (QSV_M_DENSE_R0 path)
    uint8_t pad[2];
    uint32_t cmask;             // control mask over tile bits (0 = no controls)
};

// complex128 op: the same fields with FP64 matrices. In the complex128 layout tile bits 0-2 are lane bits
// 0-2 (one 16-byte amplitude per slot), so there is no QSV_SLOT_COMP and cm_c is always 0.
struct QsvOpD {
    double m0[8];
    double m1[8];
    uint32_t cmask;
    uint32_t cm_thr;
    uint8_t cm_reg;
    uint8_t cm_c;
    uint8_t kind;
    uint8_t cls;
    uint8_t cls0, cls1;
    uint8_t slot;
    uint8_t tbit;
    uint8_t variant;
    uint8_t r00;
    uint8_t pad[6];
};


// A phase's thread layout: lane bits 0-2 sit on tile bits lane_lo[0..2] (1, 2, 3 for complex64 unless the
// sweep is swizzled, see QsvSweepT::swz; 0, 1, 2 for complex128), lane bits 3-4 on lane_bits[0..1].
struct QsvPhase {
    uint8_t reg_bits[QSV_RB_MAX];
    uint8_t lane_bits[2];
    uint8_t warp_bits[QSV_WB_MAX];
    uint8_t op_begin, op_end;
    uint8_t lane_lo[3];
    uint8_t pad[1];
};

// phase with 32-bit op indices (whole-circuit programs of the batch kernel can exceed 255 ops)
struct QsvPhaseX {
    uint8_t reg_bits[QSV_RB_MAX];
    uint8_t lane_bits[2];
    uint8_t warp_bits[QSV_WB_MAX];
    uint8_t lane_lo[3];
    uint8_t pad[3];
    int32_t op_begin, op_end;
};

// Streaming interpreter (qsv_sweep.cu): a group of consecutive ops that runs as one shared-memory round
// trip of the tile. A thread takes items of 8 float4 = 16 amplitudes, tile bits {0, q[0], q[1], q[2]}; the
// group's ops target tile bit 0 or an item bit (register index bits 0-2 of the item), or are diagonal on
// another tile bit (QSV_SLOT_BASE: the factor depends on a bit of the item's base).
#define QSV_MAX_GROUPS 40       // every group but the last holds ops on three distinct target bits
struct QsvGroup {
    uint8_t q[3];               // item bits: distinct, in [1, kw)
    uint8_t op_begin, op_end;
    uint8_t pad;
    int16_t type;               // group-type library: case of this group's op sequence (-1: none)
};

template <class OpT>
struct QsvSweepT {
    typedef OpT op_type;
    int32_t n;                  // state qubits
    int32_t kw;                 // window size (tile = 2^kw amplitudes)
    int32_t lo;                 // contiguous low bits of the window
    int32_t nh;                 // |H|
    uint8_t H[QSV_KW_MAX];      // high window qubits, ascending
    uint8_t tma_rank;           // 0: bulk copies per sub-block; 2..5: one tensor-map box per tile
    uint8_t tdim_free[QSV_TMA_MAX_RANK];   // free bits of T folded into each tensor dim (low dim first)
    uint8_t tdim_box[QSV_TMA_MAX_RANK];    // log2 box extent of each tensor dim
    // 1: the tile sits in shared memory with the 128-byte swizzle of the tensor-map copies (16-byte chunk
    // index = tile bits 1-3 XOR tile bits 4-6), so lane bit l may sit on tile bit 1+l or 4+l without bank
    // conflicts and ops on tile bits 1-3 can run in registers (complex64 tensor-map sweeps only)
    uint8_t swz;
    uint8_t pad[3];
    int64_t ntiles;             // 2^(n - kw)
    int32_t nphases;
    int32_t nops;
    uint32_t wait_us;           // bounded waits give up after this many microseconds (0: QSV_WAIT_US_DEFAULT)
    int32_t skip_load;          // fault injection for tests: 1 = block 0 never loads its first tile (0: off)
    QsvPhase phases[QSV_MAX_PHASES];
    OpT ops[QSV_MAX_SWEEP_OPS];
    int32_t ngroups;            // streaming plan (plan_stream; 0 until planned)
    QsvGroup groups[QSV_MAX_GROUPS];
};
typedef QsvSweepT<QsvOp> QsvSweep;      // complex64 state, fp32 matrices
typedef QsvSweepT<QsvOpD> QsvSweepD;    // complex128 state, fp64 matrices
