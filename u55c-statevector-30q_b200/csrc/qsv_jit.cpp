// qsv_jit.cpp -- sweep kernels specialised to one sweep structure, generated and compiled at run time.
//
// No reference counterpart (the reference's engine is one fixed HLS kernel). The interpreter kernel
// (qsv_sweep.cu) reads every op's slot, variant and controls at run time; a specialised kernel has them as
// template arguments (qsv_jit_ops.cuh), so per-op dispatch, control tests on register bits and layout
// arithmetic vanish from the inner loop. A sweep's *structure* is everything but its matrices, window and
// tile addressing: window size, phase layouts, and per op the target slot, code variant and control masks.
// Circuits repeat structures (a 30-qubit random-layer circuit of depth 24 has 84 sweeps of 7 structures),
// so each structure is compiled once per process with NVRTC (sm_100a cubin from the engine's own device
// headers, embedded at build time) and loaded into every device that runs it. Matrices, window and tile
// addressing stay kernel parameters. Specialised and interpreted sweeps compute the same values.
//
// Coarse structures: many sweeps differ only in which ops happen to be diagonal, dense or identity (a
// random circuit picks its one-qubit gates per qubit and layer), so their exact structures never repeat.
// A sweep's coarse structure keeps its layouts, and per op the slot, the control masks, the kind (uniform /
// controlled / general) and whether the matrix is a swap, and drops everything that depends on the matrix
// values: every other op runs the dense fused-multiply-add chain, which gives the same values on diagonal
// and identity matrices (the skipped terms are exact zeros). A coarse kernel serves every sweep with that
// coarse structure (a 30-qubit random circuit of depth 10 has 35 sweeps of 35 exact structures but 7
// coarse ones, the same 7 for other seeds), at the cost of dense arithmetic for the diagonal ops.
//
// Modes: 0 = interpreter only; 1 = eager (a new structure is compiled before its first launch);
// 2 = automatic (default): a structure is compiled in the background once the amplitudes its launches
// have swept add up to kWorkThreshold (a compilation costs about a second of one host core, worth it
// for sweeps that run often or over large states), with at most kMaxQueued compilations waiting; until
// then a sweep runs the kernel of its coarse structure, compiled by the same rule with the work of every
// sweep that shares it (kCoarseThreshold, 2^30 amplitudes), or the interpreter; 3 = eager, coarse
// structures only (tests and measurements of the coarse kernels).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <algorithm>
#include <cstdio>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "qsv_planner.h"
#include "_gen/qsv_jit_headers.inc"

namespace qsv {
namespace dev {
cudaError_t make_tmap(CUtensorMap *map, float2 *state, const QsvSweep &sw);
}
cudaError_t status_word_ptr(int **out);

namespace {

constexpr double kWorkThreshold = 2147483648.0;   // 2^31 amplitudes: 2 sweeps at 30 qubits, 512 at 22
constexpr double kCoarseThreshold = 1073741824.0; // 2^30, summed over the sweeps of a coarse key: a coarse
                                                  // kernel serves many sweeps, so it is worth compiling once
                                                  // one 30-qubit sweep (or 64 at 24 qubits) has used it
constexpr size_t kMaxQueued = 64;
constexpr size_t kMaxEntries = 8192;   // structures tracked; past it, the ones never queued are forgotten
constexpr int kMaxDevices = 64;
constexpr int kStages = 3;         // tile buffers in flight (as the interpreter)

// Consumer groups per CTA for a sweep. Two groups (16 consumer warps taking alternate tiles, registers
// capped at 96 per thread: 17 warps share the four schedulers' register files) overlap one group's phase
// round trips with the other's arithmetic. Warp-shuffle ops need the most registers: with more than three
// the kernel spills, so it takes one group. Measured on the 30-qubit random-layer program: 3.05 -> 2.96 ms
// for sweeps with 7-8 dense ops; with swizzled layouts, 4.65-4.69 -> 4.46-4.53 ms for the FP32-bound
// sweeps with 12 dense ops and 0-3 shuffle ops (before swizzled layouts those had 5-6 shuffle ops and ran
// slower with two groups, 4.4 -> 5.3 ms). QSV_JIT_GROUPS13=1 or 2 forces one choice.
int groups_for(const QsvSweep &sw, int wb) {
    static const int forced = [] {
        const char *e = std::getenv("QSV_JIT_GROUPS13");
        return e ? std::atoi(e) : 0;
    }();
    if (sw.kw != 13 || wb > 3) return 1;
    if (forced == 1 || forced == 2) return forced;
    int lane = 0;
    for (int o = 0; o < sw.nops; o++) {
        const QsvOp &op = sw.ops[o];
        lane += op.slot >= QSV_SLOT_LANE0 && op.variant != QSV_V_SKIP;
    }
    return lane <= 3 ? 2 : 1;
}

// Whether a sweep's kernel interleaves the phases of two tiles per consumer thread (sweep_pipeline IL).
// Off by default: on the 30-qubit random-layer program it made the tensor-map sweeps with 7-8 dense ops
// 0.5-2 % faster and the FP32-bound sweeps over qubits 0-12 5-15 % slower (their prefetch depth drops from
// two tiles to one). QSV_JIT_INTERLEAVE=1: multi-phase tensor-map sweeps of one consumer group; =2: every
// multi-phase sweep of one consumer group.
// Whether uncontrolled dense ops on register bits use the coefficient-major form (jit_reg_cm). Tuning
// switch QSV_JIT_CM=1; off by default.
bool coef_major() {
    static const bool on = [] {
        const char *e = std::getenv("QSV_JIT_CM");
        return e && std::atoi(e) == 1;
    }();
    return on;
}

int interleave_for(const QsvSweep &sw, int groups) {
    static const int mode = [] {
        const char *e = std::getenv("QSV_JIT_INTERLEAVE");
        return e ? std::atoi(e) : 0;
    }();
    if (mode == 0 || groups != 1 || sw.nphases < 2) return 0;
    return mode == 2 || sw.tma_rank > 0 ? 1 : 0;
}

struct Drv {
    PFN_cuModuleLoadData_v2000 module_load = nullptr;
    PFN_cuModuleGetFunction_v2000 get_function = nullptr;
    PFN_cuFuncSetAttribute_v9000 set_attribute = nullptr;
    PFN_cuLaunchKernel_v4000 launch = nullptr;
    PFN_cuOccupancyMaxActiveBlocksPerMultiprocessor_v6050 occupancy = nullptr;
    bool ok = false;
};

const Drv &drv() {
    static const Drv d = [] {
        Drv x;
        auto get = [](const char *name, void **p) {
            cudaDriverEntryPointQueryResult q;
            return cudaGetDriverEntryPoint(name, p, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess;
        };
        x.ok = get("cuModuleLoadData", reinterpret_cast<void **>(&x.module_load)) &&
               get("cuModuleGetFunction", reinterpret_cast<void **>(&x.get_function)) &&
               get("cuFuncSetAttribute", reinterpret_cast<void **>(&x.set_attribute)) &&
               get("cuLaunchKernel", reinterpret_cast<void **>(&x.launch)) &&
               get("cuOccupancyMaxActiveBlocksPerMultiprocessor", reinterpret_cast<void **>(&x.occupancy));
        return x;
    }();
    return d;
}

enum State { kNew, kQueued, kReady, kFailed };

struct Entry {
    int kw = 0, rb = 0, wb = 0, groups = 1;
    std::string src;
    State state = kNew;
    std::vector<char> cubin;
    std::string log;
    long long uses = 0;
    bool coarse = false;        // a coarse structure's kernel (coarse_of)
    bool stream = false;        // a streaming-form kernel (gen_source_stream; op table in shared memory)
    double work = 0.0;          // amplitudes swept by this structure's launches
    CUfunction fn[kMaxDevices] = {nullptr};
    int per_sm[kMaxDevices] = {0};
};

// a compiled (or compiling) group-type library: its cases in order
struct Lib {
    int rb = 0, wb = 0;
    std::vector<std::string> types;
    std::unordered_map<std::string, int> index;
    std::shared_ptr<Entry> entry;
};

// the libraries of one build
struct LibSet {
    std::vector<std::shared_ptr<Lib>> libs;
    int types = 0;              // distinct group types over the libraries
};

struct Jit {
    std::mutex mu;
    std::condition_variable work, done;
    std::unordered_map<std::string, std::shared_ptr<Entry>> map;
    std::deque<std::shared_ptr<Entry>> queue;
    int threads = 0, busy = 0;
    bool stopping = false;      // set at process exit: workers take no new work
    int mode = 2;
    long long jit_launches = 0, interp_launches = 0, coarse_launches = 0, compiled = 0, failed = 0;
    // group-type libraries: amplitudes swept per group type, the set in use and the one being built
    std::unordered_map<std::string, double> gweight;
    std::shared_ptr<LibSet> lib, lib_next;
    double lib_uncovered = 0.0;
    long long lib_launches = 0;
    double compile_ms = 0.0;
    std::string last_log;
};

// process-lifetime state (never destroyed: detached compile threads may still wait on it at exit)
Jit &J() {
    static Jit *j = new Jit;
    return *j;
}

bool is_swap_variant(int v) {
    return v == QSV_V_UNI_SWAP || v == QSV_V_CTRL_SWAP || v == QSV_V_CTRL_SWAP_SEL;
}

// The coarse structure of sw: a copy whose ops keep slot, controls, kind and the swap / non-swap split,
// with every value-dependent field replaced by its dense form (generated code reads only these fields).
QsvSweep coarse_of(const QsvSweep &sw) {
    QsvSweep c = sw;
    for (int o = 0; o < c.nops; o++) {
        QsvOp &op = c.ops[o];
        const bool swap = is_swap_variant(op.variant) ||
                          (op.variant == QSV_V_MUX && op.kind == QSV_K_CTRL && op.cls1 == QSV_M_XSWAP);
        const bool sel = op.variant == QSV_V_CTRL_DENSE_SEL || op.variant == QSV_V_CTRL_DIAG1_SEL ||
                         op.variant == QSV_V_CTRL_SWAP_SEL;
        op.r00 = 0;
        if (op.kind == QSV_K_UNI) {
            op.cls = op.cls0 = op.cls1 = swap ? QSV_M_XSWAP : QSV_M_DENSE;
            op.variant = swap ? QSV_V_UNI_SWAP : QSV_V_UNI_DENSE;
        } else if (op.kind == QSV_K_CTRL) {
            op.cls0 = QSV_M_IDENT;
            op.cls = op.cls1 = swap ? QSV_M_XSWAP : QSV_M_DENSE;
            if (op.variant != QSV_V_MUX)       // the tile-bit-0-control form stays MUX (its own code path)
                op.variant = swap ? (sel ? QSV_V_CTRL_SWAP_SEL : QSV_V_CTRL_SWAP)
                                  : (sel ? QSV_V_CTRL_DENSE_SEL : QSV_V_CTRL_DENSE);
        } else {
            op.cls = op.cls0 = op.cls1 = QSV_M_DENSE;
            op.variant = QSV_V_MUX;
        }
    }
    return c;
}

std::string key_of(const QsvSweep &sw, int rb, int wb) {
    std::string k;
    auto put = [&](int v) { k.push_back((char)(v & 0xff)); };
    auto put32 = [&](uint32_t v) { k.append(reinterpret_cast<const char *>(&v), 4); };
    put(sw.kw); put(rb); put(wb); put(sw.nphases); put(sw.nops); put(sw.swz);
    for (int p = 0; p < sw.nphases; p++) {
        const QsvPhase &ph = sw.phases[p];
        for (int r = 0; r < rb; r++) put(ph.reg_bits[r]);
        for (int l = 0; l < 3; l++) put(ph.lane_lo[l]);
        put(ph.lane_bits[0]); put(ph.lane_bits[1]);
        for (int w = 0; w < wb; w++) put(ph.warp_bits[w]);
        put(ph.op_begin); put(ph.op_end);
    }
    for (int o = 0; o < sw.nops; o++) {
        const QsvOp &op = sw.ops[o];
        put(op.slot); put(op.variant); put(op.cm_reg); put32(op.cm_thr);
        put(op.kind); put(op.cls0); put(op.cls1); put(op.cm_c); put(op.r00);
    }
    return k;
}

// Streaming form (QSV_JIT_STREAM=1; sw planned by plan_stream): a kernel per sequence of groups, each group
// straight-line code for its ops' slots, variants, kinds, matrix classes and r00; item bits, control masks,
// target bits and matrices are read at run time, so every sweep with the same sequence shares the kernel.
bool stream_form() {
    static const bool on = [] {
        const char *e = std::getenv("QSV_JIT_STREAM");
        return e && std::atoi(e) == 1;
    }();
    return on;
}

std::string stream_key_of(const QsvSweep &sw, int rb, int wb) {
    std::string k;
    auto put = [&](int v) { k.push_back((char)(v & 0xff)); };
    put(sw.kw); put(rb); put(wb); put(sw.swz); put(sw.ngroups); put(sw.nops);
    for (int g = 0; g < sw.ngroups; g++) { put(sw.groups[g].op_begin); put(sw.groups[g].op_end); }
    for (int o = 0; o < sw.nops; o++) {
        const QsvOp &op = sw.ops[o];
        put(op.slot); put(op.variant); put(op.kind); put(op.cls0); put(op.cls1); put(op.r00);
    }
    return k;
}

std::string gen_source_stream(const QsvSweep &sw, int rb, int wb) {
    const int nc = 1 << (5 + wb), nt = nc + 32, minb = sw.kw >= 13 ? 1 : 2;
    std::ostringstream s;
    s << "#include \"qsv_sweep_body.cuh\"\n#include \"qsv_stream.cuh\"\n"
      << "namespace qsv {\nnamespace dev {\nstruct JitBody {\n"
      << "    using Amp = float2;\n"
      << "    static constexpr int kHalfBits = 1;\n"
      << "    static constexpr bool kSmemOps = true;\n"
      << "    template <int NV, int RB, int WB>\n"
      << "    static __device__ __forceinline__ void tile(float2 *tile, const QsvSweep &P, const QsvOp *ops, int lane, int warp,\n"
      << "                                                int bar) {\n"
      << "        const int ctid = warp * 32 + lane;\n";
    for (int g = 0; g < sw.ngroups; g++) {
        const QsvGroup &G = sw.groups[g];
        if (g > 0) s << "        named_bar_sync(bar, " << nc << ");\n";
        s << "        stream_items<" << sw.kw << ", " << nc << ", " << (g > 0 ? "true" : "false") << ", "
          << (g + 1 < sw.ngroups ? "true" : "false") << ">(tile, P.groups[" << g << "], ctid, "
          << (sw.swz ? "true" : "false") << ", [&](float2 (&R)[8], float2 (&I)[8], uint32_t x) {\n";
        for (int o = G.op_begin; o < G.op_end; o++) {
            const QsvOp &op = sw.ops[o];
            if (op.variant == QSV_V_SKIP) continue;
            s << "            stream_op_fixed<true, " << (int)op.slot << ", " << (int)op.variant << ", " << (int)op.kind
              << ", " << (int)op.cls0 << ", " << (int)op.cls1 << ", " << (int)op.r00 << ">(ops + " << o
              << ", R, I, x);\n";
        }
        s << "        });\n";
    }
    s << "    }\n};\n}  // namespace dev\n}  // namespace qsv\n"
      << "extern \"C\" __global__ void __launch_bounds__(" << nt << ", " << minb << ")\n"
      << "    qsv_sweep_jit(float2 *__restrict__ state, const __grid_constant__ QsvSweep P,\n"
      << "                  const __grid_constant__ CUtensorMap tmap, int *status) {\n"
      << "    qsv::dev::sweep_pipeline<" << sw.kw << ", " << rb << ", " << wb << ", " << kStages
      << ", 1, qsv::dev::JitBody, QsvSweep, 0>(state, P, &tmap, status);\n}\n";
    return s.str();
}

// ---------------------------------------------------------------- group-type library
// Sweeps whose exact and coarse structures never repeat (random gate choices, random Toffoli positions)
// still repeat at the level of one group of the streaming form: the op sequence of a group (per op: slot
// among the item bits, variant, kind, matrix classes, r00) recurs across sweeps and circuits. A library
// is ONE kernel for 13-qubit windows with straight-line code for each of its group types and a
// run-time-dispatch path for the others, selected per group; a set of libraries is rebuilt, in the
// background, from the types that have swept the most amplitudes. Item bits, control masks and matrices
// are read at run time.
// A library holds kLibCommon + kLibBand cases: front-end compile time grows faster than linearly with the
// cases (10 / 20 / 40 / 86 cases: 4 / 7 / 17 / ~80 s), so wider coverage comes from several libraries
// compiled in parallel. The 16 / 64 most swept group types cover 87 / 94 % of the groups of a mixed batch.
constexpr int kLibCommon = 16;          // the most swept types, in every library
constexpr int kLibBand = 16;            // then a band of its own
constexpr int kLibSets = 8;             // libraries per build
constexpr double kLibThreshold = 2147483648.0;   // amplitudes swept by groups outside the library before a rebuild
constexpr size_t kLibMaxSeen = 1u << 16;          // group types tracked
constexpr double kLibMinCover = 0.75;             // share of a sweep's ops in library cases to use the kernel

std::string group_key(const QsvSweep &sw, const QsvGroup &g) {
    std::string k;
    for (int o = g.op_begin; o < g.op_end; o++) {
        const QsvOp &op = sw.ops[o];
        const char c[6] = {(char)op.slot, (char)op.variant, (char)op.kind, (char)op.cls0, (char)op.cls1, (char)op.r00};
        k.append(c, 6);
    }
    return k;
}

std::string gen_source_lib(const std::vector<std::string> &types, int rb, int wb) {
    const int nc = 1 << (5 + wb), nt = nc + 32;
    std::ostringstream s;
    s << "#include \"qsv_sweep_body.cuh\"\n#include \"qsv_stream.cuh\"\n"
      << "namespace qsv {\nnamespace dev {\nstruct JitBody {\n"
      << "    using Amp = float2;\n"
      << "    static constexpr int kHalfBits = 1;\n"
      << "    static constexpr bool kSmemOps = true;\n"
      << "    template <int NV, int RB, int WB>\n"
      << "    static __device__ __forceinline__ void tile(float2 *tile, const QsvSweep &P, const QsvOp *ops, int lane, int warp,\n"
      << "                                                int bar) {\n"
      << "        const int ctid = warp * 32 + lane;\n"
      << "        const bool swz = P.swz != 0;\n"
      << "        const int ng = P.ngroups;\n"
      << "        for (int gi = 0; gi < ng; gi++) {\n"
      << "            if (gi > 0) named_bar_sync(bar, " << nc << ");\n"
      << "            const QsvGroup g = P.groups[gi];\n"
      << "            const bool sin = gi > 0, sout = gi + 1 < ng;\n"
      << "            const QsvOp *gops = ops + g.op_begin;\n"
      << "            switch (g.type) {\n";
    for (size_t t = 0; t < types.size(); t++) {
        const std::string &k = types[t];
        s << "            case " << t << ":\n                stream_items_rt<13, " << nc
          << ">(tile, g, ctid, swz, sin, sout, [&](float2 (&R)[8], float2 (&I)[8], uint32_t x) {\n";
        for (size_t o = 0; o * 6 < k.size(); o++) {
            const unsigned char *c = reinterpret_cast<const unsigned char *>(k.data()) + 6 * o;
            if (c[1] == QSV_V_SKIP) continue;
            s << "                    stream_op_fixed<true, " << (int)c[0] << ", " << (int)c[1] << ", " << (int)c[2]
              << ", " << (int)c[3] << ", " << (int)c[4] << ", " << (int)c[5] << ">(gops + " << o << ", R, I, x);\n";
        }
        s << "                });\n                break;\n";
    }
    s << "            default: {\n"
      << "                const int n = g.op_end - g.op_begin;\n"
      << "                stream_items_rt<13, " << nc
      << ">(tile, g, ctid, swz, sin, sout, [&](float2 (&R)[8], float2 (&I)[8], uint32_t x) {\n"
      << "                    for (int o = 0; o < n; o++) stream_op<true>(gops + o, R, I, x);\n"
      << "                });\n                break;\n            }\n"
      << "            }\n        }\n    }\n};\n}  // namespace dev\n}  // namespace qsv\n"
      << "extern \"C\" __global__ void __launch_bounds__(" << nt << ", 1)\n"
      << "    qsv_sweep_jit(float2 *__restrict__ state, const __grid_constant__ QsvSweep P,\n"
      << "                  const __grid_constant__ CUtensorMap tmap, int *status) {\n"
      << "    qsv::dev::sweep_pipeline<13, " << rb << ", " << wb << ", " << kStages
      << ", 1, qsv::dev::JitBody, QsvSweep, 0>(state, P, &tmap, status);\n}\n";
    return s.str();
}

// CUDA source of the kernel specialised to sw's structure
std::string gen_source(const QsvSweep &sw, int rb, int wb) {
    const int groups = groups_for(sw, wb);
    const int nc = 1 << (5 + wb), nt = groups * nc + 32, minb = sw.kw >= 13 ? 1 : 2;
    std::ostringstream s;
    s << "#include \"qsv_sweep_body.cuh\"\n#include \"qsv_jit_ops.cuh\"\n"
      << "namespace qsv {\nnamespace dev {\nstruct JitBody {\n"
      << "    using Amp = float2;\n"
      << "    static constexpr int kHalfBits = 1;\n"
      << "    static constexpr bool kSmemOps = false;\n"
      << "    static constexpr int kPhases = " << sw.nphases << ";\n"
      << "    // one phase of a tile: load in the phase's layout, apply its ops, store\n"
      << "    template <int NV, int RB, int WB>\n"
      << "    static __device__ __forceinline__ void phase(int p, float2 *tile, const QsvSweep &P, const QsvOp *, int lane,\n"
      << "                                                 int warp) {\n"
      << "        switch (p) {\n";
    for (int p = 0; p < sw.nphases; p++) {
        const QsvPhase &ph = sw.phases[p];
        s << "        case " << p << ": {\n            const uint32_t tb = jit_lane_base<" << (int)ph.lane_lo[0] << ", "
          << (int)ph.lane_lo[1] << ", " << (int)ph.lane_lo[2] << ", " << (int)ph.lane_bits[0] << ", "
          << (int)ph.lane_bits[1] << ">(lane)";
        for (int w = 0; w < wb; w++) s << " | jit_warp_bit<" << (int)ph.warp_bits[w] << ">(warp, " << w << ")";
        s << ";\n            float2 R[NV], I[NV];\n";
        std::string rbits;
        for (int r = 0; r < rb; r++) rbits += (r ? ", " : "") + std::to_string((int)ph.reg_bits[r]);
        s << "            jit_load<NV, " << (int)sw.swz << ", " << (p > 0 ? 1 : 0) << ", " << rbits
          << ">(tile, tb, R, I);\n";
        for (int o = ph.op_begin; o < ph.op_end; o++) {
            const QsvOp &op = sw.ops[o];
            const std::string thr = std::to_string(op.cm_thr) + "u";
            // m00-real dense ops take the QSV_M_DENSE_R0 / QSV_V_UNI_DENSE_R0 code paths
            const bool r0 = op.r00 && op.kind == QSV_K_UNI;
            const int cls0 = r0 ? QSV_M_DENSE_R0 : op.cls0;
            const int var = (r0 && op.variant == QSV_V_UNI_DENSE) ? QSV_V_UNI_DENSE_R0 : op.variant;
            const std::string cls = std::to_string((int)op.kind) + ", " + std::to_string(cls0) + ", " +
                                    std::to_string((int)op.cls1) + ", ";
            const std::string ctl = std::to_string((int)op.cm_reg) + ", " + thr;
            const std::string mux = std::to_string((int)op.kind) + ", " + std::to_string((int)op.cls1) + ", " +
                                    std::to_string((int)op.cm_c) + ", " + ctl;
            if (op.slot == QSV_SLOT_COMP)
                s << "            jit_comp<NV, " << cls << ctl << ">(R, I, P.ops[" << o << "], tb);\n";
            else if (op.slot < QSV_SLOT_LANE0 && op.variant == QSV_V_MUX)
                s << "            jit_reg_mux<NV, " << (op.slot - QSV_SLOT_REG0) << ", " << mux << ">(R, I, P.ops[" << o
                  << "], tb);\n";
            else if (op.slot < QSV_SLOT_LANE0 && coef_major() &&
                     (var == QSV_V_UNI_DENSE || var == QSV_V_UNI_DENSE_R0))
                s << "            jit_reg_cm<NV, " << (op.slot - QSV_SLOT_REG0) << ", " << var << ">(R, I, P.ops[" << o
                  << "]);\n";
            else if (op.slot < QSV_SLOT_LANE0)
                s << "            jit_reg<NV, " << (op.slot - QSV_SLOT_REG0) << ", " << var << ", " << ctl
                  << ">(R, I, P.ops[" << o << "], tb);\n";
            else if (op.variant == QSV_V_MUX)
                s << "            jit_lane_mux<NV, " << (op.slot - QSV_SLOT_LANE0) << ", " << mux << ">(R, I, P.ops["
                  << o << "], tb, lane);\n";
            else
                s << "            jit_lane<NV, " << (op.slot - QSV_SLOT_LANE0) << ", " << (int)op.variant << ", " << ctl
                  << ">(R, I, P.ops[" << o << "], tb, lane);\n";
        }
        s << "            jit_store<NV, " << (int)sw.swz << ", " << (p + 1 < sw.nphases ? 1 : 0) << ", " << rbits
          << ">(tile, tb, R, I);\n            break;\n        }\n";
    }
    s << "        default: break;\n        }\n    }\n"
      << "    template <int NV, int RB, int WB>\n"
      << "    static __device__ __forceinline__ void tile(float2 *tile, const QsvSweep &P, const QsvOp *ops, int lane, int warp,\n"
      << "                                                int bar) {\n"
      << "#pragma unroll\n"
      << "        for (int p = 0; p < kPhases; p++) {\n"
      << "            if (p > 0) named_bar_sync(bar, " << nc << ");\n"
      << "            phase<NV, RB, WB>(p, tile, P, ops, lane, warp);\n"
      << "        }\n    }\n";
    s << "};\n}  // namespace dev\n}  // namespace qsv\n"
      << "extern \"C\" __global__ void __launch_bounds__(" << nt << ", " << minb << ")\n"
      << "    qsv_sweep_jit(float2 *__restrict__ state, const __grid_constant__ QsvSweep P,\n"
      << "                  const __grid_constant__ CUtensorMap tmap, int *status) {\n"
      << "    qsv::dev::sweep_pipeline<" << sw.kw << ", " << rb << ", " << wb << ", " << kStages << ", " << groups
      << ", qsv::dev::JitBody, QsvSweep, " << interleave_for(sw, groups) << ">(state, P, &tmap, status);\n}\n";
    return s.str();
}

bool nvrtc_compile(const std::string &src, std::vector<char> &cubin, std::string &log) {
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "qsv_sweep_jit.cu", kJitNumHeaders, kJitHeaderSources,
                           kJitHeaderNames) != NVRTC_SUCCESS) {
        log = "nvrtcCreateProgram failed";
        return false;
    }
    // QSV_JIT_PTXAS_VERBOSE=1 keeps ptxas's resource report (registers, spills) in the compile log;
    // QSV_JIT_EXTRA_OPTS adds NVRTC options (space separated), for compile-time / code-quality studies
    std::vector<std::string> extra;
    if (const char *x = std::getenv("QSV_JIT_EXTRA_OPTS")) {
        std::istringstream is(x);
        for (std::string o; is >> o;) extra.push_back(o);
    }
    std::vector<const char *> opts = {"--gpu-architecture=sm_100a", "-std=c++17", "-DQSV_JIT=1"};
    if (std::getenv("QSV_JIT_PTXAS_VERBOSE")) opts.push_back("--ptxas-options=-v");
    for (const std::string &o : extra) opts.push_back(o.c_str());
    const nvrtcResult r = nvrtcCompileProgram(prog, (int)opts.size(), opts.data());
    size_t ls = 0;
    nvrtcGetProgramLogSize(prog, &ls);
    log.assign(ls, '\0');
    if (ls) nvrtcGetProgramLog(prog, &log[0]);
    while (!log.empty() && log.back() == '\0') log.pop_back();   // the size counts the terminator
    bool ok = r == NVRTC_SUCCESS;
    if (ok) {
        size_t n = 0;
        ok = nvrtcGetCUBINSize(prog, &n) == NVRTC_SUCCESS && n > 0;
        if (ok) {
            cubin.resize(n);
            ok = nvrtcGetCUBIN(prog, cubin.data()) == NVRTC_SUCCESS;
        }
    } else {
        log = std::string(nvrtcGetErrorString(r)) + ": " + log;
    }
    nvrtcDestroyProgram(&prog);
    return ok;
}

void worker() {
    Jit &j = J();
    std::unique_lock<std::mutex> lk(j.mu);
    for (;;) {
        j.work.wait(lk, [&] { return j.stopping || !j.queue.empty(); });
        if (j.stopping) {
            // park for good: a thread that exits during process teardown runs its thread-local destructors
            // after the libraries it used may be gone
            j.work.wait(lk, [] { return false; });
        }
        std::shared_ptr<Entry> e = j.queue.front();
        j.queue.pop_front();
        j.busy++;
        const std::string src = e->src;
        lk.unlock();
        // QSV_JIT_DUMP_DIR (tuning): write each generated source there before compiling it
        if (const char *dir = std::getenv("QSV_JIT_DUMP_DIR")) {
            const std::string path = std::string(dir) + "/qsv_jit_" + std::to_string(std::hash<std::string>()(src)) + ".cu";
            if (FILE *f = std::fopen(path.c_str(), "w")) {
                std::fwrite(src.data(), 1, src.size(), f);
                std::fclose(f);
            }
        }
        std::vector<char> cubin;
        std::string log;
        const auto t0 = std::chrono::steady_clock::now();
        const bool ok = nvrtc_compile(src, cubin, log);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        lk.lock();
        e->cubin = std::move(cubin);
        e->log = log;
        e->state = ok ? kReady : kFailed;
        if (ok) j.compiled++;
        else j.failed++;
        if (!ok) j.last_log = log;
        else if (std::getenv("QSV_JIT_PTXAS_VERBOSE") && j.last_log.size() < (1u << 20)) j.last_log += log;  // all reports
        j.compile_ms += ms;
        j.busy--;
        j.done.notify_all();
    }
}

// Drop queued compilations and wait (up to 60 s) for running ones; with j.mu held by lk.
void drain(Jit &j, std::unique_lock<std::mutex> &lk) {
    for (auto &e : j.queue) e->state = kNew;
    j.queue.clear();
    j.done.notify_all();
    j.done.wait_for(lk, std::chrono::seconds(60), [&] { return j.busy == 0; });
}

// Process exit with a compilation in flight would tear NVRTC down under a running compile. This handler
// drops the queue and waits for running compilations to finish. It is registered after a first (tiny)
// compilation has loaded NVRTC's run-time parts, so that it runs before their teardown (exit handlers
// run in reverse order of registration).
void stop_workers_at_exit() {
    Jit &j = J();
    std::unique_lock<std::mutex> lk(j.mu);
    j.stopping = true;
    j.work.notify_all();
    drain(j, lk);
}

void warm_up_nvrtc() {
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, "extern \"C\" __global__ void qsv_warm_up() {}\n", "warm_up.cu", 0, nullptr,
                           nullptr) != NVRTC_SUCCESS)
        return;
    const char *opts[] = {"--gpu-architecture=sm_100a", "-std=c++17"};
    nvrtcCompileProgram(prog, 2, opts);
    nvrtcDestroyProgram(&prog);
}

// with j.mu held: queue e for compilation (starts the compile threads on first use)
void enqueue_src(Jit &j, const std::shared_ptr<Entry> &e) {
    if (e->state != kNew) return;
    e->state = kQueued;
    j.queue.push_back(e);
    if (j.stopping) {
        e->state = kNew;
        j.queue.pop_back();
        return;
    }
    if (j.threads == 0) {
        warm_up_nvrtc();
        std::atexit(stop_workers_at_exit);
        const unsigned hw = std::thread::hardware_concurrency();
        const int n = std::max(1, std::min(8, (int)(hw ? hw / 2 : 2)));
        for (int i = 0; i < n; i++) std::thread(worker).detach();
        j.threads = n;
    }
    j.work.notify_one();
}

void enqueue(Jit &j, const std::shared_ptr<Entry> &e, const QsvSweep &sw) {
    if (e->state != kNew) return;
    e->src = e->stream ? gen_source_stream(sw, e->rb, e->wb) : gen_source(sw, e->rb, e->wb);
    enqueue_src(j, e);
}

// with j.mu held: adopt a finished build (the libraries of it that compiled), forget a dropped one
void lib_poll(Jit &j) {
    if (!j.lib_next) return;
    for (auto &L : j.lib_next->libs)
        if (L->entry->state == kQueued) return;               // still compiling
    auto done = std::make_shared<LibSet>();
    for (auto &L : j.lib_next->libs)
        if (L->entry->state == kReady) done->libs.push_back(L);
    if (!done->libs.empty()) {
        std::unordered_map<std::string, int> all;
        for (auto &L : done->libs)
            for (auto &k : L->types) all.emplace(k, 0);
        done->types = (int)all.size();
        j.lib = done;
    }
    j.lib_next = nullptr;
}

bool lib_building(Jit &j) {
    if (!j.lib_next) return false;
    for (auto &L : j.lib_next->libs)
        if (L->entry->state == kQueued) return true;
    return false;
}

// with j.mu held: queue a build. The group types are ranked by swept amplitudes, `must` (the types of the
// sweeps at hand) first; the kLibCommon first ones go into every library, each library adds its own band of
// the next kLibBand, up to kLibSets libraries compiled in parallel (a sweep takes the one that covers most
// of its ops, so its common groups and one rarer group are covered together).
void lib_build(Jit &j, int rb, int wb, const std::vector<std::string> &must) {
    std::vector<std::string> ranked;
    std::unordered_map<std::string, int> seen;
    auto by_weight = [](std::vector<std::pair<double, const std::string *>> &v) {
        std::sort(v.begin(), v.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
    };
    auto add = [&](const std::string &k) {
        if (!seen.count(k)) { seen.emplace(k, 0); ranked.push_back(k); }
    };
    std::vector<std::pair<double, const std::string *>> m, v;
    for (const std::string &k : must) {
        auto it = j.gweight.find(k);
        m.push_back({it != j.gweight.end() ? it->second : 0.0, &k});
    }
    by_weight(m);
    for (auto &p : m) add(*p.second);
    v.reserve(j.gweight.size());
    for (auto &kv : j.gweight) v.push_back({kv.second, &kv.first});
    by_weight(v);
    for (auto &p : v) add(*p.second);
    auto set = std::make_shared<LibSet>();
    const size_t common = std::min(ranked.size(), (size_t)kLibCommon);
    for (int b = 0; b < kLibSets; b++) {
        const size_t lo = common + (size_t)b * kLibBand;
        if (b > 0 && lo >= ranked.size()) break;
        auto L = std::make_shared<Lib>();
        L->rb = rb;
        L->wb = wb;
        auto put = [&](const std::string &k) {
            if (!L->index.count(k)) { L->index.emplace(k, (int)L->types.size()); L->types.push_back(k); }
        };
        for (size_t i = 0; i < common; i++) put(ranked[i]);
        for (size_t i = lo; i < std::min(ranked.size(), lo + kLibBand); i++) put(ranked[i]);
        L->entry = std::make_shared<Entry>();
        L->entry->kw = 13;
        L->entry->rb = rb;
        L->entry->wb = wb;
        L->entry->groups = 1;
        L->entry->stream = true;
        L->entry->src = gen_source_lib(L->types, rb, wb);
        set->libs.push_back(L);
    }
    j.lib_next = set;
    for (auto &L : set->libs) enqueue_src(j, L->entry);
}

// with j.mu held: wait (j.done) until the build in progress has finished, then adopt it
void lib_wait(Jit &j, std::unique_lock<std::mutex> &lk) {
    j.done.wait(lk, [&] { return !lib_building(j); });
    lib_poll(j);
}

// with j.mu held: give s2's groups their cases in the library (of those in use) that covers most of its ops
// (type -1: run-time dispatch) and, with work > 0, add work to each group type's swept amplitudes (and the
// uncovered share to lib_uncovered). Returns the share of the sweep's ops in that library's cases (*best:
// the library, or null); keys (if given) receives the group types.
double lib_annotate(Jit &j, QsvSweep &s2, double work, std::vector<std::string> *keys, const Lib **best) {
    std::string k[QSV_MAX_GROUPS];
    int n[QSV_MAX_GROUPS], total = 0;
    for (int g = 0; g < s2.ngroups; g++) {
        const QsvGroup &G = s2.groups[g];
        k[g] = group_key(s2, G);
        n[g] = 0;
        for (int o = G.op_begin; o < G.op_end; o++) n[g] += s2.ops[o].variant != QSV_V_SKIP;
        total += n[g];
        if (work > 0) {
            auto it = j.gweight.find(k[g]);
            if (it != j.gweight.end()) it->second += work;
            else if (j.gweight.size() < kLibMaxSeen) j.gweight.emplace(k[g], work);
        }
        if (keys) keys->push_back(k[g]);
    }
    // the streaming form does not depend on the phase layouts: any library serves any 13-qubit sweep
    const Lib *L = nullptr;
    int covered = 0;
    if (j.lib) {
        for (auto &C : j.lib->libs) {
            int c = 0;
            for (int g = 0; g < s2.ngroups; g++) c += C->index.count(k[g]) ? n[g] : 0;
            if (!L || c > covered) { L = C.get(); covered = c; }
        }
    }
    for (int g = 0; g < s2.ngroups; g++) {
        int idx = -1;
        if (L) {
            auto f = L->index.find(k[g]);
            if (f != L->index.end()) idx = f->second;
        }
        s2.groups[g].type = (int16_t)idx;
    }
    if (best) *best = L;
    const double cover = total ? (double)covered / (double)total : 1.0;
    if (work > 0) j.lib_uncovered += work * (1.0 - cover);
    return cover;
}

std::shared_ptr<Entry> find_or_add(Jit &j, const QsvSweep &sw, int rb, int wb, bool coarse = false,
                                   bool stream = false) {
    const std::string key = stream ? "S" + stream_key_of(sw, rb, wb) : (coarse ? "C" : "E") + key_of(sw, rb, wb);
    auto it = j.map.find(key);
    if (it != j.map.end()) return it->second;
    if (j.map.size() >= kMaxEntries) {
        // a long-running process that meets many one-off structures: drop the ones that were never queued
        // (their work counts restart); queued, compiled and failed ones stay
        for (auto m = j.map.begin(); m != j.map.end();) {
            if (m->second->state == kNew && m->second.use_count() == 1) m = j.map.erase(m);
            else ++m;
        }
    }
    auto e = std::make_shared<Entry>();
    e->kw = sw.kw;
    e->rb = rb;
    e->wb = wb;
    e->groups = stream ? 1 : groups_for(sw, wb);
    e->coarse = coarse;
    e->stream = stream;
    j.map.emplace(key, e);
    return e;
}

}  // namespace

int jit_set_mode(int mode) {
    if (mode < 0 || mode > 4) return -1;
    Jit &j = J();
    std::unique_lock<std::mutex> lk(j.mu);
    const int old = j.mode;
    j.mode = mode;
    if (mode == 0) drain(j, lk);       // interpreter only: queued compilations are dropped
    return old;
}

// Compile (in parallel, blocking) every structure of the given sweeps that is not compiled yet.
// Returns the number of those structures whose kernel is ready.
int jit_prepare(const std::vector<QsvSweep> &sweeps) {
    Jit &j = J();
    std::unique_lock<std::mutex> lk(j.mu);
    std::vector<std::shared_ptr<Entry>> mine;
    if (j.mode == 4 && !stream_form()) {
        // group-type libraries: one build (blocking) from the group types of the 13-qubit sweeps (the most
        // swept 144 of them, these first)
        int rb = 0, wb = 0;
        layout_for_kw(13, &rb, &wb);
        std::vector<QsvSweep> s13;
        std::vector<std::string> keys;
        bool all = true;
        for (const QsvSweep &sw : sweeps) {
            if (sw.kw != 13) continue;
            s13.push_back(sw);
            std::string err;
            if (plan_stream(s13.back(), err) != QSV_OK) { s13.pop_back(); continue; }
            const double work = (double)sw.ntiles * (double)(1 << sw.kw);
            all = lib_annotate(j, s13.back(), work, &keys, nullptr) >= 1.0 && all;
        }
        if (!all) {
            lib_wait(j, lk);
            lib_build(j, rb, wb, keys);
            lib_wait(j, lk);
        }
        int ready = 0;
        for (QsvSweep &s2 : s13) ready += lib_annotate(j, s2, 0.0, nullptr, nullptr) >= 1.0;
        return ready;
    }
    for (const QsvSweep &sw : sweeps) {
        int rb = 0, wb = 0;
        if (layout_for_kw(sw.kw, &rb, &wb)) continue;
        if (stream_form()) {
            QsvSweep s2 = sw;
            std::string err;
            if (plan_stream(s2, err) != QSV_OK) continue;
            auto e = find_or_add(j, s2, rb, wb, false, true);
            enqueue(j, e, s2);
            mine.push_back(e);
            continue;
        }
        if (j.mode == 3) {
            const QsvSweep c = coarse_of(sw);
            auto e = find_or_add(j, c, rb, wb, true);
            enqueue(j, e, c);
            mine.push_back(e);
            continue;
        }
        auto e = find_or_add(j, sw, rb, wb);
        enqueue(j, e, sw);
        mine.push_back(e);
    }
    j.done.wait(lk, [&] {
        for (auto &e : mine)
            if (e->state == kQueued) return false;
        return true;
    });
    int ready = 0;
    for (auto &e : mine) ready += e->state == kReady;
    return ready;
}

// Build (blocking) a group-type library from the 13-qubit sweeps of many programs: their group types'
// swept amplitudes are recorded and the libraries take the most swept of every type seen so far (lib_build).
// Returns the number of distinct types in the libraries in use, or -1 if a library failed to compile.
int jit_prepare_library(const std::vector<QsvSweep> &sweeps) {
    Jit &j = J();
    std::unique_lock<std::mutex> lk(j.mu);
    int rb = 0, wb = 0;
    layout_for_kw(13, &rb, &wb);
    QsvSweep s2;
    for (const QsvSweep &sw : sweeps) {
        if (sw.kw != 13) continue;
        std::memcpy(&s2, &sw, sizeof(QsvSweep));
        std::string err;
        if (plan_stream(s2, err) != QSV_OK) continue;
        lib_annotate(j, s2, (double)sw.ntiles * (double)(1 << sw.kw), nullptr, nullptr);
    }
    lib_wait(j, lk);
    lib_build(j, rb, wb, {});
    const std::shared_ptr<LibSet> built = j.lib_next;
    lib_wait(j, lk);
    j.lib_uncovered = 0.0;
    for (auto &L : built->libs)
        if (L->entry->state != kReady) return -1;
    return j.lib ? j.lib->types : 0;
}

void jit_wait() {
    Jit &j = J();
    std::unique_lock<std::mutex> lk(j.mu);
    j.done.wait(lk, [&] { return (j.queue.empty() && j.busy == 0) || j.stopping; });
}

// stats: mode, structures, ready, failed, launches specialised (exact or coarse), launches interpreted,
// compile ms, queued, launches of coarse kernels, coarse structures
int jit_info(long long *out, int cap) {
    Jit &j = J();
    std::lock_guard<std::mutex> lk(j.mu);
    long long ready = 0, coarse = 0;
    for (auto &kv : j.map) {
        ready += kv.second->state == kReady;
        coarse += kv.second->coarse;
    }
    lib_poll(j);
    const long long v[12] = {j.mode, (long long)j.map.size(), ready, j.failed, j.jit_launches, j.interp_launches,
                             (long long)j.compile_ms, (long long)(j.queue.size() + j.busy), j.coarse_launches,
                             coarse, j.lib_launches, j.lib ? (long long)j.lib->types : 0};
    const int n = std::min(cap, 12);
    for (int i = 0; i < n; i++) out[i] = v[i];
    return 12;
}

std::string jit_last_log() {
    Jit &j = J();
    std::lock_guard<std::mutex> lk(j.mu);
    return j.last_log;
}

// Launch sw with its specialised kernel if that kernel is ready (compiling it first in eager mode).
// Returns 1 if launched, 0 if the caller should run the interpreter, -1 on a CUDA error (*err set).
int jit_try_launch(float2 *state, const QsvSweep &sw_in, int nsm, cudaStream_t stream, cudaError_t *err) {
    Jit &j = J();
    int rb = 0, wb = 0;
    if (layout_for_kw(sw_in.kw, &rb, &wb)) return 0;
    // streaming form: the kernel runs the sweep re-planned into groups
    thread_local QsvSweep s2;
    const bool sf = stream_form();
    if (sf) {
        std::memcpy(&s2, &sw_in, sizeof(QsvSweep));
        std::string perr;
        if (plan_stream(s2, perr) != QSV_OK) return 0;
    }
    const QsvSweep &sw = sf ? s2 : sw_in;
    thread_local QsvSweep sl;          // the sweep in streaming form for the group-type library
    const QsvSweep *lp = &sw;          // what the kernel runs
    const Drv &d = drv();
    std::shared_ptr<Entry> e;
    {
        std::unique_lock<std::mutex> lk(j.mu);
        if (j.mode == 0 || !d.ok) { j.interp_launches++; return 0; }
        const double work = (double)sw.ntiles * (double)(1 << sw.kw);
        if ((j.mode != 3 && j.mode != 4) || sf) {
            e = find_or_add(j, sw, rb, wb, false, sf);
            e->uses++;
            e->work += work;
            if (e->state == kNew &&
                (j.mode == 1 || (e->work >= kWorkThreshold && j.queue.size() < kMaxQueued)))
                enqueue(j, e, sw);
            if (j.mode == 1) j.done.wait(lk, [&] { return e->state != kQueued; });
        }
        if (!sf && (!e || e->state != kReady) && (j.mode == 2 || j.mode == 3)) {
            // the kernel of the sweep's coarse structure, shared with every sweep of that structure
            const QsvSweep c = coarse_of(sw);
            std::shared_ptr<Entry> ce = find_or_add(j, c, rb, wb, true);
            ce->uses++;
            ce->work += work;
            if (ce->state == kNew &&
                (j.mode == 3 || (ce->work >= kCoarseThreshold && j.queue.size() < kMaxQueued)))
                enqueue(j, ce, c);
            if (j.mode == 3) j.done.wait(lk, [&] { return ce->state != kQueued; });
            if (ce->state == kReady) e = ce;
        }
        if ((!e || e->state != kReady) && !sf && sw.kw == 13 && (j.mode == 2 || j.mode == 4)) {
            // the group-type library, with this sweep's groups annotated with their cases
            lib_poll(j);
            std::memcpy(&sl, &sw, sizeof(QsvSweep));
            std::string perr;
            if (plan_stream(sl, perr) == QSV_OK) {
                const Lib *best = nullptr;
                const double cover = lib_annotate(j, sl, work, nullptr, &best);
                if (j.lib_uncovered >= kLibThreshold && !j.lib_next && j.queue.size() < kMaxQueued) {
                    lib_build(j, rb, wb, {});
                    j.lib_uncovered = 0.0;
                }
                if (best && best->entry->state == kReady && cover >= kLibMinCover) {
                    e = best->entry;
                    lp = &sl;
                }
            }
        }
        if (!e || e->state != kReady) { j.interp_launches++; return 0; }
    }
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess || dev < 0 || dev >= kMaxDevices) { *err = ce != cudaSuccess ? ce : cudaErrorInvalidDevice; return -1; }
    // the block the kernel was compiled for (a library kernel keeps the layout it was built with)
    const int NT = e->groups * (1 << (5 + e->wb)) + 32;
    // sweep_smem_bytes of the generated body: the tile buffers plus 1 KiB for their 1024-byte alignment
    const size_t smem = ((size_t)kStages << sw.kw) * sizeof(float2) + QSV_SMEM_ALIGN +
                        (e->stream ? sizeof(QsvOp) * QSV_MAX_SWEEP_OPS : 0);
    if (!e->fn[dev]) {
        // loading a module is not a stream operation: keep it out of stream captures
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
            cudaGetLastError();
            std::lock_guard<std::mutex> lk(j.mu);
            j.interp_launches++;
            return 0;
        }
        ce = cudaSetDevice(dev);      // makes the device's primary context current on this thread
        if (ce != cudaSuccess) { *err = ce; return -1; }
        CUmodule mod = nullptr;
        CUfunction fn = nullptr;
        int per_sm = 0;
        if (d.module_load(&mod, e->cubin.data()) != CUDA_SUCCESS ||
            d.get_function(&fn, mod, "qsv_sweep_jit") != CUDA_SUCCESS ||
            d.set_attribute(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, (int)smem) != CUDA_SUCCESS ||
            d.occupancy(&per_sm, fn, NT, smem) != CUDA_SUCCESS) {
            *err = cudaErrorInvalidKernelImage;
            return -1;
        }
        std::lock_guard<std::mutex> lk(j.mu);
        e->per_sm[dev] = per_sm < 1 ? 1 : per_sm;
        e->fn[dev] = fn;
    }
    alignas(64) CUtensorMap map;
    ce = dev::make_tmap(&map, state, *lp);
    if (ce != cudaSuccess) { *err = ce; return -1; }
    int *status = nullptr;
    ce = status_word_ptr(&status);
    if (ce != cudaSuccess) { *err = ce; return -1; }
    int64_t grid = (int64_t)nsm * e->per_sm[dev];
    if (grid > sw.ntiles) grid = sw.ntiles;
    void *args[] = {&state, const_cast<QsvSweep *>(lp), &map, &status};
    if (d.launch(e->fn[dev], (unsigned)grid, 1, 1, (unsigned)NT, 1, 1, (unsigned)smem, (CUstream)stream, args,
                 nullptr) != CUDA_SUCCESS) {
        *err = cudaErrorLaunchFailure;
        return -1;
    }
    std::lock_guard<std::mutex> lk(j.mu);
    if (lp == &sl) j.lib_launches++;
    else j.jit_launches++;
    if (e->coarse) j.coarse_launches++;
    return 1;
}

}  // namespace qsv
