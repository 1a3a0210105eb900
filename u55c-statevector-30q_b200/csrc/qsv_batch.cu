// qsv_batch.cu -- whole-circuit batch kernel: many small circuits per persistent launch (sm_100a).
//
// No reference counterpart: the reference runs one circuit per launch and names batching as future work.
// A circuit of n <= 13 qubits is one 2^n-amplitude tile, so its entire program (every op of every pass of
// every segment, in order) runs inside one CTA's shared memory: one HBM read and one HBM write per
// circuit instead of one per pass. The kernel is the sweep kernel's pipeline with circuits in place of
// tiles: a producer warp streams circuit states in and out with bulk-async copies (three in flight), the
// consumer warps run each circuit's phases with the shared op code (qsv_ops.cuh). The per-circuit programs
// (phases and ops) live in a caller-provided device workspace, uploaded once and replayable (the launch is
// capturable in a CUDA graph).
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "../../include/qsv_b200.h"
#include "qsv_device.cuh"
#include "qsv_ops.cuh"
#include "qsv_planner.h"

namespace qsv {

struct BatchItem {
    float2 *state;
    int32_t ph_begin, ph_end;   // phase range in the batch's phase table
};

namespace dev {

template <int KW, int RB, int WB, int S>
__global__ void __launch_bounds__((1 << (5 + WB)) + 32, (KW >= 13 ? 1 : 2))
    batch_kernel(const BatchItem *__restrict__ items, int nitems, const QsvPhaseX *__restrict__ phases,
                 const QsvOp *__restrict__ ops, int *status) {
    constexpr int NC = 1 << (5 + WB);
    constexpr int NV = 1 << RB;
    constexpr int TILE = 1 << KW;
    static_assert(1 + 3 + 2 + RB + WB == KW, "layout must cover the window");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    float2 *bufs = reinterpret_cast<float2 *>(smem_raw);
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t done[S];
    __shared__ volatile int abort_flag;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&done[s], NC);
        }
        abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();
    const int64_t first = blockIdx.x, stride = gridDim.x;
    const int64_t nmine = first < nitems ? (nitems - 1 - first) / stride + 1 : 0;

    if (tid >= NC) {
        if ((tid & 31) != 0) return;          // one producer thread: one bulk copy per circuit
        auto load = [&](int64_t j, int b) {
            const BatchItem &it = items[first + j * stride];
            mbar_arrive_expect_tx(&full[b], (uint32_t)TILE * 8u);
            bulk_g2s(bufs + (size_t)b * TILE, it.state, (uint32_t)TILE * 8u, &full[b]);
        };
        for (int64_t j = 0; j < S && j < nmine; j++) load(j, (int)j);
        for (int64_t j = 0; j < nmine; j++) {
            const int b = (int)(j % S);
            if (!mbar_wait(&done[b], (uint32_t)((j / S) & 1), &abort_flag, status)) break;
            bulk_s2g(items[first + j * stride].state, bufs + (size_t)b * TILE, (uint32_t)TILE * 8u);
            bulk_commit();
            if (j + S < nmine) {
                bulk_wait_read_all();
                load(j + S, b);
            }
        }
        bulk_wait_all();
        return;
    }
    const int lane = tid & 31, warp = tid >> 5;
    for (int64_t j = 0; j < nmine; j++) {
        const int b = (int)(j % S);
        if (!mbar_wait(&full[b], (uint32_t)((j / S) & 1), &abort_flag, status)) break;
        float2 *tile = bufs + (size_t)b * TILE;
        const BatchItem &it = items[first + j * stride];
        for (int ph = it.ph_begin; ph < it.ph_end; ph++) {
            if (ph > it.ph_begin) named_bar_sync(1, NC);
            const QsvPhaseX &Q = phases[ph];
            run_phase<NV, RB, WB>(tile, Q, ops, Q.op_begin, Q.op_end, lane, warp, false, ph > it.ph_begin,
                                  ph + 1 < it.ph_end);
        }
        fence_proxy_async_smem();
        mbar_arrive(&done[b]);
    }
}

template <int KW, int RB, int WB, int S>
static cudaError_t launch_batch_t(const BatchItem *items, int nitems, const QsvPhaseX *phases, const QsvOp *ops,
                                  int *status, int nsm, cudaStream_t stream) {
    constexpr int NT = (1 << (5 + WB)) + 32;
    const size_t smem = ((size_t)S << KW) * sizeof(float2);
    static int configured_dev = -1;
    static int per_sm = 1;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (configured_dev != dev) {
        e = cudaFuncSetAttribute(batch_kernel<KW, RB, WB, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel<KW, RB, WB, S>, NT, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        configured_dev = dev;
    }
    int64_t grid = (int64_t)nsm * per_sm;
    if (grid > nitems) grid = nitems;
    batch_kernel<KW, RB, WB, S><<<(unsigned)grid, NT, smem, stream>>>(items, nitems, phases, ops, status);
    return cudaGetLastError();
}

}  // namespace dev

cudaError_t status_word_ptr(int **out);

// ---------------------------------------------------------------- host batch object
struct Batch {
    struct Circ {
        float2 *state;
        int n;
        int32_t ph_begin, ph_end;
    };
    std::vector<Circ> circs;
    std::vector<QsvPhaseX> phases;
    std::vector<QsvOp> ops;
    // finalized layout (items grouped by n, then phases, then ops, in the device workspace)
    std::vector<BatchItem> items;
    int group_off[QSV_KW_MAX + 1] = {0}, group_cnt[QSV_KW_MAX + 1] = {0};
    size_t off_phases = 0, off_ops = 0, bytes = 0;
    bool finalized = false;
    int rb13 = 0;               // register bits of the 13-qubit layout the circuits were planned with
};

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int batch_add(Batch *b, void *state, int n, int nseg, const int32_t *const *segs, const size_t *nwords,
              std::string &err) {
    if (n < 10 || n > QSV_KW_MAX) { err = "batch circuits must have 10..13 qubits"; return QSV_ERR_INVALID_ARG; }
    std::vector<PhysPass> all, one;
    for (int s = 0; s < nseg; s++) {
        int rc = decode_segment(segs[s], nwords[s], n, one, err);
        if (rc) return rc;
        all.insert(all.end(), one.begin(), one.end());
    }
    if (n == 13) {
        int rb = 4, wb = 3;
        layout_for_kw(13, &rb, &wb);
        if (b->rb13 && b->rb13 != rb) { err = "13-qubit layout changed while building the batch"; return QSV_ERR_INVALID_ARG; }
        b->rb13 = rb;
    }
    std::vector<QsvOp> ops;
    std::vector<QsvPhaseX> phases;
    int rc = plan_whole_state(all, n, ops, phases, err);
    if (rc) return rc;
    const int32_t op_base = (int32_t)b->ops.size();
    for (QsvPhaseX &p : phases) { p.op_begin += op_base; p.op_end += op_base; }
    Batch::Circ c;
    c.state = static_cast<float2 *>(state);
    c.n = n;
    c.ph_begin = (int32_t)b->phases.size();
    c.ph_end = c.ph_begin + (int32_t)phases.size();
    b->phases.insert(b->phases.end(), phases.begin(), phases.end());
    b->ops.insert(b->ops.end(), ops.begin(), ops.end());
    b->circs.push_back(c);
    b->finalized = false;
    return QSV_OK;
}

static void batch_finalize(Batch *b) {
    if (b->finalized) return;
    b->items.clear();
    for (int n = 0; n <= QSV_KW_MAX; n++) { b->group_off[n] = 0; b->group_cnt[n] = 0; }
    for (int n = 10; n <= QSV_KW_MAX; n++) {
        b->group_off[n] = (int)b->items.size();
        for (const Batch::Circ &c : b->circs)
            if (c.n == n) b->items.push_back(BatchItem{c.state, c.ph_begin, c.ph_end});
        b->group_cnt[n] = (int)b->items.size() - b->group_off[n];
    }
    b->off_phases = align_up(b->items.size() * sizeof(BatchItem), 256);
    b->off_ops = align_up(b->off_phases + b->phases.size() * sizeof(QsvPhaseX), 256);
    b->bytes = align_up(b->off_ops + b->ops.size() * sizeof(QsvOp), 256);
    b->finalized = true;
}

size_t batch_workspace_bytes(Batch *b) {
    batch_finalize(b);
    return b->bytes;
}

cudaError_t batch_upload(Batch *b, void *ws, cudaStream_t stream) {
    batch_finalize(b);
    char *base = static_cast<char *>(ws);
    cudaError_t e = cudaSuccess;
    if (!b->items.empty())
        e = cudaMemcpyAsync(base, b->items.data(), b->items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && !b->phases.empty())
        e = cudaMemcpyAsync(base + b->off_phases, b->phases.data(), b->phases.size() * sizeof(QsvPhaseX),
                            cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && !b->ops.empty())
        e = cudaMemcpyAsync(base + b->off_ops, b->ops.data(), b->ops.size() * sizeof(QsvOp), cudaMemcpyHostToDevice,
                            stream);
    return e;
}

cudaError_t batch_launch(Batch *b, void *ws, int nsm, cudaStream_t stream, int *launches) {
    batch_finalize(b);
    char *base = static_cast<char *>(ws);
    const BatchItem *items = reinterpret_cast<const BatchItem *>(base);
    const QsvPhaseX *phases = reinterpret_cast<const QsvPhaseX *>(base + b->off_phases);
    const QsvOp *ops = reinterpret_cast<const QsvOp *>(base + b->off_ops);
    int *status = nullptr;
    cudaError_t e = status_word_ptr(&status);
    if (e != cudaSuccess) return e;
    *launches = 0;
    for (int n = 10; n <= QSV_KW_MAX; n++) {
        const int cnt = b->group_cnt[n];
        if (!cnt) continue;
        const BatchItem *it = items + b->group_off[n];
        const int rb = b->rb13 ? b->rb13 : 4;
        switch (n) {
            case 13:
                e = rb == 3 ? dev::launch_batch_t<13, 3, 4, 3>(it, cnt, phases, ops, status, nsm, stream)
                            : dev::launch_batch_t<13, 4, 3, 3>(it, cnt, phases, ops, status, nsm, stream);
                break;
            case 12: e = dev::launch_batch_t<12, 4, 2, 3>(it, cnt, phases, ops, status, nsm, stream); break;
            case 11: e = dev::launch_batch_t<11, 3, 2, 3>(it, cnt, phases, ops, status, nsm, stream); break;
            default: e = dev::launch_batch_t<10, 2, 2, 3>(it, cnt, phases, ops, status, nsm, stream); break;
        }
        if (e != cudaSuccess) return e;
        (*launches)++;
    }
    return cudaSuccess;
}

Batch *batch_new() { return new Batch(); }
void batch_free(Batch *b) { delete b; }
int batch_size(const Batch *b) { return (int)b->circs.size(); }

}  // namespace qsv
