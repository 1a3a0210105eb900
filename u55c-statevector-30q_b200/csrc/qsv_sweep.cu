// qsv_sweep.cu -- the pass engine: one persistent, warp-specialised launch per sweep (sm_100a).
//
// Replaces the reference's HLS engine kernels/sv/sv_engine.cpp (reader :86-118 / compute :164-279 /
// writer :120-152 DATAFLOW per pass). B200 design:
//   * one CTA per SM (KW = 13: three 64 KiB tile buffers), grid-strided over the 2^(n-13) tiles;
//   * a producer warp streams every tile's 2^(13-lo) sub-blocks HBM -> shared memory with bulk-async
//     copies (the TMA engine; completion counted on an mbarrier) and, once the consumers are done,
//     shared memory -> HBM with bulk-async stores, keeping up to three tiles in flight;
//   * consumer warps apply the sweep's ops in registers: each thread holds 2^RB float4 (two amplitudes
//     each); ops on tile bit 0 pair the halves of a float4, ops on register bits pair two float4, ops
//     on lane bits exchange with warp shuffles; an op whose target is on a warp bit starts a new phase
//     (shared-memory round trip in another layout). Controls may sit anywhere in the window.
// The tile addressing is the reference's (model.py:25-40 / sv_engine.cpp:61-84,116): tile T's base is
// pdep(T, free bits) and sub-block s sits at base | pdep(s, H).
#include "qsv_device.cuh"

namespace qsv {
namespace dev {

// Device status word: kernels OR a bit in when a bounded wait gives up (1 = mbarrier wait timeout).
__device__ int g_status = 0;

// ---------------------------------------------------------------- per-thread pair iteration
// pairs across the two halves of each float4 (target = tile bit 0); i0 = position of the .xy half
template <int NV, class F>
__device__ __forceinline__ void pairs_comp(float4 (&v)[NV], uint32_t tb, const uint32_t (&off)[NV], F &f) {
#pragma unroll
    for (int r = 0; r < NV; r++) f(v[r].x, v[r].y, v[r].z, v[r].w, tb | off[r]);
}
// pairs between float4 r and r | 2^R (target = register bit R), both halves
template <int NV, int R, class F>
__device__ __forceinline__ void pairs_reg(float4 (&v)[NV], uint32_t tb, const uint32_t (&off)[NV], F &f) {
#pragma unroll
    for (int r = 0; r < NV; r++) {
        if (r & (1 << R)) continue;
        const int r2 = r | (1 << R);
        f(v[r].x, v[r].y, v[r2].x, v[r2].y, tb | off[r]);
        f(v[r].z, v[r].w, v[r2].z, v[r2].w, tb | off[r] | 1u);
    }
}

template <int NV, int RB, class F>
__device__ __forceinline__ void pairs_slot(int slot, float4 (&v)[NV], uint32_t tb, const uint32_t (&off)[NV], F &f) {
    switch (slot) {
        case QSV_SLOT_COMP: pairs_comp<NV>(v, tb, off, f); break;
        case QSV_SLOT_REG0 + 0: pairs_reg<NV, 0>(v, tb, off, f); break;
        case QSV_SLOT_REG0 + 1: if constexpr (RB > 1) pairs_reg<NV, (RB > 1 ? 1 : 0)>(v, tb, off, f); break;
        case QSV_SLOT_REG0 + 2: if constexpr (RB > 2) pairs_reg<NV, (RB > 2 ? 2 : 0)>(v, tb, off, f); break;
        case QSV_SLOT_REG0 + 3: if constexpr (RB > 3) pairs_reg<NV, (RB > 3 ? 3 : 0)>(v, tb, off, f); break;
        default: break;
    }
}

struct FUni {          // same matrix for every pair
    const float *m;
    int cls;
    __device__ __forceinline__ void operator()(float &a, float &b, float &c, float &d, uint32_t) const {
        pair_apply(a, b, c, d, m, cls);
    }
};
struct FDense {
    const float *m;
    __device__ __forceinline__ void operator()(float &a, float &b, float &c, float &d, uint32_t) const {
        pair_apply(a, b, c, d, m, QSV_M_DENSE);
    }
};
struct FCtrl {         // M0 = identity: only pairs whose controls are all set change
    const float *m1;
    int cls1;
    uint32_t cm;
    __device__ __forceinline__ void operator()(float &a, float &b, float &c, float &d, uint32_t i0) const {
        if ((i0 & cm) == cm) pair_apply(a, b, c, d, m1, cls1);
    }
};
struct FMux {          // general MUX2
    const float *m0, *m1;
    int cls0, cls1;
    uint32_t cm;
    __device__ __forceinline__ void operator()(float &a, float &b, float &c, float &d, uint32_t i0) const {
        if ((i0 & cm) == cm) pair_apply(a, b, c, d, m1, cls1);
        else pair_apply(a, b, c, d, m0, cls0);
    }
};

// op on a lane bit: exchange with the partner lane, each thread computes its own amplitude
template <int NV>
__device__ __forceinline__ void lane_op(float4 (&v)[NV], uint32_t tb, const uint32_t (&off)[NV], int lanebit,
                                        uint32_t tmask, const float *m0, const float *m1, int cls0, int cls1,
                                        uint32_t cm, int lane) {
    const int mine = (lane >> lanebit) & 1;
    const int xm = 1 << lanebit;
#pragma unroll
    for (int r = 0; r < NV; r++) {
        float4 o;
        o.x = __shfl_xor_sync(0xffffffffu, v[r].x, xm);
        o.y = __shfl_xor_sync(0xffffffffu, v[r].y, xm);
        o.z = __shfl_xor_sync(0xffffffffu, v[r].z, xm);
        o.w = __shfl_xor_sync(0xffffffffu, v[r].w, xm);
#pragma unroll
        for (int c = 0; c < 2; c++) {
            const uint32_t i0 = (tb | off[r] | (uint32_t)c) & ~tmask;
            const bool sel = cm != 0 && (i0 & cm) == cm;
            const int cls = sel ? cls1 : cls0;
            float &owr = c ? v[r].z : v[r].x;
            float &owi = c ? v[r].w : v[r].y;
            const float otr = c ? o.z : o.x;
            const float oti = c ? o.w : o.y;
            if (cls == QSV_M_IDENT) continue;
            if (cls == QSV_M_XSWAP) { owr = otr; owi = oti; continue; }
            // (a, b) = (m00, m01) for the bit-0 amplitude, (m11, m10) for the bit-1 amplitude; selected by
            // value (constant register indices keep the matrices in registers)
            const float ar = sel ? (mine ? m1[6] : m1[0]) : (mine ? m0[6] : m0[0]);
            const float ai = sel ? (mine ? m1[7] : m1[1]) : (mine ? m0[7] : m0[1]);
            float yr, yi;
            if (cls == QSV_M_DIAG) {
                diag_own(yr, yi, ar, ai, owr, owi);
            } else {
                const float br = sel ? (mine ? m1[4] : m1[2]) : (mine ? m0[4] : m0[2]);
                const float bi = sel ? (mine ? m1[5] : m1[3]) : (mine ? m0[5] : m0[3]);
                lin_own(yr, yi, ar, ai, br, bi, owr, owi, otr, oti);
            }
            owr = yr; owi = yi;
        }
    }
}

template <int NV, int RB>
__device__ __forceinline__ void apply_op(const QsvOp &op, float4 (&v)[NV], uint32_t tb, const uint32_t (&off)[NV],
                                         uint32_t lane34, int lane) {
    float m0[8], m1[8];
#pragma unroll
    for (int e = 0; e < 8; e++) { m0[e] = op.m0[e]; m1[e] = op.m1[e]; }
    const uint32_t cm = op.cmask;
    const int c0 = op.cls0, c1 = op.cls1, slot = op.slot;
    if (slot >= QSV_SLOT_LANE0) {
        const int l = slot - QSV_SLOT_LANE0;
        // tile bit of lane bit l: lane bits 0..2 hold tile bits 1..3, lane bits 3, 4 the phase's choice
        const uint32_t tbit = l < 3 ? (uint32_t)(l + 1) : ((lane34 >> (8 * (l - 3))) & 0xffu);
        lane_op<NV>(v, tb, off, l, 1u << tbit, m0, m1, c0, c1, cm, lane);
        return;
    }
    if (cm == 0) {
        if (c0 == QSV_M_DENSE) { FDense f{m0}; pairs_slot<NV, RB>(slot, v, tb, off, f); }
        else if (c0 != QSV_M_IDENT) { FUni f{m0, c0}; pairs_slot<NV, RB>(slot, v, tb, off, f); }
    } else if (c0 == QSV_M_IDENT) {
        if (c1 != QSV_M_IDENT) { FCtrl f{m1, c1, cm}; pairs_slot<NV, RB>(slot, v, tb, off, f); }
    } else {
        FMux f{m0, m1, c0, c1, cm};
        pairs_slot<NV, RB>(slot, v, tb, off, f);
    }
}

// ---------------------------------------------------------------- the sweep kernel
template <int KW, int RB, int WB, int S>
__global__ void __launch_bounds__((1 << (5 + WB)) + 32, (KW >= 13 ? 1 : 2))
    sweep_kernel(float2 *__restrict__ state, const __grid_constant__ QsvSweep P) {
    constexpr int NC = 1 << (5 + WB);        // consumer threads
    constexpr int NV = 1 << RB;              // float4 per consumer thread
    constexpr int TILE = 1 << KW;            // amplitudes per tile
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

    const int64_t ntiles = P.ntiles;
    const int64_t first = blockIdx.x, stride = gridDim.x;
    const int64_t nmine = first < ntiles ? (ntiles - 1 - first) / stride + 1 : 0;

    if (tid >= NC) {
        // ------------------------------------------------------------ producer warp
        const int lane = tid & 31;
        const int lo = P.lo;
        const int nsub = 1 << (KW - lo);
        const uint32_t subbytes = 8u << lo;
        const int nh = P.nh;
        auto tile_base = [&](int64_t T) -> int64_t {
            int64_t x = T << lo;                      // free bits are the bits outside [0, lo) U H
            for (int i = 0; i < nh; i++) {
                const int h = P.H[i];
                x = ((x >> h) << (h + 1)) | (x & ((1ll << h) - 1));
            }
            return x;
        };
        auto sub_off = [&](int s) -> int64_t {
            int64_t o = 0;
            for (int i = 0; i < KW - lo; i++)
                if ((s >> i) & 1) o |= 1ll << P.H[i];
            return o;
        };
        auto issue_load = [&](int64_t j, int b) {
            const int64_t base = tile_base(first + j * stride);
            if (lane == 0) mbar_arrive_expect_tx(&full[b], (uint32_t)TILE * 8u);
            __syncwarp();
            float2 *dst = bufs + (size_t)b * TILE;
            for (int s = lane; s < nsub; s += 32) bulk_g2s(dst + (s << lo), state + (base | sub_off(s)), subbytes, &full[b]);
        };
        auto issue_store = [&](int64_t j, int b) {
            const int64_t base = tile_base(first + j * stride);
            const float2 *src = bufs + (size_t)b * TILE;
            for (int s = lane; s < nsub; s += 32) bulk_s2g(state + (base | sub_off(s)), src + (s << lo), subbytes);
            bulk_commit();
        };
        for (int64_t j = 0; j < S && j < nmine; j++) issue_load(j, (int)j);
        for (int64_t j = 0; j < nmine; j++) {
            const int b = (int)(j % S);
            const uint32_t par = (uint32_t)((j / S) & 1);
            if (!mbar_wait(&done[b], par, &abort_flag, &g_status)) break;
            issue_store(j, b);
            if (j + S < nmine) {
                bulk_wait_read_all();                 // this lane's stores have read the buffer
                __syncwarp();
                issue_load(j + S, b);
            }
        }
        bulk_wait_all();
        return;
    }

    // ---------------------------------------------------------------- consumer warps
    const int lane = tid & 31, warp = tid >> 5;
    for (int64_t j = 0; j < nmine; j++) {
        const int b = (int)(j % S);
        const uint32_t par = (uint32_t)((j / S) & 1);
        if (!mbar_wait(&full[b], par, &abort_flag, &g_status)) break;
        float2 *tile = bufs + (size_t)b * TILE;
        for (int ph = 0; ph < P.nphases; ph++) {
            if (ph > 0) named_bar_sync(1, NC);
            const QsvPhase &Q = P.phases[ph];
            uint32_t tb = ((uint32_t)(lane & 7) << 1) | ((uint32_t)((lane >> 3) & 1) << Q.lane_bits[0]) |
                          ((uint32_t)((lane >> 4) & 1) << Q.lane_bits[1]);
#pragma unroll
            for (int w = 0; w < WB; w++) tb |= (uint32_t)((warp >> w) & 1) << Q.warp_bits[w];
            uint32_t rbit[RB];
#pragma unroll
            for (int r = 0; r < RB; r++) rbit[r] = 1u << Q.reg_bits[r];
            uint32_t off[NV];
#pragma unroll
            for (int r = 0; r < NV; r++) {
                uint32_t o = 0;
#pragma unroll
                for (int q = 0; q < RB; q++)
                    if ((r >> q) & 1) o |= rbit[q];
                off[r] = o;
            }
            const uint32_t lane34 = (uint32_t)Q.lane_bits[0] | ((uint32_t)Q.lane_bits[1] << 8);
            float4 v[NV];
#pragma unroll
            for (int r = 0; r < NV; r++) v[r] = *reinterpret_cast<const float4 *>(tile + (tb | off[r]));
            for (int o = Q.op_begin; o < Q.op_end; o++) apply_op<NV, RB>(P.ops[o], v, tb, off, lane34, lane);
#pragma unroll
            for (int r = 0; r < NV; r++) *reinterpret_cast<float4 *>(tile + (tb | off[r])) = v[r];
        }
        fence_proxy_async_smem();
        mbar_arrive(&done[b]);
    }
}

// ---------------------------------------------------------------- host launchers
template <int KW, int RB, int WB, int S>
static cudaError_t launch_sweep_t(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream) {
    constexpr int NT = (1 << (5 + WB)) + 32;
    const size_t smem = ((size_t)S << KW) * sizeof(float2);
    static int configured_dev = -1;     // attribute set once per device (first-use; not thread-raced in
    int dev = 0;                        // practice: set under the engine's launch lock)
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (configured_dev != dev) {
        e = cudaFuncSetAttribute(sweep_kernel<KW, RB, WB, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured_dev = dev;
    }
    int per_sm = 1;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_kernel<KW, RB, WB, S>, NT, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int64_t grid = (int64_t)nsm * per_sm;
    if (grid > sw.ntiles) grid = sw.ntiles;
    sweep_kernel<KW, RB, WB, S><<<(unsigned)grid, NT, smem, stream>>>(state, sw);
    return cudaGetLastError();
}

}  // namespace dev

cudaError_t take_device_status(int *out) {
    int zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(out, dev::g_status, sizeof(int));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(dev::g_status, &zero, sizeof(int));
}

cudaError_t launch_sweep(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream) {
    switch (sw.kw) {
        case 13: return dev::launch_sweep_t<13, 4, 3, 3>(state, sw, nsm, stream);
        case 12: return dev::launch_sweep_t<12, 4, 2, 3>(state, sw, nsm, stream);
        case 11: return dev::launch_sweep_t<11, 3, 2, 3>(state, sw, nsm, stream);
        case 10: return dev::launch_sweep_t<10, 2, 2, 3>(state, sw, nsm, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace qsv
