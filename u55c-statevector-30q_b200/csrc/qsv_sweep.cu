// qsv_sweep.cu -- the pass engine: one persistent, warp-specialised launch per sweep (sm_100a).
//
// Replaces the reference's HLS engine kernels/sv/sv_engine.cpp (reader :86-118 / compute :164-279 /
// writer :120-152 DATAFLOW per pass). B200 design:
//   * one CTA per SM (KW = 13: three 64 KiB tile buffers), grid-strided over the 2^(n-13) tiles;
//   * a producer warp streams tiles HBM -> shared memory and back with the TMA engine: one tensor-map
//     box per tile when the window's contiguous runs are short, one bulk-async copy per sub-block when
//     they are long; completion is counted on mbarriers, up to three tiles are in flight;
//   * consumer warps apply the sweep's ops in registers. A thread keeps 2^RB float4 (the two halves of
//     each float4 = tile bit 0) repacked as float2 (re, re) / (im, im) pairs so that every register-bit op
//     runs on two amplitude pairs per packed FP32x2 FMA; ops on lane bits exchange with warp shuffles; an op
//     whose target is on a warp bit starts a new phase (shared-memory round trip in another layout).
// The tile addressing is the reference's (model.py:25-40 / sv_engine.cpp:61-84,116): tile T's base is
// pdep(T, free bits) and sub-block s sits at base | pdep(s, H).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>

#include "qsv_device.cuh"
#include "qsv_ops.cuh"
#include "qsv_planner.h"

namespace qsv {
namespace dev {

// Device status word: kernels OR a bit in when a bounded wait gives up (1 = mbarrier wait timeout).
__device__ int g_status = 0;

// ---------------------------------------------------------------- tensor-map TMA
__device__ __forceinline__ void tma_load(void *sdst, const CUtensorMap *map, const int32_t *c, int rank, uint64_t *bar) {
    const uint64_t m = reinterpret_cast<uint64_t>(map);
    const uint32_t d = smem_u32(sdst), b = smem_u32(bar);
    switch (rank) {
        case 2:
            asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                         ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(b) : "memory");
            break;
        case 3:
            asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                         ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(b) : "memory");
            break;
        case 4:
            asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
                         ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(b) : "memory");
            break;
        default:
            asm volatile("cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
                         ::"r"(d), "l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(b) : "memory");
            break;
    }
}
__device__ __forceinline__ void tma_store(const CUtensorMap *map, const int32_t *c, int rank, const void *ssrc) {
    const uint64_t m = reinterpret_cast<uint64_t>(map);
    const uint32_t s = smem_u32(ssrc);
    switch (rank) {
        case 2:
            asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
                         ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(s) : "memory");
            break;
        case 3:
            asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];"
                         ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(s) : "memory");
            break;
        case 4:
            asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4}], [%5];"
                         ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(s) : "memory");
            break;
        default:
            asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];"
                         ::"l"(m), "r"(c[0]), "r"(c[1]), "r"(c[2]), "r"(c[3]), "r"(c[4]), "r"(s) : "memory");
            break;
    }
}

// ---------------------------------------------------------------- the sweep kernel
template <int KW, int RB, int WB, int S>
__global__ void __launch_bounds__((1 << (5 + WB)) + 32, (KW >= 13 ? 1 : 2))
    sweep_kernel(float2 *__restrict__ state, const __grid_constant__ QsvSweep P, const __grid_constant__ CUtensorMap tmap) {
    constexpr int NC = 1 << (5 + WB);        // consumer threads
    constexpr int NV = 1 << RB;              // float4 per consumer thread
    constexpr int TILE = 1 << KW;            // amplitudes per tile
    static_assert(1 + 3 + 2 + RB + WB == KW, "layout must cover the window");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    float2 *bufs = reinterpret_cast<float2 *>(smem_raw);
    // the sweep's op table, copied once from the parameter block: shared-memory reads of an op's fields
    // are independent short-latency loads (the constant-bank path serialises them per op)
    QsvOp *sops = reinterpret_cast<QsvOp *>(smem_raw + ((size_t)S << KW) * sizeof(float2));
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t done[S];
    __shared__ volatile int abort_flag;

    const int tid = threadIdx.x;
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(P.ops);
        uint32_t *dst = reinterpret_cast<uint32_t *>(sops);
        const int words = P.nops * (int)(sizeof(QsvOp) / 4);
        for (int i = tid; i < words; i += blockDim.x) dst[i] = src[i];
    }
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
        const int rank = P.tma_rank;
        auto coords = [&](int64_t T, int32_t *c) {
            int pos = 0;
            for (int d = 0; d < rank; d++) {
                const int f = P.tdim_free[d];
                c[d] = (int32_t)(((T >> pos) & ((1ll << f) - 1)) << P.tdim_box[d]);
                pos += f;
            }
        };
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
            const int64_t T = first + j * stride;
            float2 *dst = bufs + (size_t)b * TILE;
            if (rank) {
                if (lane == 0) {
                    int32_t c[QSV_TMA_MAX_RANK];
                    coords(T, c);
                    mbar_arrive_expect_tx(&full[b], (uint32_t)TILE * 8u);
                    tma_load(dst, &tmap, c, rank, &full[b]);
                }
                return;
            }
            const int64_t base = tile_base(T);
            if (lane == 0) mbar_arrive_expect_tx(&full[b], (uint32_t)TILE * 8u);
            __syncwarp();
            for (int s = lane; s < nsub; s += 32) bulk_g2s(dst + (s << lo), state + (base | sub_off(s)), subbytes, &full[b]);
        };
        auto issue_store = [&](int64_t j, int b) {
            const int64_t T = first + j * stride;
            const float2 *src = bufs + (size_t)b * TILE;
            if (rank) {
                if (lane == 0) {
                    int32_t c[QSV_TMA_MAX_RANK];
                    coords(T, c);
                    tma_store(&tmap, c, rank, src);
                    bulk_commit();
                }
                return;
            }
            const int64_t base = tile_base(T);
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
            run_phase<NV, RB, WB>(tile, Q, sops, Q.op_begin, Q.op_end, lane, warp);
        }
        fence_proxy_async_smem();
        mbar_arrive(&done[b]);
    }
}

// ---------------------------------------------------------------- host launchers
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// tensor map of the state for a sweep staged with one box per tile (see qsv_plan.h)
static cudaError_t make_tmap(CUtensorMap *map, float2 *state, const QsvSweep &sw) {
    std::memset(map, 0, sizeof(*map));
    if (!sw.tma_rank) return cudaSuccess;
    auto fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    cuuint64_t dims[QSV_TMA_MAX_RANK], strides[QSV_TMA_MAX_RANK];
    cuuint32_t box[QSV_TMA_MAX_RANK], estr[QSV_TMA_MAX_RANK];
    // dim d starts at the window bit following the previous dim's box + free bits
    int start = 0;
    for (int d = 0; d < sw.tma_rank; d++) {
        if (d > 0) strides[d - 1] = (cuuint64_t)8 << start;
        dims[d] = (cuuint64_t)1 << (sw.tdim_box[d] + sw.tdim_free[d]);
        box[d] = 1u << sw.tdim_box[d];
        estr[d] = 1;
        start += sw.tdim_box[d] + sw.tdim_free[d];
    }
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_INT64, sw.tma_rank, state, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int KW, int RB, int WB, int S>
static cudaError_t launch_sweep_t(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream) {
    constexpr int NT = (1 << (5 + WB)) + 32;
    const size_t smem = ((size_t)S << KW) * sizeof(float2) + sizeof(QsvOp) * QSV_MAX_SWEEP_OPS;
    static int configured_dev = -1;     // attribute set once per device (under the engine's launch lock)
    static int per_sm = 1;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (configured_dev != dev) {
        e = cudaFuncSetAttribute(sweep_kernel<KW, RB, WB, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sweep_kernel<KW, RB, WB, S>, NT, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        configured_dev = dev;
    }
    alignas(64) CUtensorMap map;
    e = make_tmap(&map, state, sw);
    if (e != cudaSuccess) return e;
    int64_t grid = (int64_t)nsm * per_sm;
    if (grid > sw.ntiles) grid = sw.ntiles;
    sweep_kernel<KW, RB, WB, S><<<(unsigned)grid, NT, smem, stream>>>(state, sw, map);
    return cudaGetLastError();
}

}  // namespace dev

// device address of the status word, for kernels in other translation units
cudaError_t status_word_ptr(int **out) {
    static int *ptr[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, dev::g_status);
        if (e != cudaSuccess) return e;
        ptr[dev] = static_cast<int *>(p);
    }
    *out = ptr[dev];
    return cudaSuccess;
}

cudaError_t take_device_status(int *out) {
    int zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(out, dev::g_status, sizeof(int));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(dev::g_status, &zero, sizeof(int));
}

cudaError_t launch_sweep(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream) {
    int rb = 4, wb = 3;
    layout_for_kw(sw.kw, &rb, &wb);
    switch (sw.kw) {
        case 13:
            if (rb == 3) return dev::launch_sweep_t<13, 3, 4, 3>(state, sw, nsm, stream);
            return dev::launch_sweep_t<13, 4, 3, 3>(state, sw, nsm, stream);
        case 12: return dev::launch_sweep_t<12, 4, 2, 3>(state, sw, nsm, stream);
        case 11: return dev::launch_sweep_t<11, 3, 2, 3>(state, sw, nsm, stream);
        case 10: return dev::launch_sweep_t<10, 2, 2, 3>(state, sw, nsm, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace qsv
