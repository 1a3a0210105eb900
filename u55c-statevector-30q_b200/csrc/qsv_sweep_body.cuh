// qsv_sweep_body.cuh -- the sweep pipeline shared by every sweep kernel (sm_100a).
//
// Replaces the reader / writer stages of the reference's HLS engine (kernels/sv/sv_engine.cpp:86-152,
// DATAFLOW per pass). One persistent CTA per SM, grid-strided over the 2^(n-KW) tiles of a sweep:
//   * a producer warp streams tiles HBM -> shared memory and back with the TMA engine: one tensor-map box
//     per tile when the window's contiguous runs are short, one bulk-async copy per sub-block when they
//     are long; completion is counted on mbarriers, up to S tiles are in flight;
//   * G groups of consumer warps run Body::tile on the staged tiles (the ops of the sweep, in registers);
//     with G = 2 the groups take alternate tiles, so one group's phase barriers and shared-memory round
//     trips overlap the other group's arithmetic;
//   * or (IL = 1, one group) every consumer thread keeps two tiles in flight and interleaves their phases
//     (Body::phase), with an mbarrier per tile slot in place of the block-wide barrier between two phases of
//     a tile: a thread runs a phase of the other tile while the slowest threads finish their stores, so the
//     phase round trips of one tile overlap the arithmetic of the other without a second register set.
// Body is the interpreter (qsv_sweep.cu: op table read at run time) or a kernel specialised to one sweep
// structure (qsv_jit.cpp: ops fixed at compile time). Both run the same arithmetic (qsv_ops.cuh).
// The tile addressing is the reference's (host/sv/model.py:25-40, sv_engine.cpp:61-84,116): tile T's
// base is pdep(T, free bits) and sub-block s sits at base | pdep(s, H).
#pragma once
#include "qsv_device.cuh"

namespace qsv {
namespace dev {

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

// Dynamic shared memory a sweep kernel needs: S tile buffers, plus the op table when Body reads it there,
// plus 1 KiB to align the buffers to 1024 bytes (the 128-byte swizzle pattern repeats every 1024 bytes of
// shared-memory address, and the consumers' addressing assumes it starts at each buffer).
template <int KW, int S, class Body, class SW = QsvSweep>
__host__ __device__ constexpr size_t sweep_smem_bytes() {
    return ((size_t)S << KW) * sizeof(typename Body::Amp) +
           (Body::kSmemOps ? sizeof(typename SW::op_type) * QSV_MAX_SWEEP_OPS : 0) + QSV_SMEM_ALIGN;
}

// The pipeline. Launch with G * (1 << (5 + WB)) + 32 threads and sweep_smem_bytes<KW, S, Body, SW>() bytes
// of dynamic shared memory. status: device word that bounded waits OR their failure bit into.
// Body::Amp is the amplitude type (float2: complex64, double2: complex128); Body::kHalfBits is 1 when a
// thread's 16-byte slot packs two amplitudes (tile bit 0), 0 when it holds one. IL = 1 needs G = 1 and a
// Body with kPhases and phase(p, ...) (one phase of a tile: load in its layout, apply its ops, store).
template <int KW, int RB, int WB, int S, int G, class Body, class SW = QsvSweep, int IL = 0>
__device__ __forceinline__ void sweep_pipeline(typename Body::Amp *__restrict__ state, const SW &P,
                                               const CUtensorMap *tmap, int *status) {
    using Amp = typename Body::Amp;
    using Op = typename SW::op_type;
    constexpr int NCG = 1 << (5 + WB);       // consumer threads of one group
    constexpr int NC = G * NCG;              // consumer threads
    constexpr int NV = 1 << RB;              // 16-byte slots per consumer thread
    constexpr int TILE = 1 << KW;            // amplitudes per tile
    constexpr uint32_t TILE_BYTES = (uint32_t)TILE * (uint32_t)sizeof(Amp);
    static_assert(Body::kHalfBits + 3 + 2 + RB + WB == KW, "layout must cover the window");
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    static_assert(QSV_SMEM_ALIGN == 1024, "the 128-byte swizzle repeats every 1024 bytes");
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    Amp *bufs = reinterpret_cast<Amp *>(smem);
    // the interpreter's op table, copied once from the parameter block: shared-memory reads of an op's
    // fields are independent short-latency loads (the constant-bank path serialises run-time indices)
    Op *sops = reinterpret_cast<Op *>(smem + ((size_t)S << KW) * sizeof(Amp));
    // full barrier of tile j: full[j % (S * G)]. Tiles sharing a full barrier share a buffer (j % S) and a
    // consumer group (j % G), so each full barrier is waited on by one group, phase after phase (a parity
    // wait never meets a phase two steps old). done[b] is waited on by the producer alone, tile by tile.
    constexpr int NF = S * G;
    __shared__ __align__(8) uint64_t full[NF];
    __shared__ __align__(8) uint64_t done[S];
    __shared__ __align__(8) uint64_t pbar[2];     // IL: phase barriers of the two tiles in flight
    __shared__ volatile int abort_flag;

    const int tid = threadIdx.x;
    if (Body::kSmemOps) {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(P.ops);
        uint32_t *dst = reinterpret_cast<uint32_t *>(sops);
        const int words = P.nops * (int)(sizeof(Op) / 4);
        for (int i = tid; i < words; i += blockDim.x) dst[i] = src[i];
    }
    if (tid == 0) {
        for (int f = 0; f < NF; f++) mbar_init(&full[f], 1);
        for (int s = 0; s < S; s++) mbar_init(&done[s], NCG);
        for (int u = 0; u < 2; u++) mbar_init(&pbar[u], NCG);
        abort_flag = 0;
        fence_mbar_init();
    }
    __syncthreads();

    const int64_t ntiles = P.ntiles;
    const int64_t first = blockIdx.x, stride = gridDim.x;
    const int64_t nmine = first < ntiles ? (ntiles - 1 - first) / stride + 1 : 0;
    const uint64_t limit = wait_limit_ns(P.wait_us);

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
        const uint32_t subbytes = (uint32_t)sizeof(Amp) << lo;
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
        // fault injection (tests of the bounded waits): block 0 never loads its first tile
        const bool skip_first = P.skip_load != 0 && blockIdx.x == 0;
        auto issue_load = [&](int64_t j, int b) {
            const int64_t T = first + j * stride;
            Amp *dst = bufs + (size_t)b * TILE;
            uint64_t *fb = &full[j % NF];
            if (skip_first && j == 0) return;
            if (rank) {
                if (lane == 0) {
                    int32_t c[QSV_TMA_MAX_RANK];
                    coords(T, c);
                    mbar_arrive_expect_tx(fb, TILE_BYTES);
                    tma_load(dst, tmap, c, rank, fb);
                }
                return;
            }
            const int64_t base = tile_base(T);
            if (lane == 0) mbar_arrive_expect_tx(fb, TILE_BYTES);
            __syncwarp();
            for (int s = lane; s < nsub; s += 32) bulk_g2s(dst + (s << lo), state + (base | sub_off(s)), subbytes, fb);
        };
        auto issue_store = [&](int64_t j, int b) {
            const int64_t T = first + j * stride;
            const Amp *src = bufs + (size_t)b * TILE;
            if (rank) {
                if (lane == 0) {
                    int32_t c[QSV_TMA_MAX_RANK];
                    coords(T, c);
                    tma_store(tmap, c, rank, src);
                    bulk_commit();
                }
                return;
            }
            const int64_t base = tile_base(T);
            for (int s = lane; s < nsub; s += 32) bulk_s2g(state + (base | sub_off(s)), src + (s << lo), subbytes);
            bulk_commit();
        };
        int64_t issued = 0, j = 0;                    // loads issued for tiles [0, issued)
        for (; issued < S && issued < nmine; issued++) issue_load(issued, (int)issued);
        for (; j < nmine; j++) {
            const int b = (int)(j % S);
            const uint32_t par = (uint32_t)((j / S) & 1);
            if (!mbar_wait(&done[b], par, &abort_flag, status, limit)) break;
            issue_store(j, b);
            if (j + S < nmine) {
                bulk_wait_read_all();                 // this lane's stores have read the buffer
                __syncwarp();
                issue_load(j + S, b);
                issued = j + S + 1;
            }
        }
        if (j < nmine && lane == 0) {
            // aborted: loads of tiles [j, issued) may still be in flight into this CTA's shared memory;
            // wait for them (bounded) before the CTA exits
            for (int64_t k = j; k < issued; k++)
                if (!(skip_first && k == 0)) mbar_wait_drain(&full[k % NF], (uint32_t)((k / NF) & 1), limit);
        }
        bulk_wait_all();
        return;
    }

    // ---------------------------------------------------------------- consumer warps
    if constexpr (IL != 0) {
        static_assert(G == 1, "interleaved phases run one consumer group");
        // tiles j0 and j0 + 1 (slots u = 0, 1): phase p of both, then phase p + 1 of both. Every consumer
        // thread arrives on pbar[u] after its stores of a phase and waits on it before its loads of the next
        // phase of the same tile; it waits on each completion of pbar[u] in order, so its count of waits gives
        // the parity, and no thread can fall two completions behind (each completion needs its arrival).
        const int lane = tid & 31, warp = tid >> 5;
        uint32_t waits[2] = {0u, 0u};
        bool ok = true;
        for (int64_t j0 = 0; ok && j0 < nmine; j0 += 2) {
            const int cnt = j0 + 1 < nmine ? 2 : 1;
#pragma unroll
            for (int p = 0; p < Body::kPhases; p++) {
                for (int u = 0; u < cnt; u++) {
                    const int64_t j = j0 + u;
                    const int b = (int)(j % S);
                    if (p == 0) {
                        ok = mbar_wait(&full[j % NF], (uint32_t)((j / NF) & 1), &abort_flag, status, limit);
                    } else {
                        ok = mbar_wait(&pbar[u], waits[u] & 1u, &abort_flag, status, limit);
                        waits[u]++;
                    }
                    if (!ok) break;
                    Body::template phase<NV, RB, WB>(p, bufs + (size_t)b * TILE, P, sops, lane, warp);
                    if (p + 1 < Body::kPhases) {
                        mbar_arrive(&pbar[u]);
                    } else {
                        fence_proxy_async_smem();
                        mbar_arrive(&done[b]);
                    }
                }
                if (!ok) break;
            }
        }
        return;
    }
    const int grp = tid / NCG;                   // group grp takes tiles grp, grp + G, ...
    const int lane = tid & 31, warp = (tid % NCG) >> 5;
    for (int64_t j = grp; j < nmine; j += G) {
        const int b = (int)(j % S);
        const uint32_t par = (uint32_t)((j / NF) & 1);
        if (!mbar_wait(&full[j % NF], par, &abort_flag, status, limit)) break;
        Amp *tile = bufs + (size_t)b * TILE;
        Body::template tile<NV, RB, WB>(tile, P, sops, lane, warp, 1 + grp);
        fence_proxy_async_smem();
        mbar_arrive(&done[b]);
    }
}

}  // namespace dev
}  // namespace qsv
