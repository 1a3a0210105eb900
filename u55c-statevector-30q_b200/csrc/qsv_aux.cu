// qsv_aux.cu -- the remap (qubit permutation) kernel, |0..0> init, FP64 reductions and the Born sampler.
//
// remap: replaces the reference's exchange path -- sv_swap (kernels/sv/sv_swap.cpp:10-39) for
// bank<->local transpositions and the host permutes of host/sv/runtime.py:261-268 -- with one in-HBM
// sweep for an arbitrary bit permutation perm[new] = old (host/sv/model.py:74-78). Each CTA moves tiles
// of 2^10 amplitudes that are contiguous in 32-amplitude runs on both sides: the tile holds source bits
// 0..4 (coalesced reads) and the source bits that land on destination bits 0..4 (coalesced writes),
// padded with the lowest remaining source bits; the transpose happens in shared memory.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <mutex>

#include "qsv_device.cuh"

namespace qsv {
namespace dev {

#define REMAP_TB 11                 // tile bits: 2^11 amplitudes per tile (2^10 for a 10-qubit state)
#define REMAP_RUN 5                 // contiguous run bits on each side (32 amplitudes per warp access)
#define REMAP_THREADS 256

struct RemapParams {
    int n;
    int nfree;
    uint8_t ubits[REMAP_TB];        // source bits of the tile, ascending (tile position bit i <-> ubits[i])
    uint8_t fx[40];                 // free source bits, ascending
    uint8_t fy[40];                 // destination position of free source bit fx[i]
    uint8_t ypos[REMAP_TB];         // destination position of tile source bit ubits[i]
    int8_t swz[REMAP_TB];           // shared-memory swizzle: tile bit b >= REMAP_RUN is XORed into low bit swz[b]
};

// Bit permutation of the state, one HBM read and one write per amplitude. A tile is 2^11 amplitudes that
// share the free bits (the source bits outside the tile); it holds source bits 0..4, so a warp's 32 reads
// are contiguous, and the source bits that land on destination bits 0..4, so a warp's 32 writes are
// contiguous. Shared memory holds the tile as 32-bit planes (W = sizeof(A) / 4 words per amplitude) at a
// swizzled position: a warp's stores vary tile bits 0..4 and its loads vary the tile bits of destination
// bits 0..4; the swizzle (host-chosen, linear) moves each such bit above bit 4 onto a low bit the other
// four leave free, so both sides hit 32 distinct banks. Each thread's tile-invariant offsets are computed
// once; the loads of the next tile are issued before the stores of the current one.
// (three CTAs per SM: 80 registers, three tiles of loads in flight per SM plus each CTA's next tile)
template <class A, int TB>
__global__ void __launch_bounds__(REMAP_THREADS, 3)
    remap_kernel(const A *__restrict__ src, A *__restrict__ dst, const __grid_constant__ RemapParams P) {
    constexpr int TS = 1 << TB;
    constexpr int REMAP_EPT = TS / REMAP_THREADS;     // amplitudes per thread per tile
    constexpr int W = sizeof(A) / 4;
    using Word = uint32_t;
    __shared__ Word plane[W * TS];
    const int t = threadIdx.x;
    // destination enumeration: bit q of k walks the tile bit with the q-th smallest destination position
    uint8_t order[TB];
    {
        bool used[TB] = {false};
        for (int q = 0; q < TB; q++) {
            int best = -1;
            for (int i = 0; i < TB; i++)
                if (!used[i] && (best < 0 || P.ypos[i] < P.ypos[best])) best = i;
            used[best] = true;
            order[q] = (uint8_t)best;
        }
    }
    auto swz = [&](uint32_t j) -> uint32_t {
        uint32_t m = 0;
        for (int b = REMAP_RUN; b < TB; b++)
            if (P.swz[b] >= 0 && ((j >> b) & 1)) m |= 1u << P.swz[b];
        return j ^ m;
    };
    uint64_t ro[REMAP_EPT], wo[REMAP_EPT];
    uint32_t sp_in[REMAP_EPT], sp_out[REMAP_EPT];
#pragma unroll
    for (int e = 0; e < REMAP_EPT; e++) {
        const uint32_t j = (uint32_t)(t + e * REMAP_THREADS);        // source-ordered tile position
        uint64_t o = 0;
        for (int i = 0; i < TB; i++)
            if ((j >> i) & 1) o |= 1ull << P.ubits[i];
        ro[e] = o;
        sp_in[e] = swz(j);
        const uint32_t k = j;                                         // destination-ordered enumeration
        uint64_t w = 0;
        uint32_t pos = 0;
        for (int q = 0; q < TB; q++)
            if ((k >> q) & 1) {
                w |= 1ull << P.ypos[order[q]];
                pos |= 1u << order[q];
            }
        wo[e] = w;
        sp_out[e] = swz(pos);
    }
    auto bases = [&](int64_t T, uint64_t &xb, uint64_t &yb) {
        xb = 0;
        yb = 0;
        for (uint64_t r = (uint64_t)T; r; r &= r - 1) {
            const int i = __ffsll((long long)r) - 1;
            xb |= 1ull << P.fx[i];
            yb |= 1ull << P.fy[i];
        }
    };
    const int64_t ntiles = 1ll << P.nfree;
    int64_t T = blockIdx.x;
    if (T >= ntiles) return;
    A v[REMAP_EPT];
    uint64_t xb, yb;
    bases(T, xb, yb);
#pragma unroll
    for (int e = 0; e < REMAP_EPT; e++) v[e] = src[xb | ro[e]];
    while (true) {
#pragma unroll
        for (int e = 0; e < REMAP_EPT; e++) {
            const Word *w = reinterpret_cast<const Word *>(&v[e]);
#pragma unroll
            for (int p = 0; p < W; p++) plane[p * TS + sp_in[e]] = w[p];
        }
        __syncthreads();
        const uint64_t ycur = yb;
        const int64_t Tn = T + gridDim.x;
        if (Tn < ntiles) {                      // next tile's loads in flight during this tile's stores
            bases(Tn, xb, yb);
#pragma unroll
            for (int e = 0; e < REMAP_EPT; e++) v[e] = src[xb | ro[e]];
        }
#pragma unroll
        for (int e = 0; e < REMAP_EPT; e++) {
            A a;
            Word *w = reinterpret_cast<Word *>(&a);
#pragma unroll
            for (int p = 0; p < W; p++) w[p] = plane[p * TS + sp_out[e]];
            dst[ycur | wo[e]] = a;
        }
        if (Tn >= ntiles) break;
        T = Tn;
        __syncthreads();                        // this tile's shared-memory reads are done
    }
}

// ---------------------------------------------------------------- HBM copy probe
// The achievable-bandwidth denominator (the B200 counterpart of the reference's FPGA HBM stream
// microbenchmark, kernels/hbm_stream/): a grid-stride 16-byte copy, every byte read once and written once.
__global__ void __launch_bounds__(512) copy_probe_kernel(const float4 *__restrict__ src, float4 *__restrict__ dst,
                                                         int64_t n16) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n16; i += 4 * stride) {
        const float4 a = __ldcs(src + i), b = __ldcs(src + i + stride), c = __ldcs(src + i + 2 * stride),
                     d = __ldcs(src + i + 3 * stride);
        __stcs(dst + i, a);
        __stcs(dst + i + stride, b);
        __stcs(dst + i + 2 * stride, c);
        __stcs(dst + i + 3 * stride, d);
    }
    for (; i < n16; i += stride) __stcs(dst + i, __ldcs(src + i));
}

// ---------------------------------------------------------------- |0...0>
__global__ void set_amp0_kernel(float2 *state) { state[0] = make_float2(1.0f, 0.0f); }
__global__ void set_amp0_kernel_d(double2 *state) { state[0] = make_double2(1.0, 0.0); }

// ---------------------------------------------------------------- FP64 reductions
// Block b covers amplitudes [b << B, (b+1) << B). Thread t visits i = (b << B) + t + 256 * it. The
// per-block result is 1 + B doubles: the block total and, for each bit q < B of the index, the sum of
// |a_i|^2 over the block's i with bit q set. Fixed summation order (deterministic).
#define RED_THREADS 256
template <class A>
__global__ void __launch_bounds__(RED_THREADS)
    reduce_block_kernel(const A *__restrict__ state, int B, double *__restrict__ partials) {
    __shared__ double s_tot[RED_THREADS];
    __shared__ double s_bits[RED_THREADS][17];
    const int t = threadIdx.x;
    const int64_t base = (int64_t)blockIdx.x << B;
    const int niter = 1 << (B - 8);
    double tot = 0.0;
    double hb[17];                  // bits 8..B-1 of i (from it)
#pragma unroll
    for (int q = 0; q < 17; q++) hb[q] = 0.0;
    // it = (g << 4) | k: the 16 values of k are summed per bit in registers, group totals feed the
    // bits above
    const int ng = niter >= 16 ? niter >> 4 : 1;
    const int gk = niter >= 16 ? 16 : niter;
    for (int g = 0; g < ng; g++) {
        double u[16];
#pragma unroll
        for (int k = 0; k < 16; k++) {
            u[k] = 0.0;
            if (k < gk) {
                const A a = state[base + t + ((int64_t)((g << 4) | k) << 8)];
                u[k] = (double)a.x * a.x + (double)a.y * a.y;
            }
        }
        double gt = 0.0;
#pragma unroll
        for (int k = 0; k < 16; k++) gt += u[k];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 16; k++)
                if ((k >> q) & 1) s += u[k];
            hb[q] += s;
        }
        for (int q = 4; q < B - 8; q++)
            if ((g >> (q - 4)) & 1) hb[q] += gt;
        tot += gt;
    }
    s_tot[t] = tot;
    for (int q = 0; q < 17; q++) s_bits[t][q] = hb[q];
    __syncthreads();
    double *out = partials + (int64_t)blockIdx.x * (B + 1);
    if (t == 0) {
        double s = 0.0;
        for (int i = 0; i < RED_THREADS; i++) s += s_tot[i];
        out[0] = s;
    } else if (t <= B) {
        const int q = t - 1;        // index bit q
        double s = 0.0;
        if (q < 8) {
            for (int i = 0; i < RED_THREADS; i++)
                if ((i >> q) & 1) s += s_tot[i];
        } else {
            for (int i = 0; i < RED_THREADS; i++) s += s_bits[i][q - 8];
        }
        out[1 + q] = s;
    }
}

// out[0] = total, out[1 + q] = total - 2 * (sum over i with bit q set)
__global__ void reduce_final_kernel(const double *__restrict__ partials, int nblocks, int B, int n,
                                    double *__restrict__ out) {
    const int t = threadIdx.x;
    if (t > n) return;
    double tot = 0.0, s = 0.0;
    for (int b = 0; b < nblocks; b++) {
        const double *p = partials + (int64_t)b * (B + 1);
        tot += p[0];
        if (t >= 1) {
            const int q = t - 1;
            if (q < B) s += p[1 + q];
            else if ((b >> (q - B)) & 1) s += p[0];
        }
    }
    if (t == 0) out[0] = tot;
    else out[t] = tot - 2.0 * s;
}

// chunk probabilities: one block per chunk of 2^cb amplitudes
template <class A>
__global__ void __launch_bounds__(RED_THREADS)
    chunk_probs_kernel(const A *__restrict__ state, int cb, double *__restrict__ out) {
    __shared__ double s[RED_THREADS];
    const int64_t base = (int64_t)blockIdx.x << cb;
    const int len = 1 << cb;
    double acc = 0.0;
    for (int i = threadIdx.x; i < len; i += RED_THREADS) {
        const A a = state[base + i];
        acc += (double)a.x * a.x + (double)a.y * a.y;
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

// inclusive prefix sum of nc doubles in one block (sequential per thread slice, fixed order)
__global__ void scan_kernel(double *__restrict__ v, int64_t nc) {
    __shared__ double part[1024];
    const int t = threadIdx.x, nt = blockDim.x;
    const int64_t per = (nc + nt - 1) / nt;
    const int64_t b = t * per, e = b + per < nc ? b + per : nc;
    double s = 0.0;
    for (int64_t i = b; i < e; i++) s += v[i];
    part[t] = s;
    __syncthreads();
    if (t == 0) {
        double run = 0.0;
        for (int i = 0; i < nt; i++) {
            const double x = part[i];
            part[i] = run;
            run += x;
        }
    }
    __syncthreads();
    double run = part[t];
    for (int64_t i = b; i < e; i++) {
        run += v[i];
        v[i] = run;
    }
}

// one thread per shot: chunk by binary search on the FP64 chunk cdf, then a linear FP64 scan inside
// the chunk (first index whose running sum exceeds the remainder, clipped to the chunk)
template <class A>
__global__ void sample_kernel(const A *__restrict__ state, int cb, const double *__restrict__ cdf, int64_t nc,
                              const double *__restrict__ uni, int shots, int64_t *__restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= shots) return;
    const double total = cdf[nc - 1];
    const double x = uni[s] * total;
    int64_t lo = 0, hi = nc;        // first c with cdf[c] > x
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (cdf[mid] > x) hi = mid;
        else lo = mid + 1;
    }
    int64_t c = lo < nc ? lo : nc - 1;
    const double rem = x - (c > 0 ? cdf[c - 1] : 0.0);
    const int len = 1 << cb;
    const A *p = state + (c << cb);
    double run = 0.0;
    int j = 0;
    for (; j < len; j++) {
        const A a = p[j];
        run += (double)a.x * a.x + (double)a.y * a.y;
        if (run > rem) break;
    }
    if (j >= len) j = len - 1;
    out[s] = (c << cb) + j;
}

}  // namespace dev

// ---------------------------------------------------------------- host launchers
// dtype: 0 = complex64 (float2 amplitudes), 1 = complex128 (double2)
cudaError_t launch_remap(const void *src, void *dst, int n, const int32_t *perm, int dtype, int nsm,
                         cudaStream_t stream) {
    dev::RemapParams P;
    memset(&P, 0, sizeof(P));
    P.n = n;
    int inv[64];
    for (int j = 0; j < n; j++) inv[perm[j]] = j;          // source bit perm[j] -> destination bit j
    bool in_tile[64] = {false};
    int cnt = 0;
    for (int b = 0; b < REMAP_RUN; b++) { in_tile[b] = true; cnt++; }
    for (int j = 0; j < REMAP_RUN; j++)
        if (!in_tile[perm[j]]) { in_tile[perm[j]] = true; cnt++; }
    const int tbits = n < REMAP_TB ? n : REMAP_TB;
    for (int b = 0; b < n && cnt < tbits; b++)
        if (!in_tile[b]) { in_tile[b] = true; cnt++; }
    int nu = 0, nf = 0;
    for (int b = 0; b < n; b++) {
        if (in_tile[b]) {
            P.ubits[nu] = (uint8_t)b;
            P.ypos[nu] = (uint8_t)inv[b];
            nu++;
        } else {
            P.fx[nf] = (uint8_t)b;
            P.fy[nf] = (uint8_t)inv[b];
            nf++;
        }
    }
    P.nfree = nf;
    // swizzle: the tile bits carrying destination bits 0..4 vary across a warp's shared-memory loads; each of
    // them above bit 4 is XORed onto a low bit (0..4) that none of the others occupies
    for (int b = 0; b < REMAP_TB; b++) P.swz[b] = -1;
    bool low_used[REMAP_RUN] = {false};
    int hi[REMAP_RUN], nhi = 0;
    for (int j = 0; j < REMAP_RUN; j++) {
        int tb = -1;
        for (int i = 0; i < nu; i++)
            if (P.ubits[i] == perm[j]) tb = i;
        if (tb < REMAP_RUN) low_used[tb] = true;
        else hi[nhi++] = tb;
    }
    for (int h = 0, slot = 0; h < nhi; h++) {
        while (low_used[slot]) slot++;
        P.swz[hi[h]] = (int8_t)slot;
        low_used[slot] = true;
    }
    const int64_t ntiles = 1ll << nf;
    int64_t grid = (int64_t)nsm * 3;
    if (grid > ntiles) grid = ntiles;
    const unsigned g = (unsigned)grid;
    if (tbits == REMAP_TB) {
        if (dtype) dev::remap_kernel<double2, REMAP_TB><<<g, REMAP_THREADS, 0, stream>>>((const double2 *)src, (double2 *)dst, P);
        else dev::remap_kernel<float2, REMAP_TB><<<g, REMAP_THREADS, 0, stream>>>((const float2 *)src, (float2 *)dst, P);
    } else {                                  // a 10-qubit state is one tile of 2^10
        if (dtype) dev::remap_kernel<double2, 10><<<g, REMAP_THREADS, 0, stream>>>((const double2 *)src, (double2 *)dst, P);
        else dev::remap_kernel<float2, 10><<<g, REMAP_THREADS, 0, stream>>>((const float2 *)src, (float2 *)dst, P);
    }
    return cudaGetLastError();
}

cudaError_t launch_copy_probe(void *dst, const void *src, size_t bytes, int nsm, cudaStream_t stream) {
    const int64_t n16 = (int64_t)(bytes / 16);
    int64_t grid = (int64_t)nsm * 4;
    if (grid > (n16 + 511) / 512) grid = (n16 + 511) / 512;
    if (grid < 1) grid = 1;
    dev::copy_probe_kernel<<<(unsigned)grid, 512, 0, stream>>>((const float4 *)src, (float4 *)dst, n16);
    return cudaGetLastError();
}

cudaError_t launch_set_amp0(void *state, int dtype, cudaStream_t stream) {
    if (dtype) dev::set_amp0_kernel_d<<<1, 1, 0, stream>>>((double2 *)state);
    else dev::set_amp0_kernel<<<1, 1, 0, stream>>>((float2 *)state);
    return cudaGetLastError();
}

constexpr int reduce_bits_of(int n) {
    int B = n - 10;
    if (B < 13) B = 13;
    if (B > n) B = n;
    if (B > 25) B = 25;
    return B;
}
int reduce_bits(int n) { return reduce_bits_of(n); }

size_t reduce_scratch_bytes(int n, int chunk_bits) {
    const int B = reduce_bits(n);
    const size_t red = ((size_t)1 << (n - B)) * (B + 1) * sizeof(double);
    const size_t smp = ((size_t)1 << (n - chunk_bits)) * sizeof(double);
    return red > smp ? red : smp;
}

cudaError_t launch_reduce(const void *state, int n, int dtype, double *out, void *scratch, cudaStream_t stream) {
    const int B = reduce_bits(n);
    const int nblocks = 1 << (n - B);
    double *partials = (double *)scratch;
    if (dtype) dev::reduce_block_kernel<double2><<<nblocks, RED_THREADS, 0, stream>>>((const double2 *)state, B, partials);
    else dev::reduce_block_kernel<float2><<<nblocks, RED_THREADS, 0, stream>>>((const float2 *)state, B, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dev::reduce_final_kernel<<<1, 64, 0, stream>>>(partials, nblocks, B, n, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- reduction without caller scratch
// Fixed-size scratch for reduce_f64_noalloc: a 2^n state needs 2^(n-B) * (B+1) doubles of block partials
// (B = reduce_bits(n)); the largest supported state (n = 34, B = 24) needs 1024 * 25 = 25600. The array
// holds 32768 doubles (256 KiB). It is part of the module image, so every GPU that loads the library keeps
// it until the process exits. The partial count does not depend on the amplitude type.
#define QSV_NOALLOC_REDUCE_DOUBLES 32768
#define QSV_NOALLOC_N_MIN 10
#define QSV_NOALLOC_N_MAX 34
static __device__ __align__(256) double g_noalloc_reduce_scratch[QSV_NOALLOC_REDUCE_DOUBLES];

constexpr long long noalloc_partials(int n) { return (1ll << (n - reduce_bits_of(n))) * (reduce_bits_of(n) + 1); }
constexpr bool noalloc_fits_every_n() {
    for (int n = QSV_NOALLOC_N_MIN; n <= QSV_NOALLOC_N_MAX; n++)
        if (noalloc_partials(n) > QSV_NOALLOC_REDUCE_DOUBLES) return false;
    return true;
}
static_assert(noalloc_fits_every_n(), "the fixed reduction scratch must hold the partials of every supported n");

size_t noalloc_reduce_capacity() { return QSV_NOALLOC_REDUCE_DOUBLES * sizeof(double); }

// Device address of the fixed scratch for the current device. Looked up once per device (the host-side
// name of the array is only a stand-in for it, never a device address) and cached for the life of the
// process: the cache assumes the device's primary context is not reset (cudaDeviceReset) while the library
// is loaded, since a reset unloads the module and the cached address would then be stale.
static cudaError_t noalloc_scratch_ptr(double **out) {
    static std::mutex mu;
    static double *ptr[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    if (!ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_reduce_scratch);
        if (e != cudaSuccess) return e;
        ptr[dev] = static_cast<double *>(p);
    }
    *out = ptr[dev];
    return cudaSuccess;
}

cudaError_t launch_reduce_noalloc(const void *state, int n, int dtype, double *out, cudaStream_t stream,
                                  size_t *need) {
    const size_t doubles = (size_t)noalloc_partials(n);
    *need = doubles * sizeof(double);
    if (doubles > QSV_NOALLOC_REDUCE_DOUBLES) return cudaErrorInvalidValue;
    double *scratch = nullptr;
    cudaError_t e = noalloc_scratch_ptr(&scratch);
    if (e != cudaSuccess) return e;
    return launch_reduce(state, n, dtype, out, scratch, stream);
}

cudaError_t launch_chunk_probs(const void *state, int n, int dtype, int cb, double *out, cudaStream_t stream) {
    const unsigned nc = (unsigned)(1ll << (n - cb));
    if (dtype) dev::chunk_probs_kernel<double2><<<nc, RED_THREADS, 0, stream>>>((const double2 *)state, cb, out);
    else dev::chunk_probs_kernel<float2><<<nc, RED_THREADS, 0, stream>>>((const float2 *)state, cb, out);
    return cudaGetLastError();
}

cudaError_t launch_sample(const void *state, int n, int dtype, int cb, const double *uni, int shots, int64_t *out,
                          void *scratch, cudaStream_t stream) {
    double *cdf = (double *)scratch;
    const int64_t nc = 1ll << (n - cb);
    cudaError_t e0 = launch_chunk_probs(state, n, dtype, cb, cdf, stream);
    if (e0 != cudaSuccess) return e0;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dev::scan_kernel<<<1, 1024, 0, stream>>>(cdf, nc);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (shots > 0) {
        if (dtype)
            dev::sample_kernel<double2><<<(shots + 127) / 128, 128, 0, stream>>>((const double2 *)state, cb, cdf, nc, uni,
                                                                                 shots, out);
        else
            dev::sample_kernel<float2><<<(shots + 127) / 128, 128, 0, stream>>>((const float2 *)state, cb, cdf, nc, uni,
                                                                                shots, out);
    }
    return cudaGetLastError();
}

}  // namespace qsv
