// qsv_capi.cu -- the extern "C" boundary of libqsv_b200.so (declared in include/qsv_b200.h).
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/qsv_b200.h"
#include "qsv_planner.h"

namespace qsv {
cudaError_t launch_sweep(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream);
int set_interp(int mode);
cudaError_t launch_sweep_c128(double2 *state, const QsvSweepD &sw, int nsm, cudaStream_t stream);
cudaError_t launch_remap(const void *src, void *dst, int n, const int32_t *perm, int dtype, int nsm,
                         cudaStream_t stream);
cudaError_t launch_set_amp0(void *state, int dtype, cudaStream_t stream);
cudaError_t launch_copy_probe(void *dst, const void *src, size_t bytes, int nsm, cudaStream_t stream);
cudaError_t launch_reduce(const void *state, int n, int dtype, double *out, void *scratch, cudaStream_t stream);
cudaError_t launch_chunk_probs(const void *state, int n, int dtype, int cb, double *out, cudaStream_t stream);
cudaError_t launch_sample(const void *state, int n, int dtype, int cb, const double *uni, int shots, int64_t *out,
                          void *scratch, cudaStream_t stream);
size_t reduce_scratch_bytes(int n, int chunk_bits);
cudaError_t take_device_status(int *out);
struct Batch;
Batch *batch_new();
void batch_free(Batch *b);
int batch_add(Batch *b, void *state, int n, int nseg, const int32_t *const *segs, const size_t *nwords, std::string &err);
size_t batch_workspace_bytes(Batch *b);
cudaError_t batch_upload(Batch *b, void *ws, cudaStream_t stream);
cudaError_t batch_launch(Batch *b, void *ws, int nsm, cudaStream_t stream, int *launches);
cudaError_t launch_reduce_noalloc(const void *state, int n, int dtype, double *out, cudaStream_t stream, size_t *need);
size_t noalloc_reduce_capacity();
int jit_set_mode(int mode);
int jit_prepare(const std::vector<QsvSweep> &sweeps);
int jit_prepare_library(const std::vector<QsvSweep> &sweeps);
void jit_wait();
int jit_info(long long *out, int cap);
std::string jit_last_log();
int jit_try_launch(float2 *state, const QsvSweep &sw, int nsm, cudaStream_t stream, cudaError_t *err);
}  // namespace qsv

static std::atomic<unsigned> g_wait_us{0};     // bounded-wait limit of the sweep kernels (0: 2 s default)
static std::atomic<int> g_inject_skip{0};      // fault injection: sweep launches left that skip a tile load

// one armed fault injection, if any (consumed by the launch that takes it)
static int take_injection() {
    int c = g_inject_skip.load();
    while (c > 0 && !g_inject_skip.compare_exchange_weak(c, c - 1)) {
    }
    return c > 0 ? 1 : 0;
}

static thread_local std::string t_err;
static thread_local long long t_launches = 0;
static std::mutex g_launch_mu;         // serialises first-use kernel attribute setup
static int g_lo_merge = 4;             // merged sweeps keep sub-blocks of >= 2^4 amplitudes (128 B)

static const int QSV_CHUNK_BITS = 12;  // sampler chunk: 2^12 amplitudes (host/sv/runtime.py:47 chunk_bits=12)
static int chunk_bits_for(int n) { return n < QSV_CHUNK_BITS ? n : QSV_CHUNK_BITS; }
static bool dtype_ok(int dtype) { return dtype == QSV_C64 || dtype == QSV_C128; }
static size_t amp_bytes(int dtype) { return dtype == QSV_C128 ? 16 : 8; }
static const int QSV_N_MIN = 10;
static const int QSV_N_MAX = 34;

static int fail(int code, const std::string &msg) {
    t_err = msg;
    return code;
}
static int cuda_fail(cudaError_t e, const char *what) {
    return fail(QSV_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
static int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cached[dev] = v;
    }
    return cached[dev];
}

extern "C" {

int qsv_version(void) { return 100; }

const char *qsv_last_error(void) { return t_err.c_str(); }

int qsv_set_lo_merge(int lo) {
    if (lo < QSV_LO_MIN || lo > 13) return fail(QSV_ERR_INVALID_ARG, "lo_merge out of [3, 13]");
    g_lo_merge = lo;
    return QSV_OK;
}

int qsv_set_layout13(int rb) {
    if (qsv::set_rb13(rb)) return fail(QSV_ERR_INVALID_ARG, "13-qubit layout takes 3 or 4 register bits");
    return QSV_OK;
}

int qsv_set_interp(int mode) {
    const int prev = qsv::set_interp(mode);
    if (prev < 0) return fail(QSV_ERR_INVALID_ARG, "interpreter mode must be 0 (phase layouts) or 1 (streaming)");
    return prev;
}

int qsv_set_phase_lanes(int k) {
    if (qsv::set_phase_lanes(k)) return fail(QSV_ERR_INVALID_ARG, "phase lane targets must be 0, 1 or 2");
    return QSV_OK;
}

int qsv_set_wait_limit_us(unsigned int us) {
    g_wait_us.store(us);
    return QSV_OK;
}

int qsv_inject_skip_load(int count) {
    if (count < 0) return fail(QSV_ERR_INVALID_ARG, "count must be >= 0");
    g_inject_skip.store(count);
    return QSV_OK;
}

int qsv_plan_segment(const int32_t *seg, size_t nwords, int n, int32_t *out, size_t cap) {
    if (n < QSV_N_MIN || n > QSV_N_MAX) return fail(QSV_ERR_INVALID_ARG, "n out of [10, 34]");
    std::vector<qsv::PhysPass> passes;
    std::string err;
    int rc = qsv::decode_segment(seg, nwords, n, passes, err);
    if (rc) return fail(rc, err);
    std::vector<QsvSweep> sweeps;
    const int kw = n < QSV_KW_MAX ? n : QSV_KW_MAX;
    rc = qsv::build_sweeps<QsvOp>(passes, n, kw, g_lo_merge, sweeps, err);
    if (rc) return fail(rc, err);
    return qsv::serialize(sweeps, out, cap);
}

int qsv_plan_stream(const int32_t *seg, size_t nwords, int n, int32_t *out, size_t cap) {
    if (n < QSV_N_MIN || n > QSV_N_MAX) return fail(QSV_ERR_INVALID_ARG, "n out of [10, 34]");
    std::vector<qsv::PhysPass> passes;
    std::string err;
    int rc = qsv::decode_segment(seg, nwords, n, passes, err);
    if (rc) return fail(rc, err);
    std::vector<QsvSweep> sweeps;
    const int kw = n < QSV_KW_MAX ? n : QSV_KW_MAX;
    rc = qsv::build_sweeps<QsvOp>(passes, n, kw, g_lo_merge, sweeps, err);
    if (rc) return fail(rc, err);
    for (QsvSweep &sw : sweeps) {
        rc = qsv::plan_stream(sw, err);
        if (rc) return fail(rc, err);
    }
    return qsv::serialize_stream(sweeps, out, cap);
}

int qsv_run_segment(void *state, int n, const int32_t *seg, size_t nwords, int dtype, void *stream) {
    if (!state) return fail(QSV_ERR_INVALID_ARG, "state is null");
    if (!dtype_ok(dtype)) return fail(QSV_ERR_UNSUPPORTED, "dtype must be QSV_C64 or QSV_C128");
    if (n < QSV_N_MIN || n > QSV_N_MAX) return fail(QSV_ERR_INVALID_ARG, "n out of [10, 34]");
    std::vector<qsv::PhysPass> passes;
    std::string err;
    int rc = qsv::decode_segment(seg, nwords, n, passes, err, dtype);
    if (rc) return fail(rc, err);
    const int nsm = sm_count();
    if (dtype == QSV_C128) {
        std::vector<QsvSweepD> sweeps;
        const int kw = n < 12 ? n : 12;
        rc = qsv::build_sweeps<QsvOpD>(passes, n, kw, g_lo_merge, sweeps, err);
        if (rc) return fail(rc, err);
        std::lock_guard<std::mutex> lk(g_launch_mu);
        for (QsvSweepD &sw : sweeps) {
            sw.wait_us = g_wait_us.load();
            sw.skip_load = take_injection();
            cudaError_t e = qsv::launch_sweep_c128((double2 *)state, sw, nsm, (cudaStream_t)stream);
            if (e != cudaSuccess) return cuda_fail(e, "complex128 sweep launch");
            t_launches++;
        }
        return QSV_OK;
    }
    std::vector<QsvSweep> sweeps;
    const int kw = n < QSV_KW_MAX ? n : QSV_KW_MAX;
    rc = qsv::build_sweeps<QsvOp>(passes, n, kw, g_lo_merge, sweeps, err);
    if (rc) return fail(rc, err);
    std::lock_guard<std::mutex> lk(g_launch_mu);
    for (QsvSweep &sw : sweeps) {
        sw.wait_us = g_wait_us.load();
        sw.skip_load = take_injection();
        cudaError_t e = cudaSuccess;
        const int r = qsv::jit_try_launch((float2 *)state, sw, nsm, (cudaStream_t)stream, &e);
        if (r < 0) return cuda_fail(e, "specialised sweep launch");
        if (r == 0) {
            e = qsv::launch_sweep((float2 *)state, sw, nsm, (cudaStream_t)stream);
            if (e != cudaSuccess) return cuda_fail(e, "sweep launch");
        }
        t_launches++;
    }
    return QSV_OK;
}

int qsv_set_jit(int mode) {
    const int old = qsv::jit_set_mode(mode);
    if (old < 0) return fail(QSV_ERR_INVALID_ARG, "jit mode must be 0, 1, 2, 3 or 4");
    return old;
}

int qsv_jit_prepare(const int32_t *seg, size_t nwords, int n) {
    if (n < QSV_N_MIN || n > QSV_N_MAX) return fail(QSV_ERR_INVALID_ARG, "n out of [10, 34]");
    std::vector<qsv::PhysPass> passes;
    std::string err;
    int rc = qsv::decode_segment(seg, nwords, n, passes, err);
    if (rc) return fail(rc, err);
    std::vector<QsvSweep> sweeps;
    const int kw = n < QSV_KW_MAX ? n : QSV_KW_MAX;
    rc = qsv::build_sweeps<QsvOp>(passes, n, kw, g_lo_merge, sweeps, err);
    if (rc) return fail(rc, err);
    const int ready = qsv::jit_prepare(sweeps);
    const std::string log = qsv::jit_last_log();
    if (!log.empty()) t_err = log;
    return ready;
}

int qsv_jit_prepare_library(const int32_t *const *segs, const size_t *nwords, const int *ns, int count) {
    if (count < 0 || (count > 0 && (!segs || !nwords || !ns))) return fail(QSV_ERR_INVALID_ARG, "null segment list");
    std::vector<QsvSweep> all;
    for (int i = 0; i < count; i++) {
        const int n = ns[i];
        if (n < QSV_N_MIN || n > QSV_N_MAX) return fail(QSV_ERR_INVALID_ARG, "n out of [10, 34]");
        std::vector<qsv::PhysPass> passes;
        std::string err;
        int rc = qsv::decode_segment(segs[i], nwords[i], n, passes, err);
        if (rc) return fail(rc, err);
        std::vector<QsvSweep> sweeps;
        const int kw = n < QSV_KW_MAX ? n : QSV_KW_MAX;
        rc = qsv::build_sweeps<QsvOp>(passes, n, kw, g_lo_merge, sweeps, err);
        if (rc) return fail(rc, err);
        all.insert(all.end(), sweeps.begin(), sweeps.end());
    }
    const int types = qsv::jit_prepare_library(all);
    if (types < 0) return fail(QSV_ERR_CUDA, "group-type library failed to compile: " + qsv::jit_last_log());
    return types;
}

int qsv_jit_wait(void) {
    qsv::jit_wait();
    return QSV_OK;
}

int qsv_jit_info(long long *out, int cap) {
    if (!out || cap < 0) return fail(QSV_ERR_INVALID_ARG, "null output");
    return qsv::jit_info(out, cap);
}

int qsv_remap(const void *src, void *dst, int n, const int32_t *perm, int dtype, void *stream) {
    if (!src || !dst || !perm) return fail(QSV_ERR_INVALID_ARG, "null pointer");
    if (!dtype_ok(dtype)) return fail(QSV_ERR_UNSUPPORTED, "dtype must be QSV_C64 or QSV_C128");
    if (n < QSV_N_MIN || n > QSV_N_MAX) return fail(QSV_ERR_INVALID_ARG, "n out of [10, 34]");
    if (src == dst) return fail(QSV_ERR_INVALID_ARG, "remap is out of place: src == dst");
    bool seen[64] = {false};
    for (int j = 0; j < n; j++) {
        if (perm[j] < 0 || perm[j] >= n || seen[perm[j]]) return fail(QSV_ERR_INVALID_ARG, "perm is not a permutation");
        seen[perm[j]] = true;
    }
    cudaError_t e = qsv::launch_remap(src, dst, n, perm, dtype, sm_count(), (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "remap launch");
    t_launches++;
    return QSV_OK;
}

int qsv_zero_state(void *state, int n, int dtype, void *stream) {
    if (!state) return fail(QSV_ERR_INVALID_ARG, "state is null");
    if (!dtype_ok(dtype)) return fail(QSV_ERR_UNSUPPORTED, "dtype must be QSV_C64 or QSV_C128");
    if (n < 1 || n > QSV_N_MAX) return fail(QSV_ERR_INVALID_ARG, "n out of range");
    cudaError_t e = cudaMemsetAsync(state, 0, amp_bytes(dtype) << n, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "memset");
    e = qsv::launch_set_amp0(state, dtype, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "init launch");
    t_launches++;
    return QSV_OK;
}

size_t qsv_reduce_scratch_bytes(int n) {
    if (n < QSV_N_MIN || n > QSV_N_MAX) return 0;
    return qsv::reduce_scratch_bytes(n, chunk_bits_for(n));
}

int qsv_reduce_f64(const void *state, int n, int dtype, double *out_dev, void *scratch, size_t scratch_bytes,
                   void *stream) {
    if (!state || !out_dev || !scratch) return fail(QSV_ERR_INVALID_ARG, "null pointer");
    if (!dtype_ok(dtype)) return fail(QSV_ERR_UNSUPPORTED, "dtype must be QSV_C64 or QSV_C128");
    if (n < QSV_N_MIN || n > QSV_N_MAX) return fail(QSV_ERR_INVALID_ARG, "n out of [10, 34]");
    if (scratch_bytes < qsv_reduce_scratch_bytes(n)) return fail(QSV_ERR_SCRATCH, "scratch too small");
    cudaError_t e = qsv::launch_reduce(state, n, dtype, out_dev, scratch, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "reduce launch");
    t_launches += 2;
    return QSV_OK;
}

int qsv_reduce_f64_noalloc(const void *state, int n, int dtype, double *out_dev, void *stream) {
    if (!state || !out_dev) return fail(QSV_ERR_INVALID_ARG, "null pointer");
    if (!dtype_ok(dtype)) return fail(QSV_ERR_UNSUPPORTED, "dtype must be QSV_C64 or QSV_C128");
    if (n < QSV_N_MIN || n > QSV_N_MAX)
        return fail(QSV_ERR_INVALID_ARG, "n out of [10, 34] for the fixed-scratch reduction");
    size_t need = 0;
    cudaError_t e = qsv::launch_reduce_noalloc(state, n, dtype, out_dev, (cudaStream_t)stream, &need);
    if (need > qsv::noalloc_reduce_capacity())
        return fail(QSV_ERR_SCRATCH, "state needs " + std::to_string(need) + " B of block partials, fixed scratch holds " +
                                         std::to_string(qsv::noalloc_reduce_capacity()) + " B");
    if (e != cudaSuccess) return cuda_fail(e, "fixed-scratch reduce");
    t_launches += 2;
    return QSV_OK;
}

int qsv_chunk_probs_f64(const void *state, int n, int dtype, int chunk_bits, double *out_dev, void *stream) {
    if (!state || !out_dev) return fail(QSV_ERR_INVALID_ARG, "null pointer");
    if (!dtype_ok(dtype)) return fail(QSV_ERR_UNSUPPORTED, "dtype must be QSV_C64 or QSV_C128");
    if (n < QSV_N_MIN || n > QSV_N_MAX || chunk_bits < 0 || chunk_bits > n)
        return fail(QSV_ERR_INVALID_ARG, "n or chunk_bits out of range");
    cudaError_t e = qsv::launch_chunk_probs(state, n, dtype, chunk_bits, out_dev, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "chunk launch");
    t_launches++;
    return QSV_OK;
}

int qsv_sample_f64(const void *state, int n, int dtype, const double *uniforms_dev, int shots, int64_t *out_dev,
                   void *scratch, size_t scratch_bytes, void *stream) {
    if (!state || !scratch || (shots > 0 && (!uniforms_dev || !out_dev))) return fail(QSV_ERR_INVALID_ARG, "null pointer");
    if (!dtype_ok(dtype)) return fail(QSV_ERR_UNSUPPORTED, "dtype must be QSV_C64 or QSV_C128");
    if (n < QSV_N_MIN || n > QSV_N_MAX || shots < 0) return fail(QSV_ERR_INVALID_ARG, "n or shots out of range");
    if (scratch_bytes < qsv_reduce_scratch_bytes(n)) return fail(QSV_ERR_SCRATCH, "scratch too small");
    cudaError_t e = qsv::launch_sample(state, n, dtype, chunk_bits_for(n), uniforms_dev, shots, out_dev, scratch,
                                       (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "sample launch");
    t_launches += 3;
    return QSV_OK;
}

int qsv_hbm_copy(void *dst, const void *src, size_t bytes, void *stream) {
    if (!dst || !src) return fail(QSV_ERR_INVALID_ARG, "null pointer");
    if (bytes % 16 || ((uintptr_t)dst % 16) || ((uintptr_t)src % 16))
        return fail(QSV_ERR_INVALID_ARG, "copy probe needs 16-byte aligned buffers and a multiple of 16 bytes");
    const char *d = (const char *)dst, *s = (const char *)src;
    if (d < s + bytes && s < d + bytes) return fail(QSV_ERR_INVALID_ARG, "copy probe buffers overlap");
    cudaError_t e = qsv::launch_copy_probe(dst, src, bytes, sm_count(), (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "copy probe launch");
    t_launches++;
    return QSV_OK;
}

int qsv_device_status(int *status) {
    if (!status) return fail(QSV_ERR_INVALID_ARG, "null pointer");
    int v = 0;
    cudaError_t e = qsv::take_device_status(&v);
    if (e != cudaSuccess) return cuda_fail(e, "device status");
    *status = v;
    return QSV_OK;
}

struct qsv_batch {
    qsv::Batch *impl;
};

qsv_batch *qsv_batch_new(void) {
    qsv_batch *b = new (std::nothrow) qsv_batch;
    if (!b) { fail(QSV_ERR_INVALID_ARG, "out of host memory"); return nullptr; }
    b->impl = qsv::batch_new();
    return b;
}

void qsv_batch_free(qsv_batch *b) {
    if (!b) return;
    qsv::batch_free(b->impl);
    delete b;
}

int qsv_batch_add(qsv_batch *b, void *state, int n, int nseg, const int32_t *const *segs, const size_t *nwords) {
    if (!b || !state || (nseg > 0 && (!segs || !nwords)) || nseg < 0) return fail(QSV_ERR_INVALID_ARG, "null pointer");
    std::string err;
    int rc = qsv::batch_add(b->impl, state, n, nseg, segs, nwords, err);
    if (rc) return fail(rc, err);
    return QSV_OK;
}

size_t qsv_batch_workspace_bytes(qsv_batch *b) { return b ? qsv::batch_workspace_bytes(b->impl) : 0; }

int qsv_batch_upload(qsv_batch *b, void *workspace, size_t bytes, void *stream) {
    if (!b || !workspace) return fail(QSV_ERR_INVALID_ARG, "null pointer");
    if (bytes < qsv::batch_workspace_bytes(b->impl)) return fail(QSV_ERR_SCRATCH, "batch workspace too small");
    cudaError_t e = qsv::batch_upload(b->impl, workspace, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch upload");
    return QSV_OK;
}

int qsv_batch_launch(qsv_batch *b, void *workspace, size_t bytes, void *stream) {
    if (!b || !workspace) return fail(QSV_ERR_INVALID_ARG, "null pointer");
    if (bytes < qsv::batch_workspace_bytes(b->impl)) return fail(QSV_ERR_SCRATCH, "batch workspace too small");
    int launches = 0;
    std::lock_guard<std::mutex> lk(g_launch_mu);
    cudaError_t e = qsv::batch_launch(b->impl, workspace, sm_count(), (cudaStream_t)stream, &launches);
    if (e != cudaSuccess) return cuda_fail(e, "batch launch");
    t_launches += launches;
    return QSV_OK;
}

long long qsv_take_launch_count(void) {
    long long v = t_launches;
    t_launches = 0;
    return v;
}

}  // extern "C"
