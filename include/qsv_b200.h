/*
 * qsv_b200.h -- C ABI of libqsv_b200.so, the B200 (sm_100a) QSV2 statevector engine.
 *
 * The entry points replace the reference's device calls one for one (paths are within the reference
 * project nasir26/u55c-statevector-30q):
 *   qsv_run_segment   <- sv_engine(st, ins_off)            kernels/sv/sv_engine.cpp:302-331,
 *                        launched per slice at host/sv/runtime.py:227-233 (_run_segment)
 *   qsv_remap         <- sv_swap(a, b, offa, offb, nw)     kernels/sv/sv_swap.cpp:10-39 and the host
 *                        exchange of host/sv/runtime.py:235-284 (_swap_bank_local/_swap_local_local/_remap)
 *   qsv_zero_state    <- _zero_segment/_init_zero_state    host/sv/runtime.py:205-217
 *   qsv_chunk_probs_f64, qsv_sample_f64
 *                     <- sample_slices (host Born sampling) host/sv/runtime.py:47-80, moved on device
 *   qsv_reduce_f64    <- the norm check of tests/functional_suite.py:92-94 and the per-qubit <Z>
 *                        outputs of the batched workload; no device counterpart in the reference
 *   qsv_plan_segment  <- model.decode (host/sv/model.py:7-22): exposes how a segment is executed
 *
 * Conventions: every function returns QSV_OK (0) or a negative QSV_ERR_* code and never throws;
 * qsv_last_error() gives a message for the calling thread's last failure. Device pointers are plain
 * CUDA device addresses (the Python runtime passes PyTorch tensor storage); `stream` is a cudaStream_t
 * (NULL = legacy default stream). Calls are asynchronous on `stream` unless stated otherwise; the host
 * arrays they read (segment words, permutations) may be reused as soon as the call returns. The library
 * allocates no device memory on these paths: scratch is passed in by the caller.
 * State layout: 2^n amplitudes, little-endian qubit order (qubit q = index bit q), complex64 as
 * interleaved float32 (re, im) -- the numpy complex64 layout the reference uses (sv_engine.cpp:4-5).
 */
#ifndef QSV_B200_H
#define QSV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define QSV_API __attribute__((visibility("default")))
#else
#define QSV_API
#endif

#define QSV_OK 0
#define QSV_ERR_INVALID_ARG (-1)   /* null pointer, size out of range, bad permutation */
#define QSV_ERR_BAD_STREAM (-2)    /* malformed QSV2 segment (magic, header, record bounds) */
#define QSV_ERR_UNSUPPORTED (-3)   /* well-formed but beyond this engine (window wider than 13 qubits) */
#define QSV_ERR_CUDA (-4)          /* a CUDA runtime call failed; see qsv_last_error() */
#define QSV_ERR_DEVICE (-5)        /* a kernel reported a fault through the device status word */
#define QSV_ERR_SCRATCH (-6)       /* caller-provided scratch smaller than required */

#define QSV_C64 0                  /* complex64 amplitudes (QSV2, fp32 matrices) */
#define QSV_C128 1                 /* complex128 amplitudes (QSV2 with FP64 matrices, header word 4 = 1;
                                      an extension with no reference counterpart: the FPGA engine is
                                      complex64 only). Accepted by run_segment, remap, zero_state,
                                      reduce_f64, reduce_f64_noalloc, chunk_probs_f64 and sample_f64. */

/* Library version (major * 10000 + minor * 100 + patch). */
QSV_API int qsv_version(void);

/* Message of the calling thread's last error ("" if none). */
QSV_API const char *qsv_last_error(void);

/* Execute one QSV2 segment (every pass, in order) on the device state in place.
 * Replaces sv_engine (kernels/sv/sv_engine.cpp:302); `seg` is the host copy of the words the reference
 * runtime uploads behind each slice (host/sv/runtime.py:218-225). The segment's L must equal n.
 * Consecutive passes are merged into sweeps whose qubit window fits the engine's 13-qubit tile (12 for
 * QSV_C128); the result equals pass-by-pass execution value for value. n in [10, 34]. dtype QSV_C128
 * needs a segment with FP64 matrices (header word 4 = 1); a segment of the other element type is
 * rejected with QSV_ERR_BAD_STREAM. */
QSV_API int qsv_run_segment(void *state, int n, const int32_t *seg, size_t nwords, int dtype, void *stream);

/* Qubit permutation, out of place: dst[y] = src[x] with bit j of y = bit perm[j] of x
 * (perm[new_phys] = old_phys, host/sv/model.py:74-78). Replaces the sv_swap exchange and the host
 * remaps of host/sv/runtime.py:235-284 with one in-HBM sweep. src and dst must not overlap. */
QSV_API int qsv_remap(const void *src, void *dst, int n, const int32_t *perm, int dtype, void *stream);

/* |0...0>: zero the state and set amplitude 0 to 1 (host/sv/runtime.py:205-217). */
QSV_API int qsv_zero_state(void *state, int n, int dtype, void *stream);

/* Bytes of scratch the reductions and the sampler need for a 2^n state. */
QSV_API size_t qsv_reduce_scratch_bytes(int n);

/* FP64 reductions over |a_i|^2: out_dev[0] = sum |a_i|^2, out_dev[1 + q] = <Z_q> = sum (1 - 2 bit_q(i))
 * |a_i|^2 for q < n (n + 1 doubles, device memory). */
QSV_API int qsv_reduce_f64(const void *state, int n, int dtype, double *out_dev, void *scratch, size_t scratch_bytes,
                   void *stream);

/* The same FP64 reductions as qsv_reduce_f64 (complex64 or complex128 states), for callers that cannot
 * allocate device memory: code that runs where the device heap belongs to another allocator, or that must
 * keep a fixed footprint once it is running (a long-lived service), or that reaches this library through an
 * FFI with no CUDA allocator of its own. No counterpart in the reference. It takes no scratch argument and
 * allocates nothing: the block partials go to a fixed 256 KiB array compiled into the library (file scope),
 * which every GPU that loads the library holds until the process exits. The array covers every supported
 * size (at most 25,600 doubles, at n = 34); n outside [10, 34] is rejected with QSV_ERR_INVALID_ARG and a
 * message, a dtype other than QSV_C64 / QSV_C128 with QSV_ERR_UNSUPPORTED. The first call on a device looks
 * up the array's device address (once per device, with that device current) and caches it, so make that
 * first call before any stream capture, and do not reset the device (cudaDeviceReset) while the library is
 * loaded. All calls share the one array and it keeps the last call's partials; every call overwrites each
 * partial it reads, so nothing needs clearing, but calls whose kernels overlap on the GPU (two streams, two
 * host threads) race on it: order them on one stream or synchronise between them. */
QSV_API int qsv_reduce_f64_noalloc(const void *state, int n, int dtype, double *out_dev, void *stream);

/* Probability of each chunk of 2^chunk_bits consecutive amplitudes, FP64 (2^(n - chunk_bits) doubles).
 * The first level of the reference's hierarchical sampler (host/sv/runtime.py:59-63). */
QSV_API int qsv_chunk_probs_f64(const void *state, int n, int dtype, int chunk_bits, double *out_dev, void *stream);

/* Born-rule sampling on the device: for each of `shots` uniforms u in [0, 1) (device array), the
 * physical index i with cdf(i-1) <= u * total < cdf(i), cdf in FP64 over chunk sums then within the
 * chosen chunk (the search of host/sv/runtime.py:64-75). Writes int64 indices to out_dev. */
QSV_API int qsv_sample_f64(const void *state, int n, int dtype, const double *uniforms_dev, int shots, int64_t *out_dev,
                   void *scratch, size_t scratch_bytes, void *stream);

/* ---------------------------------------------------------------- batched execution
 * Many small circuits per launch (no reference counterpart: the reference runs one circuit per launch,
 * paper/revised/sections/discussion.tex:8 lists batching as future work). A circuit of n in [10, 13] qubits
 * is one tile: its whole program runs inside one CTA's shared memory, one HBM read and one write per
 * circuit. Build on the host (qsv_batch_new / qsv_batch_add, one call per circuit with all its QSV2
 * segments, L = n each), copy the tables once into a caller-provided device workspace (qsv_batch_upload),
 * then qsv_batch_launch runs every circuit in place on its state (one kernel launch per qubit count
 * present; capturable in a CUDA graph and replayable as long as the states and the workspace stay). */
typedef struct qsv_batch qsv_batch;
QSV_API qsv_batch *qsv_batch_new(void);
QSV_API void qsv_batch_free(qsv_batch *batch);
QSV_API int qsv_batch_add(qsv_batch *batch, void *state, int n, int nseg, const int32_t *const *segs,
                          const size_t *nwords);
QSV_API size_t qsv_batch_workspace_bytes(qsv_batch *batch);
QSV_API int qsv_batch_upload(qsv_batch *batch, void *workspace, size_t bytes, void *stream);
QSV_API int qsv_batch_launch(qsv_batch *batch, void *workspace, size_t bytes, void *stream);

/* Host-side decode of a segment into the sweep plan the engine launches, for inspection and tests.
 * Writes at most `cap` int32 words to `out` (layout in csrc/qsv_plan.h, qsv_plan_serialize) and returns
 * the number of words of the full plan, or a negative error code. Pure host code, no device work. */
QSV_API int qsv_plan_segment(const int32_t *seg, size_t nwords, int n, int32_t *out, size_t cap);

/* The streaming form of the same sweeps (no reference counterpart): how the streaming interpreter and the
 * group-type library run them. Writes at most `cap` int32 words: the sweep count, then per sweep kw,
 * ngroups, nops, per group its three item bits and op range, per op tbit, slot (0 = tile bit 0, 1 + k =
 * item bit k, 7 = a base bit, diagonal ops only), variant, cmask, cm_reg (controls on item bits), cm_thr
 * (controls on base bits), kind. Returns the number of words of the full plan, or a negative error code.
 * Pure host code. */
QSV_API int qsv_plan_stream(const int32_t *seg, size_t nwords, int n, int32_t *out, size_t cap);

/* HBM copy probe: dst <- src, `bytes` (a multiple of 16, 16-byte aligned, not overlapping), a grid-stride
 * 16-byte copy that reads and writes every byte once. The measured achievable-bandwidth denominator for the
 * sweep roofline; the B200 counterpart of the reference's FPGA HBM stream microbenchmark
 * (kernels/hbm_stream/hbm1.cpp:38-60). Asynchronous on `stream`. */
QSV_API int qsv_hbm_copy(void *dst, const void *src, size_t bytes, void *stream);

/* Read and clear the device status word that kernels set when a bounded wait gives up (0 = clean).
 * Synchronous. */
QSV_API int qsv_device_status(int *status);

/* Failure-detection knob (no reference counterpart): every mbarrier wait of the sweep kernels launched after
 * this call gives up after `us` microseconds (0 = the default, 2 s), ORs bit 0 into the device status word,
 * waits (bounded) for its CTA's copies in flight and returns, so a stuck pipeline ends the kernel instead of
 * hanging the GPU. Process-wide. */
QSV_API int qsv_set_wait_limit_us(unsigned int us);

/* Fault injection for tests of that path (no reference counterpart): the next `count` sweep launches of
 * qsv_run_segment have block 0 never issue the load of its first tile, so its waits run out after the wait
 * limit; the kernel then sets status bit 0 and returns with that block's tiles not updated (the state must
 * be rebuilt). count 0 disarms it. A host-side switch: no fault, trap or endless wait is involved. */
QSV_API int qsv_inject_skip_load(int count);

/* Number of kernel launches this thread issued through this library since the last call (and reset
 * the count). No reference counterpart: launch accounting for the benchmark. */
QSV_API long long qsv_take_launch_count(void);

/* Tuning knob (no reference counterpart): merged sweeps keep sub-blocks of at least 2^lo amplitudes
 * contiguous (lo in [3, 13]; default 4 = 128 bytes). Larger values merge fewer passes. Process-wide. */
QSV_API int qsv_set_lo_merge(int lo);

/* Tuning knob (no reference counterpart): consumer layout of the 13-qubit sweep kernel, 4 register bits
 * per thread with 8 consumer warps (default) or 3 with 16. Values are identical either way. */
QSV_API int qsv_set_layout13(int rb);

/* Interpreter kernel for sweeps without a specialised kernel (no reference counterpart): 1 = streaming:
 * the tile stays in shared memory and each group of consecutive ops touching at most three target qubits
 * (plus ops on the lowest tile bit and diagonal ops anywhere) is one pass over it, 16 amplitudes per thread
 * at a time; 0 = phase layouts (default): a thread keeps 32 amplitudes in registers per phase and exchanges
 * lane bits with warp shuffles. Values are identical either way. Returns the previous mode; process-wide. */
QSV_API int qsv_set_interp(int mode);

/* Tuning knob (no reference counterpart): how many op targets a phase may place on lane bits (warp
 * shuffles) instead of starting a new phase, 0..2 (default 1). Values are identical either way. */
QSV_API int qsv_set_phase_lanes(int k);

/* Specialised sweep kernels (no reference counterpart; the reference's engine is one fixed HLS kernel).
 * qsv_run_segment can launch, instead of the interpreter kernel, a kernel compiled at run time (NVRTC,
 * sm_100a) for the sweep's structure: its phase layouts and, per op, target slot, code variant and control
 * masks (everything but the matrices and the window). Values are identical either way.
 * A coarse structure keeps the layouts and, per op, slot, control masks, kind and whether the matrix is a
 * swap; its kernel runs every other op with the dense arithmetic (same values) and serves every sweep of
 * that coarse structure, so sweeps whose exact structure never repeats (random gate choices) still share it.
 * mode 0 = interpreter only; 1 = eager: a new structure is compiled (blocking) before its first launch;
 * 2 = automatic (default): a structure is compiled in background threads once its launches have swept
 * 2^31 amplitudes in total (two sweeps of a 30-qubit state, 512 of a 22-qubit one; at most 64 compilations
 * wait at a time), and used from the first launch after its kernel is ready; until then the sweep runs its
 * coarse structure's kernel, compiled once the sweeps sharing it have swept 2^30 amplitudes, or (13-qubit
 * windows) the group-type library, or the interpreter; 3 = eager with coarse structures only; 4 = the
 * group-type library only (qsv_jit_prepare builds it, blocking, to cover a segment's 13-qubit sweeps).
 * The group-type library is a set of up to 8 kernels, each with straight-line code for 32 op sequences of
 * one group of the streaming form (per op: slot among the group's three item bits, code variant, kind,
 * matrix classes): the 16 that have swept the most amplitudes and a band of 16 more, with item bits,
 * control masks and matrices read at run time. A sweep whose exact and coarse structures never repeat
 * takes the kernel that covers most of its ops, once 3/4 of them fall in its cases; the set is rebuilt in
 * the background after groups outside it have swept 2^31 amplitudes.
 * Switching to mode 0 drops waiting compilations and waits for running ones. Returns the previous mode.
 * Process-wide. */
QSV_API int qsv_set_jit(int mode);

/* Compile, in parallel and blocking, the specialised kernels of every sweep of a segment for an n-qubit
 * state (host work only; no device is touched): exact structures, coarse ones in mode 3, a group-type
 * library covering the segment's 13-qubit sweeps in mode 4. Returns how many of the segment's sweeps have a
 * ready kernel, or a negative error code for a malformed segment. */
QSV_API int qsv_jit_prepare(const int32_t *seg, size_t nwords, int n);

/* Build (blocking, host work only) the group-type library (qsv_set_jit) from the 13-qubit sweeps of count
 * programs (segment i: segs[i], nwords[i] words, for an ns[i]-qubit state): their group types' swept
 * amplitudes are recorded and the libraries take the most swept types seen so far (up to 144). A batch or a service
 * calls it once before its timed or latency-bound work. Returns the number of types in the library, or a
 * negative error code (malformed segment; QSV_ERR_CUDA if the library does not compile). */
QSV_API int qsv_jit_prepare_library(const int32_t *const *segs, const size_t *nwords, const int *ns, int count);

/* Block until every queued background compilation has finished. */
QSV_API int qsv_jit_wait(void);

/* Counters of the specialised-kernel cache, written to out[0 .. min(cap, 12)): mode, structures seen
 * (exact and coarse), kernels ready, compilations failed, sweeps launched specialised (exact or coarse),
 * sweeps launched interpreted, total compile milliseconds, compilations queued or running, sweeps launched
 * with a coarse structure's kernel, coarse structures seen, sweeps launched with the group-type library,
 * group types in the library in use. Returns 12. */
QSV_API int qsv_jit_info(long long *out, int cap);

#ifdef __cplusplus
}
#endif
#endif /* QSV_B200_H */
