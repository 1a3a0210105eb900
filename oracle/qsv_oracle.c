/*
 * qsv_oracle.c -- CPU restatement of the QSV2 engine, used as TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker for the CUDA engine; nothing on the product path links or calls it. Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark load it.
 *
 * Semantics follow the reference's golden model (host/sv/model.py):
 *   decode             model.py:7-22     stream header / pass header / MUX2 records
 *   tile addressing    model.py:25-40    tile t base = pdep(t, free bits); tile element j ->
 *                                        low bits of j | high bit i of j at physical h_i
 *   apply_op_tile      model.py:43-56    pair (i0, i0|1<<t) uses M1 iff cmask && (i0 & cmask) == cmask
 *   run_segment        model.py:59-71    passes in order, every tile independent
 *   remap / unpermute  model.py:74-84    perm[new] = old on index bits
 * The arithmetic of one pair update is written as an explicit fused-multiply-add chain, the canonical
 * order that the CUDA engine uses too, so the two agree value for value (the numpy model rounds each
 * complex product separately and agrees with both to float32 rounding):
 *   y0.re = fma(m00.re, x0.re, fma(-m00.im, x0.im, fma(m01.re, x1.re, -(m01.im * x1.im))))
 *   y0.im = fma(m00.re, x0.im, fma( m00.im, x0.re, fma(m01.re, x1.im,   m01.im * x1.re)))
 *   y1.re = fma(m11.re, x1.re, fma(-m11.im, x1.im, fma(m10.re, x0.re, -(m10.im * x0.im))))
 *   y1.im = fma(m11.re, x1.im, fma( m11.im, x1.re, fma(m10.re, x0.im,   m10.im * x0.re)))
 * Also here: an FP64 dense gate-by-gate simulator (the "Qiskit-style statevector" oracle) and FP64
 * reductions used to check the device reductions, and the complex128 engine (streams with header word
 * 4 = 1 carry FP64 matrices, 40-word op records; same addressing, the same chain in double precision).
 *
 * Build: gcc -O2 -fPIC -shared -fopenmp -ffp-contract=off (see oracle/Makefile).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define QSV_MAGIC 0x51535632
#define HDR_WORDS 8
#define PASS_WORDS 8
#define OP_WORDS 24
#define OP_WORDS_C128 40

typedef struct { float re, im; } c64;

static inline float f_of(int32_t w) { float f; memcpy(&f, &w, 4); return f; }

/* one pair update with matrix m[8] = m00 m01 m10 m11 (re, im), canonical fma order */
static inline void pair_update(const float *m, c64 *a, c64 *b) {
    const float x0r = a->re, x0i = a->im, x1r = b->re, x1i = b->im;
    const float y0r = fmaf(m[0], x0r, fmaf(-m[1], x0i, fmaf(m[2], x1r, -(m[3] * x1i))));
    const float y0i = fmaf(m[0], x0i, fmaf(m[1], x0r, fmaf(m[2], x1i, m[3] * x1r)));
    const float y1r = fmaf(m[6], x1r, fmaf(-m[7], x1i, fmaf(m[4], x0r, -(m[5] * x0i))));
    const float y1i = fmaf(m[6], x1i, fmaf(m[7], x1r, fmaf(m[4], x0i, m[5] * x0r)));
    a->re = y0r; a->im = y0i; b->re = y1r; b->im = y1i;
}

/* Validates a segment of element type dtype (0 = complex64, 1 = complex128); returns the number of
 * passes or a negative code. */
static int check_segment_dt(const int32_t *seg, int64_t nwords, int n, int dtype) {
    const int opw = dtype ? OP_WORDS_C128 : OP_WORDS;
    if (nwords < HDR_WORDS || seg[0] != QSV_MAGIC) return -1;
    if (seg[4] != dtype) return -9;
    const int L = seg[1], np = seg[2], k = seg[3];
    if (L != n || k < 1 || k > L || np < 0) return -2;
    int64_t pos = HDR_WORDS;
    for (int p = 0; p < np; p++) {
        if (pos + PASS_WORDS > nwords) return -3;
        const int m = seg[pos], nops = seg[pos + 3];
        const int h[4] = {seg[pos + 1], seg[pos + 2], seg[pos + 4], seg[pos + 5]};
        if (m < 0 || m > 4 || m > k || nops < 0 || nops > 64) return -4;
        for (int i = 0; i < m; i++) {
            if (h[i] < k - m || h[i] >= L) return -5;
            for (int j = 0; j < i; j++) if (h[j] == h[i]) return -5;
        }
        pos += PASS_WORDS;
        for (int o = 0; o < nops; o++) {
            if (pos + opw > nwords) return -3;
            if (seg[pos] != 1) return -6;
            const int t = seg[pos + 1];
            const uint32_t cm = (uint32_t)seg[pos + 2];
            if (t < 0 || t >= k) return -7;
            if (k < 32 && (cm >> k)) return -7;
            pos += opw;
        }
    }
    if (pos != nwords) return -8;
    return np;
}

/* Validates a complex64 segment; returns number of passes or a negative code. */
int qsv_oracle_check_segment(const int32_t *seg, int64_t nwords, int n) {
    return check_segment_dt(seg, nwords, n, 0);
}

/* Execute one QSV2 segment on a complex64 state of 2^n amplitudes in place (model.py:59-71, P = 1). */
int qsv_oracle_run_segment(float *state, int n, const int32_t *seg, int64_t nwords, int nthreads) {
    const int np = qsv_oracle_check_segment(seg, nwords, n);
    if (np < 0) return np;
    const int L = seg[1], k = seg[3];
    c64 *st = (c64 *)state;
    int64_t pos = HDR_WORDS;
    for (int p = 0; p < np; p++) {
        const int m = seg[pos], nops = seg[pos + 3];
        const int h[4] = {seg[pos + 1], seg[pos + 2], seg[pos + 4], seg[pos + 5]};
        const int32_t *ops = seg + pos + PASS_WORDS;
        pos += PASS_WORDS + (int64_t)nops * OP_WORDS;
        const int low = k - m;
        /* free bits: every local bit that is neither in the low window nor a high qubit */
        int free_bits[64], nfree = 0;
        for (int b = 0; b < L; b++) {
            int used = b < low;
            for (int i = 0; i < m; i++) used |= (b == h[i]);
            if (!used) free_bits[nfree++] = b;
        }
        const int64_t ntiles = (int64_t)1 << nfree, tsize = (int64_t)1 << k;
        /* tile element j -> offset within the tile (independent of the tile) */
        int64_t *off = (int64_t *)malloc(sizeof(int64_t) * tsize);
        for (int64_t j = 0; j < tsize; j++) {
            int64_t o = j & (((int64_t)1 << low) - 1);
            for (int i = 0; i < m; i++) o |= ((j >> (low + i)) & 1) << h[i];
            off[j] = o;
        }
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
        {
            c64 *T = (c64 *)malloc(sizeof(c64) * tsize);
#pragma omp for schedule(static)
            for (int64_t t = 0; t < ntiles; t++) {
                int64_t base = 0;
                for (int i = 0; i < nfree; i++) base |= ((t >> i) & 1) << free_bits[i];
                for (int64_t j = 0; j < tsize; j++) T[j] = st[base | off[j]];
                for (int o = 0; o < nops; o++) {
                    const int32_t *rec = ops + (int64_t)o * OP_WORDS;
                    const int tq = rec[1];
                    const int64_t cm = (uint32_t)rec[2];
                    float M0[8], M1[8];
                    for (int e = 0; e < 8; e++) { M0[e] = f_of(rec[8 + e]); M1[e] = f_of(rec[16 + e]); }
                    const int64_t bit = (int64_t)1 << tq;
                    for (int64_t i0 = 0; i0 < tsize; i0++) {
                        if (i0 & bit) continue;
                        const int sel = cm != 0 && (i0 & cm) == cm;
                        pair_update(sel ? M1 : M0, &T[i0], &T[i0 | bit]);
                    }
                }
                for (int64_t j = 0; j < tsize; j++) st[base | off[j]] = T[j];
            }
            free(T);
        }
        free(off);
    }
    return 0;
}

/* dst[y] = src[x] where bit j of y is bit perm[j] of x (model.py:74-78). Out of place. */
int qsv_oracle_remap(const float *src, float *dst, int n, const int32_t *perm, int nthreads) {
    int seen[64] = {0};
    if (n < 0 || n > 40) return -1;
    for (int j = 0; j < n; j++) {
        if (perm[j] < 0 || perm[j] >= n || seen[perm[j]]) return -2;
        seen[perm[j]] = 1;
    }
    const c64 *s = (const c64 *)src;
    c64 *d = (c64 *)dst;
    const int64_t N = (int64_t)1 << n;
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(static)
    for (int64_t y = 0; y < N; y++) {
        int64_t x = 0;
        for (int j = 0; j < n; j++) x |= ((y >> j) & 1) << perm[j];
        d[y] = s[x];
    }
    return 0;
}

typedef struct { double re, im; } c128;

/* ------------------------------------------------------------------ complex128 engine */

static inline double d_of(const int32_t *w) { double d; memcpy(&d, w, 8); return d; }

/* the canonical chain in double precision */
static inline void pair_update_d(const double *m, c128 *a, c128 *b) {
    const double x0r = a->re, x0i = a->im, x1r = b->re, x1i = b->im;
    const double y0r = fma(m[0], x0r, fma(-m[1], x0i, fma(m[2], x1r, -(m[3] * x1i))));
    const double y0i = fma(m[0], x0i, fma(m[1], x0r, fma(m[2], x1i, m[3] * x1r)));
    const double y1r = fma(m[6], x1r, fma(-m[7], x1i, fma(m[4], x0r, -(m[5] * x0i))));
    const double y1i = fma(m[6], x1i, fma(m[7], x1r, fma(m[4], x0i, m[5] * x0r)));
    a->re = y0r; a->im = y0i; b->re = y1r; b->im = y1i;
}

/* Execute one complex128 segment (header word 4 = 1) on a complex128 state in place. */
int qsv_oracle_run_segment_c128(double *state, int n, const int32_t *seg, int64_t nwords, int nthreads) {
    const int np = check_segment_dt(seg, nwords, n, 1);
    if (np < 0) return np;
    const int L = seg[1], k = seg[3];
    c128 *st = (c128 *)state;
    int64_t pos = HDR_WORDS;
    for (int p = 0; p < np; p++) {
        const int m = seg[pos], nops = seg[pos + 3];
        const int h[4] = {seg[pos + 1], seg[pos + 2], seg[pos + 4], seg[pos + 5]};
        const int32_t *ops = seg + pos + PASS_WORDS;
        pos += PASS_WORDS + (int64_t)nops * OP_WORDS_C128;
        const int low = k - m;
        int free_bits[64], nfree = 0;
        for (int b = 0; b < L; b++) {
            int used = b < low;
            for (int i = 0; i < m; i++) used |= (b == h[i]);
            if (!used) free_bits[nfree++] = b;
        }
        const int64_t ntiles = (int64_t)1 << nfree, tsize = (int64_t)1 << k;
        int64_t *off = (int64_t *)malloc(sizeof(int64_t) * tsize);
        for (int64_t j = 0; j < tsize; j++) {
            int64_t o = j & (((int64_t)1 << low) - 1);
            for (int i = 0; i < m; i++) o |= ((j >> (low + i)) & 1) << h[i];
            off[j] = o;
        }
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
        {
            c128 *T = (c128 *)malloc(sizeof(c128) * tsize);
#pragma omp for schedule(static)
            for (int64_t t = 0; t < ntiles; t++) {
                int64_t base = 0;
                for (int i = 0; i < nfree; i++) base |= ((t >> i) & 1) << free_bits[i];
                for (int64_t j = 0; j < tsize; j++) T[j] = st[base | off[j]];
                for (int o = 0; o < nops; o++) {
                    const int32_t *rec = ops + (int64_t)o * OP_WORDS_C128;
                    const int tq = rec[1];
                    const int64_t cm = (uint32_t)rec[2];
                    double M0[8], M1[8];
                    for (int e = 0; e < 8; e++) { M0[e] = d_of(rec + 8 + 2 * e); M1[e] = d_of(rec + 24 + 2 * e); }
                    const int64_t bit = (int64_t)1 << tq;
                    for (int64_t i0 = 0; i0 < tsize; i0++) {
                        if (i0 & bit) continue;
                        const int sel = cm != 0 && (i0 & cm) == cm;
                        pair_update_d(sel ? M1 : M0, &T[i0], &T[i0 | bit]);
                    }
                }
                for (int64_t j = 0; j < tsize; j++) st[base | off[j]] = T[j];
            }
            free(T);
        }
        free(off);
    }
    return 0;
}

/* complex128 remap: dst[y] = src[x], bit j of y = bit perm[j] of x. */
int qsv_oracle_remap_c128(const double *src, double *dst, int n, const int32_t *perm, int nthreads) {
    const int64_t N = (int64_t)1 << n;
    const c128 *s = (const c128 *)src;
    c128 *d = (c128 *)dst;
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(static)
    for (int64_t y = 0; y < N; y++) {
        int64_t x = 0;
        for (int j = 0; j < n; j++) x |= ((y >> j) & 1) << perm[j];
        d[y] = s[x];
    }
    return 0;
}

/* Apply a dense 2^nq x 2^nq complex128 matrix (row-major, Qiskit little-endian over `qubits`) to the
 * complex128 state of 2^n amplitudes in place. */
/* ------------------------------------------------------------------ FP64 dense oracle */
int qsv_oracle_apply_dense_f64(double *state, int n, const int32_t *qubits, int nq, const double *mat,
                               int nthreads) {
    if (nq < 1 || nq > 12 || nq > n) return -1;
    int64_t qmask = 0;
    for (int i = 0; i < nq; i++) {
        if (qubits[i] < 0 || qubits[i] >= n || (qmask >> qubits[i]) & 1) return -2;
        qmask |= (int64_t)1 << qubits[i];
    }
    int rest[64], nr = 0;
    for (int b = 0; b < n; b++) if (!((qmask >> b) & 1)) rest[nr++] = b;
    const int64_t D = (int64_t)1 << nq, NB = (int64_t)1 << nr;
    int64_t *off = (int64_t *)malloc(sizeof(int64_t) * D);
    for (int64_t j = 0; j < D; j++) {
        int64_t o = 0;
        for (int i = 0; i < nq; i++) o |= ((j >> i) & 1) << qubits[i];
        off[j] = o;
    }
    c128 *st = (c128 *)state;
    const c128 *M = (const c128 *)mat;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        c128 *x = (c128 *)malloc(sizeof(c128) * D);
#pragma omp for schedule(static)
        for (int64_t b = 0; b < NB; b++) {
            int64_t base = 0;
            for (int i = 0; i < nr; i++) base |= ((b >> i) & 1) << rest[i];
            for (int64_t j = 0; j < D; j++) x[j] = st[base | off[j]];
            for (int64_t r = 0; r < D; r++) {
                double yr = 0.0, yi = 0.0;
                for (int64_t c = 0; c < D; c++) {
                    const c128 m = M[r * D + c];
                    yr += m.re * x[c].re - m.im * x[c].im;
                    yi += m.re * x[c].im + m.im * x[c].re;
                }
                st[base | off[r]].re = yr;
                st[base | off[r]].im = yi;
            }
        }
        free(x);
    }
    free(off);
    return 0;
}

/* Fidelity metrics of a complex64 state `sv` against a complex128 reference (same recipe as the
 * reference's bench/fpga/sv_maxwidth_ref.py:15-25): out[0] = |<ref|sv>|^2 / (|ref|^2 |sv|^2),
 * out[1] = 1 - F computed without cancellation as d^2 - d^4/4 (d = l2 distance of the normalised
 * states after optimal global-phase alignment), out[2] = max |delta amp| after alignment,
 * out[3] = |sv| (norm). */
int qsv_oracle_metrics(const double *ref, const float *sv, int64_t N, double *out) {
    const c128 *r = (const c128 *)ref;
    const c64 *s = (const c64 *)sv;
    double nr = 0, ns = 0, ipr = 0, ipi = 0;
#pragma omp parallel for reduction(+ : nr, ns, ipr, ipi) schedule(static)
    for (int64_t i = 0; i < N; i++) {
        const double ar = r[i].re, ai = r[i].im, br = s[i].re, bi = s[i].im;
        nr += ar * ar + ai * ai;
        ns += br * br + bi * bi;
        ipr += ar * br + ai * bi;     /* conj(ref) * sv */
        ipi += ar * bi - ai * br;
    }
    nr = sqrt(nr); ns = sqrt(ns);
    const double ipn_r = ipr / (nr * ns), ipn_i = ipi / (nr * ns);
    const double mag = sqrt(ipn_r * ipn_r + ipn_i * ipn_i);
    const double ph_r = mag > 0 ? ipn_r / mag : 1.0, ph_i = mag > 0 ? ipn_i / mag : 0.0;
    double d2 = 0, mx = 0;
#pragma omp parallel for reduction(+ : d2) reduction(max : mx) schedule(static)
    for (int64_t i = 0; i < N; i++) {
        const double ar = r[i].re / nr, ai = r[i].im / nr;
        const double er = s[i].re / ns - (ph_r * ar - ph_i * ai);
        const double ei = s[i].im / ns - (ph_r * ai + ph_i * ar);
        const double e2 = er * er + ei * ei;
        d2 += e2;
        const double e = sqrt(e2);
        if (e > mx) mx = e;
    }
    out[0] = mag * mag;
    out[1] = d2 - d2 * d2 / 4.0;
    out[2] = mx;
    out[3] = ns;
    return 0;
}

/* FP64 reductions of a complex64 state, the checker for the device reductions:
 * norm2 = sum |a|^2; zexp[q] = sum (1 - 2 bit_q(i)) |a_i|^2 for q < n. */
int qsv_oracle_reduce_f64(const float *sv, int n, double *norm2, double *zexp) {
    const c64 *s = (const c64 *)sv;
    const int64_t N = (int64_t)1 << n;
    double tot = 0;
    for (int q = 0; q < n; q++) zexp[q] = 0;
#pragma omp parallel
    {
        double loc[64] = {0}, lt = 0;
#pragma omp for schedule(static)
        for (int64_t i = 0; i < N; i++) {
            const double p = (double)s[i].re * s[i].re + (double)s[i].im * s[i].im;
            lt += p;
            for (int q = 0; q < n; q++) loc[q] += ((i >> q) & 1) ? -p : p;
        }
#pragma omp critical
        {
            tot += lt;
            for (int q = 0; q < n; q++) zexp[q] += loc[q];
        }
    }
    *norm2 = tot;
    return 0;
}

int qsv_oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
