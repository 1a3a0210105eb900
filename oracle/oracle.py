"""Oracle front end -- TEST INFRASTRUCTURE ONLY (tests, the smoke check and the benchmark's CPU-baseline
leg use it as the checker; the product path never imports it).

* ``run_segment`` / ``remap`` / ``run_program``: the C restatement of the QSV2 engine (qsv_oracle.c), whose
  fused-multiply-add order equals the CUDA engine's, so CUDA results must equal these value for value.
* ``statevector_f64``: the FP64 dense gate-by-gate simulator that stands in for Qiskit's ``Statevector``
  (Qiskit is not installed): every gate's Qiskit-convention matrix applied to a complex128 state.
* ``metrics``: 1 - F (computed without cancellation), fidelity and max |delta amp| after global-phase
  alignment, as in the reference's bench/fpga/sv_maxwidth_ref.py:15-25.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqsv_oracle.so")
_lib = None


def build(force=False):
    """Compile the C oracle in place (gcc, OpenMP)."""
    if force or not os.path.exists(LIB_PATH) or \
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "qsv_oracle.c")):
        subprocess.check_call(["make", "-s", "-C", HERE, "-B" if force else "libqsv_oracle.so"])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P, I32, I64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
        L.qsv_oracle_run_segment.argtypes = [P, ctypes.c_int, P, I64, ctypes.c_int]
        L.qsv_oracle_check_segment.argtypes = [P, I64, ctypes.c_int]
        L.qsv_oracle_remap.argtypes = [P, P, ctypes.c_int, P, ctypes.c_int]
        L.qsv_oracle_apply_dense_f64.argtypes = [P, ctypes.c_int, P, ctypes.c_int, P, ctypes.c_int]
        L.qsv_oracle_metrics.argtypes = [P, P, I64, P]
        L.qsv_oracle_reduce_f64.argtypes = [P, ctypes.c_int, P, P]
        L.qsv_oracle_run_segment_c128.argtypes = [P, ctypes.c_int, P, I64, ctypes.c_int]
        L.qsv_oracle_remap_c128.argtypes = [P, P, ctypes.c_int, P, ctypes.c_int]
        for f in ("run_segment", "check_segment", "remap", "apply_dense_f64", "metrics", "reduce_f64",
                  "run_segment_c128", "remap_c128"):
            getattr(L, "qsv_oracle_" + f).restype = I32
        _lib = L
    return _lib


def threads():
    return int(lib().qsv_oracle_max_threads())


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def run_segment(state, seg, nthreads=None):
    """Execute one QSV2 segment in place on a numpy state (single slice, L = n): complex64 with a
    reference-format segment, complex128 with an FP64-matrix segment (header word 4 = 1)."""
    assert state.dtype in (np.complex64, np.complex128) and state.flags.c_contiguous
    seg = np.ascontiguousarray(seg, dtype=np.int32)
    n = state.size.bit_length() - 1
    run = lib().qsv_oracle_run_segment_c128 if state.dtype == np.complex128 else lib().qsv_oracle_run_segment
    rc = run(_ptr(state), n, _ptr(seg), seg.size, nthreads or threads())
    if rc != 0:
        raise ValueError(f"oracle rejected segment (code {rc})")
    return state


def remap(state, perm, nthreads=None):
    n = state.size.bit_length() - 1
    perm = np.ascontiguousarray(perm, dtype=np.int32)
    out = np.empty_like(state)
    f = lib().qsv_oracle_remap_c128 if state.dtype == np.complex128 else lib().qsv_oracle_remap
    rc = f(_ptr(state), _ptr(out), n, _ptr(perm), nthreads or threads())
    if rc != 0:
        raise ValueError(f"bad permutation (code {rc})")
    return out


def unpermute(state, final_map):
    return remap(state, [final_map[q] for q in range(len(final_map))])


def run_program(prog, n, final_map, state=None, dtype=np.complex64):
    """Whole program from |0...0> with the C engine; returns the logical-order state."""
    if state is None:
        state = np.zeros(1 << n, dtype=dtype)
        state[0] = 1
    for kind, payload in prog:
        if kind == "segment":
            run_segment(state, payload)
        else:
            state = remap(state, payload)
    return unpermute(state, final_map)


def statevector_f64(qc, n=None):
    """Dense FP64 statevector of a circuit, gate by gate with Qiskit-convention matrices (the oracle
    every reference test compares against, tests/test_compiler_model.py:22)."""
    import sys
    pkg = sys.modules.get("qsv_b200")
    if pkg is None:
        raise RuntimeError("load the qsv_b200 package before the FP64 oracle (it reads its gate table)")
    n = qc.num_qubits if n is None else n
    st = np.zeros(1 << n, dtype=np.complex128)
    st[0] = 1
    skip = {"measure", "barrier", "delay", "save_statevector", "id"}
    mc_names = {"ccx", "ccz", "c3x", "c4x", "mcx", "mcx_gray", "mcx_recursive", "mcp", "mcphase", "c3sx"}
    for name, qs, params in pkg.circuit.normalize(qc):
        if name in skip:
            continue
        if name in mc_names:
            apply_controlled(st, qs[:-1], qs[-1], pkg.gates.mc_matrix(name, len(qs) - 1, params))
        else:
            apply_dense(st, qs, pkg.gates.gate_matrix(name, params, len(qs)))
    return st


def apply_controlled(st, ctrls, t, U):
    """U on qubit t for the amplitudes whose control bits are all 1 (complex128, in place)."""
    n = st.size.bit_length() - 1
    idx = np.arange(1 << n, dtype=np.int64)
    cm = 0
    for c in ctrls:
        cm |= 1 << c
    i0 = idx[((idx & cm) == cm) & (((idx >> t) & 1) == 0)]
    i1 = i0 | (1 << t)
    a0, a1 = st[i0].copy(), st[i1].copy()
    st[i0] = U[0, 0] * a0 + U[0, 1] * a1
    st[i1] = U[1, 0] * a0 + U[1, 1] * a1


def apply_dense(st, qubits, M):
    n = st.size.bit_length() - 1
    M = np.ascontiguousarray(M, dtype=np.complex128)
    q = np.ascontiguousarray(qubits, dtype=np.int32)
    rc = lib().qsv_oracle_apply_dense_f64(_ptr(st), n, _ptr(q), len(q), _ptr(M), threads())
    if rc != 0:
        raise ValueError(f"dense apply failed ({rc})")


def metrics(ref, sv):
    """dict(fidelity, one_minus_f, max_abs_err, norm) of complex64 `sv` against complex128 `ref`."""
    ref = np.ascontiguousarray(ref, dtype=np.complex128)
    sv = np.ascontiguousarray(sv, dtype=np.complex64)
    out = np.zeros(4, dtype=np.float64)
    lib().qsv_oracle_metrics(_ptr(ref), _ptr(sv), sv.size, _ptr(out))
    return dict(fidelity=float(out[0]), one_minus_f=float(out[1]), max_abs_err=float(out[2]),
                norm=float(out[3]))


def reduce_f64(sv):
    """(sum |a|^2, [<Z_q>]) of a complex64 state in FP64."""
    sv = np.ascontiguousarray(sv, dtype=np.complex64)
    n = sv.size.bit_length() - 1
    nrm = np.zeros(1, dtype=np.float64)
    z = np.zeros(max(n, 1), dtype=np.float64)
    lib().qsv_oracle_reduce_f64(_ptr(sv), n, _ptr(nrm), _ptr(z))
    return float(nrm[0]), z[:n]
