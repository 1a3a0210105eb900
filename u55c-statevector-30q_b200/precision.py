"""Precision and scale study on one GPU: complex64 at the largest size, complex128 as the FP64 reference.

No reference counterpart (the FPGA engine is complex64 only and its precision checks use Qiskit on the
host). Run A: a random-layer circuit with CZ brickwork and Toffolis at 33 qubits in complex64 (64 GiB).
Run B: the same recipe at 32 qubits in complex128 (64 GiB), the on-GPU FP64 path, against the complex64
run of the same circuit: 1 - F and max |delta amp| with the reference's recipe
(bench/fpga/sv_maxwidth_ref.py:15-25: norms, overlap, global-phase alignment, 1 - F = d^2 - d^4 / 4
without cancellation). Both runs use one compiled schedule, so the two states share their final qubit
map and are compared in physical order. The comparison is FP64 on the device, in chunks.
Run A is checked against FP64 the same way, by the pattern the reference uses at its widest sizes (save the
state, then compare chunk by chunk: bench/fpga/sv_maxwidth.py:53 with sv_maxwidth_ref.py): its 64 GiB
complex64 state goes to host memory, the 33-qubit complex128 run (128 GiB) takes the device, and the
chunks of the saved state come back one at a time for the comparison.
"""
import os
import time

from . import engine
from .compiler import compile_circuit
from .generators import random_layer_ccx


def config3_circuit(n, depth=16, seed=2):
    """U3 on every qubit (angles uniform in [0, 2pi)), CZ brickwork, n // 4 Toffolis per layer."""
    return random_layer_ccx(n, depth, seed)


def run_state(qc, dtype="c64", k=12, device=None):
    """Compile and run qc from |0...0> on the device. Returns (state, final_map, timing)."""
    import torch
    n = qc.num_qubits
    t0 = time.perf_counter()
    prog, fmap, stats = compile_circuit(qc, n, min(k, n), dtype=dtype)
    t1 = time.perf_counter()
    st = engine.new_state(n, device=device, dtype=dtype)
    alt = None
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for kind, payload in prog:
        if kind == "segment":
            engine.run_segment(st, payload)
        else:
            alt = torch.empty_like(st) if alt is None else alt
            engine.remap(st, alt, payload)
            st, alt = alt, st
    ev1.record()
    torch.cuda.synchronize()
    del alt
    status = engine.device_status()
    if status:
        raise engine.QSVError(-5, f"device status word {status:#x}")
    return st, fmap, dict(T_compile=t1 - t0, T_kernel=ev0.elapsed_time(ev1) / 1e3, passes=stats.n_passes,
                          ops=stats.n_ops)


def compare(ref, sv, chunk_bits=26):
    """1 - F, fidelity and max |delta amp| of state `sv` against `ref` (same length; `ref` on the device,
    `sv` on the device or in host memory, moved chunk by chunk), in
    FP64: F = |<ref|sv>|^2 / (|ref|^2 |sv|^2); the difference after normalising and aligning the global
    phase gives d^2 and 1 - F = d^2 - d^4 / 4."""
    import torch
    N = ref.numel()
    step = min(N, 1 << chunk_bits)
    nr = ns = 0.0
    ip = 0j
    dev = ref.device
    for i in range(0, N, step):
        a = ref[i:i + step].to(torch.complex128)
        b = sv[i:i + step].to(dev).to(torch.complex128)
        nr += float(torch.sum(a.real * a.real + a.imag * a.imag))
        ns += float(torch.sum(b.real * b.real + b.imag * b.imag))
        ip += complex(torch.sum(torch.conj(a) * b))
    nr, ns = nr ** 0.5, ns ** 0.5
    ipn = ip / (nr * ns)
    mag = abs(ipn)
    ph = ipn / mag if mag > 0 else 1.0
    d2 = 0.0
    mx = 0.0
    for i in range(0, N, step):
        a = ref[i:i + step].to(torch.complex128) / nr
        b = sv[i:i + step].to(dev).to(torch.complex128) / ns
        e = torch.abs(b - ph * a)
        d2 += float(torch.sum(e * e))
        mx = max(mx, float(torch.max(e)))
    return dict(fidelity=mag * mag, one_minus_f=d2 - d2 * d2 / 4.0, max_abs_err=mx, norm=ns)


def _host_bytes_available():
    try:
        import psutil
        return psutil.virtual_memory().available
    except Exception:
        return os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")


def study(n_a=33, n_b=32, depth=16, seed=2, device=None, run_a_vs_fp64=True):
    """Run A (n_a qubits, complex64, against complex128 when host memory can hold its state) and Run B
    (n_b qubits, complex128 vs complex64). Returns a dict."""
    import torch
    out = {}
    qa = config3_circuit(n_a, depth, seed)
    st, fmap, t = run_state(qa, "c64", device=device)
    z = engine.reduce_f64(st).cpu().numpy()
    out["run_a"] = dict(n=n_a, dtype="complex64", state_gib=(8 << n_a) / 2 ** 30, norm=float(z[0]), **t)
    need = (8 << n_a) + (16 << 30)
    if run_a_vs_fp64 and _host_bytes_available() > need:
        saved = torch.empty(st.numel(), dtype=st.dtype)
        step = 1 << 26
        for i in range(0, st.numel(), step):
            saved[i:i + step].copy_(st[i:i + step])
        del st
        torch.cuda.empty_cache()
        s128, f128, t128 = run_state(qa, "c128", device=device)
        if f128 != fmap:
            raise RuntimeError("complex64 and complex128 schedules differ")
        out["run_a"]["vs_c128"] = compare(s128, saved)
        out["run_a"]["c128_T_kernel"] = t128["T_kernel"]
        del s128, saved
    else:
        out["run_a"]["vs_c128"] = None
        out["run_a"]["vs_c128_skipped"] = f"host memory below {need / 2 ** 30:.0f} GiB"
        del st
    torch.cuda.empty_cache()
    qb = config3_circuit(n_b, depth, seed)
    s128, f128, t128 = run_state(qb, "c128", device=device)
    s64, f64, t64 = run_state(qb, "c64", device=device)
    if f128 != f64:
        raise RuntimeError("complex64 and complex128 schedules differ")
    m = compare(s128, s64)
    out["run_b"] = dict(n=n_b, dtype="complex128", state_gib=(16 << n_b) / 2 ** 30, **t128,
                        c64_T_kernel=t64["T_kernel"], c64_vs_c128=m)
    del s128, s64
    torch.cuda.empty_cache()
    return out
