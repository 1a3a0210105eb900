"""SVRuntime: drop-in for the reference's XRT host runtime (host/sv/runtime.py:83-334) on one B200.

Same entry point and result: ``SVRuntime(...).run(qc, shots, k, p_max, fuse, tiling, initial_map,
return_state, seed)`` returns ``dict(timing, P, L, k, n_run, stats, counts[, state])`` with the
reference's timing keys (runtime.py:3-12). What changes underneath:
  * the whole 2^n state is one HBM buffer (P = 1, L = n): no slices, bank qubits or virtual slices;
  * each segment goes to ``qsv_run_segment`` (sm_100a sweep kernels) instead of ``sv_engine`` CUs;
  * remaps run as one in-HBM permutation sweep (``qsv_remap``) instead of sv_swap / host exchanges;
  * Born sampling runs on the device (``qsv_sample_f64``) on the same uniforms the reference draws
    (``default_rng(seed).random(shots)``), so only the sampled indices cross PCIe;
  * the logical-order state (return_state) is produced by one device remap before the read-back.
"""
import time

import numpy as np

from . import engine
from .circuit import Circuit
from .compiler import compile_circuit
from .isa import MAX_HIGH

KMAX = 12              # default tile exponent of the compiled stream (the reference's build constant)
LMIN = engine.N_MIN    # smaller circuits are padded to this many qubits (the engine's smallest state)


def transpositions(perm):
    """perm[new] = old -> list of (a, b) bit transpositions whose product is perm (runtime.py:35-44)."""
    p = list(perm)
    out = []
    for i in range(len(p)):
        while p[i] != i:
            j = p[i]
            out.append((min(i, j), max(i, j)))
            p[i], p[j] = p[j], p[i]
    return out


def logical_counts(phys, fmap, n):
    """Map sampled physical indices to logical bitstrings (fmap[l] = physical position of logical qubit l),
    dropping padded qubits l >= n, and count them (runtime.py:76-80)."""
    phys = np.asarray(phys, dtype=np.int64)
    logical = np.zeros(phys.shape, dtype=np.int64)
    for q in range(n):
        logical |= ((phys >> fmap[q]) & 1) << q
    vals, cnt = np.unique(logical, return_counts=True)
    return {int(v): int(c) for v, c in zip(vals, cnt)}


class SVRuntime:
    """One GPU. The FPGA-specific constructor arguments of the reference (bdf, xclbin, n_engines, n_swap,
    use_device_swap) are accepted and ignored so call sites keep working. dtype="c128" (no reference
    counterpart) runs complex128 states with FP64 matrices, the on-GPU FP64 path."""

    def __init__(self, bdf=None, xclbin=None, n_engines=None, n_swap=0, use_device_swap=True, max_high=None,
                 device=None, dtype="c64"):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("SVRuntime needs a CUDA device (B200); none is available")
        engine.load()
        t0 = time.perf_counter()
        self.device = torch.device(device if device is not None else "cuda")
        if max_high is not None and max_high > MAX_HIGH:
            raise ValueError(f"max_high={max_high} exceeds the QSV2 pass header's {MAX_HIGH} slots")
        self.max_high = MAX_HIGH if max_high is None else max_high
        if dtype not in ("c64", "c128"):
            raise ValueError(f"dtype must be 'c64' or 'c128', not {dtype!r}")
        self.dtype = dtype
        self.stream = torch.cuda.current_stream(self.device)
        self.L = None
        self.P = 1
        self.st = None          # current state tensor
        self.alt = None         # second buffer for out-of-place remaps (allocated on first use)
        self.scratch = None
        self.log = []
        self.T_setup = time.perf_counter() - t0

    # ------------------------------------------------------------------ planning / allocation
    def plan(self, n, p_max=None):
        """(P, n_run, L): one slice covering the whole state; small circuits are padded to LMIN qubits."""
        n_run = max(n, LMIN)
        if n_run > engine.N_MAX:
            raise ValueError(f"{n} qubits exceed this engine's {engine.N_MAX}")
        return 1, n_run, n_run

    def _alloc(self, L):
        import torch
        if self.L == L and self.st is not None:
            return
        self.st = self.alt = self.scratch = None
        torch.cuda.empty_cache()
        self.st = torch.empty(1 << L, dtype=torch.complex128 if self.dtype == "c128" else torch.complex64,
                              device=self.device)
        self.scratch = engine.new_scratch(L, self.device)
        self.L = L

    def _other(self):
        import torch
        if self.alt is None:
            self.alt = torch.empty_like(self.st)
        return self.alt

    def _remap(self, perm):
        dst = self._other()
        engine.remap(self.st, dst, perm, self.stream)
        self.st, self.alt = dst, self.st

    # ------------------------------------------------------------------ public
    def run(self, qc, shots=1024, k=KMAX, p_max=None, fuse=True, tiling=True, initial_map=None,
            return_state=True, seed=None):
        import torch
        if isinstance(qc, str):          # OpenQASM 2 text or a .qasm path (the reference's circuit files)
            from .qasm import from_qasm
            qc = from_qasm(qc)
        n = qc.num_qubits
        P, n_run, L = self.plan(n, p_max)
        k = min(k, L)
        t0 = time.perf_counter()
        if n_run != n:
            q2 = Circuit(n_run, name=getattr(qc, "name", "circuit"))
            src = qc if isinstance(qc, Circuit) else _from_foreign(qc)
            q2.compose(src.remove_final_measurements(inplace=False), range(n), inplace=True)
            qrun = q2
        else:
            qrun = qc.remove_final_measurements(inplace=False)
        prog, fmap, stats = compile_circuit(qrun, L, k, fuse_1q=fuse, tiling=tiling, initial_map=initial_map,
                                            max_high=self.max_high, dtype=self.dtype)
        t1 = time.perf_counter()
        self._alloc(L)
        t1b = time.perf_counter()
        engine.zero_state(self.st, self.stream)
        ev = []
        started = False
        for kind, payload in prog:
            if kind == "remap" and not started:
                continue          # |0...0> is unchanged by any qubit permutation (runtime.py:308-309)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            if kind == "segment":
                started = True
                engine.run_segment(self.st, payload, self.stream)
            else:
                self._remap(payload)
            e1.record(self.stream)
            ev.append((kind, e0, e1))
        t2 = time.perf_counter()
        counts = {}
        rng = np.random.default_rng(seed)
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(self.stream)
        idx = None
        if shots > 0:
            u = torch.from_numpy(rng.random(shots)).pin_memory().to(self.device, non_blocking=True)
            idx = engine.sample_f64(self.st, u, self.scratch, self.stream)
        s1.record(self.stream)
        self.stream.synchronize()
        t3 = time.perf_counter()
        phys = idx.cpu().numpy() if idx is not None else None
        t4 = time.perf_counter()
        if phys is not None:
            counts = logical_counts(phys, fmap, n)
        t5 = time.perf_counter()
        # T_h2d: host enqueue of the zero-init and every segment (sweep plans travel as kernel
        # parameters); T_kernel / T_exchange: device time of the segments / remaps (CUDA events);
        # T_post: device sampling + host mapping to logical bitstrings; T_e2e: wall clock of the whole
        # call (host enqueue overlaps device execution, so the parts do not add up to it)
        T = dict(T_compile=t1 - t0, T_alloc=t1b - t1, T_h2d=t2 - t1b, T_kernel=0.0, T_exchange=0.0)
        for kind, e0, e1 in ev:
            sec = e0.elapsed_time(e1) / 1e3
            T["T_kernel" if kind == "segment" else "T_exchange"] += sec
        T["T_d2h"] = t4 - t3
        T["T_post"] = s0.elapsed_time(s1) / 1e3 + (t5 - t4)
        T["T_e2e"] = t5 - t0
        status = engine.device_status()
        if status:
            raise engine.QSVError(-5, f"device status word {status:#x} after the run")
        out = dict(timing=T, P=P, L=L, k=k, n_run=n_run, stats=stats.__dict__, counts=counts)
        if return_state:
            perm = [fmap[q] for q in range(n_run)]
            if perm != list(range(n_run)):
                self._remap(perm)        # the state stays in logical order until the next run
            full = self.st.cpu().numpy()
            out["state"] = full[: 1 << n]
            T["T_state_reorder"] = time.perf_counter() - t5
        return out


def _from_foreign(qc):
    """A Qiskit circuit (duck-typed) as this package's Circuit."""
    from .circuit import normalize
    c = Circuit(qc.num_qubits, name=getattr(qc, "name", "circuit"))
    for name, qs, params in normalize(qc):
        c.append(name, qs, params)
    return c
