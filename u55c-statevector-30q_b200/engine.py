"""ctypes binding of libqsv_b200.so (the C ABI in include/qsv_b200.h) plus device-state helpers.

PyTorch only holds device memory and streams here: states are complex64 CUDA tensors whose storage is
handed to the C ABI as raw pointers, on the current PyTorch stream. There is no CPU execution path: if
the library cannot be loaded, or no CUDA device is present, every call raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqsv_b200.so")

QSV_OK = 0
QSV_C64 = 0
QSV_C128 = 1            # complex128 states with FP64-matrix segments (header word 4 = 1)
CHUNK_BITS = 12
N_MIN, N_MAX = 10, 34

_ERRORS = {-1: "invalid argument", -2: "bad QSV2 stream", -3: "unsupported", -4: "CUDA error", -5: "device fault",
           -6: "scratch too small"}


class QSVError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


class BadStream(QSVError, ValueError):
    pass


_lib = None


def load(path=LIB_PATH):
    """Load the engine library (built by build.py). Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libqsv_b200.so not found at {path}; build it with build.py (nvcc, sm_100a)")
    L = ctypes.CDLL(path)
    P, I32, SZ, I64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_size_t, ctypes.c_int64
    sig = {
        "qsv_version": ([], I32),
        "qsv_last_error": ([], ctypes.c_char_p),
        "qsv_run_segment": ([P, ctypes.c_int, P, SZ, ctypes.c_int, P], I32),
        "qsv_remap": ([P, P, ctypes.c_int, P, ctypes.c_int, P], I32),
        "qsv_zero_state": ([P, ctypes.c_int, ctypes.c_int, P], I32),
        "qsv_reduce_scratch_bytes": ([ctypes.c_int], SZ),
        "qsv_reduce_f64": ([P, ctypes.c_int, ctypes.c_int, P, P, SZ, P], I32),
        "qsv_reduce_f64_noalloc": ([P, ctypes.c_int, ctypes.c_int, P, P], I32),
        "qsv_chunk_probs_f64": ([P, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P], I32),
        "qsv_sample_f64": ([P, ctypes.c_int, ctypes.c_int, P, ctypes.c_int, P, P, SZ, P], I32),
        "qsv_plan_segment": ([P, SZ, ctypes.c_int, P, SZ], I32),
        "qsv_device_status": ([P], I32),
        "qsv_take_launch_count": ([], ctypes.c_longlong),
        "qsv_set_lo_merge": ([ctypes.c_int], I32),
        "qsv_set_layout13": ([ctypes.c_int], I32),
        "qsv_batch_new": ([], P),
        "qsv_batch_free": ([P], None),
        "qsv_batch_add": ([P, P, ctypes.c_int, ctypes.c_int, P, P], I32),
        "qsv_batch_workspace_bytes": ([P], SZ),
        "qsv_batch_upload": ([P, P, SZ, P], I32),
        "qsv_batch_launch": ([P, P, SZ, P], I32),
        "qsv_set_phase_lanes": ([ctypes.c_int], I32),
        "qsv_set_interp": ([ctypes.c_int], I32),
        "qsv_set_jit": ([ctypes.c_int], I32),
        "qsv_set_wait_limit_us": ([ctypes.c_uint], I32),
        "qsv_inject_skip_load": ([ctypes.c_int], I32),
        "qsv_jit_prepare": ([P, SZ, ctypes.c_int], I32),
        "qsv_jit_wait": ([], I32),
        "qsv_plan_stream": ([P, SZ, ctypes.c_int, P, SZ], I32),
        "qsv_jit_prepare_library": ([P, P, P, ctypes.c_int], I32),
        "qsv_jit_info": ([P, ctypes.c_int], I32),
        "qsv_hbm_copy": ([P, P, SZ, P], I32),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    # before the interpreter shuts down: drop queued specialised-kernel compilations and let running ones
    # finish (the library also does this from its own exit handler)
    import atexit
    atexit.register(L.qsv_set_jit, 0)
    return L


def exported_symbols():
    """Names of the C ABI functions declared in include/qsv_b200.h."""
    return ["qsv_version", "qsv_last_error", "qsv_run_segment", "qsv_remap", "qsv_zero_state",
            "qsv_reduce_scratch_bytes", "qsv_reduce_f64", "qsv_reduce_f64_noalloc", "qsv_chunk_probs_f64",
            "qsv_sample_f64",
            "qsv_plan_segment", "qsv_plan_stream", "qsv_device_status", "qsv_take_launch_count", "qsv_set_lo_merge",
            "qsv_set_layout13", "qsv_set_phase_lanes", "qsv_set_interp", "qsv_set_wait_limit_us",
            "qsv_inject_skip_load", "qsv_batch_new", "qsv_batch_free", "qsv_batch_add",
            "qsv_batch_workspace_bytes", "qsv_batch_upload", "qsv_batch_launch", "qsv_set_jit", "qsv_jit_prepare",
            "qsv_jit_wait", "qsv_jit_prepare_library", "qsv_jit_info", "qsv_hbm_copy"]


def _check(rc):
    if rc != QSV_OK:
        msg = load().qsv_last_error().decode()
        if rc == -2:
            raise BadStream(rc, msg)
        raise QSVError(rc, msg)


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("qsv_b200 needs a CUDA device (B200); none is available")
    return torch


def _stream(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _qubits(state):
    n = state.numel().bit_length() - 1
    if state.numel() != 1 << n:
        raise ValueError("state length is not a power of two")
    return n


def _dt(state):
    """Element-type code of a state tensor: QSV_C64 (complex64) or QSV_C128 (complex128)."""
    torch = _torch()
    if state.dtype == torch.complex64:
        return QSV_C64
    if state.dtype == torch.complex128:
        return QSV_C128
    raise TypeError(f"states are complex64 or complex128 tensors, not {state.dtype}")


def new_state(n, device=None, zero=True, stream=None, dtype=None):
    """Allocate a device state of 2^n amplitudes (complex64 unless dtype=torch.complex128 or "c128";
    |0...0> unless zero=False)."""
    torch = _torch()
    if dtype in (None, "c64"):
        dtype = torch.complex64
    elif dtype == "c128":
        dtype = torch.complex128
    t = torch.empty(1 << n, dtype=dtype, device=device or "cuda")
    if zero:
        zero_state(t, stream)
    return t


def zero_state(state, stream=None):
    _check(load().qsv_zero_state(_ptr(state), _qubits(state), _dt(state), _stream(stream)))


def run_segment(state, seg, stream=None):
    """Execute one QSV2 segment (np.int32 words) in place on a CUDA state: complex64 with a reference
    format segment, complex128 with an FP64-matrix segment (compile_circuit(..., dtype="c128"))."""
    assert state.is_cuda and state.is_contiguous()
    w = np.ascontiguousarray(seg, dtype=np.int32)
    _check(load().qsv_run_segment(_ptr(state), _qubits(state), w.ctypes.data_as(ctypes.c_void_p), w.size,
                                  _dt(state), _stream(stream)))


def remap(src, dst, perm, stream=None):
    """dst <- src with index bits permuted, perm[new] = old. src and dst are distinct tensors."""
    p = np.ascontiguousarray(perm, dtype=np.int32)
    n = _qubits(src)
    if len(p) != n or dst.numel() != src.numel():
        raise ValueError("permutation length / state size mismatch")
    if dst.dtype != src.dtype:
        raise ValueError("remap source and destination differ in element type")
    _check(load().qsv_remap(_ptr(src), _ptr(dst), n, p.ctypes.data_as(ctypes.c_void_p), _dt(src), _stream(stream)))


def scratch_bytes(n):
    return int(load().qsv_reduce_scratch_bytes(n))


def new_scratch(n, device=None):
    torch = _torch()
    return torch.empty(scratch_bytes(n), dtype=torch.uint8, device=device or "cuda")


def reduce_f64(state, out=None, scratch=None, stream=None):
    """Device FP64 reductions: tensor [sum |a|^2, <Z_0>, ..., <Z_{n-1}>] (float64, on the device)."""
    torch = _torch()
    n = _qubits(state)
    out = torch.empty(n + 1, dtype=torch.float64, device=state.device) if out is None else out
    scratch = new_scratch(n, state.device) if scratch is None else scratch
    _check(load().qsv_reduce_f64(_ptr(state), n, _dt(state), _ptr(out), _ptr(scratch), scratch.numel(),
                                 _stream(stream)))
    return out


def chunk_probs_f64(state, chunk_bits=CHUNK_BITS, stream=None):
    torch = _torch()
    n = _qubits(state)
    out = torch.empty(1 << (n - chunk_bits), dtype=torch.float64, device=state.device)
    _check(load().qsv_chunk_probs_f64(_ptr(state), n, _dt(state), chunk_bits, _ptr(out), _stream(stream)))
    return out


def sample_f64(state, uniforms, scratch=None, stream=None):
    """Physical indices (int64 device tensor) of Born-rule samples, one per uniform in [0, 1)."""
    torch = _torch()
    n = _qubits(state)
    u = uniforms if isinstance(uniforms, torch.Tensor) else torch.as_tensor(np.asarray(uniforms, dtype=np.float64))
    u = u.to(device=state.device, dtype=torch.float64).contiguous()
    out = torch.empty(u.numel(), dtype=torch.int64, device=state.device)
    scratch = new_scratch(n, state.device) if scratch is None else scratch
    _check(load().qsv_sample_f64(_ptr(state), n, _dt(state), _ptr(u), u.numel(), _ptr(out), _ptr(scratch),
                                 scratch.numel(), _stream(stream)))
    return out


def plan_segment(seg, n):
    """Decode a segment into the engine's sweep plan (host only): list of dicts."""
    L = load()
    w = np.ascontiguousarray(seg, dtype=np.int32)
    need = L.qsv_plan_segment(w.ctypes.data_as(ctypes.c_void_p), w.size, n, None, 0)
    if need < 0:
        _check(need)
    buf = np.zeros(need, dtype=np.int32)
    L.qsv_plan_segment(w.ctypes.data_as(ctypes.c_void_p), w.size, n, buf.ctypes.data_as(ctypes.c_void_p), need)
    return _parse_plan(buf, n)


def plan_stream(seg, n):
    """The streaming form of a segment's sweeps (host only): per sweep a dict with kw, its groups (item bits
    q, op range) and per op the slot and control split in that form."""
    L = load()
    w = np.ascontiguousarray(seg, dtype=np.int32)
    need = L.qsv_plan_stream(w.ctypes.data_as(ctypes.c_void_p), w.size, n, None, 0)
    if need < 0:
        _check(need)
    buf = np.zeros(need, dtype=np.int32)
    L.qsv_plan_stream(w.ctypes.data_as(ctypes.c_void_p), w.size, n, buf.ctypes.data_as(ctypes.c_void_p), need)
    pos, out = 1, []
    for _ in range(int(buf[0])):
        kw, ng, nops = (int(x) for x in buf[pos:pos + 3])
        pos += 3
        groups = []
        for _ in range(ng):
            r = [int(x) for x in buf[pos:pos + 5]]
            pos += 5
            groups.append(dict(q=r[:3], op_begin=r[3], op_end=r[4]))
        ops = []
        for _ in range(nops):
            tbit, slot, variant, cmask, cm_reg, cm_thr, kind = (int(x) for x in buf[pos:pos + 7])
            pos += 7
            ops.append(dict(tbit=tbit, slot=slot, variant=variant, cmask=cmask & 0xFFFFFFFF, cm_reg=cm_reg,
                            cm_thr=cm_thr & 0xFFFFFFFF, kind=kind))
        out.append(dict(kw=kw, groups=groups, ops=ops))
    return out


def _parse_plan(w, n):
    pos = 1
    sweeps = []
    for _ in range(int(w[0])):
        kw, lo, nh = (int(x) for x in w[pos:pos + 3])
        pos += 3
        H = [int(x) for x in w[pos:pos + 13] if x >= 0]
        pos += 13
        rank = int(w[pos])
        tfree = [int(x) for x in w[pos + 1:pos + 1 + rank]]
        tbox = [int(x) for x in w[pos + 6:pos + 6 + rank]]
        pos += 11
        swz = int(w[pos])
        nph, nops = int(w[pos + 1]), int(w[pos + 2])
        pos += 3
        phases = []
        for _ in range(nph):
            rec = [int(x) for x in w[pos:pos + 15]]
            pos += 15
            phases.append(dict(reg_bits=[r for r in rec[:4] if r >= 0], lane_bits=rec[4:6],
                               warp_bits=[r for r in rec[6:10] if r >= 0], op_begin=rec[10], op_end=rec[11],
                               lane_lo=rec[12:15]))
        ops = []
        for _ in range(nops):
            tbit, slot, cmask, c0, c1, kind, cls, cm_reg, cm_c, cm_thr, variant = (int(x) for x in w[pos:pos + 11])
            m = w[pos + 11:pos + 27].view(np.float32).copy()
            pos += 27
            ops.append(dict(tbit=tbit, slot=slot, cmask=cmask & 0xFFFFFFFF, cls0=c0, cls1=c1, kind=kind, cls=cls,
                            cm_reg=cm_reg, cm_c=cm_c, cm_thr=cm_thr & 0xFFFFFFFF, variant=variant, m0=m[:8], m1=m[8:]))
        sweeps.append(dict(kw=kw, lo=lo, H=H, window=list(range(lo)) + H, phases=phases, ops=ops,
                           tma_rank=rank, tdim_free=tfree, tdim_box=tbox, swizzled=bool(swz)))
    return sweeps


class SmallBatch:
    """Whole-circuit batch for circuits of 10..13 qubits (qsv_batch_* in the C ABI): each circuit's entire
    program runs inside one CTA's shared memory. Add circuits (state tensor + QSV2 segments), upload the
    tables once into a device workspace, then launch (capturable in a CUDA graph, replayable)."""

    def __init__(self):
        self._lib = load()
        self._h = self._lib.qsv_batch_new()
        if not self._h:
            raise QSVError(-1, self._lib.qsv_last_error().decode())
        self.workspace = None
        self.count = 0
        self._keep = []

    def add(self, state, segments):
        n = _qubits(state)
        words = [np.ascontiguousarray(s, dtype=np.int32) for s in segments]
        ptrs = (ctypes.c_void_p * len(words))(*[w.ctypes.data for w in words])
        sizes = (ctypes.c_size_t * len(words))(*[w.size for w in words])
        _check(self._lib.qsv_batch_add(self._h, _ptr(state), n, len(words), ptrs, sizes))
        self._keep.append(state)
        self.count += 1

    def upload(self, stream=None):
        torch = _torch()
        nbytes = int(self._lib.qsv_batch_workspace_bytes(self._h))
        self.workspace = torch.empty(max(nbytes, 256), dtype=torch.uint8, device="cuda")
        _check(self._lib.qsv_batch_upload(self._h, _ptr(self.workspace), self.workspace.numel(), _stream(stream)))

    def launch(self, stream=None):
        if self.workspace is None:
            self.upload(stream)
        _check(self._lib.qsv_batch_launch(self._h, _ptr(self.workspace), self.workspace.numel(), _stream(stream)))

    def __del__(self):
        try:
            if self._h:
                self._lib.qsv_batch_free(self._h)
                self._h = None
        except Exception:
            pass


def device_status():
    v = ctypes.c_int(0)
    _check(load().qsv_device_status(ctypes.byref(v)))
    return v.value


def take_launch_count():
    return int(load().qsv_take_launch_count())


def set_lo_merge(lo):
    _check(load().qsv_set_lo_merge(int(lo)))


def set_layout13(rb):
    _check(load().qsv_set_layout13(int(rb)))


def set_phase_lanes(k):
    _check(load().qsv_set_phase_lanes(int(k)))


INTERP_MODES = {"phase": 0, "stream": 1}


def set_interp(mode):
    """Interpreter kernel for sweeps without a specialised kernel: "phase" (phase layouts in registers) or
    "stream" (the tile stays in shared memory; groups of ops touching at most three target qubits run as
    one pass over it). Values are identical. Returns the previous mode's name."""
    rc = load().qsv_set_interp(INTERP_MODES[mode] if isinstance(mode, str) else int(mode))
    if rc < 0:
        _check(rc)
    return {v: k for k, v in INTERP_MODES.items()}[rc]


def hbm_copy(dst, src, stream=None):
    """dst <- src with the HBM copy probe kernel (same byte size, 16-byte aligned, distinct tensors)."""
    nb = src.numel() * src.element_size()
    if dst.numel() * dst.element_size() != nb:
        raise ValueError("copy probe tensors differ in size")
    _check(load().qsv_hbm_copy(_ptr(dst), _ptr(src), nb, _stream(stream)))


JIT_MODES = {"off": 0, "eager": 1, "auto": 2, "coarse": 3, "library": 4}


def set_wait_limit_us(us):
    """Bounded mbarrier waits of the sweep kernels give up after `us` microseconds (0 = default, 2 s)."""
    _check(load().qsv_set_wait_limit_us(int(us)))


def inject_skip_load(count=1):
    """Fault injection for tests: the next `count` sweep launches have block 0 skip its first tile load, so
    their bounded waits run out and the device status word records it (0 disarms)."""
    _check(load().qsv_inject_skip_load(int(count)))


def set_jit(mode):
    """Specialised sweep kernels: "off" (interpreter only), "eager" (compile each new sweep structure before
    its first launch), "auto" (default: compile in the background once a structure's launches have swept
    2^31 amplitudes; meanwhile use the kernel of its coarse structure or, on 13-qubit windows, the group-type
    library when ready), "coarse" (eager, coarse structures only) or "library" (the group-type library only;
    jit_prepare builds it for a segment, jit_prepare_library for many programs). Values are identical in
    every mode. Returns the previous mode's name."""
    rc = load().qsv_set_jit(JIT_MODES[mode] if isinstance(mode, str) else int(mode))
    if rc < 0:
        _check(rc)
    return {v: k for k, v in JIT_MODES.items()}[rc]


def jit_prepare(seg, n):
    """Compile (blocking, in parallel) the specialised kernels of every sweep of a segment. Host only.
    Returns the number of the segment's sweep structures whose kernel is ready."""
    w = np.ascontiguousarray(seg, dtype=np.int32)
    rc = load().qsv_jit_prepare(w.ctypes.data_as(ctypes.c_void_p), w.size, int(n))
    if rc < 0:
        _check(rc)
    return rc


def jit_prepare_library(programs):
    """Build (blocking) the group-type library from the 13-qubit sweeps of many programs: `programs` is a
    list of (segment words, n). Returns the number of group types in the library."""
    segs = [np.ascontiguousarray(seg, dtype=np.int32) for seg, _ in programs]
    count = len(segs)
    ptrs = (ctypes.c_void_p * max(1, count))(*[s.ctypes.data for s in segs])
    sizes = (ctypes.c_size_t * max(1, count))(*[s.size for s in segs])
    ns = (ctypes.c_int * max(1, count))(*[int(n) for _, n in programs])
    rc = load().qsv_jit_prepare_library(ctypes.cast(ptrs, ctypes.c_void_p), ctypes.cast(sizes, ctypes.c_void_p),
                                        ctypes.cast(ns, ctypes.c_void_p), count)
    if rc < 0:
        _check(rc)
    return rc


def jit_wait():
    _check(load().qsv_jit_wait())


def jit_info():
    """Counters of the specialised-kernel cache."""
    buf = (ctypes.c_longlong * 12)()
    load().qsv_jit_info(ctypes.cast(buf, ctypes.c_void_p), 12)
    keys = ["mode", "structures", "ready", "failed", "jit_launches", "interp_launches", "compile_ms", "pending",
            "coarse_launches", "coarse_structures", "lib_launches", "lib_types"]
    return dict(zip(keys, [int(x) for x in buf]))
