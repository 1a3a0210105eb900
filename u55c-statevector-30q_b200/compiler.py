"""Host compiler: circuit -> MUX2 ops -> passes -> QSV2 segments.

This is the front end of the hot path. It follows the reference compiler (host/sv/compiler.py) step for
step, because the program it emits (which ops, in which order, grouped into which passes, encoded into
which words) defines the arithmetic the engine performs; the same circuit compiled here and by the
reference yields the same QSV2 words (the golden-stream tests check this word for word). It does not use
Qiskit: gate matrices come from ``gates.py`` and wide gates are lowered by ``_lower`` below instead of
``qiskit.transpile``.

Multi-controlled gates wider than the tile window become several narrower controlled gates (``_mc_plan``,
the constructions of Barenco et al. 1995), where the reference transpiles them to CX and one-qubit gates.

Program = list of steps, executed in order by the runtime:
  ("segment", int32 words)  one engine launch (every pass of the segment over the whole state)
  ("remap", perm)           qubit permutation, perm[new_phys] = old_phys
"""
from dataclasses import dataclass, field

import numpy as np
from scipy.linalg import cossin, schur

from .isa import MAGIC, OP_MUX2, MAX_OPS_PER_PASS, MAX_HIGH, DTYPE_C64, DTYPE_C128
from .gates import DEFINITIONS, I2, X, Z, definition, gate_matrix, mc_matrix, phase
from .circuit import normalize

SKIP = {"measure", "barrier", "delay", "save_statevector", "id"}   # compiler.py:20
# multi-controlled gates built directly as one MUX2 (controls all-ones select U), compiler.py:25-29
# ("_mcu" is the compiler's own: a controlled 2x2 matrix produced by _mc_plan, carried as its parameter)
MC_NAMES = {"ccx", "c3x", "c4x", "mcx", "mcx_gray", "mcx_recursive", "ccz", "mcphase", "mcp", "c3sx", "_mcu"}
MAX_DENSE_QUBITS = 10     # wider gates are never expanded to a dense matrix (compiler.py:132)


@dataclass
class Op:
    """One MUX2 record before encoding: target storage qubit ``t``, control storage qubits ``ctrls``
    (all set -> M1), 2x2 matrices M0 / M1 in complex128 (compiler.py:33-42)."""
    t: int
    ctrls: tuple
    M0: np.ndarray
    M1: np.ndarray
    src: object = None

    @property
    def q(self):
        return (self.t,) + tuple(self.ctrls)


@dataclass
class Stats:
    """Per-circuit compile statistics; the field names are the reference's (compiler.py:45-56) so the
    runtime's ``stats`` dictionary reads the same."""
    n_input_gates: int = 0
    native: dict = field(default_factory=dict)
    relabel: int = 0
    lowered: dict = field(default_factory=dict)
    csd_2q: int = 0
    fused_1q: int = 0
    n_ops: int = 0
    n_passes: int = 0
    n_remaps: int = 0
    n_segments: int = 0


def _count(d, key, inc=1):
    d[key] = d.get(key, 0) + inc


def _close_to_identity(R):
    """np.allclose(R, I, atol=1e-12) (rtol 1e-5): off-diagonal |R_ij| <= 1e-12, |R_ii - 1| <= 1e-12 + 1e-5."""
    d = np.diagonal(R)
    if np.any(np.abs(d - 1.0) > 1e-12 + 1e-5):
        return False
    off = R - np.diag(d)
    return not np.any(np.abs(off) > 1e-12)


def controlled_target(M, nq):
    """If M (2^nq, Qiskit order) is a 2x2 on one gate qubit j controlled by all the others being 1,
    return (j, U); else None (compiler.py:63-75)."""
    full = (1 << nq) - 1
    for j in range(nq):
        i1 = full
        i0 = full & ~(1 << j)
        sel = [i0, i1]
        U = M[np.ix_(sel, sel)].copy()
        rest = np.array(M, dtype=complex)
        rest[np.ix_(sel, sel)] = I2
        if _close_to_identity(rest):
            return j, U
    return None


def _ops_2q_records(M):
    """The MUX2 records of a 4x4 gate, independent of its qubits: ([(target_is_a, M0, M1), ...], csd)."""
    d = np.diag(M)
    if not np.any(np.abs(M - np.diag(d)) > 1e-12):      # np.allclose(M, diag(M), atol=1e-12)
        return [(False, np.diag([d[0], d[2]]), np.diag([d[1], d[3]]))], False
    ct = controlled_target(M, 2)
    if ct is not None:
        j, U = ct
        return [(j == 0, I2, U)], False
    (u1, u2), theta, (v1h, v2h) = cossin(M, p=2, q=2, separate=True)
    c, s = np.cos(theta), np.sin(theta)
    R0 = np.array([[c[0], -s[0]], [s[0], c[0]]])
    R1 = np.array([[c[1], -s[1]], [s[1], c[1]]])
    return [(True, v1h, v2h), (False, R0, R1), (True, u1, u2)], True


# records of recently seen 4x4 matrices (CX / CZ and other fixed gates repeat in every layer); the
# matrices are shared between ops and never modified in place
_OPS_2Q_CACHE = {}


def ops_2q(M, a, b, stats):
    """4x4 gate on storage qubits (a, b), basis bit_a + 2*bit_b -> MUX2 ops (compiler.py:78-92):
    diagonal -> one MUX2 on b selected by a; controlled-U -> one MUX2; otherwise the cosine-sine
    decomposition into three MUX2 (block-diag on a | rotation on b | block-diag on a)."""
    M = np.asarray(M)
    key = (M.dtype.str, M.shape, M.tobytes())
    hit = _OPS_2Q_CACHE.get(key)
    if hit is None:
        hit = _ops_2q_records(M)
        if len(_OPS_2Q_CACHE) >= 4096:
            _OPS_2Q_CACHE.clear()
        _OPS_2Q_CACHE[key] = hit
    recs, csd = hit
    if csd:
        stats.csd_2q += 1
    return [Op(a, (b,), m0, m1) if ta else Op(b, (a,), m0, m1) for ta, m0, m1 in recs]


def _lower(name, nq, params):
    """Decomposition of a gate that cannot become MUX2 records directly, into gates that can.
    Replaces the reference's ``transpile(..., basis_gates=["u", "cx"])`` (compiler.py:159-166); the
    gate sequence differs from Qiskit's but implements the same unitary. Qubits are gate-local."""
    if name == "cswap":
        return [("cx", (2, 1), ()), ("ccx", (0, 1, 2), ()), ("cx", (2, 1), ())]
    if name in DEFINITIONS:             # rccx, rcccx: their basis-gate definitions
        return definition(name)
    if name == "ms":                    # global Molmer-Sorensen: rxx(theta) on every pair (they commute)
        return [("rxx", (i, j), (params[0],)) for i in range(nq) for j in range(i + 1, nq)]
    raise NotImplementedError(
        f"gate {name!r} on {nq} qubits is neither a (multi-)controlled 2x2 nor wide-gate lowerable here")


def _sqrt2(U):
    """Principal square root of a 2x2 unitary (complex Schur form: U = Z diag(l) Z^dag, unitary Z)."""
    T, Zm = schur(np.asarray(U, dtype=complex), output="complex")
    return Zm @ np.diag(np.sqrt(np.diag(T))) @ Zm.conj().T


def _is_x(U):
    return np.array_equal(np.asarray(U), X)


def _mc_plan(ctrls, t, U, width, spare):
    """A multi-controlled 2x2 gate (U on qubit t when every qubit of `ctrls` is 1) as a sequence of
    controlled 2x2 gates of at most `width` qubits each: [(controls, target, 2x2 matrix)], in time order.
    `spare`: qubits outside the gate; they may be borrowed in any state and are returned unchanged.

    Constructions of Barenco et al., "Elementary gates for quantum computation", Phys. Rev. A 52, 3457
    (1995):
      * with a borrowed qubit g and the controls split into A and B (Lemma 7.2's one-ancilla form):
            C_{A+B}(X)_t = C_A(X)_g . C_{B+g}(X)_t . C_A(X)_g . C_{B+g}(X)_t     (time order)
        -- the first and third flip g by AND(A), so the two C_{B+g}(X) together flip t by AND(A)AND(B)
        whatever g held, and g ends as it started;
      * with no qubit to borrow, or a target matrix other than X (Lemma 7.5), V^2 = U, q one control, R the
        others:
            C_{R+q}(U)_t = C_q(V)_t . C_R(X)_q . C_q(V^dag)_t . C_R(X)_q . C_R(V)_t   (time order)
        -- the two C_R(X)_q may borrow t; C_R(V)_t has one control fewer and q becomes free.
    Both are exact identities, so the plan implements U exactly (up to the rounding of V to FP32 when
    the ops are encoded)."""
    ctrls = list(ctrls)
    if len(ctrls) + 1 <= width:
        return [(tuple(ctrls), t, U)]
    if _is_x(U) and spare:
        g = spare[0]
        rest = spare[1:]
        a = max(1, min(width - 1, len(ctrls) - 1))       # A fills a native gate; B keeps the rest
        A, B = ctrls[:a], ctrls[a:]
        on_g = _mc_plan(A, g, X, width, [t] + B + rest)
        on_t = _mc_plan(B + [g], t, X, width, A + rest)
        return on_g + on_t + on_g + on_t
    q, R = ctrls[-1], ctrls[:-1]
    V = _sqrt2(U)
    flip = _mc_plan(R, q, X, width, [t] + list(spare))
    return ([((q,), t, V)] + flip + [((q,), t, V.conj().T)] + flip +
            _mc_plan(R, t, V, width, [q] + list(spare)))


def circuit_to_ops(qc, stats, fuse_1q=True, max_width=None):
    """Gates -> MUX2 ops (compiler.py:95-173). SWAPs become a relabelling (relab[l] = storage qubit of
    logical qubit l); 1q gates on a qubit are multiplied together (complex128) until another gate
    touches that qubit. Returns (ops, relab)."""
    instrs = normalize(qc)
    n = qc.num_qubits
    relab = list(range(n))
    ops = []
    pending = {}

    def flush(q):
        if q in pending:
            U = pending.pop(q)
            ops.append(Op(q, (), U, U))

    def emit(new_ops):
        for op in new_ops:
            for q in op.q:
                flush(q)
            ops.append(op)

    def handle(name, qs, params, lowered):
        if name in SKIP:
            return
        if not lowered:
            stats.n_input_gates += 1
        if name == "swap":
            a, b = qs
            relab[a], relab[b] = relab[b], relab[a]
            stats.relabel += 1
            return
        st = [relab[q] for q in qs]
        nq = len(qs)
        if nq > 2 and name in MC_NAMES and (max_width is None or nq <= max_width):
            if not lowered:
                _count(stats.native, name)
            U = mc_matrix(name, nq - 1, params)
            emit([Op(st[-1], tuple(st[:-1]), I2, U, src=(name, qs))])
            return
        if nq > 2 and ((max_width is not None and nq > max_width) or nq > MAX_DENSE_QUBITS):
            if not lowered:
                _count(stats.native, name)
            lower(name, qs, params)
            return
        M = gate_matrix(name, params, nq)
        if not lowered:
            _count(stats.native, name)
        if nq == 1:
            s = st[0]
            if fuse_1q and s in pending:
                pending[s] = M @ pending[s]
                stats.fused_1q += 1
            elif fuse_1q:
                pending[s] = M
            else:
                ops.append(Op(s, (), M, M))
            return
        if nq == 2:
            emit(ops_2q(M, st[0], st[1], stats))
            return
        ct = controlled_target(M, nq)
        if ct is not None:
            j, U = ct
            emit([Op(st[j], tuple(x for i, x in enumerate(st) if i != j), I2, U, src=(name, qs))])
            return
        lower(name, qs, params)

    def lower(name, qs, params):
        _count(stats.native, name, -1)
        _count(stats.lowered, name)
        if name in MC_NAMES:
            # wider than the window: narrower controlled gates (the circuit's other qubits may be borrowed)
            width = max_width if max_width is not None else MAX_DENSE_QUBITS
            inside = set(qs)
            spare = [x for x in range(n) if x not in inside]
            U = mc_matrix(name, len(qs) - 1, params)
            for ctrls, t, M in _mc_plan(list(qs[:-1]), qs[-1], U, width, spare):
                sub = "_u1m" if not ctrls else "_cum" if len(ctrls) == 1 else "_mcu"
                handle(sub, list(ctrls) + [t], (M,), True)
            return
        for sub_name, sub_qs, sub_params in _lower(name, len(qs), params):
            handle(sub_name, [qs[i] for i in sub_qs], sub_params, True)

    for name, qs, params in instrs:
        handle(name, list(qs), params, False)
    for q in list(pending):
        flush(q)
    stats.n_ops = len(ops)
    return ops, relab


def pass_window(qubits, k, max_high=MAX_HIGH):
    """Smallest m in 0..max_high such that at most m of `qubits` lie at or above k - m; returns
    (m, sorted high qubits), or None when no m fits (compiler.py:176-183)."""
    qs = sorted(q for q in qubits if q >= k - max_high)
    for m in range(max_high + 1):
        hi = [q for q in qs if q >= k - m]
        if len(hi) <= m:
            return m, hi
    return None


def _fits(hi, k, M):
    """pass_window(...) is not None for a pass whose qubits at or above k - M are the sorted list hi."""
    for m in range(M + 1):
        lim = k - m
        c = 0
        for q in hi:
            if q >= lim:
                c += 1
        if c <= m:
            return True
    return False


def schedule(ops, n, L, k, stats, remap_policy="lru", tiling=True, l2p0=None, M=MAX_HIGH):
    """Greedy pass packing with remap insertion (compiler.py:186-260).

    Ops are taken in program order. An op joins the open pass while the pass's qubits still fit one tile
    window (k - m low qubits plus m <= M high qubits) and the pass holds fewer than 64 ops. An op that
    touches a bank qubit (>= L) or cannot fit any window closes the segment and emits a remap that brings
    its qubits into the window, evicting the qubits whose next use is furthest away.
    Returns (steps, l2p) with steps [("segment", [pass, ...]) | ("remap", perm)], a pass being a list of
    (op, physical qubits)."""
    l2p = list(l2p0) if l2p0 is not None else list(range(n))
    k = min(k, L)
    steps = []
    seg = []
    lim = k - M                       # only qubits from here on decide whether a pass window fits
    cur, cur_hi = [], set()

    def close_pass():
        nonlocal cur, cur_hi
        if cur:
            seg.append(cur)
        cur, cur_hi = [], set()

    def close_segment():
        close_pass()
        if seg:
            steps.append(("segment", list(seg)))
            seg.clear()

    def next_use(p, idx):
        logical = l2p.index(p)
        for j in range(idx, len(ops)):
            if logical in ops[j].q:
                return j - idx
        return 10 ** 9

    for idx, op in enumerate(ops):
        phys = [l2p[q] for q in op.q]
        hi_new = [p for p in phys if p >= lim]    # qubits below k - M always fit (and are below L)
        if hi_new and (any(p >= L for p in hi_new) or not _fits(sorted(set(hi_new)), k, M)):
            low = k - M
            assert len(phys) <= low + M, "op wider than the tile window"
            by_far = lambda p: -next_use(p, idx)          # noqa: E731  furthest next use first
            bank = [p for p in phys if p >= L]
            high_local = [p for p in phys if low <= p < L]
            hi_slots = sorted((p for p in range(max(k, L - 6), L) if p not in phys), key=by_far)
            if bank and len(high_local) + len(bank) <= M and len(hi_slots) >= len(bank):
                move, victims = bank, hi_slots[:len(bank)]
            else:
                keep = high_local[:M]
                move = [p for p in phys if p >= low and p not in keep]
                low_slots = sorted((p for p in range(low) if p not in phys), key=by_far)
                high_slots = sorted((p for p in range(low, L) if p not in phys), key=by_far)
                high_free = M - len(keep)
                victims = []
                for _ in move:
                    if low_slots:
                        victims.append(low_slots.pop(0))
                    elif high_free > 0 and high_slots:
                        victims.append(high_slots.pop(0))
                        high_free -= 1
                    else:
                        raise RuntimeError("cannot fit op into tile window")
            close_segment()
            perm = list(range(n))
            for a, b in zip(move, victims):
                perm[a], perm[b] = b, a
            steps.append(("remap", perm))
            stats.n_remaps += 1
            new_of_old = {old: new for new, old in enumerate(perm)}
            l2p = [new_of_old[p] for p in l2p]
            phys = [l2p[q] for q in op.q]
            hi_new = [p for p in phys if p >= lim]
        if hi_new:
            grown = cur_hi.union(hi_new)
            widened = len(grown) > len(cur_hi)
        else:
            grown, widened = cur_hi, False
        if (not tiling and cur) or len(cur) >= MAX_OPS_PER_PASS or (widened and not _fits(sorted(grown), k, M)):
            close_pass()
            grown = set(hi_new)
        cur.append((op, phys))
        cur_hi = grown
    close_segment()
    return steps, l2p


def encode_segment(passes, L, k, M=MAX_HIGH, dtype="c64"):
    """QSV2 words of one segment (compiler.py:263-285). For dtype "c64" (the reference's format) the
    matrices are rounded to complex64 here: this is the single FP64 -> FP32 rounding point of the program.
    For "c128" (complex128 states; header word 4 = DTYPE_C128) the FP64 matrices are stored as they are."""
    c128 = dtype == "c128"
    if dtype not in ("c64", "c128"):
        raise ValueError(f"dtype must be 'c64' or 'c128', not {dtype!r}")
    parts = [np.array([MAGIC, L, len(passes), k, DTYPE_C128 if c128 else DTYPE_C64, 0, 0, 0], dtype=np.int32)]
    for p in passes:
        qubits = set(q for _, ph in p for q in ph)
        m, hi = pass_window(qubits, k, M)
        slots = hi + [0] * (4 - len(hi))
        tile_of = {q: q for q in qubits if q < k - m}
        for i, q in enumerate(hi):
            tile_of[q] = k - m + i
        nops = len(p)
        parts.append(np.array([m, slots[0], slots[1], nops, slots[2], slots[3], 0, 0], dtype=np.int32))
        # op records: matrices rounded to complex64 together (same per-entry rounding as one by one)
        mats = np.empty((nops, 2, 4), dtype=np.complex128)
        mats[:, 0] = np.array([op.M0 for op, _ in p], dtype=complex).reshape(nops, 4)
        mats[:, 1] = np.array([op.M1 for op, _ in p], dtype=complex).reshape(nops, 4)
        if c128:
            fl = np.empty((nops, 16), dtype=np.float64)
            fl[:, 0:8:2], fl[:, 1:8:2] = mats[:, 0].real, mats[:, 0].imag
            fl[:, 8:16:2], fl[:, 9:16:2] = mats[:, 1].real, mats[:, 1].imag
        else:
            c64 = mats.astype(np.complex64)
            fl = np.empty((nops, 16), dtype=np.float32)
            fl[:, 0:8:2], fl[:, 1:8:2] = c64[:, 0].real, c64[:, 0].imag
            fl[:, 8:16:2], fl[:, 9:16:2] = c64[:, 1].real, c64[:, 1].imag
        fbits = np.ascontiguousarray(fl).view(np.int32)
        rec = np.zeros((nops, 8 + fbits.shape[1]), dtype=np.int32)
        rec[:, 0] = OP_MUX2
        for j, (op, ph) in enumerate(p):
            cmask = 0
            for c in ph[1:]:
                cmask |= 1 << tile_of[c]
            rec[j, 1] = tile_of[ph[0]]
            rec[j, 2] = cmask
        rec[:, 8:] = fbits
        parts.append(rec.reshape(-1))
    return np.concatenate(parts)


def segment_dtype(seg):
    """"c64" or "c128" from a segment's header word 4."""
    return "c128" if int(np.asarray(seg)[4]) == DTYPE_C128 else "c64"


def compile_circuit(qc, L, k, fuse_1q=True, tiling=True, remap_policy="lru", initial_map=None,
                    max_high=MAX_HIGH, dtype="c64"):
    """Full pipeline (compiler.py:288-314). Returns (prog, final_map, stats); final_map[l] is the
    physical position of logical qubit l after the program. dtype "c128" emits segments with FP64
    matrices for complex128 states (an extension of the stream, see isa.py)."""
    k = min(k, L)
    max_high = max(0, min(max_high, k - 3))      # sub-blocks of at least 2^3 amplitudes
    stats = Stats()
    ops, relab = circuit_to_ops(qc, stats, fuse_1q, max_width=k)
    n = qc.num_qubits
    steps, l2p_end = schedule(ops, n, L, k, stats, remap_policy, tiling, initial_map, max_high)
    prog = []
    if initial_map is not None and list(initial_map) != list(range(n)):
        perm = [0] * n
        for logical, p in enumerate(initial_map):
            perm[p] = logical
        prog.append(("remap", perm))
    for kind, payload in steps:
        if kind == "segment":
            prog.append(("segment", encode_segment(payload, L, k, max_high, dtype)))
            stats.n_segments += 1
            stats.n_passes += len(payload)
        else:
            prog.append(("remap", payload))
    final_map = [l2p_end[relab[q]] for q in range(n)]
    return prog, final_map, stats
