"""Gate matrices in the Qiskit convention (complex128).

For a gate applied to qubits (q0, q1, ...), basis index = bit(q0) + 2*bit(q1) + 4*bit(q2) ...
(the little-endian order that Qiskit's ``Operator(gate).data`` uses, and that the reference compiler
relies on in ``ops_2q``: "M: 4x4, basis bit_a + 2*bit_b", host/sv/compiler.py:79). Controlled gates
put their controls first and the target last, as Qiskit does.
"""
import cmath
import math

import numpy as np

I2 = np.eye(2, dtype=complex)
X = np.array([[0, 1], [1, 0]], dtype=complex)
Y = np.array([[0, -1j], [1j, 0]], dtype=complex)
Z = np.diag([1, -1]).astype(complex)
H = np.array([[1, 1], [1, -1]], dtype=complex) / math.sqrt(2)
S = np.diag([1, 1j]).astype(complex)
SDG = np.diag([1, -1j]).astype(complex)
T = np.diag([1, cmath.exp(1j * math.pi / 4)]).astype(complex)
TDG = np.diag([1, cmath.exp(-1j * math.pi / 4)]).astype(complex)
SX = 0.5 * np.array([[1 + 1j, 1 - 1j], [1 - 1j, 1 + 1j]], dtype=complex)
SXDG = 0.5 * np.array([[1 - 1j, 1 + 1j], [1 + 1j, 1 - 1j]], dtype=complex)


def u3(theta, phi, lam):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    return np.array([[c, -cmath.exp(1j * lam) * s],
                     [cmath.exp(1j * phi) * s, cmath.exp(1j * (phi + lam)) * c]], dtype=complex)


def rx(th):
    c, s = math.cos(th / 2), math.sin(th / 2)
    return np.array([[c, -1j * s], [-1j * s, c]], dtype=complex)


def ry(th):
    c, s = math.cos(th / 2), math.sin(th / 2)
    return np.array([[c, -s], [s, c]], dtype=complex)


def rz(th):
    return np.diag([cmath.exp(-0.5j * th), cmath.exp(0.5j * th)]).astype(complex)


def phase(lam):
    return np.diag([1, cmath.exp(1j * lam)]).astype(complex)


def r_gate(theta, phi):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    return np.array([[c, -1j * cmath.exp(-1j * phi) * s],
                     [-1j * cmath.exp(1j * phi) * s, c]], dtype=complex)


def controlled(U, n_ctrl=1):
    """Controls on gate qubits 0..n_ctrl-1, target on the last gate qubit."""
    nq = n_ctrl + 1
    d = 1 << nq
    M = np.eye(d, dtype=complex)
    on = (1 << n_ctrl) - 1
    i0, i1 = on, on | (1 << n_ctrl)
    M[np.ix_([i0, i1], [i0, i1])] = U
    return M


def _kron_le(*ops):
    """Little-endian tensor product: ops[0] acts on gate qubit 0 (least significant)."""
    out = np.array([[1]], dtype=complex)
    for op in ops:
        out = np.kron(op, out)
    return out


def _expm_herm(G, th):
    """exp(-i th/2 G) for G with G @ G = I."""
    return math.cos(th / 2) * np.eye(G.shape[0]) - 1j * math.sin(th / 2) * G


SWAP = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=complex)
ISWAP = np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]], dtype=complex)
ECR = np.array([[0, 1, 0, 1j], [1, 0, -1j, 0], [0, 1j, 0, 1], [-1j, 0, 1, 0]], dtype=complex) / math.sqrt(2)
DCX = np.array([[1, 0, 0, 0], [0, 0, 0, 1], [0, 1, 0, 0], [0, 0, 1, 0]], dtype=complex)


def cswap():
    M = np.eye(8, dtype=complex)
    # control = gate qubit 0; swap gate qubits 1 and 2 when it is set: |c=1,a=1,b=0> <-> |c=1,a=0,b=1>
    i, j = 0b011, 0b101
    M[[i, j]] = M[[j, i]]
    return M


def xx_plus_yy(theta, beta=0.0):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    M = np.eye(4, dtype=complex)
    M[1, 1] = c
    M[2, 2] = c
    M[1, 2] = -1j * s * cmath.exp(-1j * beta)
    M[2, 1] = -1j * s * cmath.exp(1j * beta)
    return M


# name -> (number of qubits, number of params, matrix builder)
_ONE = {
    "id": (0, lambda: I2), "x": (0, lambda: X), "y": (0, lambda: Y), "z": (0, lambda: Z),
    "h": (0, lambda: H), "s": (0, lambda: S), "sdg": (0, lambda: SDG), "t": (0, lambda: T),
    "tdg": (0, lambda: TDG), "sx": (0, lambda: SX), "sxdg": (0, lambda: SXDG),
    "rx": (1, rx), "ry": (1, ry), "rz": (1, rz), "p": (1, phase), "u1": (1, phase),
    "u": (3, u3), "u3": (3, u3), "u2": (2, lambda phi, lam: u3(math.pi / 2, phi, lam)),
    "r": (2, r_gate),
}


def _const(M):
    M = np.array(M, dtype=complex)
    M.setflags(write=False)
    return M


# parameterless multi-qubit gates: built once (read-only; callers never modify gate matrices)
_FIXED = {
    "cx": _const(controlled(X)), "cy": _const(controlled(Y)), "cz": _const(controlled(Z)),
    "ch": _const(controlled(H)), "csx": _const(controlled(SX)), "cs": _const(controlled(S)),
    "csdg": _const(controlled(SDG)), "swap": _const(SWAP), "iswap": _const(ISWAP), "ecr": _const(ECR),
    "dcx": _const(DCX), "ccx": _const(controlled(X, 2)), "ccz": _const(controlled(Z, 2)),
    "cswap": _const(cswap()), "c3x": _const(controlled(X, 3)), "c4x": _const(controlled(X, 4)),
    "c3sx": _const(controlled(SX, 3)),
}
_DEFINED = {}
_XX, _YY, _ZZ, _ZX = _kron_le(X, X), _kron_le(Y, Y), _kron_le(Z, Z), _kron_le(Z, X)
# parameterised multi-qubit gates: name -> builder(params)
_PARAM = {
    "cp": lambda p: controlled(phase(p[0])), "cu1": lambda p: controlled(phase(p[0])),
    "crx": lambda p: controlled(rx(p[0])), "cry": lambda p: controlled(ry(p[0])),
    "crz": lambda p: controlled(rz(p[0])),
    "cu": lambda p: controlled(cmath.exp(1j * p[3]) * u3(p[0], p[1], p[2])),
    "cu3": lambda p: controlled(u3(p[0], p[1], p[2])),
    "rxx": lambda p: _expm_herm(_XX, p[0]), "ryy": lambda p: _expm_herm(_YY, p[0]),
    "rzz": lambda p: _expm_herm(_ZZ, p[0]), "rzx": lambda p: _expm_herm(_ZX, p[0]),
    "xx_plus_yy": lambda p: xx_plus_yy(p[0], p[1] if len(p) > 1 else 0.0),
}


# Gates defined by a short sequence of basis gates (OpenQASM 2's qelib1.inc definitions): the relative-
# phase Toffolis. Gate-local qubits; the dense matrix is the product of the sequence, and the compiler lowers
# the gate to the sequence itself (neither is a controlled 2x2).
_U2_0PI = ("u2", (0.0, math.pi))
_T_ = ("u1", (math.pi / 4,))
_TDG_ = ("u1", (-math.pi / 4,))
DEFINITIONS = {
    # rccx a, b, c: simplified (Margolus) Toffoli, equal to ccx up to relative phases
    "rccx": (3, [(_U2_0PI, (2,)), (_T_, (2,)), (("cx", ()), (1, 2)), (_TDG_, (2,)), (("cx", ()), (0, 2)),
                 (_T_, (2,)), (("cx", ()), (1, 2)), (_TDG_, (2,)), (_U2_0PI, (2,))]),
    # rcccx (rc3x) a, b, c, d: relative-phase 3-controlled X
    "rcccx": (4, [(_U2_0PI, (3,)), (_T_, (3,)), (("cx", ()), (2, 3)), (_TDG_, (3,)), (_U2_0PI, (3,)),
                  (("cx", ()), (0, 3)), (_T_, (3,)), (("cx", ()), (1, 3)), (_TDG_, (3,)), (("cx", ()), (0, 3)),
                  (_T_, (3,)), (("cx", ()), (1, 3)), (_TDG_, (3,)), (_U2_0PI, (3,)), (_T_, (3,)),
                  (("cx", ()), (2, 3)), (_TDG_, (3,)), (_U2_0PI, (3,))]),
}


def definition(name):
    """[(gate name, gate-local qubits, params), ...] of a gate in DEFINITIONS."""
    return [(g, qs, p) for (g, p), qs in DEFINITIONS[name][1]]


def _embed(M, qubits, nq):
    """Dense 2^nq matrix of gate M acting on the given gate-local qubits (little-endian order)."""
    d = 1 << nq
    k = len(qubits)
    out = np.zeros((d, d), dtype=complex)
    for col in range(d):
        sub = sum(((col >> q) & 1) << i for i, q in enumerate(qubits))
        rest = col & ~sum(1 << q for q in qubits)
        for row_sub in range(1 << k):
            v = M[row_sub, sub]
            if v != 0:
                row = rest | sum(((row_sub >> i) & 1) << q for i, q in enumerate(qubits))
                out[row, col] += v
    return out


def _defined_matrix(name):
    nq = DEFINITIONS[name][0]
    M = np.eye(1 << nq, dtype=complex)
    for g, qs, p in definition(name):
        M = _embed(gate_matrix(g, p), qs, nq) @ M
    return _const(M)


def ms_matrix(nq, theta):
    """Global Molmer-Sorensen gate on nq qubits: the product of rxx(theta) over every qubit pair (the pair
    terms commute)."""
    M = np.eye(1 << nq, dtype=complex)
    R = _expm_herm(_XX, theta)
    for i in range(nq):
        for j in range(i + 1, nq):
            M = _embed(R, (i, j), nq) @ M
    return M


def gate_matrix(name, params=(), nq=None):
    """Dense Qiskit-convention matrix of a named gate (1q, 2q and the supported multi-qubit gates). nq is
    needed only by gates of variable width (ms)."""
    if name == "_u1m":                  # compiler-internal: a 2x2 matrix carried as the parameter
        return params[0]
    if name == "_cum":                  # compiler-internal: the 2x2 parameter controlled by gate qubit 0
        return controlled(params[0])
    if name in DEFINITIONS:
        M = _DEFINED.get(name)
        if M is None:
            M = _DEFINED[name] = _defined_matrix(name)
        return M
    if name == "ms":
        if nq is None:
            raise KeyError("ms needs its number of qubits")
        return ms_matrix(nq, float(params[0]))
    if name in _ONE:
        npar, f = _ONE[name]
        return f(*[float(x) for x in params[:npar]]) if npar else f()
    M = _FIXED.get(name)
    if M is not None:
        return M
    f = _PARAM.get(name)
    if f is not None:
        return f([float(x) for x in params])
    raise KeyError(f"no matrix for gate {name!r}")


def mc_matrix(name, n_ctrl, params=()):
    """Target matrix U of a multi-controlled gate (controls all-ones select U)."""
    if name in ("mcx", "ccx", "c3x", "c4x", "mcx_gray", "mcx_recursive"):
        return X
    if name == "ccz":
        return Z
    if name == "c3sx":
        return SX
    if name in ("mcp", "mcphase"):
        return phase(float(params[0]))
    if name == "_mcu":                  # compiler-internal: the 2x2 target matrix carried as the parameter
        return params[0]
    raise KeyError(name)
