"""A small, qiskit-free circuit container with the part of Qiskit's ``QuantumCircuit`` surface that the
compiler and the runtime read: ``num_qubits``, ``name``, ``data`` (instructions with ``operation.name``,
``operation.params`` and qubit indices), ``remove_final_measurements`` and the usual gate methods.

A real Qiskit circuit is accepted by the compiler as well (see ``normalize``); this class exists because
the simulator itself must not depend on Qiskit.
"""
from dataclasses import dataclass, field


@dataclass(frozen=True)
class Operation:
    name: str
    params: tuple = ()
    num_qubits: int = 1


@dataclass(frozen=True)
class Instruction:
    operation: Operation
    qubits: tuple          # qubit indices (ints)

    @property
    def name(self):
        return self.operation.name

    @property
    def params(self):
        return self.operation.params


class Circuit:
    def __init__(self, num_qubits, name="circuit"):
        self.num_qubits = int(num_qubits)
        self.name = name
        self.data = []
        self.num_clbits = 0

    # ------------------------------------------------------------------ construction
    def append(self, name, qubits, params=()):
        qs = tuple(int(q) for q in qubits)
        if len(set(qs)) != len(qs):
            raise ValueError(f"{name}: repeated qubit in {qs}")
        for q in qs:
            if not 0 <= q < self.num_qubits:
                raise ValueError(f"{name}: qubit {q} out of range for {self.num_qubits} qubits")
        self.data.append(Instruction(Operation(name, tuple(float(p) for p in params), len(qs)), qs))
        return self

    def __getattr__(self, name):
        # gate methods: qc.h(q), qc.rx(theta, q), qc.cx(c, t), qc.u(th, ph, lam, q), ...
        from .gates import _ONE
        npar = None
        if name in _ONE:
            npar = _ONE[name][0]
        elif name in _TWO_PARAMS:
            npar = _TWO_PARAMS[name]
        if npar is None:
            raise AttributeError(name)

        def method(*args):
            params, qubits = args[:npar], args[npar:]
            if len(qubits) == 1 and not isinstance(qubits[0], int) and hasattr(qubits[0], "__iter__"):
                for q in qubits[0]:
                    self.append(name, (q,), params)
                return self
            return self.append(name, qubits, params)
        return method

    def mcx(self, controls, target):
        controls = tuple(controls)
        if len(controls) == 1:          # as Qiskit's mcx: one control is a CX
            return self.append("cx", controls + (target,))
        return self.append("mcx", controls + (target,))

    def mcp(self, lam, controls, target):
        controls = tuple(controls)
        if len(controls) == 1:
            return self.append("cp", controls + (target,), (lam,))
        return self.append("mcp", controls + (target,), (lam,))

    def barrier(self, *qs):
        return self.append("barrier", qs or range(self.num_qubits))

    def measure_all(self):
        for q in range(self.num_qubits):
            self.append("measure", (q,))
        return self

    def remove_final_measurements(self, inplace=False):
        out = self if inplace else self.copy()
        while out.data and out.data[-1].name in ("measure", "barrier"):
            out.data.pop()
        return out

    def copy(self, name=None):
        c = Circuit(self.num_qubits, name or self.name)
        c.data = list(self.data)
        return c

    def compose(self, other, qubits=None, inplace=False):
        out = self if inplace else self.copy()
        qmap = list(range(other.num_qubits)) if qubits is None else list(qubits)
        for ins in other.data:
            out.data.append(Instruction(ins.operation, tuple(qmap[q] for q in ins.qubits)))
        return out

    def size(self):
        return sum(1 for i in self.data if i.name not in ("barrier", "measure"))

    def find_bit(self, q):
        """Qiskit-style bit lookup; qubits here are plain indices."""
        return _BitLocation(int(q))

    def __repr__(self):
        return f"Circuit({self.name!r}, n={self.num_qubits}, gates={len(self.data)})"


@dataclass(frozen=True)
class _BitLocation:
    index: int


_TWO_PARAMS = {
    "cx": 0, "cy": 0, "cz": 0, "ch": 0, "csx": 0, "cs": 0, "csdg": 0, "swap": 0, "iswap": 0, "ecr": 0,
    "dcx": 0, "cp": 1, "cu1": 1, "crx": 1, "cry": 1, "crz": 1, "cu": 4, "cu3": 3, "rxx": 1, "ryy": 1,
    "rzz": 1, "rzx": 1, "xx_plus_yy": 2, "ccx": 0, "ccz": 0, "cswap": 0, "c3x": 0, "c4x": 0,
}


def normalize(qc):
    """Instruction list [(name, qubits, params)] of a Circuit or of a Qiskit QuantumCircuit."""
    out = []
    if isinstance(qc, Circuit):
        for ins in qc.data:
            out.append((ins.name, tuple(ins.qubits), tuple(ins.params)))
        return out
    # Qiskit (duck-typed): instructions carry Qubit objects that the circuit resolves with find_bit
    for ins in qc.data:
        op = ins.operation
        qs = tuple(qc.find_bit(q).index for q in ins.qubits)
        params = []
        for p in op.params:
            try:
                params.append(float(p))
            except TypeError:
                params.append(p)
        out.append((op.name, qs, tuple(params)))
    return out
