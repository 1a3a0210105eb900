"""OpenQASM 2.0 front end: round trips through text compile to the same QSV2 words, parameter expressions,
broadcast, register layout and gate definitions are read as OpenQASM 2 specifies, and the reference's
own circuit files (when the reference tree is present) parse into the circuits of the generators."""
import math
import os

import numpy as np
import pytest

import qsv_b200 as q
from qsv_b200 import generators as gen
from qsv_b200.qasm import QasmError, from_qasm, to_qasm
from oracle import oracle as orc

# the reference's exported circuit files, when a copy of the reference tree is named by QSV_REFERENCE_ROOT
REF_QASM = os.path.join(os.environ.get("QSV_REFERENCE_ROOT", "-"), "circuits", "qasm")


@pytest.mark.parametrize("qc", [gen.qft(10), gen.ghz(12), gen.rqc(10, 6, 3), gen.vqe(11, 2, 4),
                                gen.random_layer_ccx(10, 3, 1), gen.zoo(10, 2)], ids=lambda c: c.name)
def test_round_trip_same_program(qc):
    back = from_qasm(to_qasm(qc))
    n = qc.num_qubits
    p1, f1, _ = q.compile_circuit(qc, n, 8)
    p2, f2, _ = q.compile_circuit(back, n, 8)
    assert f1 == f2 and len(p1) == len(p2)
    for (k1, a), (k2, b) in zip(p1, p2):
        assert k1 == k2 and np.array_equal(np.asarray(a), np.asarray(b))


def test_expressions_broadcast_registers_and_definitions():
    text = """
    OPENQASM 2.0;
    include "qelib1.inc";
    // two registers: a -> qubits 0..1, b -> 2..4
    qreg a[2];
    qreg b[3];
    creg c[5];
    gate mix(theta) x, y { h x; cp(theta / 2) x, y; rz(-theta) y; }
    h b;
    rx(-2*pi/3) a[0];
    u3(pi/2, 0.25, -(1+2)^2/9) a[1];
    u2(0, pi) b[0];
    mix(sin(pi/6) * 4) a[1], b[2];
    cx a, b[1];
    barrier a, b;
    measure b[0] -> c[0];
    """
    qc = from_qasm(text)
    ref = q.Circuit(5)
    for t in (2, 3, 4):
        ref.h(t)
    ref.rx(-2 * math.pi / 3, 0)
    ref.u(math.pi / 2, 0.25, -1.0, 1)
    ref.u(math.pi / 2, 0.0, math.pi, 2)
    th = math.sin(math.pi / 6) * 4
    ref.h(1)
    ref.cp(th / 2, 1, 4)
    ref.rz(-th, 4)
    ref.cx(0, 3)
    ref.cx(1, 3)
    assert qc.num_qubits == 5
    a = orc.statevector_f64(qc.remove_final_measurements())
    b = orc.statevector_f64(ref)
    assert np.max(np.abs(a - b)) < 1e-12


@pytest.mark.parametrize("bad", ["OPENQASM 2.0; qreg q[2]; foo q[0];", "OPENQASM 2.0; qreg q[2]; h q[2];",
                                 "OPENQASM 2.0; qreg q[2]; rx(bar) q[0];", "OPENQASM 2.0; qreg q[2]; reset q[0];",
                                 "OPENQASM 2.0; qreg q[2]; qreg r[3]; cx q, r;"])
def test_rejects(bad):
    with pytest.raises(QasmError):
        from_qasm(bad)


@pytest.mark.skipif(not os.path.isdir(REF_QASM), reason="reference circuit files not present")
@pytest.mark.parametrize("fname,make", [("qft_12.qasm", lambda: gen.qft(12)), ("ghz_16.qasm", lambda: gen.ghz(16))])
def test_reference_files_parse_to_the_generators(fname, make):
    qc = from_qasm(os.path.join(REF_QASM, fname))
    ref = make()
    n = ref.num_qubits
    p1, f1, _ = q.compile_circuit(qc, n, 10)
    p2, f2, _ = q.compile_circuit(ref, n, 10)
    assert f1 == f2
    for (k1, a), (k2, b) in zip(p1, p2):
        assert k1 == k2 and np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.skipif(not os.path.isdir(REF_QASM), reason="reference circuit files not present")
def test_every_reference_file_parses():
    for fname in sorted(os.listdir(REF_QASM)):
        qc = from_qasm(os.path.join(REF_QASM, fname))
        assert qc.num_qubits == int(fname.split("_")[1].split(".")[0]) and qc.size() > 0
