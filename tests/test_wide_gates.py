"""Multi-controlled gates wider than the tile window, and the gates defined by basis-gate sequences (rccx,
rcccx, ms) or as controlled 2x2 (c3sx): the compiler's lowering (Barenco et al. 1995 constructions; the
reference transpiles instead, host/sv/compiler.py:132-136,159-166) gives the circuit's unitary. Checked on
the CPU: the compiled QSV2 program is run by the C oracle's exact engine and compared with the dense FP64
statevector, 1 - F <= 1e-5 (the reference's pass rule, tests/test_compiler_model.py:31)."""
import numpy as np
import pytest

import qsv_b200 as q
from qsv_b200 import generators as gen
from qsv_b200.compiler import _mc_plan
from qsv_b200.gates import X, _embed, controlled, mc_matrix
from oracle import oracle as orc


def _run(qc, n, k):
    prog, fmap, st = q.compile_circuit(qc, n, k)
    x = np.zeros(1 << n, np.complex64)
    x[0] = 1
    for kind, seg in prog:
        x = orc.run_segment(x, seg) if kind == "segment" else orc.remap(x, seg)
    return orc.metrics(orc.statevector_f64(qc), orc.unpermute(x, fmap)), st


def _prep(n, seed):
    rng = np.random.default_rng(seed)
    qc = q.Circuit(n)
    for i in range(n):
        qc.u(*[float(v) for v in rng.uniform(0, 2 * np.pi, 3)], i)
    return qc, rng


@pytest.mark.parametrize("n,k,nctrl,name", [(16, 12, 15, "mcx"), (14, 8, 11, "mcx"), (13, 6, 12, "mcp"),
                                            (12, 5, 9, "mcx"), (15, 10, 13, "mcp")])
def test_wide_multicontrolled_gate(n, k, nctrl, name):
    qc, rng = _prep(n, n + k)
    qs = [int(x) for x in rng.permutation(n)[: nctrl + 1]]
    if name == "mcx":
        qc.mcx(qs[:-1], qs[-1])
    else:
        qc.append("mcp", qs, (0.77,))
    for i in range(n):
        qc.ry(0.1 * i + 0.2, i)
    m, st = _run(qc, n, k)
    assert st.lowered.get(name) == 1
    assert m["one_minus_f"] <= 1e-5 and m["max_abs_err"] <= 1e-5, m


@pytest.mark.parametrize("n", [13, 14])
def test_grover_wider_than_window(n):
    """Grover at n > k (its oracle and diffusion are mcx over all n qubits, no qubit to borrow)."""
    m, st = _run(gen.grover(n), n, 12)
    assert st.lowered.get("mcx", 0) > 0
    assert m["one_minus_f"] <= 1e-5, m


@pytest.mark.parametrize("name,nq,params", [("rccx", 3, ()), ("rcccx", 4, ()), ("c3sx", 4, ()), ("ms", 3, (0.4,)),
                                            ("ms", 6, (-1.1,))])
@pytest.mark.parametrize("k", [8, 4])
def test_defined_and_controlled_gates(name, nq, params, k):
    n = 8
    qc, rng = _prep(n, nq + k)
    qc.append(name, [int(x) for x in rng.permutation(n)[:nq]], params)
    qc.cx(0, 7)
    m, _ = _run(qc, n, k)
    assert m["one_minus_f"] <= 1e-5, m


def _plan_unitary(plan, nq):
    """Dense matrix of a _mc_plan result on nq qubits (time order)."""
    M = np.eye(1 << nq, dtype=complex)
    for ctrls, t, U in plan:
        G = controlled(U, len(ctrls)) if ctrls else U
        M = _embed(G, list(ctrls) + [t], nq) @ M
    return M


@pytest.mark.parametrize("nctrl,width,spare", [(5, 4, 0), (5, 4, 1), (6, 3, 1), (7, 5, 2), (6, 4, 0)])
def test_mc_plan_is_exact(nctrl, width, spare):
    """The plan implements C^nctrl(U) exactly (as a dense matrix, spare qubits included, whatever they
    hold), and every gate in it has at most `width` qubits."""
    nq = nctrl + 1 + spare
    for U in (X, mc_matrix("mcp", nctrl, (0.9,)), np.array([[0.6, 0.8j], [0.8j, 0.6]])):
        plan = _mc_plan(list(range(nctrl)), nctrl, U, width, list(range(nctrl + 1, nq)))
        assert all(len(c) + 1 <= width for c, _, _ in plan)
        want = _embed(controlled(U, nctrl), list(range(nctrl + 1)), nq)
        assert np.allclose(_plan_unitary(plan, nq), want, atol=1e-12)


def test_rccx_matrix_is_toffoli_up_to_relative_phases():
    from qsv_b200.gates import gate_matrix
    R, C = gate_matrix("rccx"), gate_matrix("ccx")
    assert np.allclose(np.abs(R), np.abs(C)) and np.allclose(R @ R.conj().T, np.eye(8))
    R4 = gate_matrix("rcccx")
    assert np.allclose(np.abs(R4), np.abs(gate_matrix("c3x"))) and np.allclose(R4 @ R4.conj().T, np.eye(16))
