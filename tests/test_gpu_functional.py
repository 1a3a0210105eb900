"""The reference's fidelity-based functional suite (tests/functional_suite.py), restated for this engine.

Every case runs through the drop-in runtime (SVRuntime.run, which pads circuits below 10 qubits) and is
compared with the FP64 dense oracle. Generic input state before each gate case (functional_suite.py:32-40):
a random U3 layer, a CZ ring, another random U3 layer (default_rng(7), angles uniform in [-pi, pi)).
Sections (functional_suite.py:43-71):
  S1 1q gates : 17 gates x every qubit position, n = 5
  S2 2q gates : 21 gates x every ordered qubit pair, n = 4
  S3 3+q gates: ccx, ccz, cswap, mcx with 3 and 4 controls, both control orders
  S4 families : ghz, qft, rqc (depth 10), vqe (2 layers), grover at n = 2..20 step 2 (grover up to 12)
  S5 large n  : analytic checks without a reference state (GHZ amplitudes, QFT|0> uniform)
Pass rule (functional_suite.py:92-94): 1 - F <= 1e-5 and |norm - 1| <= 1e-4.
"""
import math

import numpy as np
import pytest

from qsv_b200 import Circuit, engine, generators as gen
from qsv_b200.runtime import SVRuntime
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

ONE = [("h", 0), ("x", 0), ("y", 0), ("z", 0), ("s", 0), ("sdg", 0), ("t", 0), ("tdg", 0), ("sx", 0), ("sxdg", 0),
       ("rx", 1), ("ry", 1), ("rz", 1), ("p", 1), ("u", 3), ("r", 2), ("id", 0)]
TWO = [("cx", 0), ("cy", 0), ("cz", 0), ("ch", 0), ("swap", 0), ("iswap", 0), ("ecr", 0), ("dcx", 0), ("csx", 0),
       ("cp", 1), ("crx", 1), ("cry", 1), ("crz", 1), ("rxx", 1), ("ryy", 1), ("rzz", 1), ("rzx", 1), ("cu", 4),
       ("cs", 0), ("csdg", 0), ("xx_plus_yy", 2)]
PAR = [0.7311, -1.2207, 2.4113, 0.3359]
THR = 1e-5


def prep(n, seed=7):
    rng = np.random.default_rng(seed)
    qc = Circuit(n)
    for q in range(n):
        qc.u(*rng.uniform(-math.pi, math.pi, 3), q)
    if n > 1:
        for q in range(n):
            qc.cz(q, (q + 1) % n)
    for q in range(n):
        qc.u(*rng.uniform(-math.pi, math.pi, 3), q)
    return qc


def cases(section, max_n_fid=20):
    out = []
    if section == "S1":
        for g, npar in ONE:
            for q in range(5):
                qc = prep(5)
                getattr(qc, g)(*PAR[:npar], q)
                out.append((f"{g}_q{q}", qc))
    elif section == "S2":
        for g, npar in TWO:
            for a in range(4):
                for b in range(4):
                    if a != b:
                        qc = prep(4)
                        getattr(qc, g)(*PAR[:npar], a, b)
                        out.append((f"{g}_{a}{b}", qc))
    elif section == "S3":
        for name, f in [("ccx", lambda qc: qc.ccx(0, 2, 4)), ("ccx_r", lambda qc: qc.ccx(4, 1, 0)),
                        ("ccz", lambda qc: qc.ccz(1, 3, 2)), ("cswap", lambda qc: qc.cswap(0, 3, 4)),
                        ("cswap_r", lambda qc: qc.cswap(4, 1, 2)), ("mcx3", lambda qc: qc.mcx([0, 1, 3], 4)),
                        ("mcx4", lambda qc: qc.mcx([4, 3, 1, 0], 2))]:
            qc = prep(5)
            f(qc)
            out.append((name, qc))
    else:
        for fam in ("ghz", "qft", "rqc", "vqe", "grover"):
            for n in range(2, max_n_fid + 1, 2):
                if fam == "grover" and n > 12:
                    continue
                out.append((f"{fam}_{n}", getattr(gen, fam)(n)))
    return out


@pytest.fixture(scope="module")
def rt():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    engine.load()
    return SVRuntime()


@pytest.mark.timeout(1200)
@pytest.mark.parametrize("section,count", [("S1", 85), ("S2", 252), ("S3", 7), ("S4", 46)])
def test_functional_section(rt, section, count):
    cs = cases(section)
    assert len(cs) == count
    failed = []
    worst = 0.0
    for name, qc in cs:
        sv = rt.run(qc, shots=0, return_state=True)["state"].astype(np.complex128)
        ref = orc.statevector_f64(qc)
        nrm = float(np.vdot(sv, sv).real)
        one_minus_f = 1.0 - abs(np.vdot(ref, sv)) ** 2 / nrm
        worst = max(worst, one_minus_f)
        if not (one_minus_f <= THR and abs(nrm - 1) <= 1e-4):
            failed.append((name, one_minus_f, nrm))
    assert not failed, failed[:10]
    assert worst <= THR


@pytest.mark.timeout(1200)
@pytest.mark.parametrize("n", [24, 26])
def test_functional_large_analytic(rt, n):
    """S5: GHZ end amplitudes and QFT|0> uniformity, deviation < 1e-4 (functional_suite.py:74-82)."""
    sv = rt.run(gen.ghz(n), shots=0, return_state=True)["state"]
    a0, a1 = abs(sv[0]) ** 2, abs(sv[-1]) ** 2
    rest = float(np.sum(np.abs(sv.astype(np.complex128)) ** 2)) - a0 - a1
    assert 1 - (a0 + a1) + abs(a0 - 0.5) + abs(a1 - 0.5) + rest < 1e-4
    sv = rt.run(gen.qft(n), shots=0, return_state=True)["state"]
    assert float(np.max(np.abs(np.abs(sv.astype(np.complex128)) ** 2 - 1.0 / sv.size)) * sv.size) < 1e-4
