"""GPU parity of the specialised sweep kernels (compiled at run time for each sweep structure), called
through the C ABI. Bar: EXACT value equality with the C oracle and with the interpreter kernel, for every
window size, both 13-qubit layouts and every op variant; the automatic mode switches to specialised
kernels without changing a value."""
import numpy as np
import pytest

import qsv_b200 as q
from qsv_b200 import engine, generators as gen
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

def _qubit0_controls(n, seed):
    """Controlled gates with qubit 0 as control (targets on every other qubit) and as target, plus dense
    layers: exercises tile-bit-0 ops of every kind and controls on tile bit 0 for register and lane targets."""
    rng = np.random.default_rng(seed)
    qc = gen.random_layer(n, 1, seed)
    for t in range(1, n):
        th = float(rng.uniform(-np.pi, np.pi))
        qc.cx(0, t)
        qc.cz(0, t)
        qc.ch(0, t)
        qc.crx(th, 0, t)
        qc.cp(th, 0, t)
        qc.cx(t, 0)
        qc.ch(t, 0)
        qc.crz(th, t, 0)
        qc.u(th, th / 3, -th / 2, t)
    qc.ccx(0, 1, n - 1)
    qc.ccx(n - 1, 0, 2)
    return qc


CASES = [
    (14, 12, lambda: _qubit0_controls(14, 1)),
    (19, 12, lambda: _qubit0_controls(19, 2)),
    (10, 8, lambda: gen.random_layer(10, 6, 11)),
    (11, 9, lambda: gen.random_layer_ccx(11, 5, 12)),
    (12, 12, lambda: gen.zoo(12, 3)),
    (13, 10, lambda: gen.qft(13)),
    (14, 12, lambda: gen.random_layer(14, 8, 13)),
    (16, 12, lambda: gen.random_layer_ccx(16, 6, 14)),
    (17, 7, lambda: gen.zoo(17, 4)),
    (18, 12, lambda: gen.qft(18)),
    (20, 12, lambda: gen.random_layer(20, 10, 0)),
    (22, 12, lambda: gen.random_layer_ccx(22, 4, 15)),
]


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    engine.load()
    return t


@pytest.fixture
def jit_mode():
    old = engine.set_jit("auto")
    yield engine.set_jit
    engine.set_jit(old)


def _rand_state(n, seed):
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(np.complex64)
    return (x / np.float32(np.linalg.norm(x))).astype(np.complex64)


def _run(torch, x, seg):
    t = torch.from_numpy(x.copy()).cuda()
    engine.run_segment(t, seg)
    torch.cuda.synchronize()
    assert engine.device_status() == 0
    return t.cpu().numpy()


@pytest.mark.timeout(900)
@pytest.mark.parametrize("rb", [4, 3])
@pytest.mark.parametrize("n,k,maker", CASES)
def test_specialised_exact_vs_oracle(torch, jit_mode, rb, n, k, maker):
    jit_mode("eager")
    engine.set_layout13(rb)
    try:
        prog, _, _ = q.compile_circuit(maker(), n, k)
        x = _rand_state(n, n + rb)
        before = engine.jit_info()["jit_launches"]
        nsw = 0
        for kind, seg in prog:
            if kind == "segment":
                nsw += len(engine.plan_segment(seg, n))
                y = _run(torch, x, seg)
                ref = orc.run_segment(x.copy(), seg)
                assert np.array_equal(y, ref), f"n={n} rb={rb} max diff {np.max(np.abs(y - ref))}"
                x = y
            else:
                x = orc.remap(x, seg)
        info = engine.jit_info()
        assert info["failed"] == 0 and info["jit_launches"] - before == nsw
    finally:
        engine.set_layout13(4)


@pytest.mark.timeout(900)
def test_specialised_equals_interpreter_large(torch, jit_mode):
    """26 qubits (2^13 tiles per sweep, tensor-map and bulk staging): specialised == interpreter."""
    n = 26
    prog, _, _ = q.compile_circuit(gen.random_layer_ccx(n, 6, 5), n, 12)
    segs = [s for kind, s in prog if kind == "segment"]
    outs = []
    for mode in ("off", "eager"):
        jit_mode(mode)
        t = engine.new_state(n)
        for s in segs:
            engine.run_segment(t, s)
        torch.cuda.synchronize()
        outs.append(t)
    assert engine.device_status() == 0
    assert torch.equal(outs[0], outs[1])


@pytest.mark.timeout(900)
def test_auto_mode_switches_without_changing_values(torch, jit_mode):
    """Automatic mode compiles a structure once its launches have swept 2^31 amplitudes (here: 32 sweeps
    of a 26-qubit state) and switches to it between runs; every run equals the interpreter's."""
    n = 26
    prog, _, _ = q.compile_circuit(gen.random_layer(n, 12, 77), n, 12)
    segs = [s for kind, s in prog if kind == "segment"]
    x = torch.from_numpy(_rand_state(n, 5)).cuda()
    jit_mode("off")
    ref = x.clone()
    for s in segs:
        engine.run_segment(ref, s)
    jit_mode("auto")
    before = engine.jit_info()["jit_launches"]
    for it in range(6):
        t = x.clone()
        for s in segs:
            engine.run_segment(t, s)
        torch.cuda.synchronize()
        assert torch.equal(t, ref), it
        engine.jit_wait()
    info = engine.jit_info()
    assert engine.device_status() == 0
    assert info["failed"] == 0 and info["jit_launches"] > before


_SWITCH_SCRIPT = r"""
import sys
sys.path.insert(0, sys.argv[1])
import conftest  # noqa: F401  (registers the package as qsv_b200)
import numpy as np, torch
import qsv_b200 as q
from qsv_b200 import engine, generators as gen
from oracle import oracle as orc
engine.load()
swizzled = 0
for n, maker in ((14, lambda: gen.random_layer(14, 8, 13)), (20, lambda: gen.random_layer(20, 10, 0)),
                 (24, lambda: gen.random_layer_ccx(24, 4, 15))):
    prog, _, _ = q.compile_circuit(maker(), n, 12)
    segs = [s for kind, s in prog if kind == "segment"]
    swizzled += sum(sw["swizzled"] for s in segs for sw in engine.plan_segment(s, n))
    rng = np.random.default_rng(n)
    x = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(np.complex64)
    outs = []
    for mode in ("off", "eager", "coarse"):
        engine.set_jit(mode)
        t = torch.from_numpy(x.copy()).cuda()
        for s in segs:
            engine.run_segment(t, s)
        torch.cuda.synchronize()
        outs.append(t.cpu().numpy())
    assert engine.device_status() == 0
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2]), n
    if n <= 20:
        ref = x.copy()
        for s in segs:
            ref = orc.run_segment(ref, s)
        assert np.array_equal(outs[1], ref), n
print("swizzled sweeps", swizzled)
"""


@pytest.mark.timeout(900)
@pytest.mark.parametrize("env", [{"QSV_JIT_INTERLEAVE": "2"}, {"QSV_SWIZZLE": "0", "QSV_JIT_INTERLEAVE": "1"},
                                 {"QSV_JIT_CM": "1"}, {"QSV_JIT_CM": "1", "QSV_JIT_GROUPS13": "1"},
                                 {"QSV_JIT_STREAM": "1"}])
def test_layout_switches_exact(torch, env, tmp_path):
    """The non-default code-generation switches (read once per process, so run in a child process): phases
    of two tiles interleaved in every multi-phase sweep; no swizzled layouts with interleaved tensor-map
    sweeps; coefficient-major dense ops, with two or one consumer groups; streaming-form kernels. Specialised (exact and coarse
    structures) == interpreter == oracle, exactly."""
    import os
    import subprocess
    import sys
    tests_dir = os.path.dirname(os.path.abspath(__file__))
    script = tmp_path / "switches.py"
    script.write_text(_SWITCH_SCRIPT)
    r = subprocess.run([sys.executable, str(script), tests_dir], env={**os.environ, **env},
                       capture_output=True, text=True, timeout=800)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    swz = int(r.stdout.split("swizzled sweeps")[1])
    assert (swz == 0) == (env.get("QSV_SWIZZLE") == "0"), r.stdout
