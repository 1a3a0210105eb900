"""Failure detection on the GPU without a GPU fault: a bounded wait runs out, the kernel reports it through
the device status word and returns, and the same GPU context keeps working.

The fault is made on the host: qsv_inject_skip_load arms the next sweep launch so that block 0 never issues
the load of its first tile (a flag that nothing sets, from the consumers' point of view). With a short wait
limit (qsv_set_wait_limit_us, 20 ms here instead of the default 2 s) the waiting threads give up, set bit 0
of the status word, the issuing thread waits (bounded) for its other loads still in flight, and the kernel
ends. The test reads the status, then runs the same segment clean and checks it against the C oracle value
for value. Covered: the interpreter, a kernel specialised to the sweep's exact structure, a coarse
structure's kernel, the complex128 kernel, and SVRuntime.run, which raises on a set status word. No test
here traps, faults or hangs a GPU.
"""
import numpy as np
import pytest

import qsv_b200 as q
from qsv_b200 import engine, generators as gen
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
LIMIT_US = 20000


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    engine.load()
    return t


def _rand_state(n, seed, dtype=np.complex64):
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(dtype)
    return (x / np.linalg.norm(x)).astype(dtype)


def _run_armed_then_clean(torch, seg, x):
    """Run seg on x with one injected skipped load, then clean; returns (status after the faulty run,
    status after the clean run, clean result)."""
    assert engine.device_status() == 0
    try:
        engine.set_wait_limit_us(LIMIT_US)
        engine.inject_skip_load(1)
        t = torch.from_numpy(x.copy()).cuda()
        engine.run_segment(t, seg)
        torch.cuda.synchronize()
        bad = engine.device_status()
    finally:
        engine.inject_skip_load(0)
        engine.set_wait_limit_us(0)
    t = torch.from_numpy(x.copy()).cuda()
    engine.run_segment(t, seg)
    torch.cuda.synchronize()
    return bad, engine.device_status(), t.cpu().numpy()


@pytest.mark.parametrize("mode", ["off", "eager", "coarse"])
def test_bounded_wait_reports_and_gpu_stays_usable(torch, mode):
    n = 20
    prog, _, _ = q.compile_circuit(gen.random_layer(n, 4, 7), n, 12)
    seg = prog[0][1]
    x = _rand_state(n, 9)
    ref = orc.run_segment(x.copy(), seg)
    old_jit = engine.set_jit(mode)
    try:
        bad, clean, y = _run_armed_then_clean(torch, seg, x)
    finally:
        engine.set_jit(old_jit)
    assert bad & 1, f"status word {bad:#x}: the injected skipped load was not reported"
    assert clean == 0
    assert np.array_equal(y, ref)


def test_bounded_wait_complex128(torch):
    n = 18
    prog, _, _ = q.compile_circuit(gen.random_layer(n, 3, 8), n, 12, dtype="c128")
    seg = prog[0][1]
    x = _rand_state(n, 10, np.complex128)
    ref = orc.run_segment(x.copy(), seg)
    bad, clean, y = _run_armed_then_clean(torch, seg, x)
    assert bad & 1 and clean == 0
    assert np.array_equal(y, ref)


def test_runtime_raises_on_reported_wait_failure(torch):
    from qsv_b200.runtime import SVRuntime
    rt = SVRuntime()
    qc = gen.random_layer(16, 3, 11)
    try:
        engine.set_wait_limit_us(LIMIT_US)
        engine.inject_skip_load(1)
        with pytest.raises(engine.QSVError) as ei:
            rt.run(qc, shots=16, seed=0)
        assert ei.value.code == -5
    finally:
        engine.inject_skip_load(0)
        engine.set_wait_limit_us(0)
    assert engine.device_status() == 0
    r = rt.run(qc, shots=16, seed=0, return_state=True)
    m = orc.metrics(orc.statevector_f64(qc), r["state"])
    assert m["one_minus_f"] <= 1e-5
