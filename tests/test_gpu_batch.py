"""GPU tests of the batching layer: the whole-circuit kernel (qsv_batch_*) equals the C oracle value for
value; BatchRunner's <Z> and sampled states match the FP64 oracle; a circuit gives bit-identical results
alone and inside a batch; CUDA-graph replays are repeatable."""
import numpy as np
import pytest

import qsv_b200 as q
from qsv_b200 import engine, generators as gen
from qsv_b200.batch import BatchRunner
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    engine.load()
    return t


def _rand(n, seed):
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(np.complex64)
    return (x / np.float32(np.linalg.norm(x))).astype(np.complex64)


def test_whole_circuit_kernel_exact(torch):
    circs = [gen.random_layer_ccx(10 + (i % 4), 4 + i % 5, 50 + i) for i in range(12)]
    circs += [gen.zoo(11, 1), gen.qft(13), gen.random_layer(12, 9, 7)]
    b = engine.SmallBatch()
    states, refs = [], []
    for i, qc in enumerate(circs):
        n = qc.num_qubits
        prog, fmap, st = q.compile_circuit(qc, n, n)
        segs = [s for k, s in prog if k == "segment"]
        assert len(segs) == len(prog)
        x = _rand(n, i)
        t = torch.from_numpy(x.copy()).cuda()
        b.add(t, segs)
        ref = x.copy()
        for s in segs:
            orc.run_segment(ref, s)
        states.append(t)
        refs.append((ref, segs))
    b.upload()
    b.launch()
    torch.cuda.synchronize()
    assert engine.device_status() == 0
    for t, (ref, segs) in zip(states, refs):
        assert np.array_equal(t.cpu().numpy(), ref)
    # a second launch applies every program again
    b.launch()
    for t, (ref, segs) in zip(states, refs):
        for s in segs:
            orc.run_segment(ref, s)
        assert np.array_equal(t.cpu().numpy(), ref)


def _z_from_state(psi):
    p = np.abs(psi) ** 2
    n = psi.size.bit_length() - 1
    idx = np.arange(psi.size)
    return np.array([np.sum(p * (1 - 2 * ((idx >> k) & 1))) for k in range(n)])


def test_batch_runner_matches_fp64_and_is_packing_independent(torch):
    rng = np.random.default_rng(11)
    circs = [gen.random_layer_ccx(int(rng.integers(10, 18)), int(rng.integers(3, 12)), 100 + i) for i in range(24)]
    runner = BatchRunner(streams=4, autotune=True)
    plan = runner.prepare(circs, sample_fraction=0.25, sample_seed=2)
    z, states = runner.run(plan)
    assert engine.device_status() == 0
    for i, qc in enumerate(circs):
        ref = orc.statevector_f64(qc)
        nrm, zq = z[i]
        assert abs(nrm - 1) < 1e-4
        assert np.max(np.abs(zq - _z_from_state(ref))) < 1e-5, i
    for i, st in states.items():
        m = orc.metrics(orc.statevector_f64(circs[i]), st)
        assert m["one_minus_f"] <= 1e-5
    # replay: identical values
    z2, _ = runner.run(plan)
    for a, b in zip(z, z2):
        assert a[0] == b[0] and np.array_equal(a[1], b[1])
    # alone vs in the mix: bit-identical
    for i in (0, 5, 17):
        alone = runner.prepare([circs[i]], sample_fraction=0)
        za, _ = runner.run(alone)
        assert za[0][0] == z[i][0] and np.array_equal(za[0][1], z[i][1])


def test_graph_capture_with_specialised_kernels(torch):
    """Sweeps whose specialised kernels are compiled and loaded before the capture are launched through
    the driver API inside the CUDA-graph capture; replays equal the interpreter-only plain path."""
    from qsv_b200.batch import plain_run, compile_many
    circs = [gen.random_layer(n, 6, 300 + n) for n in (14, 16, 18, 20)] + [gen.random_layer(16, 6, 316)]
    progs = compile_many(circs)
    old = engine.set_jit("eager")
    try:
        runner = BatchRunner(streams=3, autotune=False)
        plan = runner.prepare(circs, sample_fraction=0.0, programs=progs)
        before = engine.jit_info()["jit_launches"]
        runner.capture(plan)          # eager pass (compiles + loads), then the capture
        z1, _ = runner.run(plan)
        z2, _ = runner.run(plan)
        assert engine.jit_info()["jit_launches"] > before
    finally:
        engine.set_jit(old)
    engine.set_jit("off")
    try:
        zp = plain_run(circs, progs)
    finally:
        engine.set_jit(old)
    assert engine.device_status() == 0
    for a, b, c in zip(z1, z2, zp):
        assert a[0] == b[0] == c[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[1], c[1])
