"""GPU tests of the serving loop: overlapping, budget-admitted requests give the same results as each
request alone (bit for bit) and as the FP64 oracle; the HBM budget bounds resident memory."""
import numpy as np
import pytest

from qsv_b200 import engine, generators as gen
from qsv_b200.serve import Request, Server, latency_stats, plain_serve
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _requests(count, rate, seed):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    out = []
    for i in range(count):
        n = int(rng.integers(10, 17))
        out.append(Request(i, gen.random_layer_ccx(n, int(rng.integers(3, 10)), 900 + i), float(t[i] - t[0]),
                           want_state=(i % 7 == 0)))
    return out


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    engine.load()
    return t


@pytest.mark.timeout(600)
def test_served_results_equal_alone_and_oracle(torch):
    srv = Server(budget_bytes=2e9, max_inflight=6)
    done = srv.run(_requests(40, 3000.0, 5))
    assert len(done) == 40 and engine.device_status() == 0
    alone = {r.rid: r for r in plain_serve(_requests(40, 1e9, 5))}
    for r in done:
        a = alone[r.rid]
        assert r.result[0] == a.result[0] and np.array_equal(r.result[1], a.result[1])
        ref = orc.statevector_f64(r.circuit)
        p = np.abs(ref) ** 2
        idx = np.arange(ref.size)
        z = np.array([np.sum(p * (1 - 2 * ((idx >> q) & 1))) for q in range(r.circuit.num_qubits)])
        assert np.max(np.abs(r.result[1] - z)) < 1e-5
        if r.want_state:
            assert orc.metrics(ref, r.state)["one_minus_f"] <= 1e-5
    assert srv.stats["small_batches"] >= 1
    st = latency_stats(done)
    assert st["p99_ms"] >= st["p50_ms"] > 0


@pytest.mark.timeout(600)
def test_budget_limits_resident_memory(torch):
    budget = 3 * Server.footprint(16)
    srv = Server(budget_bytes=budget, max_inflight=8)
    done = srv.run([Request(i, gen.random_layer(16, 6, i), 0.0) for i in range(10)])
    assert len(done) == 10 and srv.stats["peak_bytes"] <= budget and srv.used == 0
    # a request whose state can never fit is rejected on its own; the server does not stop
    small = Server(budget_bytes=Server.footprint(16) - 1)
    done = small.run([Request(0, gen.random_layer(16, 2, 0), 0.0), Request(1, gen.random_layer(12, 2, 1), 0.0)])
    assert [r.rid for r in done] == [1]
    assert [r.rid for r, _ in small.failed] == [0] and "exceeds the HBM budget" in small.failed[0][1]


@pytest.mark.timeout(600)
def test_poisoned_requests_fail_alone(torch):
    """Faults injected on the host into single requests of a served mix: a program with a corrupted word
    (one small request, run in a whole-circuit batch, and one large), a circuit that does not compile (an
    unknown gate) and a request whose state is larger than the budget's largest block. Each of those fails
    alone with its reason; every other request completes with the same result as when it is served alone."""
    from qsv_b200.circuit import Circuit
    from qsv_b200.serve import _compile_request
    reqs = _requests(24, 3000.0, 11)

    def corrupt(r):
        Server._finish_compile(r, _compile_request((r.circuit, None, 12)))
        seg = np.array(r.program[0], dtype=np.int32, copy=True)
        seg[0] ^= 0x1                       # the QSV2 magic word
        r.program = [seg] + list(r.program[1:])

    small_bad = next(r for r in reqs if r.circuit.num_qubits <= 13)
    large_bad = next(r for r in reqs if r.circuit.num_qubits > 13)
    corrupt(small_bad)
    corrupt(large_bad)
    nocompile = next(r for r in reqs[5:] if r not in (small_bad, large_bad))
    bad = Circuit(nocompile.circuit.num_qubits)
    bad.append("no_such_gate", [0], [])
    nocompile.circuit = bad
    big = Request(1000, gen.random_layer_ccx(23, 3, 5), reqs[10].arrival)
    srv = Server(budget_bytes=32 << 20, max_inflight=6)         # largest block 32 MiB: at most 22 qubits
    done = srv.run(reqs + [big])
    failed = {r.rid: why for r, why in srv.failed}
    assert set(failed) == {small_bad.rid, large_bad.rid, nocompile.rid, big.rid}, failed
    assert "engine rejected" in failed[small_bad.rid] and "engine rejected" in failed[large_bad.rid]
    assert "compile" in failed[nocompile.rid] and "budget" in failed[big.rid]
    assert len(done) == len(reqs) - 3 and engine.device_status() == 0 and srv.used == 0
    skip = {small_bad.rid, large_bad.rid, nocompile.rid}
    alone = {r.rid: r for r in plain_serve([r for r in _requests(24, 1e9, 11) if r.rid not in skip])}
    for r in done:
        a = alone[r.rid]
        assert r.result[0] == a.result[0] and np.array_equal(r.result[1], a.result[1])


@pytest.mark.timeout(600)
@pytest.mark.parametrize("policy", ["sjf", "fifo"])
def test_compile_on_arrival_equals_plain(torch, policy):
    """Programs compiled as requests arrive, in a pool of worker processes started before the arrivals
    (shortest-work-first takes each finished compilation at once; FIFO keeps arrival order): every
    result equals the plain path's, which compiles in line."""
    srv = Server(budget_bytes=2e9, max_inflight=6, compile_workers=2, policy=policy)
    try:
        srv.warm()
        done = srv.run(_requests(24, 3000.0, 7))
    finally:
        srv.close()
    assert len(done) == 24 and engine.device_status() == 0
    alone = {r.rid: r for r in plain_serve(_requests(24, 1e9, 7))}
    for r in done:
        a = alone[r.rid]
        assert r.result[0] == a.result[0] and np.array_equal(r.result[1], a.result[1])
