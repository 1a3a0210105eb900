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
    with pytest.raises(MemoryError):
        Server(budget_bytes=Server.footprint(16) - 1).run([Request(0, gen.random_layer(16, 2, 0), 0.0)])


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
