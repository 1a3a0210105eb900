"""GPU parity of the complex128 path (FP64 states, FP64 matrices), called through the C ABI.
Bars: segment execution EXACT vs the C oracle's complex128 engine (same FP64 fused-multiply-add chains);
remap exact; FP64 reductions relative 1e-12; whole circuits through SVRuntime(dtype="c128"):
1 - F <= 1e-12 against the FP64 dense oracle."""
import numpy as np
import pytest

import qsv_b200 as q
from qsv_b200 import engine, generators as gen
from qsv_b200.runtime import SVRuntime
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

CASES = [
    (10, 8, lambda: gen.random_layer(10, 6, 11)),
    (11, 9, lambda: gen.random_layer_ccx(11, 5, 12)),
    (12, 12, lambda: gen.zoo(12, 3)),
    (13, 10, lambda: gen.qft(13)),
    (16, 12, lambda: gen.random_layer_ccx(16, 6, 14)),
    (17, 7, lambda: gen.zoo(17, 4)),
    (20, 12, lambda: gen.random_layer(20, 8, 0)),
]


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    engine.load()
    return t


def _rand_state(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return (x / np.linalg.norm(x)).astype(np.complex128)


@pytest.mark.parametrize("n,k,maker", CASES)
def test_c128_segments_exact_vs_oracle(torch, n, k, maker):
    prog, _, _ = q.compile_circuit(maker(), n, k, dtype="c128")
    x = _rand_state(n, n)
    for kind, seg in prog:
        if kind == "segment":
            t = torch.from_numpy(x.copy()).cuda()
            engine.run_segment(t, seg)
            torch.cuda.synchronize()
            assert engine.device_status() == 0
            y = t.cpu().numpy()
            ref = orc.run_segment(x.copy(), seg)
            assert np.array_equal(y, ref), f"n={n} max diff {np.max(np.abs(y - ref))}"
            x = y
        else:
            x = orc.remap(x, seg)


def test_c128_rejects_c64_segment(torch):
    prog, _, _ = q.compile_circuit(gen.random_layer(12, 2, 0), 12, 8)
    t = engine.new_state(12, dtype="c128")
    with pytest.raises(engine.BadStream):
        engine.run_segment(t, prog[0][1])
    h = t.cpu().numpy()
    assert h[0] == 1 and np.count_nonzero(h) == 1


@pytest.mark.parametrize("n", [10, 15, 21])
def test_c128_remap_and_reductions(torch, n):
    x = _rand_state(n, 7)
    perm = list(np.random.default_rng(n).permutation(n))
    src = torch.from_numpy(x).cuda()
    dst = torch.empty_like(src)
    engine.remap(src, dst, perm)
    assert np.array_equal(dst.cpu().numpy(), orc.remap(x, perm))
    z = engine.reduce_f64(src).cpu().numpy()
    p = np.abs(x) ** 2
    idx = np.arange(x.size)
    ref = [p.sum()] + [np.sum(p * (1 - 2 * ((idx >> b) & 1))) for b in range(n)]
    assert np.allclose(z, ref, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("qc", [gen.random_layer_ccx(14, 8, 2), gen.qft(16), gen.zoo(12, 9)], ids=lambda c: c.name)
def test_c128_runtime_fidelity(torch, qc):
    rt = SVRuntime(dtype="c128")
    r = rt.run(qc, shots=256, seed=3)
    ref = orc.statevector_f64(qc)
    s = r["state"]
    assert s.dtype == np.complex128
    assert 1 - abs(np.vdot(ref, s)) ** 2 <= 1e-12
    assert np.max(np.abs(s - ref)) < 1e-12
    assert sum(r["counts"].values()) == 256


def test_c128_large_exact(torch):
    n = 24
    prog, _, _ = q.compile_circuit(gen.random_layer_ccx(n, 3, 8), n, 12, dtype="c128")
    t = engine.new_state(n, dtype="c128")
    x = np.zeros(1 << n, dtype=np.complex128)
    x[0] = 1
    for kind, seg in prog:
        if kind == "segment":
            engine.run_segment(t, seg)
            orc.run_segment(x, seg)
        else:
            dst = torch.empty_like(t)
            engine.remap(t, dst, seg)
            t = dst
            x = orc.remap(x, seg)
    torch.cuda.synchronize()
    assert engine.device_status() == 0
    assert np.array_equal(t.cpu().numpy(), x)
