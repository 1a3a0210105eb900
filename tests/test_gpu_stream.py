"""Both interpreter kernels give the C oracle's values exactly, sweep by sweep.

The streaming interpreter (qsv_set_interp(1)) keeps the tile in shared memory and runs each group of
consecutive ops whose targets span at most three tile bits as one pass over it, 16 amplitudes per thread;
ops on tile bit 0 and diagonal ops on any bit join a group. The phase interpreter (qsv_set_interp(0)) keeps
32 amplitudes per thread in registers per phase layout. Both run the same per-variant arithmetic, so both
must equal the oracle (np.array_equal: signs of zeros aside). Cases cover every window size 10..13, plain
and swizzled tiles, tensor-map and bulk staging, controls on tile bit 0 (general MUX ops), Toffoli layers
(controls on item and base bits), diagonal runs (QFT) and long sweeps with many groups.
"""
import numpy as np
import pytest

import qsv_b200 as q
from qsv_b200 import engine, generators as gen
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    engine.load()
    return t


def _rand_state(n, seed):
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(np.complex64)
    return (x / np.float32(np.linalg.norm(x))).astype(np.complex64)


CASES = [
    (10, 8, lambda: gen.random_layer(10, 6, 41)),
    (11, 9, lambda: gen.random_layer_ccx(11, 5, 42)),
    (12, 12, lambda: gen.zoo(12, 7)),
    (13, 10, lambda: gen.qft(13)),
    (14, 12, lambda: gen.grover(14, 5)),
    (16, 12, lambda: gen.rqc(16, 10, 4)),
    (18, 12, lambda: gen.random_layer_ccx(18, 8, 44)),
    (20, 12, lambda: gen.vqe(20, 2, 6)),
    (21, 12, lambda: gen.zoo(21, 8)),
    (22, 12, lambda: gen.random_layer(22, 8, 45)),
    (24, 12, lambda: gen.qft(24)),
]


@pytest.mark.parametrize("interp", ["stream", "phase"])
@pytest.mark.parametrize("n,k,maker", CASES)
def test_interpreters_exact_vs_oracle(torch, interp, n, k, maker):
    prog, fmap, _ = q.compile_circuit(maker(), n, k)
    x = _rand_state(n, 200 + n)
    old_jit = engine.set_jit("off")
    old = engine.set_interp(interp)
    try:
        t = torch.from_numpy(x.copy()).cuda()
        ref = x.copy()
        for kind, seg in prog:
            if kind == "segment":
                engine.run_segment(t, seg)
                ref = orc.run_segment(ref, seg)
            else:
                alt = torch.empty_like(t)
                engine.remap(t, alt, seg)
                t = alt
                ref = orc.remap(ref, seg)
        torch.cuda.synchronize()
        assert engine.device_status() == 0
        y = t.cpu().numpy()
    finally:
        engine.set_interp(old)
        engine.set_jit(old_jit)
    assert np.array_equal(y, ref), f"{interp} n={n}: max diff {np.max(np.abs(y - ref))}"


def test_stream_cases_cover_swizzled_tiles_and_bit0_controls(torch):
    """The cases above include swizzled tensor-map sweeps and ops controlled on tile bit 0."""
    swz = bit0 = 0
    for n, k, maker in CASES:
        prog, _, _ = q.compile_circuit(maker(), n, k)
        for kind, seg in prog:
            if kind != "segment":
                continue
            for sw in engine.plan_segment(seg, n):
                swz += sw["swizzled"]
                bit0 += sum(o["cm_c"] for o in sw["ops"])
    assert swz > 0 and bit0 > 0, (swz, bit0)


def test_interp_mode_switch(torch):
    prev = engine.set_interp("stream")
    try:
        assert engine.set_interp("phase") == "stream"
        assert engine.set_interp("stream") == "phase"
        with pytest.raises(Exception):
            engine.set_interp(2)
    finally:
        engine.set_interp(prev)
