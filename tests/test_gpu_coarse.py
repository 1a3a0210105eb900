"""The interpreter kernel and the kernels of coarse sweep structures give the C oracle's values exactly.

A coarse structure (qsv_set_jit mode 3, "coarse") keeps a sweep's layouts and, per op, slot, controls, kind
and the swap / non-swap split; its kernel runs every other op with the dense fused-multiply-add chain, whose
skipped terms are exact zeros on diagonal and identity matrices, so the values equal the oracle's (compared
with np.array_equal, which does not tell the signs of zeros apart). Cases cover every window size 10..13,
both 13-qubit layouts (4 register bits with 8 consumer warps, 3 with 16), plain and swizzled tiles,
tensor-map and bulk staging, and every op variant the random circuits produce (uniform, controlled,
branch-free controlled, general MUX, on tile bit 0, register bits and lane bits). A second circuit with the
same coarse structures (another seed) must reuse them.
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
    (10, 8, lambda: gen.random_layer(10, 6, 31)),
    (11, 9, lambda: gen.random_layer_ccx(11, 5, 32)),
    (12, 12, lambda: gen.zoo(12, 5)),
    (13, 10, lambda: gen.qft(13)),
    (16, 12, lambda: gen.rqc(16, 10, 3)),
    (18, 12, lambda: gen.random_layer_ccx(18, 6, 34)),
    (20, 12, lambda: gen.vqe(20, 2, 5)),
    (21, 12, lambda: gen.zoo(21, 6)),
    (22, 12, lambda: gen.random_layer(22, 6, 35)),
]


@pytest.mark.parametrize("mode", ["off", "coarse"])
@pytest.mark.parametrize("rb13", [4, 3])
@pytest.mark.parametrize("n,k,maker", CASES)
def test_interpreter_and_coarse_kernels_exact_vs_oracle(torch, mode, rb13, n, k, maker):
    prog, fmap, _ = q.compile_circuit(maker(), n, k)
    x = _rand_state(n, 100 + n)
    old_jit = engine.set_jit(mode)
    try:
        engine.set_layout13(rb13)
        before = engine.jit_info()
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
        after = engine.jit_info()
    finally:
        engine.set_layout13(4)
        engine.set_jit(old_jit)
    assert np.array_equal(y, ref), f"{mode} n={n}: max diff {np.max(np.abs(y - ref))}"
    if mode == "coarse":
        assert after["coarse_launches"] > before["coarse_launches"]
        assert after["interp_launches"] == before["interp_launches"]


def test_coarse_structures_shared_across_seeds(torch):
    """Random circuits of one family and size share coarse structures: a second seed compiles nothing new."""
    old_jit = engine.set_jit("coarse")
    try:
        p1, _, _ = q.compile_circuit(gen.rqc(20, 10, 1), 20, 12)
        p2, _, _ = q.compile_circuit(gen.rqc(20, 10, 2), 20, 12)
        for kind, seg in p1:
            engine.jit_prepare(seg, 20)
        n1 = engine.jit_info()["coarse_structures"]
        for kind, seg in p2:
            engine.jit_prepare(seg, 20)
        assert engine.jit_info()["coarse_structures"] == n1
    finally:
        engine.set_jit(old_jit)
