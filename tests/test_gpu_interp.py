"""Every form of the interpreter sweep kernel gives the C oracle's values exactly.

Forms (qsv_set_interp_form): 0 = ops in place, tiles staged by a producer warp; 1 = ping-pong register sets
(ops that write every slot go from one set to the other), staged by the consumer warps (the default);
2 = ops in place, staged by the consumers. Specialised kernels are off, so every sweep runs on the
interpreter. Cases cover every window size 10..13, both 13-qubit layouts (4 register bits with 8 consumer
warps, 3 with 16), plain and swizzled tiles, tensor-map and bulk staging, and every op variant the random
circuits produce (uniform, controlled, branch-free controlled, general MUX, on tile bit 0, register bits and
lane bits).
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


@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("rb13", [4, 3])
@pytest.mark.parametrize("n,k,maker", CASES)
def test_interpreter_forms_exact_vs_oracle(torch, form, rb13, n, k, maker):
    prog, fmap, _ = q.compile_circuit(maker(), n, k)
    x = _rand_state(n, 100 + n)
    old_jit = engine.set_jit(0)
    old_form = engine.set_interp_form(form)
    try:
        engine.set_layout13(rb13)
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
        engine.set_layout13(4)
        engine.set_interp_form(old_form)
        engine.set_jit(old_jit)
    assert np.array_equal(y, ref), f"form {form} n={n}: max diff {np.max(np.abs(y - ref))}"
