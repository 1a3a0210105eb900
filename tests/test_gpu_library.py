"""The group-type library kernel gives the C oracle's values exactly.

The library (qsv_set_jit mode 4, "library") is a set of kernels for 13-qubit windows (up to 8, each with the
16 most swept group types and a band of 16 more), each with straight-line code for its group types of the
streaming form (per op: slot among the group's item bits, variant, kind, matrix classes) and a
run-time-dispatch path for groups of other types; item bits, control masks and matrices are read at run
time. Its cases and its fallback run the interpreter's per-variant arithmetic, so every value
equals the oracle's (np.array_equal: signs of zeros aside). Cases: random layers with Toffolis (controls on
item and base bits), random circuits, VQE (CX chains), the zoo (every gate family), QFT (diagonal runs),
Grover (wide multi-controlled gates); a library built from one circuit serving another (groups in cases and
in the fallback path of the same launch).
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


def _run(torch, prog, x):
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
    return t.cpu().numpy(), ref


CASES = [
    (14, 12, lambda: gen.grover(14, 3)),
    (16, 12, lambda: gen.rqc(16, 10, 8)),
    (16, 12, lambda: gen.qft(16)),
    (18, 12, lambda: gen.random_layer_ccx(18, 10, 51)),
    (20, 12, lambda: gen.vqe(20, 2, 9)),
    (21, 12, lambda: gen.zoo(21, 11)),
    (22, 12, lambda: gen.random_layer(22, 8, 52)),
]


@pytest.mark.timeout(900)
@pytest.mark.parametrize("n,k,maker", CASES)
def test_library_exact_vs_oracle(torch, n, k, maker):
    prog, _, _ = q.compile_circuit(maker(), n, k)
    old = engine.set_jit("library")
    try:
        for kind, seg in prog:
            if kind == "segment":
                engine.jit_prepare(seg, n)
        before = engine.jit_info()
        y, ref = _run(torch, prog, _rand_state(n, 300 + n))
        after = engine.jit_info()
    finally:
        engine.set_jit(old)
    assert np.array_equal(y, ref), f"n={n}: max diff {np.max(np.abs(y - ref))}"
    assert 0 < after["lib_types"] <= 144
    assert after["lib_launches"] > before["lib_launches"]


@pytest.mark.timeout(900)
def test_library_from_other_programs_with_fallback_groups(torch):
    """A library built from one random-Toffoli circuit serves another seed's circuit: its sweeps mix groups
    in library cases with groups on the run-time-dispatch path; values stay exact."""
    n = 20
    progs = [q.compile_circuit(gen.random_layer_ccx(n, 12, s), n, 12)[0] for s in (61, 62)]
    segs0 = [(seg, n) for kind, seg in progs[0] if kind == "segment"]
    old = engine.set_jit("library")
    try:
        types = engine.jit_prepare_library(segs0)
        assert 0 < types <= 144
        before = engine.jit_info()
        y, ref = _run(torch, progs[1], _rand_state(n, 77))
        after = engine.jit_info()
    finally:
        engine.set_jit(old)
    assert np.array_equal(y, ref), f"max diff {np.max(np.abs(y - ref))}"
    assert after["lib_launches"] > before["lib_launches"]
    assert after["interp_launches"] + after["lib_launches"] > before["interp_launches"] + before["lib_launches"]


def test_prepare_library_rejects_bad_segments(torch):
    with pytest.raises(Exception):
        engine.jit_prepare_library([(np.zeros(4, dtype=np.int32), 20)])
    with pytest.raises(Exception):
        engine.jit_prepare_library([(np.zeros(4, dtype=np.int32), 40)])


@pytest.mark.timeout(900)
def test_library_serves_sweeps_planned_in_either_layout(torch):
    """The streaming form does not depend on the phase layouts: a library built while 13-qubit sweeps use 4
    register bits per thread serves them when they are planned with 3 (16 consumer warps), launched with
    the block it was compiled for; values stay exact."""
    n = 19
    prog, _, _ = q.compile_circuit(gen.random_layer_ccx(n, 6, 71), n, 12)
    old = engine.set_jit("library")
    try:
        engine.set_layout13(4)
        engine.jit_prepare_library([(seg, n) for kind, seg in prog if kind == "segment"])
        engine.set_layout13(3)
        before = engine.jit_info()
        y, ref = _run(torch, prog, _rand_state(n, 78))
        after = engine.jit_info()
    finally:
        engine.set_layout13(4)
        engine.set_jit(old)
    assert np.array_equal(y, ref), f"max diff {np.max(np.abs(y - ref))}"
    assert after["lib_launches"] > before["lib_launches"]
