"""Host side of the batching layer (no GPU): the spawned compile pools (per call, and persistent) give
the same programs as compiling in-process, and the batched workload generator is seeded and within its
stated ranges."""
import numpy as np
import pytest

from qsv_b200 import generators as gen
from qsv_b200.batch import CompilePool, compile_many, config4_circuits


@pytest.mark.timeout(300)
def test_compile_pool_matches_inline():
    circs = [gen.random_layer_ccx(12, 4, i) for i in range(4)] + [gen.random_layer_ccx(15, 3, 9)]
    a = compile_many(circs, workers=0)
    b = compile_many(circs, workers=2, timeout=120)
    with CompilePool(2) as pool:              # persistent pool: two batches through the same workers
        c = compile_many(circs, pool=pool, timeout=120)
        d = compile_many(circs[::-1], pool=pool, timeout=120)[::-1]
    for other in (b, c, d):
        for (pa, fa, na, _), (pb, fb, nb, _) in zip(a, other):
            assert fa == fb and na == nb
            for (ka, sa), (kb, sb) in zip(pa, pb):
                assert ka == kb and np.array_equal(sa, sb)
    # small circuits compile as one window (k = n): no remaps, whole-state programs
    for prog, fmap, n, _ in a[:4]:
        assert all(kind == "segment" for kind, _ in prog) and np.asarray(prog[0][1])[3] == n


def test_config4_generator():
    c1 = config4_circuits(64)
    c2 = config4_circuits(64)
    assert [c.num_qubits for c in c1] == [c.num_qubits for c in c2]
    assert all(10 <= c.num_qubits <= 24 for c in c1)
    assert len(set(c.num_qubits for c in c1)) > 5
    # Toffolis on distinct qubits, one per 4 qubits per layer
    for c in c1[:8]:
        ccx = [ins for ins in c.data if ins.name == "ccx"]
        assert all(len(set(ins.qubits)) == 3 for ins in ccx)
