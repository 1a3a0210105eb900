"""complex128 path, host side: the FP64-matrix stream extension (header word 4 = 1, 40-word op records)
encodes the compiler's complex128 matrices exactly, the engine's decoder rejects a segment of the other
element type, and the oracle's complex128 engine agrees with the FP64 dense simulator to rounding."""
import numpy as np
import pytest

import qsv_b200 as q
from qsv_b200 import engine, generators as gen, isa
from oracle import oracle as orc


def test_c128_stream_layout():
    qc = gen.random_layer(12, 3, 5)
    p64, f64, _ = q.compile_circuit(qc, 12, 10)
    p128, f128, _ = q.compile_circuit(qc, 12, 10, dtype="c128")
    assert f64 == f128 and len(p64) == len(p128)
    s64, s128 = p64[0][1], p128[0][1]
    assert s64[4] == isa.DTYPE_C64 and s128[4] == isa.DTYPE_C128
    assert q.compiler.segment_dtype(s128) == "c128" and q.compiler.segment_dtype(s64) == "c64"
    # same passes and op headers, 40-word records whose FP64 matrices round to the complex64 ones
    pos64 = pos128 = isa.HDR_WORDS
    for _ in range(int(s64[2])):
        assert list(s64[pos64:pos64 + 8]) == list(s128[pos128:pos128 + 8])
        nops = int(s64[pos64 + 3])
        pos64 += 8
        pos128 += 8
        for _ in range(nops):
            assert list(s64[pos64:pos64 + 8]) == list(s128[pos128:pos128 + 8])
            m32 = s64[pos64 + 8:pos64 + 24].view(np.float32)
            m64 = np.ascontiguousarray(s128[pos128 + 8:pos128 + 40]).view(np.float64)
            assert np.array_equal(m64.astype(np.float32), m32)
            pos64 += isa.OP_WORDS
            pos128 += isa.OP_WORDS_C128
    assert pos64 == len(s64) and pos128 == len(s128)


@pytest.mark.parametrize("n,k,make", [(10, 8, lambda: gen.random_layer_ccx(10, 6, 3)),
                                      (13, 12, lambda: gen.zoo(13, 2)),
                                      (15, 12, lambda: gen.qft(15))])
def test_oracle_c128_matches_fp64_dense(n, k, make):
    qc = make()
    prog, fmap, _ = q.compile_circuit(qc, n, k, dtype="c128")
    s = orc.run_program(prog, n, fmap, dtype=np.complex128)
    ref = orc.statevector_f64(qc)
    assert np.max(np.abs(s - ref)) < 1e-13
    assert abs(np.vdot(ref, s)) ** 2 > 1 - 1e-13


def test_plan_rejects_other_element_type():
    L = engine.load()
    prog, _, _ = q.compile_circuit(gen.random_layer(12, 2, 0), 12, 10, dtype="c128")
    w = np.ascontiguousarray(prog[0][1], dtype=np.int32)
    rc = L.qsv_plan_segment(w.ctypes.data_as(engine.ctypes.c_void_p), w.size, 12, None, 0)
    assert rc == -2 and b"complex128" in L.qsv_last_error()
