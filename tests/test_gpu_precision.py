"""GPU precision study at small size: the complex128 run agrees with the FP64 dense oracle to rounding,
and the device-side comparison of the complex64 run against it equals the oracle's metrics of the
complex64 state against the FP64 dense state (1 - F <= 1e-5, the reference's pass rule)."""
import numpy as np
import pytest

from qsv_b200 import engine, precision
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    engine.load()
    return t


def test_precision_study_small(torch):
    n = 16
    qc = precision.config3_circuit(n, depth=8, seed=2)
    s128, fmap, _ = precision.run_state(qc, "c128")
    s64, fmap64, _ = precision.run_state(qc, "c64")
    assert fmap == fmap64
    ref = orc.statevector_f64(qc)
    perm = [fmap[q] for q in range(n)]
    h128 = orc.remap(s128.cpu().numpy(), perm)
    h64 = orc.remap(s64.cpu().numpy(), perm)
    assert np.max(np.abs(h128 - ref)) < 1e-12
    m = precision.compare(s128, s64)
    o = orc.metrics(ref, h64)
    assert m["one_minus_f"] <= 1e-5 and abs(m["one_minus_f"] - o["one_minus_f"]) <= 1e-9
    assert abs(m["max_abs_err"] - o["max_abs_err"]) <= 1e-7
    out = precision.study(n_a=17, n_b=16, depth=8)
    assert out["run_b"]["c64_vs_c128"]["one_minus_f"] <= 1e-5 and abs(out["run_a"]["norm"] - 1) < 1e-4
