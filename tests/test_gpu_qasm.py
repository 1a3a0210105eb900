"""OpenQASM 2 text runs through the drop-in runtime (SVRuntime.run accepts OpenQASM text or a .qasm
path, as the reference's circuits come as files): 1 - F <= 1e-5 against the FP64 oracle."""
import pytest

from qsv_b200 import engine, generators as gen
from qsv_b200.qasm import from_qasm, to_qasm
from qsv_b200.runtime import SVRuntime
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def test_runtime_runs_qasm_text():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    engine.load()
    for qc in (gen.qft(12), gen.rqc(14, 6, 2), gen.vqe(13, 2, 5)):
        text = to_qasm(qc)
        r = SVRuntime().run(text, shots=64, seed=1)
        ref = orc.statevector_f64(from_qasm(text))
        assert orc.metrics(ref, r["state"])["one_minus_f"] <= 1e-5
        assert sum(r["counts"].values()) == 64
