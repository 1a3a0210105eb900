"""The sharded runtime's GPU slice backend (CudaSlices: this package's engine) in a process group of one
rank: no exchanges, so the whole state is one slice and every result must equal the single-GPU runtime's
(state bit for bit; <Z> and norm from the state). The exchanges themselves are covered with 2 and 4 ranks
on CPU (test_sharded_host.py); runs of several GPUs are not available here."""
import os
import socket

import numpy as np
import pytest

from qsv_b200 import generators as gen
from qsv_b200.runtime import SVRuntime

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def group():
    import torch
    import torch.distributed as dist
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=0, world_size=1, timeout=timedelta(seconds=60))
    yield dist
    dist.destroy_process_group()


@pytest.mark.timeout(600)
@pytest.mark.parametrize("kind,n", [("rl", 16), ("ccx", 18), ("qft", 14)])
def test_one_rank_equals_single_gpu_runtime(group, kind, n):
    from qsv_b200.sharded import ShardedRuntime
    qc = {"rl": lambda: gen.random_layer(n, 8, 2), "ccx": lambda: gen.random_layer_ccx(n, 6, 3),
          "qft": lambda: gen.qft(n)}[kind]()
    r = ShardedRuntime().run(qc, shots=2000, return_state=True, seed=9)
    ref = SVRuntime().run(qc, shots=0, return_state=True)["state"]
    assert np.array_equal(r["state"], ref)
    p = np.abs(ref.astype(np.complex128)) ** 2
    idx = np.arange(p.size)
    z = np.array([np.sum(p * (1 - 2 * ((idx >> q) & 1))) for q in range(n)]) / p.sum()
    assert abs(r["norm"] - p.sum()) < 1e-6 and np.max(np.abs(r["expect_z"] - z)) < 1e-6
    assert sum(r["counts"].values()) == 2000 and r["exchanges"] == 0
