"""The fixed-scratch FP64 reduction (qsv_reduce_f64_noalloc) gives the same result as the scratch-taking
entry point, through the C ABI, on two calls in a row.

It exists for callers that cannot allocate device memory (their device heap belongs to another allocator,
or they must keep a fixed footprint while running); its block partials live in one array compiled into
libqsv_b200.so. Two back-to-back calls on different states check that the second call does not see the
first call's partials. This file is collected last so that a failure here never hides the other tests;
it also passes on its own in a fresh process (the first call does the per-device set-up).
"""
import ctypes
import math

import numpy as np
import pytest

from qsv_b200 import engine

pytestmark = pytest.mark.gpu


def _state(torch, n, seed, dtype=np.complex64):
    rng = np.random.default_rng(seed)
    x = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(dtype)
    return torch.from_numpy(x).cuda()


def test_noalloc_reduction_matches_scratch_reduction():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    lib = engine.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # two calls in a row: a larger state, then a smaller one (fewer partials than the first call left)
    for n, seed in ((22, 1), (14, 2)):
        st = _state(torch, n, seed)
        ref = engine.reduce_f64(st).cpu().numpy()              # entry point with caller scratch
        out = torch.full((n + 1,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.qsv_reduce_f64_noalloc(ctypes.c_void_p(st.data_ptr()), n, 0, ctypes.c_void_p(out.data_ptr()),
                                        stream)
        assert rc == 0, lib.qsv_last_error().decode()
        got = out.cpu().numpy()
        assert math.isclose(got[0], ref[0], rel_tol=1e-12)
        assert np.allclose(got[1:], ref[1:], rtol=1e-10, atol=1e-12)
    # complex128 states use the same array (the partial count does not depend on the amplitude type)
    n = 16
    st = _state(torch, n, 3, np.complex128)
    ref = engine.reduce_f64(st).cpu().numpy()
    out = torch.full((n + 1,), float("nan"), dtype=torch.float64, device="cuda")
    rc = lib.qsv_reduce_f64_noalloc(ctypes.c_void_p(st.data_ptr()), n, 1, ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == 0, lib.qsv_last_error().decode()
    got = out.cpu().numpy()
    assert math.isclose(got[0], ref[0], rel_tol=1e-12)
    assert np.allclose(got[1:], ref[1:], rtol=1e-10, atol=1e-12)
    # sizes outside the supported range, and unknown element types, are rejected before any launch
    rc = lib.qsv_reduce_f64_noalloc(ctypes.c_void_p(st.data_ptr()), 35, 0, ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == -1 and "n out of" in lib.qsv_last_error().decode()
    rc = lib.qsv_reduce_f64_noalloc(ctypes.c_void_p(st.data_ptr()), n, 2, ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == -3 and "dtype" in lib.qsv_last_error().decode()
    assert engine.device_status() == 0


def test_noalloc_capacity_covers_largest_state():
    """The fixed array (256 KiB = 32768 doubles) holds the block partials of the largest supported state,
    computed on the host from the reduction's block size (no 34-qubit state needed); the library also
    checks this at compile time."""
    def bits(n):
        return min(max(n - 10, 13), n, 25)
    need = max((1 << (n - bits(n))) * (bits(n) + 1) for n in range(10, 35))
    assert need == 25600 and need * 8 <= 256 * 1024
