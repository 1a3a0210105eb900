"""Specialised sweep kernels, host side: the generated CUDA source compiles (NVRTC, sm_100a) for every sweep
structure of a varied set of circuits -- all window sizes 10..13, both 13-qubit layouts, every op variant
and slot -- with no device involved. Their values are checked against the oracle in test_gpu_jit.py."""
import collections

import pytest

import qsv_b200 as q
from qsv_b200 import engine, generators as gen

CIRCUITS = [
    (10, 8, lambda: gen.random_layer(10, 4, 1)),
    (11, 9, lambda: gen.random_layer_ccx(11, 3, 2)),
    (12, 12, lambda: gen.zoo(12, 3)),
    (16, 12, lambda: gen.zoo(16, 5)),
    (17, 7, lambda: gen.random_layer_ccx(17, 3, 4)),
    (18, 12, lambda: gen.qft(18)),
]


@pytest.fixture(scope="module")
def lib():
    return engine.load()


def _variants(prog, n):
    seen = collections.Counter()
    for kind, seg in prog:
        if kind == "segment":
            for sw in engine.plan_segment(seg, n):
                for o in sw["ops"]:
                    slot = "comp" if o["slot"] == 0 else ("reg" if o["slot"] < 8 else "lane")
                    seen[(slot, o["variant"])] += 1
    return seen


@pytest.mark.timeout(900)
def test_specialised_kernels_compile(lib):
    variants = collections.Counter()
    for rb in (4, 3):
        engine.set_layout13(rb)
        try:
            for n, k, make in CIRCUITS:
                prog, _, _ = q.compile_circuit(make(), n, k)
                variants.update(_variants(prog, n))
                for kind, seg in prog:
                    if kind == "segment":
                        nsw = len(engine.plan_segment(seg, n))
                        assert engine.jit_prepare(seg, n) == nsw, lib.qsv_last_error().decode()
        finally:
            engine.set_layout13(4)
    info = engine.jit_info()
    assert info["failed"] == 0 and info["ready"] == info["structures"] > 10 and info["pending"] == 0
    # every slot kind and the common variants were generated
    slots = {s for s, _ in variants}
    assert slots == {"comp", "reg", "lane"}
    vs = {v for _, v in variants}
    assert {1, 2, 3, 4, 5, 6, 7}.issubset(vs), sorted(vs)


def test_jit_mode_switch(lib):
    old = engine.set_jit("off")
    try:
        assert engine.jit_info()["mode"] == 0
        assert engine.set_jit("eager") == "off"
        assert engine.jit_info()["mode"] == 1
        with pytest.raises(engine.QSVError):
            engine.set_jit(7)
    finally:
        engine.set_jit(old)


def test_exit_with_compilations_in_flight():
    """A process that exits while specialised kernels are compiling in the background exits cleanly."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys, threading, time\n"
        f"sys.path.insert(0, {os.path.join(root, 'tests')!r}); sys.path.insert(0, {root!r})\n"
        "import conftest\n"
        "import qsv_b200 as q\n"
        "from qsv_b200 import engine, generators as gen\n"
        "prog, _, _ = q.compile_circuit(gen.qft(20), 20, 12)\n"
        "segs = [s for k, s in prog if k == 'segment']\n"
        "def bg():\n"
        "    for s in segs: engine.jit_prepare(s, 20)\n"
        "threading.Thread(target=bg, daemon=True).start()\n"
        "time.sleep(0.5)\n"
        "assert engine.jit_info()['pending'] > 0\n"
    )
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]


@pytest.mark.timeout(900)
def test_group_type_library_compiles(lib):
    """The group-type library (one kernel with a case per group type of the streaming form) compiles for the
    types of a random-Toffoli circuit and a Grover circuit (up to 8 kernels of 32 cases: the 16 most swept
    types and a band of 16 more each), and is the library in use afterwards (host work only)."""
    progs = []
    for n, maker in ((18, lambda: gen.random_layer_ccx(18, 8, 5)), (14, lambda: gen.grover(14, 2))):
        prog, _, _ = q.compile_circuit(maker(), n, 12)
        progs += [(seg, n) for kind, seg in prog if kind == "segment"]
    old = engine.set_jit("library")
    try:
        types = engine.jit_prepare_library(progs)
        info = engine.jit_info()
    finally:
        engine.set_jit(old)
    assert 0 < types <= 144
    assert info["lib_types"] == types and info["failed"] == 0


@pytest.mark.timeout(900)
def test_group_type_library_bands(lib):
    """A mix with more group types than one library holds gets several libraries (compiled in parallel on the
    host): the 16 most swept types in each and a band of 16 more, up to 144 distinct types."""
    progs = []
    for s in range(6):
        n = 18 + s % 3
        prog, _, _ = q.compile_circuit(gen.random_layer_ccx(n, 12, 90 + s), n, 12)
        progs += [(seg, n) for kind, seg in prog if kind == "segment"]
    old = engine.set_jit("library")
    try:
        types = engine.jit_prepare_library(progs)
        info = engine.jit_info()
    finally:
        engine.set_jit(old)
    assert 32 < types <= 144, types
    assert info["lib_types"] == types and info["failed"] == 0
