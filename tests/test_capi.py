"""The C ABI library builds for sm_100a, loads without a GPU, exports every symbol include/qsv_b200.h
declares, and its host-side planner (QSV2 decode -> sweep plan) keeps the program's semantics:
the plan's ops, read back in physical qubits, are the segment's ops in the same order with the same
matrices, every op fits its sweep window, and every target has a slot in its phase."""
import ctypes
import os
import re

import numpy as np
import pytest

import qsv_b200 as q
from qsv_b200 import engine, generators as gen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    from importlib import import_module
    b = import_module("qsv_b200.build")
    b.build()
    return engine.load()


def test_header_symbols_exported(lib):
    hdr = open(os.path.join(ROOT, "include", "qsv_b200.h")).read()
    declared = set(re.findall(r"^QSV_API\s+[\w\s\*]*?\b(qsv_\w+)\s*\(", hdr, re.M))
    assert {"qsv_run_segment", "qsv_remap", "qsv_zero_state", "qsv_last_error"} <= declared
    for name in declared:
        assert hasattr(lib, name), name
    assert set(engine.exported_symbols()) == declared
    assert lib.qsv_version() >= 100


def _segment_ops_phys(seg):
    """Ops of a QSV2 segment in physical coordinates, in order: (t, ctrl set, m0 bits, m1 bits)."""
    w = np.asarray(seg, dtype=np.int32)
    k = int(w[3])
    pos = 8
    out = []
    for _ in range(int(w[2])):
        m, nops = int(w[pos]), int(w[pos + 3])
        h = [int(w[pos + 1]), int(w[pos + 2]), int(w[pos + 4]), int(w[pos + 5])]
        pos += 8
        phys = lambda tq: tq if tq < k - m else h[tq - (k - m)]  # noqa: E731
        for _ in range(nops):
            t, cm = int(w[pos + 1]), int(w[pos + 2])
            ctrls = frozenset(phys(b) for b in range(k) if (cm >> b) & 1)
            out.append((phys(t), ctrls, tuple(w[pos + 8:pos + 16]), tuple(w[pos + 16:pos + 24])))
            pos += 24
    return out


def _plan_ops_phys(plan):
    out = []
    for sw in plan:
        W = sw["window"]
        rb = len(sw["phases"][0]["reg_bits"])
        for ph in sw["phases"]:
            for o in range(ph["op_begin"], ph["op_end"]):
                op = sw["ops"][o]
                tb = op["tbit"]
                # lane bits 0-2: tile bits 1-3, or in a swizzled sweep one of each pair (1+l, 4+l)
                if sw["swizzled"]:
                    assert all(ph["lane_lo"][l] in (1 + l, 4 + l) for l in range(3)), ph["lane_lo"]
                else:
                    assert ph["lane_lo"] == [1, 2, 3]
                # slot placement
                if tb == 0:
                    assert op["slot"] == 0
                elif tb in ph["lane_lo"]:
                    assert op["slot"] == 8 + ph["lane_lo"].index(tb)
                elif tb in ph["reg_bits"]:
                    assert op["slot"] == 1 + ph["reg_bits"].index(tb)
                else:
                    assert tb in ph["lane_bits"] and op["slot"] == 11 + ph["lane_bits"].index(tb)
                # the phase layout covers every tile bit exactly once
                bits = sorted([0] + ph["lane_lo"] + ph["reg_bits"] + ph["lane_bits"] + ph["warp_bits"])
                assert bits == list(range(sw["kw"])), bits
                assert len(ph["reg_bits"]) == rb
                ctrls = frozenset(W[b] for b in range(sw["kw"]) if (op["cmask"] >> b) & 1)
                out.append((W[tb], ctrls, tuple(op["m0"].view(np.int32)), tuple(op["m1"].view(np.int32))))
        if sw["swizzled"]:                       # staged by 128-byte-swizzled tensor-map boxes
            assert sw["tma_rank"] > 0 and sw["tdim_box"][0] == 4 and sw["lo"] >= 4
        assert sw["lo"] >= 3 and len(W) == sw["kw"] and len(set(W)) == sw["kw"]
        assert W == sorted(W)
    return out


@pytest.mark.parametrize("n,k,M,maker", [
    (16, 12, 4, lambda: gen.random_layer(16, 8, 3)),
    (14, 10, 4, lambda: gen.random_layer_ccx(14, 5, 4)),
    (13, 8, 3, lambda: gen.qft(13)),
    (12, 12, 4, lambda: gen.zoo(12, 5)),
    (20, 12, 4, lambda: gen.random_layer(20, 6, 0)),
    (11, 5, 2, lambda: gen.vqe(11, 3)),
])
def test_plan_preserves_program(lib, n, k, M, maker):
    prog, fmap, st = q.compile_circuit(maker(), n, k, max_high=M)
    for kind, seg in prog:
        if kind != "segment":
            continue
        plan = engine.plan_segment(seg, n)
        seg_ops = _segment_ops_phys(seg)
        plan_ops = _plan_ops_phys(plan)
        assert len(plan) <= int(np.asarray(seg)[2])
        # ops with identical M0/M1 may have had their (irrelevant) controls dropped
        assert len(seg_ops) == len(plan_ops)
        for a, b in zip(seg_ops, plan_ops):
            assert a[0] == b[0] and a[2] == b[2] and a[3] == b[3]
            assert a[1] == b[1] or (a[2] == a[3] and not b[1])


def test_plan_merges_passes(lib):
    qc = gen.random_layer(30, 24, 1)
    prog, fmap, st = q.compile_circuit(qc, 30, 12)
    plan = engine.plan_segment(prog[0][1], 30)
    assert st.n_passes == 133
    assert len(plan) < 0.7 * st.n_passes        # 13-qubit windows absorb neighbouring 12-qubit passes


def test_bad_streams_rejected(lib):
    qc = gen.random_layer(12, 3, 0)
    prog, _, _ = q.compile_circuit(qc, 12, 8)
    seg = np.array(prog[0][1])
    bad = seg.copy(); bad[0] = 7
    with pytest.raises(engine.BadStream):
        engine.plan_segment(bad, 12)
    with pytest.raises(engine.BadStream):
        engine.plan_segment(seg[:-3], 12)
    with pytest.raises(engine.BadStream):
        engine.plan_segment(seg, 13)                 # L mismatch
    bad = seg.copy(); bad[8 + 8] = 5                # opcode of the first record
    with pytest.raises(engine.BadStream):
        engine.plan_segment(bad, 12)
    bad = seg.copy(); bad[8] = 9                    # m > MAX_HIGH
    with pytest.raises(engine.BadStream):
        engine.plan_segment(bad, 12)
    with pytest.raises(engine.QSVError):
        engine.plan_segment(seg, 40)


def test_wide_window_unsupported(lib):
    # a 14-qubit controlled op cannot fit one 13-qubit window
    qc = q.Circuit(16)
    qc.mcx(list(range(13)), 15)
    prog, _, _ = q.compile_circuit(qc, 16, 16, max_high=2)
    with pytest.raises(engine.QSVError) as ei:
        engine.plan_segment(prog[0][1], 16)
    assert ei.value.code == -3


def test_no_gpu_calls_fail_loudly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(RuntimeError):
        engine.new_state(12)


def test_swizzled_plans_remove_shuffles(lib):
    """RL-30: most sweeps take the swizzled layout, and the ones over qubits 0-12 (12-13 dense ops) keep at
    most three warp-shuffle ops (with lane bits fixed on tile bits 1-3 they had five or six)."""
    prog, fmap, st = q.compile_circuit(gen.random_layer(30, 24, 1), 30, 12)
    plan = engine.plan_segment(prog[0][1], 30)
    assert len(plan) == 84
    assert sum(sw["swizzled"] for sw in plan) >= 60
    for sw in plan:
        if sw["lo"] >= 9 and len(sw["ops"]) >= 12:
            shuffles = sum(1 for o in sw["ops"] if o["slot"] >= 8 and o["variant"] != 0)
            assert sw["swizzled"] and shuffles <= 3, (sw["lo"], shuffles)
