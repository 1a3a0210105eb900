"""The streaming plan (qsv_plan_stream), host side: structure and meaning, with no device involved.

plan_stream cuts each sweep's ops into groups of consecutive ops whose targets span at most three tile bits
(item bits q0..q2); ops on tile bit 0, and diagonal ops on any other bit, ride along. The streaming kernels
(interpreter and group-type library) then run a group on items of 16 amplitudes (tile bits 0, q0, q1, q2)
and read each op's controls split into cm_reg (item bits) and cm_thr (the item base). This test checks the
structure of the plan against the phase plan of the same sweeps and, in float64, that applying every group
item by item with that split gives what applying the ops one by one on the whole tile gives (the
pass semantics of host/sv/model.py:43-70: pairs along the target, M1 where every control is set). The
kernels' values are checked against the oracle on the GPU in test_gpu_stream.py and test_gpu_library.py.
"""
import numpy as np
import pytest

import qsv_b200 as q
from qsv_b200 import engine, generators as gen

CIRCUITS = [
    (10, 8, lambda: gen.random_layer(10, 4, 1)),
    (11, 9, lambda: gen.random_layer_ccx(11, 3, 2)),
    (12, 12, lambda: gen.zoo(12, 3)),
    (14, 12, lambda: gen.grover(14, 2, 1)),
    (16, 12, lambda: gen.zoo(16, 5)),
    (16, 12, lambda: gen.rqc(16, 6, 3)),
    (16, 12, lambda: gen.vqe(16, 2, 4)),
    (17, 12, lambda: gen.qft(17)),
    (18, 12, lambda: gen.random_layer_ccx(18, 6, 5)),
]

SKIP, UNI_DIAG, CTRL_DIAG1 = 0, 2, 5
UNI, CTRL, MUX = 0, 1, 2


@pytest.fixture(scope="module")
def lib():
    return engine.load()


def _mats(op):
    m0 = op["m0"].astype(np.float64)
    m1 = op["m1"].astype(np.float64)
    M0 = np.array([[m0[0] + 1j * m0[1], m0[2] + 1j * m0[3]], [m0[4] + 1j * m0[5], m0[6] + 1j * m0[7]]])
    M1 = np.array([[m1[0] + 1j * m1[1], m1[2] + 1j * m1[3]], [m1[4] + 1j * m1[5], m1[6] + 1j * m1[7]]])
    return M0, M1


def _pair_update(x0, x1, sel, kind, M0, M1):
    """y = M1 x where sel, else M0 x (identity for CTRL ops): the same float64 arithmetic on both paths."""
    A = np.where(sel[..., None, None], M1, np.eye(2) if kind == CTRL else M0)
    if kind == UNI:
        A = np.broadcast_to(M0, A.shape)
    y0 = A[..., 0, 0] * x0 + A[..., 0, 1] * x1
    y1 = A[..., 1, 0] * x0 + A[..., 1, 1] * x1
    return y0, y1


def _apply_tile(T, op, M0, M1, kw):
    """One op on the whole tile, as the pass semantics define it."""
    t, cm = op["tbit"], op["cmask"]
    idx = np.arange(1 << kw)
    lo = idx[((idx >> t) & 1) == 0]
    hi = lo | (1 << t)
    sel = (lo & cm) == cm
    T[lo], T[hi] = _pair_update(T[lo], T[hi], sel, op["kind"], M0, M1)


def _apply_groups(T, sp, phase_ops, kw):
    """Every group item by item, with the streaming plan's slots and control split."""
    for g in sp["groups"]:
        qb = g["q"]
        mask = 1 | (1 << qb[0]) | (1 << qb[1]) | (1 << qb[2])
        all_idx = np.arange(1 << kw)
        bases = all_idx[(all_idx & mask) == 0]
        # local index l = h + 2 r (h: tile bit 0, r: item bits q0 q1 q2)
        loc = np.array([(l & 1) | (((l >> 1) & 1) << qb[0]) | (((l >> 2) & 1) << qb[1]) | (((l >> 3) & 1) << qb[2])
                        for l in range(16)])
        X = T[bases[:, None] | loc[None, :]]
        for o in range(g["op_begin"], g["op_end"]):
            so, po = sp["ops"][o], phase_ops[o]
            if so["variant"] == SKIP:
                continue
            M0, M1 = _mats(po)
            base_ok = (bases & so["cm_thr"]) == so["cm_thr"]
            cm0 = po["cmask"] & 1
            slot = so["slot"]
            if slot == 7:
                assert so["variant"] in (UNI_DIAG, CTRL_DIAG1)
                one = ((bases >> so["tbit"]) & 1).astype(bool)
                for l in range(16):
                    r = l >> 1
                    if so["variant"] == UNI_DIAG:
                        X[:, l] *= np.where(one, M0[1, 1], M0[0, 0])
                    else:
                        ok = base_ok & one & ((r & so["cm_reg"]) == so["cm_reg"]) & (not cm0 or (l & 1) == 1)
                        X[:, l] = np.where(ok, M1[1, 1] * X[:, l], X[:, l])
                continue
            bit = 0 if slot == 0 else slot          # local bit of the target: 0 (tile bit 0) or 1 + k
            for l in range(16):
                if (l >> bit) & 1:
                    continue
                r = l >> 1
                sel = base_ok & ((r & so["cm_reg"]) == so["cm_reg"]) & (not cm0 or (l & 1) == 1)
                X[:, l], X[:, l | (1 << bit)] = _pair_update(X[:, l], X[:, l | (1 << bit)], sel, po["kind"], M0, M1)
        T[bases[:, None] | loc[None, :]] = X


@pytest.mark.timeout(900)
@pytest.mark.parametrize("n,k,maker", CIRCUITS)
def test_stream_plan_structure_and_meaning(lib, n, k, maker):
    prog, _, _ = q.compile_circuit(maker(), n, k)
    rng = np.random.default_rng(n)
    for kind, seg in prog:
        if kind != "segment":
            continue
        phase = engine.plan_segment(seg, n)
        stream = engine.plan_stream(seg, n)
        assert len(phase) == len(stream)
        for ph, sp in zip(phase, stream):
            kw, ops = sp["kw"], sp["ops"]
            assert kw == ph["kw"] and len(ops) == len(ph["ops"])
            groups = sp["groups"]
            # groups partition the ops in order; at most nops / 3 + 1 of them
            assert groups[0]["op_begin"] == 0 and groups[-1]["op_end"] == len(ops)
            for a, b in zip(groups, groups[1:]):
                assert a["op_end"] == b["op_begin"] and a["op_begin"] < a["op_end"]
            assert len(groups) <= len(ops) // 3 + 1
            for gi, g in enumerate(groups):
                qb = g["q"]
                assert len(set(qb)) == 3 and all(1 <= x < kw for x in qb)
                item = 1 | sum(1 << x for x in qb)
                targets = set()
                for o in range(g["op_begin"], g["op_end"]):
                    so, po = ops[o], ph["ops"][o]
                    assert (so["tbit"], so["cmask"], so["kind"]) == (po["tbit"], po["cmask"], po["kind"])
                    t = so["tbit"]
                    want = 0 if t == 0 else (1 + qb.index(t) if t in qb else 7)
                    assert so["slot"] == want
                    if want == 7:
                        assert so["variant"] in (SKIP, UNI_DIAG, CTRL_DIAG1)
                    elif t != 0 and so["variant"] not in (SKIP, UNI_DIAG, CTRL_DIAG1):
                        targets.add(t)
                    assert so["cm_reg"] == sum(((so["cmask"] >> x) & 1) << i for i, x in enumerate(qb))
                    assert so["cm_thr"] == so["cmask"] & ~item
                # greedy: a group closes only when a fourth distinct target arrives
                if gi + 1 < len(groups):
                    nxt = ops[g["op_end"]]
                    assert len(targets) == 3 and nxt["tbit"] not in targets and nxt["tbit"] != 0
                    assert nxt["variant"] not in (SKIP, UNI_DIAG, CTRL_DIAG1)
            # meaning: item by item with the plan's split == op by op on the whole tile (float64)
            T0 = rng.standard_normal(1 << kw) + 1j * rng.standard_normal(1 << kw)
            A = T0.copy()
            for po in ph["ops"]:
                M0, M1 = _mats(po)
                _apply_tile(A, po, M0, M1, kw)
            B = T0.copy()
            _apply_groups(B, sp, ph["ops"], kw)
            # the two paths differ only in numpy's rounding (a broadcast scalar factor against an elementwise
            # one: ~1e-15); a misplaced item bit or control split changes amplitudes by O(1)
            assert np.allclose(A, B, rtol=0, atol=1e-10), np.max(np.abs(A - B))
