"""The compiler's fast paths agree with the plain definitions they replace (CPU): the incremental window
test of the scheduler with pass_window, the cached 2-qubit records with a fresh decomposition, and the
scheduler's output with a plain re-statement of the reference's greedy pass packing."""
import numpy as np

from qsv_b200 import compiler as C, generators as gen
from qsv_b200.gates import gate_matrix


def test_fits_matches_pass_window():
    rng = np.random.default_rng(0)
    for _ in range(3000):
        k = int(rng.integers(4, 14))
        M = int(rng.integers(0, min(4, k - 3) + 1))
        qs = set(int(x) for x in rng.integers(0, k + 8, int(rng.integers(1, 9))))
        hi = sorted(q for q in qs if q >= k - M)
        assert C._fits(hi, k, M) == (C.pass_window(qs, k, M) is not None), (qs, k, M)


def test_cached_2q_records_equal_fresh():
    rng = np.random.default_rng(1)
    mats = [gate_matrix(g) for g in ("cx", "cz", "swap", "iswap", "ecr", "dcx", "ch", "cy", "csx")]
    mats += [gate_matrix(g, [float(rng.uniform(-3, 3))]) for g in ("cp", "crx", "cry", "crz", "rxx", "ryy", "rzz", "rzx")]
    for M in mats + mats:                                # second round: from the cache
        st = C.Stats()
        got = C.ops_2q(M, 3, 5, st)
        recs, csd = C._ops_2q_records(M)
        assert st.csd_2q == int(csd) and len(got) == len(recs)
        for op, (ta, m0, m1) in zip(got, recs):
            assert (op.t, op.ctrls) == ((3, (5,)) if ta else (5, (3,)))
            assert np.array_equal(op.M0, m0) and np.array_equal(op.M1, m1)


def _plain_passes(ops, k, M):
    """The reference's greedy packing without remaps (every op fits a window): an op joins the open pass
    while the pass's qubits fit one window and it holds fewer than 64 ops."""
    passes, cur, qs = [], [], set()
    for op in ops:
        grown = qs | set(op.q)
        if len(cur) >= C.MAX_OPS_PER_PASS or C.pass_window(grown, k, M) is None:
            passes.append(cur)
            cur, grown = [], set(op.q)
        cur.append(op)
        qs = grown
    if cur:
        passes.append(cur)
    return passes


def test_schedule_matches_plain_packing():
    for qc, n in ((gen.random_layer(20, 8, 3), 20), (gen.qft(16), 16), (gen.rqc(18), 18), (gen.vqe(14), 14)):
        st = C.Stats()
        ops, _ = C.circuit_to_ops(qc, st, True, max_width=12)
        steps, _ = C.schedule(ops, n, n, 12, C.Stats(), M=4)
        assert [kind for kind, _ in steps] == ["segment"]
        got = [[op for op, _ in p] for p in steps[0][1]]
        want = _plain_passes(ops, 12, 4)
        assert [len(p) for p in got] == [len(p) for p in want]
        assert all(a is b for pa, pb in zip(got, want) for a, b in zip(pa, pb))
