"""Generates the golden fixtures in this directory from the reference implementation itself.

Run once, in a container where the reference tree is present (it is not on GPU hosts):

    python tests/golden/make_golden.py <reference root>     (or QSV_REFERENCE_ROOT=<reference root>)

What it runs from the reference (imported from its own files, unmodified):
  * host/sv/compiler.py  compile_circuit / schedule / encode_segment -- with a minimal stand-in for the
    ``qiskit`` module (Qiskit is not installed here): QuantumCircuit is this package's Circuit and
    ``Operator(op).data`` is the gate matrix from this package's gate table, so both compilers see the
    same matrices and any difference in the emitted words comes from the lowering/scheduling/encoding.
  * host/sv/model.py     run_program / run_segment / remap / unpermute (the golden model).
What it writes:
  streams.json     sha256 of every compiled program (segment words and remaps), final maps and stats for the
                   reference test grid (tests/test_compiler_model.py:17-27 shapes), plus full words for
                   a few cases;
  model_states.npz golden-model outputs (complex64) for a subset of programs, per-segment in/out pairs
                   on random input states, and remap in/out pairs.
"""
import hashlib
import itertools
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def load_pkg():
    import importlib.util
    pkg_dir = os.path.join(ROOT, "u55c-statevector-30q_b200")
    spec = importlib.util.spec_from_file_location("qsv_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["qsv_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def install_qiskit_standin(pkg):
    from qsv_b200.gates import gate_matrix

    class Operator:
        def __init__(self, op):
            self.data = gate_matrix(op.name, op.params)

    def transpile(*a, **k):
        raise NotImplementedError("transpile is not available in the stand-in")

    qiskit = types.ModuleType("qiskit")
    qiskit.QuantumCircuit = pkg.Circuit
    qiskit.transpile = transpile
    qi = types.ModuleType("qiskit.quantum_info")
    qi.Operator = Operator
    qiskit.quantum_info = qi
    sys.modules["qiskit"] = qiskit
    sys.modules["qiskit.quantum_info"] = qi


def prog_sha(prog):
    """sha256 over the whole program: b"S" + segment words, b"R" + permutation, per step (int32 LE)."""
    h = hashlib.sha256()
    for kind, payload in prog:
        h.update(b"S" if kind == "segment" else b"R")
        h.update(np.ascontiguousarray(payload, dtype=np.int32).tobytes())
    return h.hexdigest()


def circuits(gen, n):
    out = [gen.zoo(n, s) for s in range(4)]
    out += [gen.make(f, n) for f in ("ghz", "qft", "rqc", "vqe")]
    out += [gen.random_layer(n, 6, 100 + n), gen.random_layer_ccx(n, 4, 200 + n)]
    if n <= 9:
        out.append(gen.grover(n))
    return out


def main(ref):
    pkg = load_pkg()
    gen = pkg.generators
    install_qiskit_standin(pkg)
    sys.path[:0] = [os.path.join(ref, "host", "sv")]
    import compiler as rc        # reference compiler
    import model as rm           # reference golden model

    records = []
    full = []
    states = {}
    sidx = 0
    for n in (5, 7, 9):
        for qc in circuits(gen, n):
            for P, k, fuse, tiling in itertools.product((1, 2, 4), (3, 4, 5), (True, False), (True, False)):
                L = n - int(np.log2(P))
                if k > L:
                    continue
                for init in (None, list(range(n))[::-1]):
                    try:
                        prog, fmap, st = rc.compile_circuit(qc, L, k, fuse_1q=fuse, tiling=tiling,
                                                            initial_map=init)
                    except Exception as e:   # recorded so the restatement must fail the same way
                        records.append(dict(circuit=qc.name, n=n, P=P, L=L, k=k, fuse=fuse, tiling=tiling,
                                            init=init is not None, error=type(e).__name__))
                        continue
                    rec = dict(circuit=qc.name, n=n, P=P, L=L, k=k, fuse=fuse, tiling=tiling,
                               init=init is not None, sha=prog_sha(prog), n_steps=len(prog),
                               final_map=[int(x) for x in fmap],
                               stats={a: b for a, b in st.__dict__.items() if a not in ("native", "lowered")})
                    # golden-model output for a deterministic subset (P = 1 and P = 2, fused, tiled)
                    if fuse and tiling and P in (1, 2) and k in (4, 5):
                        out = rm.run_program(prog, n, P, fmap)
                        key = f"prog{sidx}"
                        states[key] = out.astype(np.complex64)
                        rec["state_key"] = key
                        sidx += 1
                    if len(full) < 12 and P == 1 and fuse and tiling and k == 5 and init is None:
                        rec["words"] = [[kind, [int(x) for x in payload]] for kind, payload in prog]
                        full.append(rec["circuit"])
                    records.append(rec)

    # per-segment golden pairs at n = 12 on random normalised input states
    rng = np.random.default_rng(12345)
    seg_cases = []
    for j, (qc, k, M) in enumerate([(gen.random_layer(12, 4, 7), 8, 4), (gen.random_layer_ccx(12, 3, 8), 7, 4),
                                    (gen.qft(12), 6, 3), (gen.zoo(12, 9), 8, 4), (gen.grover(8), 8, 4)]):
        n = qc.num_qubits
        prog, fmap, st = rc.compile_circuit(qc, n, k, max_high=M)
        seg = next(p for kd, p in prog if kd == "segment")
        x = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(np.complex64)
        x /= np.float32(np.linalg.norm(x))
        y = x.copy()
        rm.run_segment(y, 1, seg)
        states[f"seg{j}_in"] = x
        states[f"seg{j}_out"] = y
        states[f"seg{j}_words"] = np.asarray(seg, dtype=np.int32)
        seg_cases.append(dict(key=f"seg{j}", n=n, circuit=qc.name, k=k, M=M))

    # remap golden pairs (pure permutations; exact)
    remap_cases = []
    for j, n in enumerate((6, 9, 10, 11)):
        perm = [int(v) for v in rng.permutation(n)]
        x = (np.arange(1 << n) + 1j * np.arange(1 << n)[::-1]).astype(np.complex64)
        states[f"remap{j}_in"] = x
        states[f"remap{j}_out"] = rm.remap(x, n, perm)
        fmap = [int(v) for v in rng.permutation(n)]
        states[f"unperm{j}_out"] = rm.unpermute(x, n, fmap)
        remap_cases.append(dict(key=f"remap{j}", n=n, perm=perm, final_map=fmap))

    json.dump(dict(reference="nasir26/u55c-statevector-30q host/sv/{compiler,model}.py",
                   records=records, segments=seg_cases, remaps=remap_cases),
              open(os.path.join(HERE, "streams.json"), "w"))
    np.savez_compressed(os.path.join(HERE, "model_states.npz"), **states)
    print(f"records={len(records)} full={len(full)} states={len(states)}")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("QSV_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py <reference root>  (or set QSV_REFERENCE_ROOT)")
    main(root)
