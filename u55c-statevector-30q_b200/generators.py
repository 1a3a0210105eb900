"""Seeded circuit generators.

* The workload circuits the benchmarks are quoted on: ``random_layer`` (U3 on every qubit + CX
  brickwork), ``qft`` (H + controlled phases + reversal swaps) and ``random_layer_ccx`` (U3 + CZ
  brickwork + Toffolis on random distinct triples).
* The reference's benchmark families ``ghz``, ``rqc``, ``vqe`` and ``grover``, restated from
  circuits/generators.py:13-82 with the same seeds and random-draw order, so the same instances run here.
"""
import math

import numpy as np

from .circuit import Circuit

SEED_BASE = 20261005      # circuits/generators.py:10


def random_layer(n, depth, seed):
    """n qubits, `depth` layers; each layer: U3(theta, phi, lam) on every qubit with the three angles
    drawn uniform in [0, 2pi) (default_rng(seed), qubit order, three draws per qubit), then CX(q, q+1)
    for q = layer % 2, layer % 2 + 2, ...  (even offset on even layers, odd on odd layers)."""
    rng = np.random.default_rng(seed)
    qc = Circuit(n, name=f"rl_{n}_d{depth}_s{seed}")
    for layer in range(depth):
        for q in range(n):
            th, ph, lam = (float(x) for x in rng.uniform(0.0, 2 * math.pi, 3))
            qc.u(th, ph, lam, q)
        for q in range(layer % 2, n - 1, 2):
            qc.cx(q, q + 1)
    return qc


def random_layer_ccx(n, depth, seed):
    """Per layer: U3 on every qubit (angles uniform in [0, 2pi)), CZ brickwork (offset layer % 2), then
    n // 4 Toffolis, each on three distinct qubits drawn without replacement (controls a, b; target c)."""
    rng = np.random.default_rng(seed)
    qc = Circuit(n, name=f"rlccx_{n}_d{depth}_s{seed}")
    for layer in range(depth):
        for q in range(n):
            th, ph, lam = (float(x) for x in rng.uniform(0.0, 2 * math.pi, 3))
            qc.u(th, ph, lam, q)
        for q in range(layer % 2, n - 1, 2):
            qc.cz(q, q + 1)
        for _ in range(n // 4):
            a, b, c = (int(x) for x in rng.choice(n, 3, replace=False))
            qc.ccx(a, b, c)
    return qc


def ghz(n):
    qc = Circuit(n, name=f"ghz_{n}")
    qc.h(0)
    for i in range(n - 1):
        qc.cx(i, i + 1)
    return qc


def qft(n, swaps=True):
    """H on each qubit (from the top), controlled phase R_k = diag(1, e^{2 pi i / 2^k}) for every pair
    k < j with R index j - k + 1, then reversal swaps (circuits/generators.py:21-30)."""
    qc = Circuit(n, name=f"qft_{n}")
    for j in reversed(range(n)):
        qc.h(j)
        for k in reversed(range(j)):
            qc.cp(math.pi / 2 ** (j - k), k, j)
    if swaps:
        for i in range(n // 2):
            qc.swap(i, n - 1 - i)
    return qc


def rqc(n, depth=10, seed=None):
    """Brick-wall random circuit (circuits/generators.py:33-49): per layer one of {rx, ry, rz, t, h} on
    every qubit, then CZ on alternating pairs."""
    rng = np.random.default_rng(SEED_BASE + 1000 * n + depth if seed is None else seed)
    qc = Circuit(n, name=f"rqc_{n}_d{depth}")
    for layer in range(depth):
        for q in range(n):
            g = rng.integers(5)
            th = float(rng.uniform(0, 2 * math.pi))
            if g == 0:
                qc.rx(th, q)
            elif g == 1:
                qc.ry(th, q)
            elif g == 2:
                qc.rz(th, q)
            elif g == 3:
                qc.t(q)
            else:
                qc.h(q)
        for q in range(layer % 2, n - 1, 2):
            qc.cz(q, q + 1)
    return qc


def vqe(n, layers=2, seed=None):
    """Hardware-efficient ansatz (circuits/generators.py:52-65)."""
    rng = np.random.default_rng(SEED_BASE + 7 * n + layers if seed is None else seed)
    qc = Circuit(n, name=f"vqe_{n}_L{layers}")
    for _ in range(layers):
        for q in range(n):
            qc.ry(float(rng.uniform(0, 2 * math.pi)), q)
            qc.rz(float(rng.uniform(0, 2 * math.pi)), q)
        for q in range(n - 1):
            qc.cx(q, q + 1)
    for q in range(n):
        qc.ry(float(rng.uniform(0, 2 * math.pi)), q)
        qc.rz(float(rng.uniform(0, 2 * math.pi)), q)
    return qc


def grover(n, marked=None, iters=None):
    """Grover search for one marked item (circuits/generators.py:68-82)."""
    marked = (2 ** n - 1) if marked is None else marked
    iters = int(math.floor(math.pi / 4 * math.sqrt(2 ** n))) if iters is None else iters
    qc = Circuit(n, name=f"grover_{n}")
    qc.h(range(n))
    for _ in range(iters):
        for q in range(n):
            if not (marked >> q) & 1:
                qc.x(q)
        qc.h(n - 1)
        qc.mcx(list(range(n - 1)), n - 1)
        qc.h(n - 1)
        for q in range(n):
            if not (marked >> q) & 1:
                qc.x(q)
        qc.h(range(n))
        qc.x(range(n))
        qc.h(n - 1)
        qc.mcx(list(range(n - 1)), n - 1)
        qc.h(n - 1)
        qc.x(range(n))
        qc.h(range(n))
    return qc


FAMILIES = {"ghz": ghz, "qft": qft, "rqc": rqc, "vqe": vqe, "grover": grover}


def make(family, n, **kw):
    return FAMILIES[family](n, **kw)


def zoo(n, seed):
    """Random circuit over the standard gate set plus CCX, 12*n gates (tests/circuit_zoo.py:6-22)."""
    rng = np.random.default_rng(seed)
    qc = Circuit(n, name=f"zoo_{n}_{seed}")
    one = ["h", "x", "y", "z", "s", "sdg", "t", "tdg", "sx", "sxdg"]
    par1 = ["rx", "ry", "rz", "p"]
    two = ["cx", "cy", "cz", "ch", "swap", "iswap", "ecr", "dcx", "csx"]
    par2 = ["rxx", "ryy", "rzz", "rzx", "cp", "crx", "cry", "crz"]
    for _ in range(12 * n):
        r = rng.integers(6)
        q = [int(x) for x in rng.choice(n, 3, replace=False)]
        th = float(rng.uniform(-np.pi, np.pi))
        if r == 0:
            qc.append(str(rng.choice(one)), (q[0],))
        elif r == 1:
            qc.append(str(rng.choice(par1)), (q[0],), (th,))
        elif r == 2:
            qc.append(str(rng.choice(two)), (q[0], q[1]))
        elif r == 3:
            qc.append(str(rng.choice(par2)), (q[0], q[1]), (th,))
        elif r == 4:
            qc.u(th, th / 2, -th / 3, q[0])
        else:
            qc.ccx(q[0], q[1], q[2])
    return qc
