"""Sharded runtime (one state over G ranks, the reference's multi-card runtime) on CPU: gloo process
groups of 2 and 4 ranks, each rank's slice run by the C oracle in place of the GPU engine (a stand-in
defined here, in the tests only: the product path is CudaSlices). Checks that the exchanges, relabellings
and local permutations reproduce the single-slice execution of the same ops value for value, and that the
distributed <Z>, norm and Born samples agree with the gathered state."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

import conftest  # noqa: F401  (registers the package as qsv_b200; spawned ranks import this module)
from qsv_b200 import compiler as C, generators as gen
from qsv_b200.runtime import transpositions
from oracle import oracle as orc


class OracleSlices:
    """A slice on the host, run by the C oracle (test stand-in for the GPU engine)."""

    def alloc(self, L):
        import torch
        return torch.zeros(1 << L, dtype=torch.complex64)

    def zero(self, state, one):
        state.zero_()
        if one:
            state[0] = 1

    def run_segment(self, state, seg):
        orc.run_segment(state.numpy(), seg)

    def permute(self, state, perm):
        import torch
        return torch.from_numpy(orc.remap(state.numpy(), perm))

    def reduce(self, state):
        p = np.abs(state.numpy().astype(np.complex128)) ** 2
        L = state.numel().bit_length() - 1
        idx = np.arange(p.size)
        return np.array([p.sum()] + [np.sum(p * (1 - 2 * ((idx >> q) & 1))) for q in range(L)])

    def sample(self, state, u):
        p = np.abs(state.numpy().astype(np.complex128)) ** 2
        cdf = np.cumsum(p)
        return np.minimum(np.searchsorted(cdf, np.asarray(u) * cdf[-1], side="right"), p.size - 1).astype(np.int64)

    def synchronize(self):
        pass


def _circuit(kind, n):
    return {"rl": lambda: gen.random_layer(n, 6, n), "ccx": lambda: gen.random_layer_ccx(n, 4, n + 1),
            "qft": lambda: gen.qft(n), "rqc": lambda: gen.rqc(n)}[kind]()


def _rank_main(rank, world, port, cases, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from qsv_b200.sharded import ShardedRuntime
        rt = ShardedRuntime(slices=OracleSlices(), piece_bytes=4096)      # small pieces: several per exchange
        out = []
        for kind, n, k in cases:
            r = rt.run(_circuit(kind, n), shots=4000, k=k, return_state=True, seed=5)
            if rank == 0:
                out.append((kind, n, k, r["state"], r["expect_z"], r["norm"], r["counts"], r["exchanges"]))
        # general permutations of a random state (bank <-> bank relabelling, exchanges, local permutations)
        import torch
        n = 12
        L = n - (world.bit_length() - 1)
        full = _random_state(n, 11)
        perms = []
        for t in range(4):
            perm = [int(v) for v in np.random.default_rng(100 + t).permutation(n)]
            rt.held = list(range(world))
            st = torch.from_numpy(full[rank << L:(rank + 1) << L].copy())
            st = rt._remap(st, perm, L)
            parts = [torch.empty_like(torch.view_as_real(st)) for _ in range(world)] if rank == 0 else None
            dist.gather(torch.view_as_real(st.contiguous()), parts, dst=0)
            if rank == 0:
                got = np.empty_like(full)
                for r_, p_ in enumerate(parts):
                    s_ = rt.held[r_]
                    got[s_ << L:(s_ + 1) << L] = torch.view_as_complex(p_).numpy()
                perms.append((perm, got))
        if rank == 0:
            q.put((out, perms))
    finally:
        dist.destroy_process_group()


def _random_state(n, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)).astype(np.complex64)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_world(world, cases):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, cases, q)) for r in range(world)]
    for p in procs:
        p.start()
    import queue
    import time
    out, t0 = None, time.time()
    try:
        while out is None and time.time() - t0 < 600:
            try:
                out = q.get(timeout=2)
            except queue.Empty:
                if any(p.exitcode not in (None, 0) for p in procs):
                    break                      # a rank failed: stop waiting
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert out is not None and all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return out


def _check(res):
    out, perms = res
    full = _random_state(12, 11)
    for perm, got in perms:
        assert np.array_equal(got, orc.remap(full, perm)), perm
    for kind, n, k, state, z, norm, counts, n_exch in out:
        prog, fmap, _ = C.compile_circuit(_circuit(kind, n), n, k)            # one slice, same ops
        ref = orc.run_program(prog, n, fmap)
        assert np.array_equal(state, ref), (kind, n, k, np.max(np.abs(state - ref)))
        p = np.abs(ref.astype(np.complex128)) ** 2
        idx = np.arange(p.size)
        zr = np.array([np.sum(p * (1 - 2 * ((idx >> q) & 1))) for q in range(n)]) / p.sum()
        assert abs(norm - p.sum()) < 1e-9 and np.max(np.abs(z - zr)) < 1e-9
        assert sum(counts.values()) == 4000
        # Born samples: total variation distance to the exact distribution (the reference's check)
        emp = np.zeros(p.size)
        for index, c in counts.items():                 # logical index -> count
            emp[index] += c / 4000
        assert 0.5 * np.abs(emp - p / p.sum()).sum() < 0.5
        assert n_exch > 0, "the case should exchange half slices"


@pytest.mark.timeout(900)
def test_sharded_two_ranks_equals_single_slice():
    _check(_run_world(2, [("rl", 12, 8), ("ccx", 13, 10), ("qft", 12, 11)]))


@pytest.mark.timeout(900)
def test_sharded_four_ranks_equals_single_slice():
    _check(_run_world(4, [("rl", 12, 8), ("rqc", 13, 9)]))


def test_transpositions_compose_to_the_permutation():
    """Applying the remap's transpositions last to first (as the sharded runtime does) is the permutation
    itself, for any permutation (the scheduler's remaps are disjoint transpositions, for which any order
    is)."""
    rng = np.random.default_rng(3)
    x = (rng.standard_normal(1 << 10) + 1j * rng.standard_normal(1 << 10)).astype(np.complex64)
    for _ in range(20):
        perm = [int(v) for v in rng.permutation(10)]
        y = x.copy()
        for a, b in reversed(transpositions(perm)):
            t = list(range(10))
            t[a], t[b] = b, a
            y = orc.remap(y, t)
        assert np.array_equal(y, orc.remap(x, perm))
