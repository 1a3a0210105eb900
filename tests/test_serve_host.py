"""Host side of the serving loop (no GPU): the request generator follows its stated distributions."""
import math

import numpy as np

from qsv_b200.serve import config5_requests


def test_config5_requests_distribution():
    reqs = config5_requests(count=4000, rate=200.0, seed=4)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) >= 0) and arr[0] == 0.0
    gaps = np.diff(arr)
    assert abs(gaps.mean() - 1 / 200.0) < 0.1 / 200.0           # Poisson: exponential gaps, mean 1/rate
    ns = np.array([r.spec[0] for r in reqs])
    assert ns.min() >= 12 and ns.max() <= 30
    # log-uniform: about as many requests in [12, 15] as the log-width share predicts
    share = np.mean(ns <= 15)
    expect = (math.log(16) - math.log(12)) / (math.log(31) - math.log(12))
    assert abs(share - expect) < 0.05
    assert config5_requests(count=5, seed=4)[3].spec == reqs[3].spec
    ds = np.array([r.spec[1] for r in reqs])
    assert ds.min() >= 10 and ds.max() <= 100


def test_ready_queue_orders():
    """Shortest estimated work first, but a request that waited longer than max_wait goes first; FIFO
    policy keeps arrival order."""
    from qsv_b200.serve import _ReadyQueue, Request

    def drain(q, now):
        out = []
        while (r := q.peek(now)) is not None:
            q.take(r)
            out.append(r.rid)
        return out

    def fill(q):
        for i, w in enumerate([50, 10, 30, 20, 40]):
            r = Request(i, None, 0.1 * i)
            r.work = w
            q.append(r)
        return q

    assert drain(fill(_ReadyQueue("sjf", max_wait=10.0)), 0.5) == [1, 3, 2, 4, 0]
    assert drain(fill(_ReadyQueue("sjf", max_wait=0.2)), 0.35) == [0, 1, 3, 2, 4]
    assert drain(fill(_ReadyQueue("fifo")), 0.5) == [0, 1, 2, 3, 4]


def test_state_arena_buddy_allocation():
    """The server's HBM arena (host tensors here): the budget splits into power-of-two roots; blocks are
    power-of-two sized and aligned to their size; freed buddies merge back; a block larger than every root
    never fits."""
    import torch
    from qsv_b200.serve import StateArena
    budget = (1 << 20) + (1 << 18) + 5000          # roots of 1 MiB and 256 KiB; the 5000-byte rest is unused
    ar = StateArena(budget, torch.device("cpu"))
    assert ar.capacity == (1 << 20) + (1 << 18) and ar.max_order == 20
    assert not ar.fits_ever((1 << 20) + 1) and ar.fits_ever(1 << 20)
    rng = np.random.default_rng(0)
    live = []
    for step in range(400):
        if live and (rng.random() < 0.45 or ar.used > ar.capacity * 0.8):
            h = live.pop(int(rng.integers(len(live))))
            ar.release(h)
            continue
        size = 1 << int(rng.integers(13, 19))
        h = ar.alloc(size)
        if h is None:
            continue
        root, off, o = h
        assert (1 << o) >= size and off % (1 << o) == 0 and off + (1 << o) <= (1 << ar.roots[root][1])
        for r2, off2, o2 in live:                  # no two live blocks overlap
            if r2 == root:
                assert off + (1 << o) <= off2 or off2 + (1 << o2) <= off
        live.append(h)
        assert ar.used == sum(1 << x[2] for x in live)
        v = ar.view(h, o - 3)
        assert v.dtype == torch.complex64 and v.numel() == (1 << o) // 8
    for h in live:
        ar.release(h)
    assert ar.used == 0
    # everything merged back: the two whole roots are free again
    assert ar.alloc(1 << 20) is not None and ar.alloc(1 << 18) is not None and ar.alloc(1 << 13) is None
