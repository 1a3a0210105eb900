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
