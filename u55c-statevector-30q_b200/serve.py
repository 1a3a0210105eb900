"""Serving loop: continuous batching of circuits on one B200 under an HBM budget.

No reference counterpart (the reference serves nothing; its latency study repeats one circuit,
bench/latency_jitter.py, and reports p50/p99 of T_e2e -- the statistics kept here). Requests arrive over
time; each is compiled on arrival (host), then admitted as soon as a device slot is free and its state
fits in the remaining HBM budget (states stay resident on the device until the request completes).
Admitted work overlaps on the GPU: requests of 10..13 qubits that are ready together run as one
whole-circuit batch launch, larger ones each run their sweeps on their own stream. Completion is
detected with CUDA events; the result (norm and <Z_q> per qubit, FP64, plus the state if asked) is read
back and the memory released. Each request's arithmetic is independent of the others (no cross-request
reduction, fixed op order), so a result is the same alone and in the mix.

The HBM budget is real memory: the server reserves it once as an arena and gives every admitted state a
power-of-two block of it (buddy allocation; a 2^n-amplitude complex64 state is exactly 2^(n+3) bytes), so
admission never depends on the caching allocator's fragmentation and the footprint stays fixed while the
server runs. A request that cannot be served (its state can never fit the arena, its circuit does not
compile, its program is rejected by the engine) fails alone: it is recorded in ``Server.failed`` with the
reason and every other request runs on.
"""
import heapq
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import engine
from .batch import SMALL_MAX
from .compiler import compile_circuit


@dataclass
class Request:
    rid: int
    circuit: object                 # a Circuit, or None to build it from `spec` on arrival
    arrival: float                  # seconds from the start of the run
    want_state: bool = False
    spec: tuple = None              # (n, depth, seed) of a random-layer circuit with Toffolis
    # filled in by the server
    program: object = None
    fmap: list = None
    n: int = 0                      # qubits the program runs on (at least the engine's minimum)
    n_log: int = 0                  # qubits of the request's circuit
    admitted: float = None
    done: float = None
    result: object = None
    state: object = None
    work: int = 0                   # estimated device work: 2^n x op records of the program
    error: str = None               # why the request could not be served (None: served)


class StateArena:
    """The server's HBM budget, reserved once, handed out as power-of-two blocks (binary buddy system).

    The budget is split into power-of-two root blocks (largest first, each at most 2^37 bytes); a request
    for 2^order bytes takes the smallest free block of at least that size, splitting it in halves; a freed
    block merges with its free buddy. Blocks are 2^order bytes at offsets that are multiples of 2^order
    within their root, so every state is aligned to its own size. Host-side bookkeeping only: reuse is safe
    because a block is freed only after the work on it has completed (its CUDA event)."""

    MIN_ORDER = 13               # 8 KiB: the smallest state the engine runs (2^10 complex64)
    MAX_ROOT_ORDER = 37          # 128 GiB

    def __init__(self, budget_bytes, device):
        import torch
        self.roots = []          # (tensor, order)
        self.free = {}           # order -> set of (root index, offset)
        left = int(budget_bytes)
        order = self.MAX_ROOT_ORDER
        while order >= self.MIN_ORDER and left >= (1 << self.MIN_ORDER):
            if left >= (1 << order):
                t = torch.empty(1 << order, dtype=torch.uint8, device=device)
                self.free.setdefault(order, set()).add((len(self.roots), 0))
                self.roots.append((t, order))
                left -= 1 << order
            else:
                order -= 1
        self.capacity = sum(1 << o for _, o in self.roots)
        self.used = 0
        self.max_order = max((o for _, o in self.roots), default=-1)

    @staticmethod
    def order_for(nbytes):
        return max(StateArena.MIN_ORDER, int(nbytes - 1).bit_length())

    def fits_ever(self, nbytes):
        return self.order_for(nbytes) <= self.max_order

    def alloc(self, nbytes):
        """-> (root index, offset, order), or None when no free block is large enough right now."""
        want = self.order_for(nbytes)
        o = want
        while o <= self.max_order and not self.free.get(o):
            o += 1
        if o > self.max_order:
            return None
        blk = min(self.free[o])               # lowest root / offset first: packs work toward the front
        self.free[o].discard(blk)
        root, off = blk
        while o > want:                       # split, keeping the lower half
            o -= 1
            self.free.setdefault(o, set()).add((root, off + (1 << o)))
        self.used += 1 << want
        return root, off, want

    def release(self, handle):
        root, off, o = handle
        self.used -= 1 << o
        root_order = self.roots[root][1]
        while o < root_order:
            buddy = (root, off ^ (1 << o))
            if buddy not in self.free.get(o, ()):
                break
            self.free[o].discard(buddy)
            off = min(off, buddy[1])
            o += 1
        self.free.setdefault(o, set()).add((root, off))

    def view(self, handle, n):
        """The block as a 2^n-amplitude complex64 state tensor."""
        import torch
        root, off, o = handle
        t = self.roots[root][0]
        return t[off: off + (8 << n)].view(torch.complex64)


@dataclass
class _Slot:
    req: Request
    stream: object
    state: object
    event: object
    scratch: object
    zout: object
    handle: tuple


def config5_requests(count=20000, rate=50.0, seed=4, qmin=12, qmax=30, dmin=10, dmax=100):
    """The served workload: Poisson arrivals at `rate` per second, qubit counts log-uniform in
    [qmin, qmax], depths uniform in [dmin, dmax], random-layer recipe with CZ brickwork and Toffolis,
    request i seeded seed + i."""
    gaps = np.random.default_rng(seed).exponential(1.0 / rate, count)
    arrivals = np.cumsum(gaps) - gaps[0]
    out = []
    for i, t in enumerate(arrivals):
        r = np.random.default_rng([seed, i])          # request i's shape depends on (seed, i) only
        n = int(np.clip(np.floor(np.exp(r.uniform(math.log(qmin), math.log(qmax + 1)))), qmin, qmax))
        d = int(r.integers(dmin, dmax + 1))
        out.append(Request(i, None, float(t), spec=(n, d, seed + i)))
    return out


def _circuit(req):
    if req.circuit is None:
        from .generators import random_layer_ccx
        n, d, s = req.spec
        req.circuit = random_layer_ccx(n, d, s)
    return req.circuit


def _compile_request(payload):
    """Compile one request (runs in a worker process or inline): -> (segments, final_map, n_run, n)."""
    circuit, spec, k = payload
    req = Request(-1, circuit, 0.0, spec=spec)
    qc = _circuit(req)
    n = qc.num_qubits
    m = max(n, engine.N_MIN)
    if m != n:
        from .circuit import Circuit
        q2 = Circuit(m)
        q2.compose(qc, range(n), inplace=True)
        qc = q2
    prog, fmap, _ = compile_circuit(qc, m, m if m <= SMALL_MAX else k)
    if any(kind != "segment" for kind, _ in prog):
        raise ValueError("program needs remaps, not served here")
    return [s for _, s in prog], fmap, m, n


class _ReadyQueue:
    """Requests whose program exists, waiting for admission. policy "sjf": smallest estimated work first,
    except that a request waiting longer than max_wait seconds goes first (no starvation); "fifo": arrival
    order. Admitted requests are dropped lazily from both orders."""

    def __init__(self, policy="sjf", max_wait=10.0):
        self.policy, self.max_wait = policy, max_wait
        self.fifo = deque()          # arrival order
        self.heap = []               # (work, sequence, request)
        self.seq = 0
        self.taken = set()           # sequence numbers of admitted requests

    def append(self, r):
        r._seq = self.seq
        self.fifo.append(r)
        heapq.heappush(self.heap, (r.work, self.seq, r))
        self.seq += 1

    def peek(self, now):
        while self.fifo and self.fifo[0]._seq in self.taken:
            self.fifo.popleft()
        while self.heap and self.heap[0][1] in self.taken:
            heapq.heappop(self.heap)
        if not self.fifo:
            return None
        oldest = self.fifo[0]
        if self.policy == "fifo" or now - oldest.arrival > self.max_wait:
            return oldest
        return self.heap[0][2]

    def take(self, r):
        self.taken.add(r._seq)


class Server:
    def __init__(self, budget_bytes=160e9, max_inflight=16, device=None, k=12, compile_workers=0, policy="sjf",
                 max_wait=10.0):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("Server needs a CUDA device (B200); none is available")
        engine.load()
        self.device = torch.device(device if device is not None else "cuda")
        self.budget = int(budget_bytes)
        self.arena = StateArena(self.budget, self.device)
        self.failed = []             # (request, reason) of requests that could not be served
        self.max_inflight = max_inflight
        self.k = k
        self.streams = [torch.cuda.Stream(self.device) for _ in range(max_inflight)]
        self.free_streams = deque(range(max_inflight))
        self.used = 0
        self.policy, self.max_wait = policy, max_wait
        self.stats = dict(admitted=0, small_batches=0, small_in_batches=0, peak_bytes=0, peak_inflight=0,
                          rejected=0, arena_bytes=self.arena.capacity)
        self.pool = None
        self.compile_workers = compile_workers
        if compile_workers:
            import multiprocessing as mp
            from .batch import _boot_code
            self.pool = mp.get_context("spawn").Pool(compile_workers, initializer=exec, initargs=(_boot_code(),))

    def warm(self):
        """Start the compile workers (interpreter start, imports, one small compilation each) and wait for
        them: a long-running service does this once at start-up, not while requests wait."""
        if self.pool is not None:
            from .batch import _warm_one
            self.pool.map(_warm_one, range(self.compile_workers), chunksize=1)

    def close(self):
        """Stop the compile workers and give the arena back to the device."""
        if self.pool is not None:
            self.pool.terminate()
            self.pool = None
        self.arena = None

    @staticmethod
    def footprint(n):
        """Arena bytes a request's state holds while in flight (its small reduction scratch and outputs come
        from the caching allocator, at most max_inflight of them)."""
        return 8 << max(n, engine.N_MIN)

    def _reject(self, req, reason, now):
        req.error = reason
        req.done = now
        self.failed.append((req, reason))
        self.stats["rejected"] += 1

    def _compile(self, req):
        self._finish_compile(req, _compile_request((req.circuit, req.spec, self.k)))

    @staticmethod
    def _finish_compile(req, res):
        # the circuit itself stays where it was built (a worker process): only its program comes back
        req.program, req.fmap, req.n, req.n_log = res
        req.work = (1 << req.n) * sum(len(seg) for seg in req.program)

    def _launch(self, reqs, now):
        """Start a group of admitted requests: small ones as one whole-circuit batch, large ones alone. A
        request whose program the engine rejects (checked on the host before anything of it is queued)
        fails alone; the others of its group still run."""
        import torch
        slots = []
        small = [r for r in reqs if r.n <= SMALL_MAX]
        large = [r for r in reqs if r.n > SMALL_MAX]
        groups = ([small] if small else []) + [[r] for r in large]
        for grp in groups:
            si = self.free_streams.popleft()
            st = self.streams[si]
            members = []                 # (request, arena block, state) that run
            batch = None
            # the small outputs and scratch are allocated on the group's stream, so the caching allocator
            # never hands them to other work before this stream is done with them
            with torch.cuda.stream(st):
                if grp is small:
                    batch = engine.SmallBatch()
                for r in grp:
                    h = self._handles.pop(r.rid)
                    s = self.arena.view(h, r.n)
                    try:
                        if batch is not None:
                            batch.add(s, r.program)          # host-side decode and checks
                        else:
                            engine.zero_state(s, st)
                            for seg in r.program:
                                engine.run_segment(s, seg, st)
                    except (engine.QSVError, ValueError) as e:
                        st.synchronize()                     # what was queued for it has drained
                        self.arena.release(h)
                        self._reject(r, f"engine rejected the program: {e}", now)
                        continue
                    members.append((r, h, s))
                if not members:
                    self.free_streams.append(si)
                    continue
                if batch is not None:
                    for _, _, s in members:
                        engine.zero_state(s, st)
                    batch.upload(st)
                    batch.launch(st)
                    self.stats["small_batches"] += 1
                    self.stats["small_in_batches"] += len(members)
                outs = []
                for r, _, s in members:
                    sc = engine.new_scratch(r.n, self.device)
                    outs.append((sc, engine.reduce_f64(s, scratch=sc, stream=st)))
                ev = torch.cuda.Event()
                ev.record(st)
            for (r, h, s), (sc, z) in zip(members, outs):
                r.admitted = now
                slot = _Slot(r, si, s, ev, sc, z, h)
                slot.batch = batch           # the batch tables stay alive until the group completes
                slots.append(slot)
        return slots

    def run(self, requests, realtime=True, timeout=3600.0):
        """Serve `requests` (sorted by arrival). Returns the list of completed requests."""
        import torch
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        compiling = deque()
        ready = _ReadyQueue(self.policy, self.max_wait)
        inflight = []
        done = []
        self._handles = {}
        t0 = time.perf_counter()
        while pending or compiling or ready.peek(time.perf_counter() - t0) is not None or inflight:
            now = time.perf_counter() - t0
            if now > timeout:
                raise TimeoutError("serving run exceeded its time limit")
            # arrivals: compiled on arrival (in the worker pool when there is one); a request joins the
            # ready queue, in arrival order, once its program exists
            while pending and (not realtime or pending[0].arrival <= now):
                r = pending.popleft()
                if r.program is not None:
                    ready.append(r)
                elif self.pool is None:
                    try:
                        self._compile(r)
                        ready.append(r)
                    except Exception as e:        # this request's circuit does not compile: it fails alone
                        self._reject(r, f"compile failed: {e}", now)
                else:
                    compiling.append((r, self.pool.apply_async(_compile_request, ((r.circuit, r.spec, self.k),))))
                if self.pool is None and realtime:
                    break                 # compile inline one at a time, keep the device fed meanwhile
            def take_compiled(r, fut):
                try:
                    self._finish_compile(r, fut.get())
                    ready.append(r)
                except Exception as e:            # the worker's compilation raised: this request fails alone
                    self._reject(r, f"compile failed: {e}", now)

            if self.policy == "fifo":
                while compiling and compiling[0][1].ready():      # arrival order
                    take_compiled(*compiling.popleft())
            elif compiling:
                # shortest-work-first: every finished compilation joins the ready queue at once (a long
                # compilation ahead of it does not hold it back)
                still = deque()
                for r, fut in compiling:
                    if fut.ready():
                        take_compiled(r, fut)
                    else:
                        still.append((r, fut))
                compiling = still
            # admission: free slot and memory budget; continuous -- new work joins while old runs
            admit = []
            streams_left = len(self.free_streams)
            small_group = False
            while streams_left > 0:
                r = ready.peek(now)
                if r is None:
                    break
                fp = self.footprint(r.n)
                if not self.arena.fits_ever(fp):
                    # its state is larger than any block the budget can ever give: reject it, serve the rest
                    ready.take(r)
                    self._reject(r, f"{r.n}-qubit state ({fp} B) exceeds the HBM budget's largest block", now)
                    continue
                h = self.arena.alloc(fp)
                if h is None:
                    break                 # waits for running requests to free their blocks
                ready.take(r)
                self._handles[r.rid] = h
                self.used = self.arena.used
                admit.append(r)
                if r.n <= SMALL_MAX:
                    if not small_group:
                        small_group = True
                        streams_left -= 1
                else:
                    streams_left -= 1
            if admit:
                inflight += self._launch(admit, now)
                self.stats["admitted"] += len(admit)
                self.stats["peak_bytes"] = max(self.stats["peak_bytes"], self.used)
                self.stats["peak_inflight"] = max(self.stats["peak_inflight"], len(inflight))
            # completions
            still = []
            finished_streams = set()
            for sl in inflight:
                if sl.event.query():
                    z = sl.zout.cpu().numpy()
                    r = sl.req
                    r.done = time.perf_counter() - t0
                    n_log = r.n_log
                    r.result = (float(z[0]), np.array([z[1 + r.fmap[q]] for q in range(n_log)]))
                    if r.want_state:
                        perm = [r.fmap[q] for q in range(r.n)]
                        dst = torch.empty_like(sl.state)
                        engine.remap(sl.state, dst, perm)
                        r.state = dst.cpu().numpy()[: 1 << n_log]
                    self.arena.release(sl.handle)
                    self.used = self.arena.used
                    finished_streams.add(sl.stream)
                    done.append(r)
                else:
                    still.append(sl)
            inflight = still
            live_streams = {sl.stream for sl in inflight}
            for si in finished_streams - live_streams:
                self.free_streams.append(si)
            if not admit and not finished_streams:
                # nothing to do right now: wait for the next arrival, compile or completion
                wait = 0.0005
                if pending and realtime and ready.peek(now) is None and not inflight and not compiling:
                    wait = max(0.0, min(0.05, pending[0].arrival - (time.perf_counter() - t0)))
                time.sleep(wait)
        return done


def precompile(requests, workers=0):
    """Compile every request ahead of time (optionally in spawned workers), to time the device side of
    serving without host compile."""
    payloads = [(r.circuit, r.spec, 12) for r in requests]
    if workers:
        import multiprocessing as mp
        from .batch import _boot_code
        with mp.get_context("spawn").Pool(workers, initializer=exec, initargs=(_boot_code(),)) as pool:
            res = pool.map_async(_compile_request, payloads).get(3600)
    else:
        res = [_compile_request(p) for p in payloads]
    for r, x in zip(requests, res):
        Server._finish_compile(r, x)
    return requests


def plain_serve(requests, device=None, k=12):
    """The plain sequential path: each request alone, in arrival order (a single FIFO server, no overlap;
    requests without a program are compiled when they are served). Returns the completed requests with
    admitted/done times on the same arrival clock; a request that cannot run (compile or engine error)
    gets its `error` set and is left out."""
    import torch
    dev = torch.device(device if device is not None else "cuda")
    pending = sorted(requests, key=lambda r: r.arrival)
    t0 = time.perf_counter()
    out = []
    for r in pending:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        try:
            if r.program is None:
                Server._finish_compile(r, _compile_request((r.circuit, r.spec, k)))
            r.admitted = time.perf_counter() - t0
            st = engine.new_state(r.n, device=dev)
            if r.n <= SMALL_MAX:
                b = engine.SmallBatch()
                b.add(st, r.program)
                b.upload()
                b.launch()
            else:
                for seg in r.program:
                    engine.run_segment(st, seg)
        except Exception as e:
            r.error = f"{type(e).__name__}: {e}"
            continue
        z = engine.reduce_f64(st).cpu().numpy()
        r.done = time.perf_counter() - t0
        n_log = r.n_log
        r.result = (float(z[0]), np.array([z[1 + r.fmap[q]] for q in range(n_log)]))
        out.append(r)
        del st
    torch.cuda.synchronize(dev)
    return out


def latency_stats(done):
    lat = np.array([r.done - r.arrival for r in done])
    span = max(r.done for r in done) - min(r.arrival for r in done)
    return dict(count=len(done), p50_ms=float(np.percentile(lat, 50) * 1e3),
                p99_ms=float(np.percentile(lat, 99) * 1e3), mean_ms=float(lat.mean() * 1e3),
                circuits_per_s=len(done) / span if span > 0 else float("inf"))
