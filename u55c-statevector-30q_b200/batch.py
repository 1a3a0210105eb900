"""Batched execution: many independent circuits per replay of one captured CUDA graph.

No reference counterpart (the reference runs one circuit per launch; its discussion names batching as
future work). The layer:
  * compiles every circuit to QSV2 (optionally in a pool of spawned worker processes);
  * keeps every state resident in one device arena (one complex64 tensor, 2^n slots per circuit);
  * runs circuits of 10..13 qubits through the whole-circuit kernel (qsv_batch_*: each circuit's whole
    program inside one CTA's shared memory, all of them in one persistent launch per qubit count);
  * runs larger circuits as sweeps (qsv_run_segment), spread over several streams so that small-grid
    sweeps of different circuits overlap on the GPU;
  * reduces every final state to <Z_q> (FP64, qsv_reduce_f64) and keeps the full state for a sample;
  * captures all of the above into ONE CUDA graph, replayed for every run of the same batch;
  * picks per qubit count the engine's tuning knobs with a small autotuner (timed on the device).
Each circuit's arithmetic is independent of what else is in the batch (no cross-circuit reductions,
fixed op order), so a circuit gives the same values alone and in any batch.
"""
import time
from dataclasses import dataclass, field

import numpy as np

from . import engine
from .compiler import compile_circuit

SMALL_MAX = 13          # circuits up to this many qubits run whole in one CTA's shared memory


def _compile_one(args):
    """Worker entry point: (circuit, k) -> (segments, final_map, n)."""
    qc, k = args
    n = qc.num_qubits
    prog, fmap, stats = compile_circuit(qc, n, min(k, n))
    return prog, fmap, n, stats.n_passes


def _warm_one(i):
    """A small compilation in a worker process (imports and first-use costs paid at pool start-up)."""
    from .generators import random_layer
    compile_circuit(random_layer(12, 2, i), 12, 12)
    return i


class CompilePool:
    """A persistent pool of spawned compile workers: started (and warmed) once, then used for batch after
    batch, as a service keeps its workers. Use as a context manager or close() it."""

    def __init__(self, workers):
        import multiprocessing as mp
        self.workers = max(1, int(workers))
        self.pool = mp.get_context("spawn").Pool(self.workers, initializer=exec, initargs=(_boot_code(),))
        self.pool.map(_warm_one, range(self.workers), chunksize=1)

    def compile(self, circuits, k=12, timeout=600):
        jobs = [(qc, qc.num_qubits if qc.num_qubits <= SMALL_MAX else k) for qc in circuits]
        return self.pool.map_async(_compile_one, jobs, chunksize=max(1, len(jobs) // (4 * self.workers))).get(timeout)

    def close(self):
        if self.pool is not None:
            self.pool.terminate()
            self.pool = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def compile_many(circuits, k=12, workers=0, timeout=600, pool=None):
    """Compile circuits to QSV2 programs: in a CompilePool when one is given, else in `workers` spawned
    processes started for this call (0 = in this process)."""
    if pool is not None:
        return pool.compile(circuits, k, timeout)
    jobs = [(qc, qc.num_qubits if qc.num_qubits <= SMALL_MAX else k) for qc in circuits]
    if workers and len(jobs) > 1:
        import multiprocessing as mp
        # spawned workers cannot import this package by name (its directory is not a module name): the
        # initializer registers it from its path before any task (which references it) is unpickled
        with mp.get_context("spawn").Pool(workers, initializer=exec, initargs=(_boot_code(),)) as pool:
            res = pool.map_async(_compile_one, jobs, chunksize=max(1, len(jobs) // (4 * workers)))
            return res.get(timeout)
    return [_compile_one(j) for j in jobs]


def _boot_code():
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    return ("import importlib.util, sys\n"
            "if 'qsv_b200' not in sys.modules:\n"
            f"    spec = importlib.util.spec_from_file_location('qsv_b200', {os.path.join(here, '__init__.py')!r}, "
            f"submodule_search_locations=[{here!r}])\n"
            "    mod = importlib.util.module_from_spec(spec)\n"
            "    sys.modules['qsv_b200'] = mod\n"
            "    spec.loader.exec_module(mod)\n")


class Autotuner:
    """Per qubit count, the (lo_merge, layout13, phase_lanes) knobs with the lowest measured device time
    on a representative program. Values never depend on the knobs (tested); only speed does."""

    CANDIDATES = [(4, 4, 1), (4, 3, 1), (4, 4, 2), (4, 4, 0), (6, 4, 1), (9, 4, 1)]   # first = the defaults

    def __init__(self, reps=2):
        self.reps = reps
        self.best = {}          # n -> (lo_merge, layout13, phase_lanes)
        self.timings = {}

    @staticmethod
    def apply(knobs):
        lo, lay, pl = knobs
        engine.set_lo_merge(lo)
        engine.set_layout13(lay)
        engine.set_phase_lanes(pl)

    def tune(self, n, segments, stream=None):
        import torch
        if n in self.best:
            return self.best[n]
        if n <= SMALL_MAX:
            self.best[n] = self.CANDIDATES[0]
            return self.best[n]
        state = engine.new_state(n)
        res = {}
        for knobs in self.CANDIDATES:
            self.apply(knobs)
            for s in segments:
                engine.run_segment(state, s, stream)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(self.reps):
                for s in segments:
                    engine.run_segment(state, s, stream)
            e1.record()
            torch.cuda.synchronize()
            res[knobs] = e0.elapsed_time(e1) / self.reps
        self.apply(self.CANDIDATES[0])
        self.best[n] = min(res, key=res.get)
        self.timings[n] = res
        return self.best[n]


@dataclass
class BatchPlan:
    circuits: list
    programs: list                      # (prog, fmap, n, passes) per circuit
    offsets: np.ndarray                 # amplitude offset of each circuit's state in the arena
    zoffsets: np.ndarray                # offset of each circuit's [norm, <Z_0..n-1>] in the output arena
    sample: list                        # circuit indices whose full state is returned
    arena: object = None
    zout: object = None
    small: object = None
    graph: object = None
    streams: list = field(default_factory=list)
    scratch: list = field(default_factory=list)
    sample_bufs: dict = field(default_factory=dict)
    knobs: dict = field(default_factory=dict)
    launches: int = 0


class BatchRunner:
    def __init__(self, device=None, streams=8, autotune=True, compile_workers=0):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("BatchRunner needs a CUDA device (B200); none is available")
        engine.load()
        self.device = torch.device(device if device is not None else "cuda")
        self.nstreams = streams
        self.tuner = Autotuner() if autotune else None
        self.compile_workers = compile_workers

    # ------------------------------------------------------------------ preparation
    def prepare(self, circuits, sample_fraction=0.01, sample_seed=0, programs=None):
        import torch
        progs = programs if programs is not None else compile_many(circuits, workers=self.compile_workers)
        for p in progs:
            if any(kind != "segment" for kind, _ in p[0]):
                raise ValueError("batched circuits must compile without remaps")
        ns = np.array([p[2] for p in progs])
        sizes = np.array([1 << int(n) for n in ns], dtype=np.int64)
        offsets = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
        zsz = ns + 1
        zoffsets = np.concatenate([[0], np.cumsum(zsz)[:-1]]).astype(np.int64)
        rng = np.random.default_rng(sample_seed)
        nsample = max(1, int(round(sample_fraction * len(progs)))) if sample_fraction > 0 else 0
        sample = sorted(int(i) for i in rng.choice(len(progs), nsample, replace=False)) if nsample else []
        plan = BatchPlan(list(circuits), progs, offsets, zoffsets, sample)
        plan.arena = torch.empty(int(sizes.sum()), dtype=torch.complex64, device=self.device)
        plan.zout = torch.empty(int(zsz.sum()), dtype=torch.float64, device=self.device)
        plan.streams = [torch.cuda.Stream(self.device) for _ in range(self.nstreams)]
        nmax = int(ns.max())
        plan.scratch = [engine.new_scratch(max(nmax, engine.N_MIN), self.device) for _ in range(self.nstreams)]
        for i in sample:
            plan.sample_bufs[i] = torch.empty(1 << int(ns[i]), dtype=torch.complex64, device=self.device)
        # tuning per qubit count on a representative (the deepest) program of that size
        if self.tuner is not None:
            for n in sorted(set(int(x) for x in ns)):
                idx = max((i for i in range(len(progs)) if ns[i] == n), key=lambda i: progs[i][3])
                plan.knobs[n] = self.tuner.tune(n, [s for _, s in progs[idx][0]])
            Autotuner.apply(Autotuner.CANDIDATES[0])
        # whole-circuit batch for the small ones (planned once, tables uploaded once)
        small = [i for i in range(len(progs)) if ns[i] <= SMALL_MAX]
        if small:
            plan.small = engine.SmallBatch()
            for i in small:
                plan.small.add(self.state(plan, i), [s for _, s in progs[i][0]])
            plan.small.upload()
        torch.cuda.synchronize(self.device)
        return plan

    @staticmethod
    def state(plan, i):
        n = int(plan.programs[i][2])
        o = int(plan.offsets[i])
        return plan.arena[o:o + (1 << n)]

    # ------------------------------------------------------------------ one pass over the batch
    def _enqueue(self, plan, main):
        import torch
        progs = plan.programs
        ns = [int(p[2]) for p in progs]
        # |0...0> everywhere: zero the arena, set amplitude 0 of every circuit
        plan.arena.zero_()
        if not hasattr(plan, "_amp0"):
            plan._amp0 = torch.as_tensor(plan.offsets, device=self.device)
        plan.arena.index_fill_(0, plan._amp0, 1.0)
        for s in plan.streams:
            s.wait_stream(main)
        if plan.small is not None:
            plan.small.launch(plan.streams[0])
        big = sorted((i for i in range(len(progs)) if ns[i] > SMALL_MAX), key=lambda i: -ns[i])
        lane = {i: j % len(plan.streams) for j, i in enumerate(big)}
        for i in big:
            st = plan.streams[lane[i]]
            if self.tuner is not None and ns[i] in plan.knobs:
                Autotuner.apply(plan.knobs[ns[i]])
            for _, seg in progs[i][0]:
                engine.run_segment(self.state(plan, i), seg, st)
        if self.tuner is not None:
            Autotuner.apply(Autotuner.CANDIDATES[0])
        # reductions and sampled states, each on the stream that produced the state (small circuits: the
        # whole-circuit kernel's stream 0)
        for j in range(len(progs)):
            k = lane.get(j, 0)
            z0 = int(plan.zoffsets[j])
            engine.reduce_f64(self.state(plan, j), plan.zout[z0:z0 + ns[j] + 1], plan.scratch[k], plan.streams[k])
        for i in plan.sample:
            st = plan.streams[lane.get(i, 0)]
            fmap = progs[i][1]
            perm = [fmap[q] for q in range(ns[i])]
            if perm == list(range(ns[i])):
                with torch.cuda.stream(st):
                    plan.sample_bufs[i].copy_(self.state(plan, i))
            else:
                engine.remap(self.state(plan, i), plan.sample_bufs[i], perm, st)
        for s in plan.streams:
            main.wait_stream(s)

    def capture(self, plan):
        """Capture one pass over the batch into a CUDA graph (after one eager pass that configures the
        kernels)."""
        import torch
        main = torch.cuda.current_stream(self.device)
        self._enqueue(plan, main)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream(self.device)
        cap.wait_stream(main)
        engine.take_launch_count()
        with torch.cuda.graph(g, stream=cap):
            self._enqueue(plan, cap)
        plan.launches = engine.take_launch_count()
        plan.graph = g
        torch.cuda.synchronize(self.device)
        return g

    def run(self, plan, use_graph=True):
        """One pass over the batch; returns (z, states): z[i] = (norm, <Z_q> in logical qubit order),
        states[i] = logical-order state for the sampled circuits."""
        import torch
        if use_graph:
            if plan.graph is None:
                self.capture(plan)
            plan.graph.replay()
        else:
            self._enqueue(plan, torch.cuda.current_stream(self.device))
        z_all = plan.zout.cpu().numpy()
        states = {i: plan.sample_bufs[i].cpu().numpy() for i in plan.sample}
        return self.collect(plan, z_all), states

    @staticmethod
    def collect(plan, z_all):
        out = []
        for i, (prog, fmap, n, _) in enumerate(plan.programs):
            n = int(n)
            z0 = int(plan.zoffsets[i])
            zp = z_all[z0 + 1:z0 + 1 + n]
            out.append((float(z_all[z0]), np.array([zp[fmap[q]] for q in range(n)])))
        return out


def config4_circuits(count=512, seed=3):
    """The batched workload: `count` circuits, qubit counts uniform in [10, 24], depths uniform in
    [5, 40], random-layer recipe with CZ brickwork and Toffolis (U3 / CZ / CCX), circuit i seeded seed+i."""
    from .generators import random_layer_ccx
    rng = np.random.default_rng(seed)
    ns = rng.integers(10, 25, count)
    ds = rng.integers(5, 41, count)
    return [random_layer_ccx(int(n), int(d), seed + i) for i, (n, d) in enumerate(zip(ns, ds))]


def plain_run(circuits, programs, device=None):
    """The plain one-circuit-at-a-time GPU path for comparison: per circuit, zero a state, run its
    segments, reduce, read back, synchronise. Returns the same per-circuit (norm, <Z>) list."""
    import torch
    dev = torch.device(device if device is not None else "cuda")
    out = []
    for qc, (prog, fmap, n, _) in zip(circuits, programs):
        n = int(n)
        st = engine.new_state(n, device=dev)
        for _, seg in prog:
            engine.run_segment(st, seg)
        z = engine.reduce_f64(st).cpu().numpy()
        out.append((float(z[0]), np.array([z[1 + fmap[q]] for q in range(n)])))
    return out
