"""Benchmark: QSV2 pass-sweep bandwidth of the 30-qubit random-layer circuit on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: random-layer circuit, 30 qubits, depth 24, seed 1 (U3 with angles uniform in [0, 2pi) on every
qubit, CX brickwork), complex64 (8 GiB state), compiled to QSV2 by the reference scheduler (k = 12,
M = 4). One step = the whole program (every sweep of every segment) over the resident state; the state
(8 GiB) is far larger than L2 (126 MB), so no flush is needed between steps.

value: algorithmic bytes (16 B per amplitude per sweep: one complex64 read + one write) over device time
(CUDA events on the launch stream, max over ranks). e2e: the same metric through the public API
(SVRuntime.run with host-side circuit, compile, instruction upload, device execution, device sampling
and the read-back of 1024 sampled indices), per step.

--gpus N > 1 runs N independent replicas (one process per GPU under torchrun): the path does not
partition one state across GPUs, so there is no collective; value is the aggregate.
--impl reference times the reference's own CPU implementation of the path (the numpy golden model,
host/sv/model.py, restated in oracle/golden_model.py) on a bounded sample of the same workload, with
every host core (spawned worker processes over disjoint tiles).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "u55c-statevector-30q_b200")
METRIC = "30q pass sweep GB/s (random-layer d24)"
HBM_FALLBACK_GBS = 6650.0
# dram__bytes_read.sum + dram__bytes_write.sum per sweep launch over the algorithmic 16 B x 2^n, measured
# with ncu on the 26-qubit version of this workload (specialised kernels, three launches: 1013-1015 MB of
# 1074 MB); traffic grows as 2^n
TRAFFIC_PER_ALGORITHMIC = 0.944


def _package():
    import importlib.util
    if "qsv_b200" in sys.modules:
        return sys.modules["qsv_b200"]
    spec = importlib.util.spec_from_file_location("qsv_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["qsv_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def workload(pkg, n, depth, seed, k=12, max_high=4, family="random_layer"):
    """The benchmark circuit (random_layer: the headline) or, for profiling other sweep mixes through the
    same timing path, one of the reference's families (rqc with `depth` layers, vqe, qft)."""
    gen = pkg.generators
    if family == "random_layer":
        qc = gen.random_layer(n, depth, seed)
    elif family == "rqc":
        qc = gen.rqc(n, depth, seed)
    else:
        qc = getattr(gen, family)(n)
    prog, fmap, stats = pkg.compile_circuit(qc, n, k, max_high=max_high)
    return qc, prog, fmap, stats


def accuracy_vs_fp64(qc):
    """1 - F and max |delta amp| of the complex64 result of qc against the same circuit run in complex128
    (FP64 matrices and arithmetic) on the device, from |0...0>, with the reference's recipe
    (bench/fpga/sv_maxwidth_ref.py:15-25; precision.compare). Both runs use one compiled schedule (same final
    qubit map), so the states are compared in physical order."""
    import torch
    from importlib import import_module
    precision = import_module("qsv_b200.precision")
    s128, f128, t128 = precision.run_state(qc, "c128")
    s64, f64, t64 = precision.run_state(qc, "c64")
    if f128 != f64:
        raise RuntimeError("complex64 and complex128 schedules differ")
    m = precision.compare(s128, s64)
    del s128, s64
    torch.cuda.empty_cache()
    return {"one_minus_f": m["one_minus_f"], "max_abs_err": m["max_abs_err"], "norm": m["norm"],
            "c128_T_kernel_s": t128["T_kernel"]}


# ------------------------------------------------------------------ CPU baseline (golden model)
def _cpu_worker(args):
    seg, n, tiles, npass = args
    sys.path.insert(0, ROOT)
    from oracle import golden_model as gm
    state = np.zeros(1 << n, dtype=np.complex64)     # lazily mapped: only the sampled tiles are touched
    state[0] = 1
    t0 = time.perf_counter()
    moved = gm.run_segment_tiles(state, seg, tiles, npass)
    return moved, time.perf_counter() - t0


def cpu_sample(seg, n, n_tiles_total, seconds=12.0, workers=None):
    """Golden model on a bounded sample of the workload: the first passes of the 30-qubit segment over a
    spread of tiles, in parallel worker processes. Returns (GB/s, cores, description)."""
    import multiprocessing as mp
    workers = workers or os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    # calibrate on one worker: tiles per second
    probe = np.arange(0, n_tiles_total, max(1, n_tiles_total // 16), dtype=np.int64)[:16]
    with ctx.Pool(1) as p:
        moved, dt = p.map(_cpu_worker, [(seg, n, probe, 2)])[0]
    rate = len(probe) / max(dt, 1e-6)
    per_worker = max(16, int(rate * seconds / 2))
    stride = max(1, n_tiles_total // (per_worker * workers))
    jobs = []
    for w in range(workers):
        t = (np.arange(per_worker, dtype=np.int64) * workers + w) * stride % n_tiles_total
        jobs.append((seg, n, t, 2))
    t0 = time.perf_counter()
    with ctx.Pool(workers) as p:
        res = p.map(_cpu_worker, jobs)
    wall = time.perf_counter() - t0
    moved = sum(r[0] for r in res)
    busy = max(r[1] for r in res)
    desc = (f"golden model (numpy port of host/sv/model.py), first 2 passes of the 30-qubit segment on "
            f"{per_worker * workers} of {n_tiles_total} tiles ({workers} processes), bytes = 16 B x amplitudes "
            f"touched; GB/s over the slowest worker's time")
    return moved / busy / 1e9, workers, desc, wall


# ------------------------------------------------------------------ precision study
def precision_main(a):
    """One JSON line: Run A (33 qubits, complex64) and Run B (32 qubits, complex128 against complex64)
    of the random-layer circuit with CZ brickwork and Toffolis, depth 16, seed 2."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    pkg = _package()
    import torch
    from importlib import import_module
    engine = import_module("qsv_b200.engine")
    precision = import_module("qsv_b200.precision")
    engine.load()
    torch.cuda.set_device(0)
    n_a = a.n if a.n != 30 else 33
    res = precision.study(n_a=n_a, n_b=n_a - 1, depth=16, seed=2)
    rb = res["run_b"]
    sweeps_bytes = 32 << rb["n"]
    print(json.dumps({"metric": "precision study: 1-F of complex64 vs complex128 (on-GPU FP64)",
                      "value": rb["c64_vs_c128"]["one_minus_f"], "unit": "1-F", "higher_is_better": False,
                      "n_gpus": 1, "dtype": "c64 and c128", "data": "synthetic (seeded circuit)",
                      "config": {"workload": f"random_layer_ccx depth 16 seed 2: run A {n_a}q complex64, "
                                             f"run B {n_a - 1}q complex128 vs complex64"},
                      "runs": res}))


# ------------------------------------------------------------------ batched and served workloads
def batched_main(a):
    """Batched: `count` circuits (qubits uniform in [10, 24], depths in [5, 40], U3 / CZ / Toffoli layers,
    circuit i seeded 3 + i) per replay of one captured CUDA graph, against the plain one-circuit-at-a-time
    path on the same compiled programs; results must be identical. Device work only (programs compiled
    before timing, in spawned workers); host compile time reported beside."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    pkg = _package()
    import torch
    from importlib import import_module
    engine = import_module("qsv_b200.engine")
    batch = import_module("qsv_b200.batch")
    engine.load()
    torch.cuda.set_device(0)
    engine.set_jit(a.jit)
    count = a.count or 512
    circs = batch.config4_circuits(count=count)
    # compile workers started once, before anything is timed (a batch service keeps its workers)
    cpool = batch.CompilePool(min(16, os.cpu_count() or 1))
    t0 = time.perf_counter()
    progs = batch.compile_many(circs, pool=cpool)
    t_compile = time.perf_counter() - t0
    # algorithmic bytes of one batch: a circuit of at most 13 qubits runs whole in shared memory (one read
    # and one write of its state), a larger one sweeps its state once per engine sweep (16 B per amplitude)
    work_bytes = 0
    for qc, (prog, fmap, n, npass) in zip(circs, progs):
        if n <= batch.SMALL_MAX:
            work_bytes += 16 << n
        else:
            work_bytes += sum(len(engine.plan_segment(seg, n)) for kind, seg in prog if kind == "segment") * (16 << n)
    # the group-type library for the 13-qubit sweeps of the batch's larger circuits (one build before the
    # timed work; the plain path below uses it too)
    lib_info = None
    if a.jit in ("auto", "library"):
        t0 = time.perf_counter()
        big = [(seg, n) for qc, (prog, fmap, n, npass) in zip(circs, progs) if n > batch.SMALL_MAX
               for kind, seg in prog if kind == "segment"]
        lib_info = {"types": engine.jit_prepare_library(big) if big else 0,
                    "build_s": round(time.perf_counter() - t0, 2)}
    br = batch.BatchRunner(streams=8, autotune=True)
    plan = br.prepare(circs, programs=progs)
    br.capture(plan)
    for _ in range(max(1, a.warmup)):
        br.run(plan)
    torch.cuda.synchronize()
    times = []
    with ClockSampler(0) as clk:
        for _ in range(a.steps):
            t = time.perf_counter()
            z, states = br.run(plan)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t)
    t_plain = time.perf_counter()
    zp = batch.plain_run(circs, progs)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t_plain
    equal = all(x[0] == y[0] and np.array_equal(x[1], y[1]) for x, y in zip(z, zp))
    t_b = statistics.median(times)
    # end to end from circuits (host compile included): one pass of a new batch (compile in the worker pool,
    # plan, run once without a graph) against one-at-a-time compile + run, as the reference runtime does
    t0 = time.perf_counter()
    progs2 = batch.compile_many(circs, pool=cpool)
    br2 = batch.BatchRunner(streams=8, autotune=False)
    plan2 = br2.prepare(circs, programs=progs2)
    z2, _ = br2.run(plan2, use_graph=False)
    torch.cuda.synchronize()
    t_e2e_b = time.perf_counter() - t0
    t0 = time.perf_counter()
    zp2 = batch.plain_run(circs, [batch._compile_one((qc, qc.num_qubits if qc.num_qubits <= batch.SMALL_MAX else 12))
                                  for qc in circs])
    torch.cuda.synchronize()
    t_e2e_p = time.perf_counter() - t0
    cpool.close()
    equal = equal and all(x[0] == y[0] and np.array_equal(x[1], y[1]) for x, y in zip(z2, zp2))
    print(json.dumps({"metric": "batched circuits/s (CUDA-graph replay) vs plain one-at-a-time",
                      "value": count / t_b, "unit": "circuits/s", "higher_is_better": True, "n_gpus": 1,
                      "steps": a.steps, "warmup": a.warmup, "dtype": "c64 (fp32 arithmetic)",
                      "data": "synthetic (seeded circuits)",
                      "config": {"workload": f"{count} circuits, n uniform in [10, 24], depth uniform in [5, 40], "
                                             "U3 / CZ brickwork / Toffoli layers, seeds 3 + i"},
                      "plain_circuits_per_s": count / t_plain, "speedup_vs_plain": t_plain / t_b,
                      "batched_s": t_b, "plain_s": t_plain, "results_identical": equal,
                      "end_to_end": {"batched_s": t_e2e_b, "plain_s": t_e2e_p, "speedup_vs_plain": t_e2e_p / t_e2e_b,
                                     "batched_circuits_per_s": count / t_e2e_b,
                                     "note": "new batch from circuits: compile in a running worker pool + plan + one pass, vs "
                                             "compile and run one circuit at a time"},
                      "algorithmic_bytes": work_bytes, "hbm_floor_s": work_bytes / (_peaks()[0] * 1e9),
                      "graph_launches": plan.launches, "host_compile_s": t_compile, "group_library": lib_info,
                      "specialised_kernels": engine.jit_info(), "clocks": clk.summary()}))


def served_main(a):
    """Served (config 5): a Poisson arrival stream of circuits with qubit counts log-uniform in [12, qmax]
    (default 30) and depths uniform in [10, 100] (U3 / CZ / Toffoli layers, request i seeded 4 + i),
    admitted under a 160 GB HBM budget (reserved once as the server's arena) with continuous batching, at
    each arrival rate of --rates (default 50, 200, 500, 1000, 2000 per second), against the plain sequential
    path (one request at a time, arrival order) on the same requests. Both sides run programs compiled
    before the run (compilation does not depend on the rate), so neither gains from host compile
    parallelism; --compile-on-arrival compiles in a warm worker pool on the served side and in line on the
    plain side instead. --count arrivals per rate (default 20000, the configuration's stream; every rate
    replays the first --count requests of the same seeded stream, so the requests, and their results, are
    the same at every rate). Both sides start warm: the server's compile workers are started and 24
    untimed requests of other seeds run through it first."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    pkg = _package()
    import torch
    from importlib import import_module
    engine = import_module("qsv_b200.engine")
    serve = import_module("qsv_b200.serve")
    engine.load()
    torch.cuda.set_device(0)
    engine.set_jit(a.jit)
    count = a.count or 20000
    rates = [float(x) for x in a.rates.split(",")]
    workers = min(16, os.cpu_count() or 1)
    base = serve.config5_requests(count=count, rate=rates[0], qmax=a.qmax)
    t0 = time.perf_counter()
    if not a.compile_on_arrival:
        base = serve.precompile(base, workers=workers)
    t_compile = time.perf_counter() - t0
    # algorithmic bytes of the whole stream (16 B per amplitude per sweep), from the sweep plans of every
    # request, or of a uniform sample of 400 of them for longer streams (planning is host work)
    work_bytes, work_kind = 0, None
    if not a.compile_on_arrival:
        sample = base if len(base) <= 2000 else [base[i] for i in np.random.default_rng(0).choice(len(base), 400,
                                                                                                 replace=False)]
        work_bytes = sum(sum(len(engine.plan_segment(seg, r.n)) for seg in r.program) * (16 << r.n) for r in sample)
        work_bytes *= len(base) / len(sample)
        work_kind = "exact" if len(sample) == len(base) else "estimated from 400 sampled requests"

    def stream(rate):
        """The same requests (same seeds, same programs) arriving at `rate` per second."""
        arr = serve.config5_requests(count=count, rate=rate, qmax=a.qmax)
        out = []
        for r, b in zip(arr, base):
            x = serve.Request(b.rid, None, r.arrival, spec=b.spec)
            if b.program is not None:
                x.program, x.fmap, x.n, x.n_log, x.work = b.program, b.fmap, b.n, b.n_log, b.work
            out.append(x)
        return out

    # group-type libraries for the 13-qubit sweeps, from up to 400 sampled requests (a service builds them at
    # start-up from its recent requests; both sides use them)
    lib_info = None
    if a.jit in ("auto", "library") and not a.compile_on_arrival:
        t0 = time.perf_counter()
        pick = base if len(base) <= 400 else [base[i] for i in np.random.default_rng(1).choice(len(base), 400,
                                                                                              replace=False)]
        big = [(seg, r.n) for r in pick if r.n > 13 for seg in r.program]
        lib_info = {"types": engine.jit_prepare_library(big) if big else 0,
                    "build_s": round(time.perf_counter() - t0, 2)}
    srv = serve.Server(budget_bytes=160e9, max_inflight=16, policy=a.policy,
                       compile_workers=workers if a.compile_on_arrival else 0)
    srv.warm()                      # compile workers started before the arrivals (service start-up)
    warm = serve.config5_requests(count=24, rate=1e9, seed=10 ** 6, qmax=min(a.qmax, 24))
    if not a.compile_on_arrival:
        warm = serve.precompile(warm, workers=workers)
    srv.run(warm)
    per_rate = []
    equal_all = True
    with ClockSampler(0) as clk:
        for rate in rates:
            srv.stats.update(admitted=0, small_batches=0, small_in_batches=0, peak_bytes=0, peak_inflight=0,
                             rejected=0)
            srv.failed = []
            t = time.perf_counter()
            done = srv.run(stream(rate), timeout=7 * 24 * 3600.0)
            t_served = time.perf_counter() - t
            st = serve.latency_stats(done)
            t = time.perf_counter()
            plain = serve.plain_serve(stream(rate))
            t_plain = time.perf_counter() - t
            sp = serve.latency_stats(plain)
            res = {r.rid: r.result for r in done}
            equal = len(done) == len(plain) and all(
                res[r.rid][0] == r.result[0] and np.array_equal(res[r.rid][1], r.result[1]) for r in plain)
            equal_all = equal_all and equal
            per_rate.append({"rate_per_s": rate, "served": dict(st, wall_s=t_served, **srv.stats),
                             "plain": dict(sp, wall_s=t_plain),
                             "speedup_vs_plain": st["circuits_per_s"] / sp["circuits_per_s"],
                             "failed": len(srv.failed), "results_identical_alone_and_in_mix": equal})
            print(json.dumps({"progress": per_rate[-1]}), file=sys.stderr, flush=True)
    srv.close()
    top = per_rate[-1]
    ns = [r.n_log for r in base] if not a.compile_on_arrival else [r.spec[0] for r in base]
    print(json.dumps({"metric": "served circuits/s and p50/p99 latency vs plain sequential",
                      "value": top["served"]["circuits_per_s"], "unit": f"circuits/s (at {top['rate_per_s']:g}/s)",
                      "higher_is_better": True, "n_gpus": 1, "dtype": "c64 (fp32 arithmetic)",
                      "data": "synthetic (seeded requests)",
                      "config": {"workload": f"{count} Poisson arrivals per rate, rates {a.rates} per second, n "
                                             f"log-uniform in [12, {a.qmax}], depth uniform in [10, 100], "
                                             "U3 / CZ brickwork / Toffoli layers, request i seeded 4 + i, 160 GB "
                                             "HBM budget (reserved arena)",
                                 "admission": a.policy,
                                 "compile": "on arrival (worker pool; plain path in line)" if a.compile_on_arrival
                                 else "before the run, both sides"},
                      "qubits": {"min": int(min(ns)), "max": int(max(ns)), "count_30": int(sum(x == 30 for x in ns))},
                      "algorithmic_bytes": work_bytes or None, "algorithmic_bytes_kind": work_kind,
                      "hbm_floor_s": (work_bytes / (_peaks()[0] * 1e9)) if work_bytes else None,
                      "host_compile_s": t_compile, "group_library": lib_info, "rates": per_rate,
                      "speedup_vs_plain": top["speedup_vs_plain"],
                      "results_identical_alone_and_in_mix": equal_all, "clocks": clk.summary()}))


def latency_main(a):
    """Latency distribution of repeated small circuits through the public API, the reference's determinism
    study (bench/latency_jitter.py:16-63): each family and size run 20 warm-up + `count` (default 2000)
    times with SVRuntime.run(qc, shots=1024, return_state=False); p50 / p99 / max of T_e2e and T_kernel."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    pkg = _package()
    import torch
    from importlib import import_module
    engine = import_module("qsv_b200.engine")
    runtime = import_module("qsv_b200.runtime")
    engine.load()
    torch.cuda.set_device(0)
    runs = a.count or 2000
    rt = runtime.SVRuntime()
    out = []
    for fam in ("ghz", "rqc"):
        for n in (4, 8, 12, 16):
            qc = getattr(pkg.generators, fam)(n)
            e2e, ker = [], []
            for i in range(runs + 20):
                r = rt.run(qc, shots=1024, return_state=False, seed=i)
                e2e.append(r["timing"]["T_e2e"])
                ker.append(r["timing"]["T_kernel"])
            x, k = np.array(e2e[20:]) * 1e3, np.array(ker[20:]) * 1e3
            out.append({"circuit": qc.name, "n": n, "runs": runs, "e2e_p50_ms": float(np.percentile(x, 50)),
                        "e2e_p99_ms": float(np.percentile(x, 99)), "e2e_max_ms": float(x.max()),
                        "kernel_p50_ms": float(np.percentile(k, 50)), "kernel_p99_ms": float(np.percentile(k, 99))})
    ref = {"rqc_16_d10": (32.4, 36.9), "ghz_16": (5.89, 9.15)}     # U55C, results/processed/jitter_summary.csv
    for o in out:
        if o["circuit"] in ref:
            o["reference_u55c_p50_p99_ms"] = ref[o["circuit"]]
    r16 = next(o for o in out if o["circuit"] == "rqc_16_d10")
    print(json.dumps({"metric": "T_e2e latency p50 / p99 of repeated circuits (SVRuntime.run, 1024 shots)",
                      "value": r16["e2e_p99_ms"], "unit": "ms (p99, rqc_16_d10)", "higher_is_better": False,
                      "n_gpus": 1, "dtype": "c64 (fp32 arithmetic)", "data": "synthetic (seeded circuits)",
                      "config": {"workload": f"ghz and rqc (depth 10) at 4, 8, 12, 16 qubits, {runs} runs each after "
                                             "20 warm-up runs"}, "circuits": out}))


def families_main(a):
    """The reference's 30-qubit families (GHZ, QFT, RQC depth 10, VQE 2 layers) through SVRuntime.run
    (1024 shots, no state read-back), beside its published U55C and A100 figures. Cold = first run in the
    process (specialised kernels not compiled yet: interpreter, compilation queued in the background);
    warm = median of 3 runs after the compilations finished. pass_gbs is the reference's formula
    (QSV2 passes x 16 B x 2^30 / T_kernel, analysis/make_tables.py:321); sweep_gbs counts the sweeps run."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    pkg = _package()
    import torch
    from importlib import import_module
    engine = import_module("qsv_b200.engine")
    runtime = import_module("qsv_b200.runtime")
    engine.load()
    torch.cuda.set_device(0)
    n = a.n
    rt = runtime.SVRuntime()
    # U55C pass GB/s and T_e2e (s), A100 Aer fp32 + cuStateVec T_e2e (s): paper/generated/macros.tex
    ref = {"ghz": (141, 4.1, 7.16), "qft": (102, 24.5, 7.29), "rqc": (67, 20.7, 7.24), "vqe": (80, None, 7.28)}
    out = []
    for fam in ("ghz", "qft", "rqc", "vqe"):
        qc = getattr(pkg.generators, fam)(n)
        t0 = time.perf_counter()
        cold = rt.run(qc, shots=1024, return_state=False, seed=0)
        cold_s = time.perf_counter() - t0
        engine.jit_wait()
        warm = []
        for i in range(3):
            warm.append(rt.run(qc, shots=1024, return_state=False, seed=1 + i))
        w = sorted(warm, key=lambda r: r["timing"]["T_e2e"])[1]
        tk = w["timing"]["T_kernel"]
        passes = w["stats"]["n_passes"]
        prog, _, _ = pkg.compile_circuit(qc, n, 12)
        sweeps = sum(len(engine.plan_segment(s_, n)) for k_, s_ in prog if k_ == "segment")
        rec = {"circuit": qc.name, "passes": passes, "sweeps": sweeps, "ops": w["stats"]["n_ops"],
               "cold_e2e_s": cold_s, "T_compile_s": w["timing"]["T_compile"], "T_kernel_s": tk,
               "T_exchange_s": w["timing"]["T_exchange"], "T_e2e_s": w["timing"]["T_e2e"],
               "pass_gbs": passes * (16 << n) / tk / 1e9, "sweep_gbs": sweeps * (16 << n) / tk / 1e9}
        if n == 30:
            rec["reference"] = {"u55c_pass_gbs": ref[fam][0], "u55c_T_e2e_s": ref[fam][1],
                                "a100_aer_cusv_T_e2e_s": ref[fam][2]}
        out.append(rec)
    print(json.dumps({"metric": f"{n}-qubit families through SVRuntime.run (1024 shots)",
                      "value": statistics.median(o["sweep_gbs"] for o in out), "unit": "GB/s (median sweep_gbs)",
                      "higher_is_better": True, "n_gpus": 1, "dtype": "c64 (fp32 arithmetic)",
                      "data": "synthetic (seeded circuits)", "config": {"workload": f"ghz, qft, rqc d10, vqe L2 at n={n}"},
                      "peak_gbs": _peaks()[0], "circuits": out, "specialised_kernels": engine.jit_info()}))


# ------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", "--qubits", dest="n", type=int, default=30)
    ap.add_argument("--depth", type=int, default=24)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the complex128 (FP64) comparison runs")
    ap.add_argument("--jit", default="auto", choices=["auto", "eager", "off", "coarse", "library"],
                    help="specialised sweep kernels (compiled before the warm-up unless off; coarse: kernels of "
                         "coarse sweep structures only)")
    ap.add_argument("--interp", default=None, choices=["phase", "stream"],
                    help="interpreter kernel for sweeps without a specialised kernel (default: the library's)")
    ap.add_argument("--family", default="random_layer", choices=["random_layer", "rqc", "vqe", "qft"],
                    help="rl30 workload circuit: the headline random-layer circuit (default) or, for profiles, "
                         "a reference family")
    ap.add_argument("--workload", default="rl30", choices=["rl30", "precision", "batched", "served", "latency", "families"],
                    help="rl30: the headline sweep benchmark; precision: the complex64 / complex128 study "
                         "(33 qubits complex64, 32 qubits complex128 vs complex64); batched: 512 circuits of "
                         "10..24 qubits per CUDA-graph replay vs one at a time; served: Poisson arrivals of "
                         "12..30-qubit circuits, continuous batching vs the plain sequential path")
    ap.add_argument("--count", type=int, default=0, help="circuits (batched: 512; served: 20000 per rate)")
    ap.add_argument("--rates", default="50,200,500,1000,2000", help="served: arrival rates per second")
    ap.add_argument("--qmax", type=int, default=30, help="served: largest qubit count")
    ap.add_argument("--policy", default="sjf", choices=["sjf", "fifo"], help="served: admission order")
    ap.add_argument("--compile-on-arrival", action="store_true",
                    help="served: compile each request when it arrives (spawned worker pool) instead of before "
                         "the run; the plain path then compiles in line as well")
    a = ap.parse_args()
    if a.workload == "precision":
        return precision_main(a)
    if a.workload == "batched":
        return batched_main(a)
    if a.workload == "served":
        return served_main(a)
    if a.workload == "latency":
        return latency_main(a)
    if a.workload == "families":
        return families_main(a)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pkg = _package()
    qc, prog, fmap, stats = workload(pkg, a.n, a.depth, a.seed, family=a.family)
    segs = [p for kind, p in prog if kind == "segment"]
    shape = (f"{a.family} n={a.n} depth={a.depth} seed={a.seed}" if a.family in ("random_layer", "rqc")
             else f"{a.family} n={a.n}")
    cfg = {"workload": f"{shape}, complex64 ({8 << a.n >> 30} GiB "
                       f"state), QSV2 k=12 M=4 from the reference scheduler",
           "n_qubits": a.n, "depth": a.depth, "qsv2_passes": stats.n_passes, "ops": stats.n_ops,
           "l2": "inputs larger than L2 (8 GiB state vs 126 MB), no flush", "parallelism": f"replicas x{a.gpus}"}

    if a.impl == "reference":
        if rank != 0:
            return
        tiles_total = 1 << (a.n - 12)
        vals = []
        for s in range(a.warmup + a.steps):
            gbs, cores, desc, wall = cpu_sample(segs[0], a.n, tiles_total, seconds=6.0)
            if s >= a.warmup:
                vals.append(gbs)
        v = statistics.median(vals)
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": a.gpus,
                          "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "c64 (fp32)", "data": "synthetic (seeded circuit)",
                          "config": cfg,
                          "cpu_baseline": {"value": v, "unit": "GB/s", "cores": cores, "kind": "port", "sample": desc},
                          "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from importlib import import_module
    engine = import_module("qsv_b200.engine")
    engine.load()
    sweeps = sum(len(engine.plan_segment(s, a.n)) for s in segs)
    eng_info = {"sweeps": sweeps}
    if a.interp:
        engine.set_interp(a.interp)
    engine.set_jit(a.jit)
    if a.jit != "off":
        t0 = time.perf_counter()
        ready = sum(engine.jit_prepare(s, a.n) for s in segs)
        eng_info["specialised_kernels"] = {"sweeps_ready": ready, "structures": engine.jit_info()["structures"],
                                           "compile_s": round(time.perf_counter() - t0, 2)}
    stream = torch.cuda.current_stream(dev)
    state = engine.new_state(a.n, device=dev)

    def step():
        for s in segs:
            engine.run_segment(state, s, stream)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    engine.take_launch_count()
    jit0 = engine.jit_info()["jit_launches"]
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(a.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize(dev)
    launches = engine.take_launch_count()
    jit_launches = engine.jit_info()["jit_launches"] - jit0
    sec = e0.elapsed_time(e1) / 1e3
    if dist:
        t = torch.tensor([sec], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sec = float(t.item())
        dist.barrier()
    bytes_per_sweep = 16 << a.n
    total_bytes = bytes_per_sweep * sweeps * a.steps * world
    value = total_bytes / sec / 1e9
    per_launch = sec / (sweeps * a.steps)
    peak, peak_kind = _peaks()
    achieved = bytes_per_sweep / per_launch / 1e9

    # config 2's second circuit, QFT-30 (H, controlled phases, reversal swaps), timed the same way; reported
    # beside the headline, which stays the random-layer circuit
    qft = None
    if a.n == 30 and world == 1:
        qprog, _, qstats = pkg.compile_circuit(pkg.generators.qft(a.n), a.n, 12)
        qsegs = [p for kind, p in qprog if kind == "segment"]
        if a.jit != "off":
            for s_ in qsegs:
                engine.jit_prepare(s_, a.n)
        qsweeps = sum(len(engine.plan_segment(s_, a.n)) for s_ in qsegs)
        for _ in range(2):
            for s_ in qsegs:
                engine.run_segment(state, s_, stream)
        q0 = torch.cuda.Event(enable_timing=True)
        q1 = torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        for _ in range(3):
            for s_ in qsegs:
                engine.run_segment(state, s_, stream)
        q1.record(stream)
        torch.cuda.synchronize(dev)
        qsec = q0.elapsed_time(q1) / 1e3 / 3
        qgbs = bytes_per_sweep * qsweeps / qsec / 1e9
        qft = {"workload": "qft n=30 (H, CP, reversal swaps as relabels)", "sweeps": qsweeps,
               "qsv2_passes": qstats.n_passes, "ms_per_step": qsec * 1e3, "value": qgbs, "unit": "GB/s",
               "frac": qgbs / _peaks()[0]}

    # accuracy of every reported result against FP64: the complex64 state of each circuit from |0...0>
    # against the complex128 engine's state of the same circuit (untimed, after the timed regions)
    accuracy = None
    if world == 1 and not a.no_accuracy:
        del state
        torch.cuda.empty_cache()
        accuracy = {"oracle": "complex128 engine on the device (FP64 matrices and arithmetic; value for value "
                              "equal to the C oracle's FP64 engine in the tests)",
                    "rl": accuracy_vs_fp64(qc)}
        if qft is not None:
            accuracy["qft30"] = accuracy_vs_fp64(pkg.generators.qft(a.n))
            qft["one_minus_f"] = accuracy["qft30"]["one_minus_f"]
            qft["max_abs_err"] = accuracy["qft30"]["max_abs_err"]
        state = engine.new_state(a.n, device=dev)

    # live copy-bandwidth probe (the hand-written HBM copy kernel) on the state's size: the achievable
    # ceiling measured in the same process, beside the driver-measured peak used for frac
    copy_gbs = remap = None
    if world == 1:
        dst = torch.empty_like(state)
        for _ in range(2):
            engine.hbm_copy(dst, state, stream)
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record(stream)
        for _ in range(5):
            engine.hbm_copy(dst, state, stream)
        c1.record(stream)
        torch.cuda.synchronize(dev)
        copy_gbs = 2 * (8 << a.n) * 5 / (c0.elapsed_time(c1) / 1e3) / 1e9
        # the remap kernel (replaces sv_swap and the host exchanges): one out-of-place bit permutation of
        # the whole state, 16 B per amplitude; a permutation that moves low and high qubits
        perm = [int(x) for x in np.random.default_rng(7).permutation(a.n)]
        for _ in range(2):
            engine.remap(state, dst, perm, stream)
        c0.record(stream)
        for _ in range(5):
            engine.remap(state, dst, perm, stream)
        c1.record(stream)
        torch.cuda.synchronize(dev)
        rsec = c0.elapsed_time(c1) / 1e3 / 5
        remap = {"perm": perm, "ms": rsec * 1e3, "value": (16 << a.n) / rsec / 1e9, "unit": "GB/s",
                 "frac": (16 << a.n) / rsec / 1e9 / _peaks()[0], "kernel": "qsv::dev::remap_kernel"}
        del dst

    # end to end through the public API (host circuit in, sampled counts out)
    e2e = None
    if a.e2e_steps > 0:
        from qsv_b200.runtime import SVRuntime
        rt = SVRuntime(device=dev)
        rt.run(qc, shots=1024, return_state=False, seed=0)
        torch.cuda.synchronize(dev)
        e2e_t = []
        for i in range(a.e2e_steps):
            t0 = time.perf_counter()
            r = rt.run(qc, shots=1024, return_state=False, seed=i)
            e2e_t.append(time.perf_counter() - t0)
        e2e_sec = max(statistics.median(e2e_t), 1e-9)
        if dist:
            t = torch.tensor([e2e_sec], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_sec = float(t.item())
        seg_bytes = sum(np.asarray(s).nbytes for s in segs)
        e2e = {"value": bytes_per_sweep * sweeps * world / e2e_sec / 1e9, "unit": "GB/s",
               "h2d_bytes_per_step": seg_bytes + 8 * 1024, "d2h_bytes_per_step": 8 * 1024,
               "ms_per_step": e2e_sec * 1e3, "T_kernel_s": r["timing"]["T_kernel"],
               "T_compile_s": r["timing"]["T_compile"]}

    if rank == 0:
        cpu = None
        if not a.no_cpu:
            gbs, cores, desc, wall = cpu_sample(segs[0], a.n, 1 << (a.n - 12), seconds=10.0)
            cpu = {"value": gbs, "unit": "GB/s", "cores": cores, "kind": "port", "sample": desc}
        out = {"metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": sec / a.steps * 1e3, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "c64 (fp32 arithmetic)",
               "data": "synthetic (seeded random-layer circuit)", "config": cfg, "engine": eng_info,
               "one_minus_f": accuracy["rl"]["one_minus_f"] if accuracy else None,
               "max_abs_err": accuracy["rl"]["max_abs_err"] if accuracy else None, "accuracy": accuracy,
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "peak_kind": peak_kind,
                            "traffic": TRAFFIC_PER_ALGORITHMIC * bytes_per_sweep,
                            "kernel": ("qsv_sweep_jit (specialised per sweep structure)" if jit_launches == launches
                                       else "qsv::dev::sweep_kernel<13,4,3,3>" if jit_launches == 0
                                       else f"qsv_sweep_jit x{jit_launches} + sweep_kernel x{launches - jit_launches}"),
                            "algorithmic_bytes_per_launch": bytes_per_sweep,
                            "copy_probe_gbs": copy_gbs},
               "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(), "qft30": qft,
               "remap": remap,
               # the reference's own formula (analysis/make_tables.py:321): QSV2 passes x 16 B x 2^n over
               # the kernel time; above the HBM roofline because consecutive passes share one sweep here
               "reference_formula_gbs": stats.n_passes * bytes_per_sweep * a.steps * world / sec / 1e9}
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
