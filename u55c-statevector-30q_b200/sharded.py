"""One state sharded over G = 2^g GPUs, one process per GPU: the reference's multi-card runtime
(host/sv/multicard.py) on torch.distributed.

Layout (the reference's, multicard.py:3-4): qubits 0..L-1 are local bits inside a slice of 2^L amplitudes,
qubits L..n-1 (g of them) select the slice. Rank r holds logical slice held[r]. The compiler is the same
one with L = n - g (compile_circuit(qc, L, k)): segments only touch local qubits, and the scheduler
inserts remaps that bring bank qubits (>= L) into the window (compiler.py:186-260). Execution, per step:

  segment  every rank runs it on its slice (qsv_run_segment; no communication);
  remap    decomposed into bit transpositions (runtime.py:35-44), each handled as in multicard.py:100-118:
             local <-> local : a permutation of every slice (qsv_remap), no communication;
             bank j <-> local v : the pairwise exchange of half slices between the holders of logical slices
                 s and s ^ 2^j (multicard.py:53-87): the holder of s with bit j = 0 sends its amplitudes with
                 local bit v = 1 and receives the partner's amplitudes with local bit v = 0, and the other
                 way round; over NCCL send/recv, in bounded pieces through contiguous staging buffers;
             bank <-> bank : a relabelling of the slices (held[]), no data movement.

Results: the norm and <Z_q> for every qubit (FP64 all-reduce of the slices' reductions), Born samples
(slice chosen on rank 0 from the slices' totals, then the index within the slice sampled on its holder
with qsv_sample_f64), and, for small n, the whole state gathered on rank 0. A slice holds the same values
the single-GPU engine would hold for those amplitudes: the ops are applied in the same order with the same
arithmetic and every data movement is an exact permutation.

No collective runs inside a segment (passes never touch bank qubits); the exchanges are the only
communication. Every rank takes the same collective steps in the same order.
"""
import time

import numpy as np

from .compiler import compile_circuit
from .runtime import KMAX, logical_counts, transpositions

# largest staging piece of one exchange (bytes per direction); pieces keep the extra memory bounded
EXCHANGE_PIECE_BYTES = 256 << 20


def _swap_bits(s, a, b):
    if ((s >> a) & 1) != ((s >> b) & 1):
        s ^= (1 << a) | (1 << b)
    return s


class CudaSlices:
    """A rank's slice on its GPU, run by this package's engine (the product path; there is no CPU one)."""

    def __init__(self, device=None, stream=None):
        import torch
        from . import engine
        if not torch.cuda.is_available():
            raise RuntimeError("the sharded runtime needs a CUDA device (B200); none is available")
        engine.load()
        self.engine = engine
        self.device = torch.device(device if device is not None else "cuda")
        self.stream = stream
        self.scratch = None

    def alloc(self, L):
        import torch
        state = torch.empty(1 << L, dtype=torch.complex64, device=self.device)
        self.scratch = self.engine.new_scratch(L, self.device)
        return state

    def zero(self, state, one):
        self.engine.zero_state(state, self.stream)        # |0...0> of the slice: amplitude 0 = 1
        if not one:
            state.zero_()

    def run_segment(self, state, seg):
        self.engine.run_segment(state, seg, self.stream)

    def permute(self, state, perm):
        import torch
        dst = torch.empty_like(state)
        self.engine.remap(state, dst, perm, self.stream)
        return dst

    def reduce(self, state):
        """[sum |a|^2, <Z_0>, ..., <Z_{L-1}>] of the slice (unnormalised, FP64) as a host array."""
        out = self.engine.reduce_f64(state, scratch=self.scratch, stream=self.stream)
        return out.cpu().numpy()

    def sample(self, state, uniforms):
        import torch
        if len(uniforms) == 0:
            return np.zeros(0, dtype=np.int64)
        idx = self.engine.sample_f64(state, torch.as_tensor(uniforms, dtype=torch.float64), self.scratch, self.stream)
        return idx.cpu().numpy()

    def synchronize(self):
        import torch
        torch.cuda.synchronize(self.device)


class ShardedRuntime:
    """Run a circuit on a state sharded over every rank of the default process group (world size a power
    of two). Call run() on every rank with the same arguments; rank 0 returns the counts (and the state
    when asked), every rank returns the norm and <Z_q>."""

    def __init__(self, slices=None, group=None, piece_bytes=EXCHANGE_PIECE_BYTES):
        import torch.distributed as dist
        if not dist.is_initialized():
            raise RuntimeError("initialise torch.distributed first (one process per GPU, backend nccl)")
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        if self.world & (self.world - 1):
            raise ValueError(f"world size {self.world} is not a power of two")
        self.g = self.world.bit_length() - 1
        self.slices = slices if slices is not None else CudaSlices()
        self.piece_bytes = int(piece_bytes)
        self.held = list(range(self.world))       # held[r] = logical slice on rank r

    def _global_rank(self, r):
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    # ------------------------------------------------------------------ data movement
    def _exchange(self, state, j, v):
        """Bank bit j (qubit L + j) <-> local bit v: swap half slices with the holder of held ^ 2^j."""
        import torch
        s = self.held[self.rank]
        peer = self.held.index(s ^ (1 << j))
        mine = (s >> j) & 1                       # 0: send / receive the amplitudes with local bit v = 1
        view = state.view(-1, 2, 1 << v)          # (chunks, local bit v, 2^v contiguous amplitudes)
        half = view[:, 1 - mine, :]
        nchunk = view.shape[0]
        rows = max(1, self.piece_bytes // ((1 << v) * state.element_size()))
        peer_g = self._global_rank(peer)
        for c0 in range(0, nchunk, rows):
            part = half[c0:c0 + rows]
            send = torch.view_as_real(part.contiguous())   # complex as float pairs (every backend moves these)
            recv = torch.empty_like(send)
            ops = [self.dist.P2POp(self.dist.isend, send, peer_g, self.group),
                   self.dist.P2POp(self.dist.irecv, recv, peer_g, self.group)]
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()
            part.copy_(torch.view_as_complex(recv))
        return state

    def _remap(self, state, perm, L):
        local = list(range(L))                    # pending local permutation (applied lazily, in order)

        def flush(st):
            nonlocal local
            if local != list(range(L)):
                st = self.slices.permute(st, local)
                local = list(range(L))
            return st

        # transpositions(perm) lists swaps whose product is perm when applied last to first (the scheduler's
        # remaps are disjoint transpositions, for which the order is immaterial)
        for a, b in reversed(transpositions(perm)):
            if b < L:
                # compose: the new layout swaps bits a and b of the current pending one
                local[a], local[b] = local[b], local[a]
            elif a < L:
                state = flush(state)
                state = self._exchange(state, b - L, a)
            else:
                ja, jb = a - L, b - L
                self.held = [_swap_bits(s, ja, jb) for s in self.held]
        return flush(state)

    # ------------------------------------------------------------------ public
    def run(self, qc, shots=1024, k=KMAX, fuse=True, tiling=True, return_state=False, seed=None):
        n = qc.num_qubits
        L = n - self.g
        if L < 10:
            raise ValueError(f"{n} qubits over {self.world} slices leaves {L} local qubits (the engine needs >= 10)")
        k = min(k, L)
        t0 = time.perf_counter()
        prog, fmap, stats = compile_circuit(qc.remove_final_measurements(inplace=False), L, k, fuse_1q=fuse,
                                            tiling=tiling)
        t1 = time.perf_counter()
        self.held = list(range(self.world))
        state = self.slices.alloc(L)
        self.slices.zero(state, self.held[self.rank] == 0)
        started = False
        n_exch = 0
        for kind, payload in prog:
            if kind == "remap" and not started:
                # |0...0> is unchanged by any qubit permutation; the slice labels still follow it
                for a, b in reversed(transpositions(payload)):
                    if a >= L:
                        self.held = [_swap_bits(s, a - L, b - L) for s in self.held]
                # amplitude 0 moves only if a relabelling moved logical slice 0
                self.slices.zero(state, self.held[self.rank] == 0)
                continue
            if kind == "segment":
                started = True
                self.slices.run_segment(state, payload)
            else:
                n_exch += sum(1 for a, b in transpositions(payload) if a < L <= b)
                state = self._remap(state, payload, L)
        self.slices.synchronize()
        t2 = time.perf_counter()
        out = self._results(state, n, L, fmap, shots, seed, return_state)
        out.update(P=self.world, L=L, k=k, stats=stats.__dict__, exchanges=n_exch,
                   timing=dict(T_compile=t1 - t0, T_run=t2 - t1, T_e2e=time.perf_counter() - t0))
        return out

    def _results(self, state, n, L, fmap, shots, seed, return_state):
        import torch
        dist = self.dist
        s = self.held[self.rank]
        red = self.slices.reduce(state)                               # [total, <Z_0..L-1> unnormalised]
        # physical <Z> of every qubit: local bits from the slice, bank bits from the slice label's sign
        zphys = np.zeros(n + 1, dtype=np.float64)
        zphys[0] = red[0]
        zphys[1:L + 1] = red[1:L + 1]
        for j in range(self.g):
            zphys[L + 1 + j] = red[0] * (1 - 2 * ((s >> j) & 1))
        t = torch.as_tensor(zphys)
        totals = torch.zeros(self.world, dtype=torch.float64)
        totals[s] = red[0]
        if dist.get_backend(self.group) == "nccl":
            t, totals = t.cuda(), totals.cuda()
        dist.all_reduce(t, group=self.group)
        dist.all_reduce(totals, group=self.group)
        zphys, totals = t.cpu().numpy(), totals.cpu().numpy()
        norm = zphys[0]
        z = np.array([zphys[1 + fmap[q]] for q in range(n)]) / norm
        out = dict(norm=norm, expect_z=z)
        # Born samples: slice on rank 0 (FP64 cdf over the slice totals), index within it on its holder
        counts = {}
        if shots > 0:
            rng = np.random.default_rng(seed)
            u = rng.random(shots)
            cdf = np.cumsum(totals)
            pick = np.minimum(np.searchsorted(cdf, u * cdf[-1], side="right"), self.world - 1)
            lo = np.concatenate([[0.0], cdf[:-1]])[pick]
            inner = np.clip((u * cdf[-1] - lo) / np.maximum(totals[pick], 1e-300), 0.0, np.nextafter(1.0, 0.0))
            mine = np.nonzero(pick == s)[0]
            idx_local = self.slices.sample(state, inner[mine])
            phys = np.zeros(shots, dtype=np.int64)
            phys[mine] = (np.int64(s) << L) | idx_local
            pt = torch.as_tensor(phys)
            if dist.get_backend(self.group) == "nccl":
                pt = pt.cuda()
            dist.all_reduce(pt, group=self.group)                       # each shot is set by one rank only
            if self.rank == 0:
                counts = logical_counts(pt.cpu().numpy(), fmap, n)
        out["counts"] = counts
        if return_state:
            host = torch.view_as_real(torch.as_tensor(np.ascontiguousarray(self._host(state))))
            parts = [torch.empty_like(host) for _ in range(self.world)] if self.rank == 0 else None
            if dist.get_backend(self.group) == "nccl":
                host = host.cuda()
                parts = [p.cuda() for p in parts] if parts is not None else None
            dist.gather(host, parts, dst=self._global_rank(0), group=self.group)
            if self.rank == 0:
                full = np.empty(1 << n, dtype=np.complex64)
                for r, p in enumerate(parts):
                    sl = self.held[r]
                    full[sl << L:(sl + 1) << L] = torch.view_as_complex(p.cpu()).numpy()
                perm = [fmap[q] for q in range(n)]       # logical order, on the host (small n only)
                idx = np.arange(1 << n)
                src = np.zeros_like(idx)
                for newb, oldb in enumerate(perm):
                    src |= ((idx >> newb) & 1) << oldb
                out["state"] = full[src]
        return out

    def _host(self, state):
        t = state.detach()
        return t.cpu().numpy() if hasattr(t, "cpu") else np.asarray(t)
