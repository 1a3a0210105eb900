"""NumPy restatement of the reference's golden model (host/sv/model.py) -- TEST INFRASTRUCTURE ONLY.

Executes a QSV2 segment tile by tile in complex64, with the same numpy operations in the same order as
the reference model, so its outputs equal the reference model's bit for bit (checked against fixtures
the reference produced, tests/golden/model_states.npz). It serves as the parity oracle at float32
tolerance and as the timed CPU baseline ("the reference's own CPU implementation of the path").
Nothing on the product path imports it.
"""
import numpy as np

MAGIC, HDR_WORDS, PASS_WORDS, OP_WORDS, OP_MUX2 = 0x51535632, 8, 8, 24, 1


def decode(seg):
    """Stream -> (L, k, [(m, highs, [(code, t, cmask, M0, M1)])])   (model.py:7-22)."""
    w = np.asarray(seg, dtype=np.int32)
    if int(w[0]) != MAGIC:
        raise ValueError("bad QSV2 magic")
    L, n_pass, k = int(w[1]), int(w[2]), int(w[3])
    at = HDR_WORDS
    passes = []
    for _ in range(n_pass):
        hdr = [int(v) for v in w[at:at + 6]]
        m, nops = hdr[0], hdr[3]
        highs = [hdr[1], hdr[2], hdr[4], hdr[5]][:m]
        at += PASS_WORDS
        ops = []
        for _ in range(nops):
            rec = w[at:at + OP_WORDS]
            at += OP_WORDS
            fl = rec[8:24].view(np.float32)
            cplx = (fl[0::2] + 1j * fl[1::2]).astype(np.complex64)
            ops.append((int(rec[0]), int(rec[1]), int(rec[2]), cplx[:4].reshape(2, 2), cplx[4:].reshape(2, 2)))
        passes.append((m, highs, ops))
    return L, k, passes


def tile_index_map(L, k, m, highs):
    """idx[t, j] = slice index of element j of tile t, shape (2^(L-k), 2^k)   (model.py:25-40)."""
    low = k - m
    taken = set(range(low)) | set(highs[:m])
    free = [b for b in range(L) if b not in taken]
    if len(free) != L - k:
        raise ValueError("high qubits overlap the low window")
    j = np.arange(1 << k, dtype=np.int64)
    within = j & ((1 << low) - 1)
    for i, h in enumerate(highs[:m]):
        within |= ((j >> (low + i)) & 1) << h
    t = np.arange(1 << (L - k), dtype=np.int64)
    base = np.zeros_like(t)
    for i, b in enumerate(free):
        base |= ((t >> i) & 1) << b
    return base[:, None] | within[None, :]


def apply_op_tile(T, code, t, cmask, M0, M1):
    """MUX2 along tile qubit t on every tile row of T (model.py:43-56)."""
    if code != OP_MUX2:
        raise ValueError(f"opcode {code}")
    rows, size = T.shape
    k = size.bit_length() - 1
    V = T.reshape(rows, 1 << (k - t - 1), 2, 1 << t)
    i0 = np.arange(size).reshape(1 << (k - t - 1), 2, 1 << t)[:, 0, :]
    use1 = ((i0 & cmask) == cmask) if cmask else np.zeros_like(i0, dtype=bool)
    x0 = V[:, :, 0, :].copy()
    x1 = V[:, :, 1, :].copy()
    for M, where in ((M0, ~use1), (M1, use1)):
        y0 = M[0, 0] * x0 + M[0, 1] * x1
        y1 = M[1, 0] * x0 + M[1, 1] * x1
        V[:, :, 0, :] = np.where(where[None], y0, V[:, :, 0, :])
        V[:, :, 1, :] = np.where(where[None], y1, V[:, :, 1, :])


def run_segment(state, P, seg):
    """Every pass of a segment over each of the P slices, in place (model.py:59-71)."""
    L, k, passes = decode(seg)
    if state.size != P << L:
        raise ValueError("state size does not match P * 2^L")
    for m, highs, ops in passes:
        idx = tile_index_map(L, k, m, highs)
        for p in range(P):
            part = state[p << L:(p + 1) << L]
            T = part[idx]
            for code, t, cm, M0, M1 in ops:
                apply_op_tile(T, code, t, cm, M0, M1)
            part[idx] = T
    return state


def remap(state, n, perm):
    """perm[new] = old on index bits (model.py:74-78)."""
    v = state.reshape([2] * n)               # numpy axis a holds index bit n-1-a
    axes = [n - 1 - perm[n - 1 - a] for a in range(n)]
    return np.ascontiguousarray(np.transpose(v, axes)).reshape(-1)


def unpermute(state, n, final_map):
    """State in logical qubit order, final_map[l] = physical position of l (model.py:81-84)."""
    return remap(state, n, [final_map[q] for q in range(n)])


def run_program(prog, n, P, final_map, state=None):
    """Whole program from |0...0> (model.py:87-95)."""
    if state is None:
        state = np.zeros(1 << n, dtype=np.complex64)
        state[0] = 1
    for kind, payload in prog:
        if kind == "segment":
            run_segment(state, P, payload)
        else:
            state = remap(state, n, payload)
    return unpermute(state, n, final_map)


def run_segment_tiles(state, seg, tiles, n_passes=None):
    """The golden model's run_segment restricted to the given tile numbers of every pass (same tile
    addressing and arithmetic as tile_index_map / apply_op_tile); a bounded sample of a full segment for
    timing the CPU baseline at sizes where the whole segment would take hours. Returns the amplitudes
    read + written (bytes)."""
    L, k, passes = decode(seg)
    tiles = np.asarray(tiles, dtype=np.int64)
    moved = 0
    for m, highs, ops in passes[:n_passes]:
        low = k - m
        taken = set(range(low)) | set(highs[:m])
        free = [b for b in range(L) if b not in taken]
        j = np.arange(1 << k, dtype=np.int64)
        within = j & ((1 << low) - 1)
        for i, h in enumerate(highs[:m]):
            within |= ((j >> (low + i)) & 1) << h
        base = np.zeros_like(tiles)
        for i, b in enumerate(free):
            base |= ((tiles >> i) & 1) << b
        idx = base[:, None] | within[None, :]
        T = state[idx]
        for code, t, cm, M0, M1 in ops:
            apply_op_tile(T, code, t, cm, M0, M1)
        state[idx] = T
        moved += T.size * 16
    return moved
