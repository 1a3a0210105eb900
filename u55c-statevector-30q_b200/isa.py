"""QSV2 instruction-stream layout (the contract shared by the compiler, the oracle and the CUDA engine).

The layout is the reference's (host/sv/isa.py:1-32); the numbers below are the wire format and have to
match it word for word so that a stream compiled for the FPGA engine runs unchanged here.

Stream (int32 words; fp32 matrices are stored as their bit patterns):
  header   [MAGIC, L, n_passes, k, 0, 0, 0, 0]
  pass     [m, h0, h1, n_ops, h2, h3, 0, 0]        tile qubits 0..k-m-1 = physical 0..k-m-1,
                                                  tile qubit k-m+i = physical h_i
  op       [OP_MUX2, t, cmask, 0, 0, 0, 0, 0, M0 (re,im x4), M1 (re,im x4)]
A pair (i0, i0 | 1<<t) along tile qubit t uses M1 when cmask != 0 and every cmask bit of i0 is set,
otherwise M0 (host/sv/isa.py:18-21, host/sv/model.py:50).

Extension for complex128 states (no reference counterpart; the FPGA engine is complex64 only): header
word 4 = DTYPE_C128 marks a stream whose op records carry FP64 matrices,
  op       [OP_MUX2, t, cmask, 0, 0, 0, 0, 0, M0 (re,im x4 as float64), M1 (re,im x4 as float64)]
(40 words; each float64 is two int32 words, low word first). Reference streams have word 4 = 0
(DTYPE_C64) and are unchanged.
"""
MAGIC = 0x51535632        # "QSV2"
HDR_WORDS = 8
PASS_WORDS = 8
OP_WORDS = 24
DTYPE_C64 = 0             # header word 4: fp32 matrices, complex64 state (the reference's streams)
DTYPE_C128 = 1            # header word 4: fp64 matrices, complex128 state
OP_WORDS_C128 = 40
OP_MUX2 = 1
MAX_OPS_PER_PASS = 64
MAX_HIGH = 4              # high-qubit slots in a pass header (words 1, 2, 4, 5)
