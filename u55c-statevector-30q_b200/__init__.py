"""qsv_b200: a B200-native statevector simulator that executes the reference's QSV2 MUX2 programs
with hand-written sm_100a CUDA kernels behind a C ABI (libqsv_b200.so).

Layers (host side in Python, device side in ``csrc/``):
  isa        QSV2 wire format
  circuit    qiskit-free circuit container; generators: seeded workload circuits; qasm: OpenQASM 2 text
  compiler   gates -> MUX2 ops -> passes -> QSV2 segments (the reference's lowering and scheduler)
  engine     ctypes binding of the C ABI; device state buffers held by PyTorch tensors
  runtime    SVRuntime, the drop-in for the reference's XRT runtime
  batch      many circuits per persistent launch, CUDA-graph replay, tile autotuner
  serve      continuous-batching server with HBM-budget admission
  sharded    one state over several GPUs (one process per GPU, NCCL exchanges of half slices)
"""
from . import isa, gates, circuit, generators, compiler, qasm  # noqa: F401
from .circuit import Circuit  # noqa: F401
from .compiler import compile_circuit, Stats, Op  # noqa: F401

__all__ = ["isa", "gates", "circuit", "generators", "compiler", "qasm", "Circuit", "compile_circuit"]
