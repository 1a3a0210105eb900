"""Builds libqsv_b200.so in place with nvcc for sm_100a (cross-compiles on a machine without a GPU).

    python u55c-statevector-30q_b200/build.py [--force] [--verbose]

The library links the CUDA runtime statically, so it does not depend on which libcudart the host
process (PyTorch) loaded; both talk to the driver's primary context.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libqsv_b200.so")
SOURCES = ["qsv_capi.cu", "qsv_sweep.cu", "qsv_sweep_d.cu", "qsv_aux.cu", "qsv_batch.cu", "qsv_planner.cpp",
           "qsv_jit.cpp"]
# device headers compiled into the library AND embedded in it for run-time (NVRTC) specialised kernels
JIT_HEADERS = ["qsv_plan.h", "qsv_device.cuh", "qsv_ops.cuh", "qsv_sweep_body.cuh", "qsv_jit_ops.cuh", "qsv_stream.cuh"]
HEADERS = JIT_HEADERS + ["qsv_planner.h"]
GEN = os.path.join(CSRC, "_gen", "qsv_jit_headers.inc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def cuda_root():
    exe = nvcc()
    if os.path.isabs(exe):
        return os.path.dirname(os.path.dirname(exe))
    return os.environ.get("CUDA_HOME", "/usr/local/cuda")


def gen_jit_headers():
    """Embed the device headers as string literals: NVRTC compiles specialised sweep kernels from them at
    run time, so the specialised and the prebuilt kernels always share one source."""
    names, bodies = [], []
    for h in JIT_HEADERS:
        with open(os.path.join(CSRC, h)) as f:
            text = f.read()
        if ")QSVJIT\"" in text:
            raise RuntimeError(f"{h} contains the raw-string delimiter")
        names.append(h)
        bodies.append(text)
    out = ["// generated by build.py from the device headers; do not edit", "#pragma once",
           f"static const int kJitNumHeaders = {len(names)};",
           "static const char *const kJitHeaderNames[] = {" + ", ".join(f'"{n}"' for n in names) + "};",
           "static const char *const kJitHeaderSources[] = {"]
    out += [f'R"QSVJIT({b})QSVJIT",' for b in bodies]
    out.append("};")
    text = "\n".join(out) + "\n"
    os.makedirs(os.path.dirname(GEN), exist_ok=True)
    if not os.path.exists(GEN) or open(GEN).read() != text:
        with open(GEN, "w") as f:
            f.write(text)


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "qsv_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    gen_jit_headers()
    lib64 = os.path.join(cuda_root(), "lib64")
    cmd = [nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "--shared", "-Xcompiler", "-fPIC,-fvisibility=hidden",
           "-cudart", "static", "--expt-relaxed-constexpr", "-o", LIB + ".tmp",
           "-L" + lib64, "-lnvrtc", "-Xlinker", "-rpath=" + lib64]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, f) for f in SOURCES]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print(LIB)
