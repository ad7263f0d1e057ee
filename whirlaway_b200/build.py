"""Builds the CUDA library of the prover in-tree (sm_100a) with nvcc.

The shared object lands in whirlaway_b200/_build/libwhirlaway_b200.so; the package loads
it from there, so the compiled code travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libwhirlaway_b200.so")
SOURCES = ["k_commit.cu", "k_sumcheck.cu", "k_whir.cu", "k_transcript.cu", "k_verify.cu", "k_program.cu", "prover.cu",
           "server.cu", "noalloc.cu", "verifier.cu", "capi.cu", "air_program.cu", "host_perm.cpp", "tuner.cpp"]
# Integer-pipe throughput probes: a separate library that only the benchmark loads.
PROBE_SRC = os.path.join("probe", "int_peaks.cu")
PROBE_LIB = os.path.join(OUT_DIR, "libwl_probe.so")
CXX_FLAGS = ["-std=c++17", "-O3", "-fPIC"]  # host-only sources (g++; CPU features dispatched at run time)
NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-ccbin", "g++",
]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, jobs=None):
    """Compiles every source to an object and links the shared library; returns its path."""
    os.makedirs(OUT_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "whirlaway_b200.h"))
    objs, procs = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OUT_DIR, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            if src.endswith(".cpp"):
                cmd = ["g++"] + CXX_FLAGS + ["-c", s, "-o", o]
            else:
                cmd = ["nvcc"] + NVCC_FLAGS + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"compiler failed on {src}:\n{out.decode()}")
    if _stale(LIB, objs):
        cmd = ["nvcc", "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-ccbin", "g++", "-o", LIB] + objs
        subprocess.run(cmd, check=True)
    probe = os.path.join(CSRC, PROBE_SRC)
    if _stale(PROBE_LIB, [probe] + headers):
        cmd = ["nvcc"] + NVCC_FLAGS + ["-shared", probe, "-o", PROBE_LIB]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
