"""Build recipe of the CUDA library libmaxwellfdtd_b200.so (sm_100a, in-tree).

--fmad=false keeps every a*b+c unfused: the reference's Julia arithmetic does not contract,
and the parity tests compare the device results with a CPU restatement bit for bit.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = [os.path.join(HERE, "csrc", "engine.cu")]
DEPS = SRC + sorted(os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc")) if f.endswith(".cuh")) + \
    [os.path.join(os.path.dirname(HERE), "include", "maxwellfdtd.h")]
OUT = os.path.join(HERE, "libmaxwellfdtd_b200.so")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "--fmad=false", "-Xcompiler", "-fPIC", "-shared", "-Xcompiler", "-fvisibility=hidden",
]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t for p in DEPS)


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return OUT
    cmd = [nvcc()] + NVCC_FLAGS + list(extra) + ["-o", OUT] + SRC
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"])
