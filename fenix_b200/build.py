"""Build recipe of libfenixcuda.so and libfenixcuda_fast.so (nvcc, sm_100a, in-tree).

libfenixcuda.so is the parity build. Flags that the bit-exact parity of its
kernels depends on:
  -fmad=false                 no contraction of a*b+c into FMA (explicit fmaf stays)
  -prec-div=true -prec-sqrt=true -ftz=false   IEEE division, square root, denormals
libfenixcuda_fast.so is the fast-arithmetic build of the same sources: FMA
contraction, approximate division and square root, CUDA's sinf/cosf and
products by reciprocals (FX_FAST_MATH). Its results are stated against f64, not
the oracle's bits.
"""
from __future__ import annotations

import os
import subprocess
import sys

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PACKAGE_DIR, "csrc")
SOURCES = ["fx_sim.cu", "fx_plain.cu", "fx_fused.cu", "fx_pressure.cu", "fx_vcycle.cu", "fx_render.cu", "fx_noalloc.cu", "fx_adjoint.cu"]
OUTPUT = os.path.join(PACKAGE_DIR, "libfenixcuda.so")
OUTPUT_FAST = os.path.join(PACKAGE_DIR, "libfenixcuda_fast.so")

NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-fmad=false",
    "-prec-div=true",
    "-prec-sqrt=true",
    "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off",
    "-shared",
]


def nvcc() -> str:
    if os.environ.get("NVCC"):
        return os.environ["NVCC"]
    return "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else "nvcc"


def sources() -> list[str]:
    return [os.path.join(CSRC, s) for s in SOURCES]


FAST_FLAGS = [("-fmad=true" if f == "-fmad=false" else "-prec-div=false" if f == "-prec-div=true" else
               "-prec-sqrt=false" if f == "-prec-sqrt=true" else f) for f in NVCC_FLAGS] + ["-DFX_FAST_MATH"]


def needs_build(output: str = OUTPUT) -> bool:
    if not os.path.exists(output):
        return True
    out_m = os.path.getmtime(output)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(PACKAGE_DIR, "..", "include", "fenix_cuda.h"))
    return any(os.path.getmtime(d) > out_m for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Builds both libraries (each only when a source is newer); returns the parity one."""
    for output, flags in ((OUTPUT, NVCC_FLAGS), (OUTPUT_FAST, FAST_FLAGS)):
        if not force and not needs_build(output):
            continue
        cmd = [nvcc(), *flags, "-o", output, *sources()]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return OUTPUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
