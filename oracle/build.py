"""Build recipe of the oracle library (test infrastructure; see fenix_oracle.cpp).

-ffp-contract=off keeps gcc from fusing a*b+c into FMA, so the f32
instantiation evaluates the same IEEE operations as the CUDA kernels.
The target is x86-64-v3 (AVX2 + FMA), not -march=native, because the library is
built in one container and loaded on another host.
"""
from __future__ import annotations

import os
import subprocess
import sys

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
SOURCE = os.path.join(ORACLE_DIR, "fenix_oracle.cpp")
SOURCES = [SOURCE, os.path.join(ORACLE_DIR, "raymarch.cpp")]
OUTPUT = os.path.join(ORACLE_DIR, "liboracle_fenix.so")

CXX_FLAGS = ["-O3", "-std=c++17", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared"]


def compiler() -> str:
    # The system g++ ships libgomp; some environments point $CXX at a g++ without it.
    if os.environ.get("FENIX_ORACLE_CXX"):
        return os.environ["FENIX_ORACLE_CXX"]
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def needs_build() -> bool:
    return not os.path.exists(OUTPUT) or any(os.path.getmtime(src) > os.path.getmtime(OUTPUT) for src in SOURCES)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return OUTPUT
    cmd = [compiler(), *CXX_FLAGS, "-o", OUTPUT, *SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return OUTPUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
