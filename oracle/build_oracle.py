"""Build recipe of the CPU oracle (test infrastructure).

Compiles oracle/hpvcd_oracle.cpp (the C++ restatement of the reference's
scalar reconstruction path) and oracle/cpu_simd.cpp (its AVX2 kernel set, for
the timed CPU reference arm) into oracle/_build/libhpvcd_oracle.so.  The
reference (Rust) cannot be compiled in this image, so there is no
oracle/_ref build.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "libhpvcd_oracle.so")


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "hpvcd_oracle.cpp")
    simd = os.path.join(HERE, "cpu_simd.cpp")
    deps = [src, simd, os.path.join(HERE, "hpvcd_oracle.h"), os.path.join(HERE, "cpu_simd.h"),
            os.path.join(os.path.dirname(HERE), "include", "hpvcd_gpu.h")]
    os.makedirs(OUT_DIR, exist_ok=True)
    if force or not os.path.exists(OUT) or any(os.path.getmtime(d) > os.path.getmtime(OUT) for d in deps):
        # x86-64-v3: AVX2 (the reference's avx/ kernel set) on every host that runs the GPU box
        cmd = ["g++", "-O3", "-march=x86-64-v3", "-std=c++17", "-shared", "-fPIC", "-Wall",
               "-Wextra", "-pthread", "-o", OUT, src, simd]
        print("+", " ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
