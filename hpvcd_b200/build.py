"""Build recipe for the native parts of hpvcd_b200.

* libhpvcd_b200.so -- CUDA kernels for sm_100a + the C ABI (include/hpvcd_gpu.h)
  + the host runtime (contexts, plans, staging, tickets).
* libhpvcd_synth.so -- host-only seeded generator of flat per-picture buffers.

Both are built in-tree so they travel with the repository snapshot.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd: list[str]) -> None:
    print("+", " ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_synth(force: bool = False) -> str:
    out = os.path.join(HERE, "libhpvcd_synth.so")
    srcs = [os.path.join(CSRC, "synth.cpp"), os.path.join(CSRC, "hpvcd_synth.h"),
            os.path.join(CSRC, "cabac_tables.h"), os.path.join(INCLUDE, "hpvcd_gpu.h"),
            os.path.join(INCLUDE, "hpvcd_syntax.h")]
    if force or _stale(out, srcs):
        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-Wall", "-Wextra",
              "-o", out, srcs[0]])
    return out


def cuda_sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


# host-only C++ of the main library (the syntax decode); synth.cpp is the
# separate generator library
HOST_SOURCES = ["syntax.cpp"]


def build_cuda(force: bool = False, verbose_ptxas: bool = False) -> str:
    out = os.path.join(HERE, "libhpvcd_b200.so")
    cus = cuda_sources()
    hosts = [os.path.join(CSRC, f) for f in HOST_SOURCES]
    deps = cus + hosts + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + [
        os.path.join(INCLUDE, "hpvcd_gpu.h"), os.path.join(INCLUDE, "hpvcd_syntax.h")]
    if not (force or _stale(out, deps)):
        return out
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for cu in cus:
        obj = os.path.join(objdir, os.path.basename(cu) + ".o")
        flags = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                 "-Xcompiler", "-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC,
                 "--expt-relaxed-constexpr", "-c", cu, "-o", obj]
        if verbose_ptxas:
            flags.insert(1, "-Xptxas=-v")
        if force or _stale(obj, [cu] + deps):
            _run(flags)
        objs.append(obj)
    for src in hosts:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        if force or _stale(obj, [src] + deps):
            _run(["g++", "-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-Wall", "-Wextra",
                  "-I", INCLUDE, "-I", CSRC, "-c", src, "-o", obj])
        objs.append(obj)
    # static CUDA runtime (nvcc's default): no dependency on a libcudart on
    # the library path; the driver's primary context is shared with torch.
    _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", out, *objs, "-lpthread"])
    return out


def build_all(force: bool = False) -> None:
    build_synth(force)
    build_cuda(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
