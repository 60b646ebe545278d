"""Builds the sm_100a shared library ``scadyn_b200/libscadyn_gpu.so`` in-tree
with nvcc (no JIT cache: the .so travels with the source tree)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libscadyn_gpu.so")
SOURCES = ["api.cu", "kernels_matvec.cu", "kernels_setup.cu", "setup_device.cu", "batch.cu", "server.cu", "selftest.cu", "near_mma.cu"]
HEADERS = ["common.cuh", "ctx.h", "fft_reg.cuh", "near_mma.cuh", "linear_basis.h", "fft_mixed.cuh", "fft_yz.cuh",
           "geom.cuh", "lin_setup.cuh", "layout_check.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "scadyn_gpu.h"))
    deps.append(os.path.join(HERE, "..", "include", "scadyn_server.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    objs = []
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    procs = []
    for s in SOURCES:
        o = os.path.join(HERE, "_build", s.replace(".cu", ".o"))
        cmd = [nvcc, *ARCH, *FLAGS, "-I", os.path.join(HERE, "..", "include"), "-c", os.path.join(CSRC, s), "-o", o]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(o)
    for s, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s}:\n{out.decode()}")
        if verbose and out:
            print(out.decode(), file=sys.stderr)
    cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fPIC"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
