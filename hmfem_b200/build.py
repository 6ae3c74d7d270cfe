"""Builds libhmfem_gpu.so (the C-ABI + sm_100a kernels) in-tree with nvcc.

    python -m hmfem_b200.build          # incremental
    python -m hmfem_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libhmfem_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=default", "--expt-relaxed-constexpr",
         "--extended-lambda"]
SOURCES = ["assemble.cu", "sparse.cu", "amg_setup.cu", "rap_stencil.cu", "rap19.cu", "stencil_cycle.cu", "smoother_setup.cu", "cycle.cu", "solver.cu",
           "device_abi.cu", "noalloc.cu", "conv3d.cu", "guess_ops.cu", "karst.cu", "textio.cu", "permio.cu"]


def _deps():
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    hdrs.append(os.path.join(HERE, "..", "include", "hmfem_gpu.h"))
    hdrs.append(os.path.join(HERE, "..", "include", "hmfem_guess.h"))
    hdrs.append(os.path.join(HERE, "..", "include", "hmfem_karst.h"))
    hdrs.append(os.path.join(HERE, "..", "include", "hmfem_textio.h"))
    hdrs.append(os.path.join(HERE, "..", "include", "hmfem_permio.h"))
    return max(os.path.getmtime(h) for h in hdrs)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdr_t = _deps()
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if (not force and os.path.exists(o)
                and os.path.getmtime(o) >= max(os.path.getmtime(s), hdr_t)):
            continue
        cmd = [NVCC] + ARCH + FLAGS + ["-c", s, "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or any(
            os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
