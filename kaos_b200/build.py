"""Build the CUDA library in-tree for sm_100a (no JIT, no torch extension):
kaos_b200/libkaos_gpu.so, loaded through ctypes by kaos_b200.lib."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libkaos_gpu.so")
SOURCES = ["kaos_api.cu"]
DEPS = ["kaos_api.cu", "kaos_common.cuh", "kaos_push.cuh", "kaos_tube.cuh", "kaos_f64.cuh",
        "kaos_cx.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
         "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-v"]


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, d) for d in DEPS]
    deps += [os.path.join(HERE, "..", "include", h) for h in ("kaos_gpu.h", "kaos_philox.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    cmd = [NVCC] + FLAGS + ["-o", OUT] + [os.path.join(CSRC, s) for s in SOURCES]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libkaos_gpu.so")
    if verbose:
        sys.stderr.write(r.stderr)
    with open(os.path.join(HERE, "ptxas_report.txt"), "w") as f:
        f.write(r.stderr)
    return OUT


if __name__ == "__main__":
    build(force=True, verbose=True)
