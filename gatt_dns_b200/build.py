"""Build recipe of the CUDA library (nvcc, sm_100a) -- ``python -m gatt_dns_b200.build``."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "gatt_dns.cu")
OUT = os.path.join(HERE, "libgatt_dns_b200.so")
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("sweep.cuh", "rsweep.cuh", "pointwise.cuh", "pwpipe.cuh", "bc.cuh", "arnoldi.cuh", "tangent.cuh")] + \
    [os.path.join(HERE, "..", "include", "gatt_dns.h")]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(p) > t for p in [SRC] + HEADERS if os.path.exists(p))


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", OUT, SRC]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
