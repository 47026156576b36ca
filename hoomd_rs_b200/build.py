"""Build libhmc_b200.so in-tree with nvcc for sm_100a.

    python -m hoomd_rs_b200.build

The library is a plain shared object with a C ABI (include/hmc.h); it links the CUDA
runtime statically, so loading it needs only the driver. Host code is compiled with
-ffp-contract=off because the FP64 decision path must round exactly where the
reference's Rust code rounds.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libhmc_b200.so")
SOURCES = ["hmc_kernels.cu", "hmc_lj.cu", "hmc_poly.cu", "hmc_poly2.cu", "hmc_serial.cu", "hmc_capi.cu", "hmc_gsd.cu", "hmc_noalloc.cu"]
HEADERS = ["hmc_math.cuh", "hmc_internal.cuh", "hmc_device.cuh", "hmc_host.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
         "-Xptxas", "-v", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "hmc.h"), __file__]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False, out: str = LIB, defines=()) -> str:
    if not force and out == LIB and not _stale():
        return LIB
    cmd = [nvcc(), *ARCH, *FLAGS, *[f"-D{d}" for d in defines], "-shared", "-o", out,
           *[os.path.join(CSRC, f) for f in SOURCES]]
    r = subprocess.run(cmd, capture_output=True, text=True)
    log = out + ".build.log"
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed ({r.returncode}); see {log}")
    if verbose:
        sys.stdout.write(r.stderr)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
