"""Builds libpureadsorb_b200.so in this directory: nvcc for sm_100a, host code with
-ffp-contract=off (the pose stream's strict arithmetic must not be contracted on the host)."""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "pa_capi.cu")
OUT = os.path.join(HERE, "libpureadsorb_b200.so")
DEPS = ["pa_capi.cu", "pa_kernels.cuh", "pa_energy32.cuh", "pa_grad32.cuh", "pa_chain32.cuh", "pa_build.cuh", "pa_common.cuh",
        "pa_coeffs.h"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    srcs = [os.path.join(HERE, "csrc", d) for d in DEPS] + [os.path.join(HERE, "..", "include", "pureadsorb_b200.h")]
    return any(os.path.getmtime(p) > t for p in srcs)


def build(force=False, verbose=False):
    if not force and not stale():
        return OUT
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-shared", "-o", OUT + ".tmp", SRC]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libpureadsorb_b200.so")
    os.replace(OUT + ".tmp", OUT)
    if verbose:
        sys.stderr.write(r.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
