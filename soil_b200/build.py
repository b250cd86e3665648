"""Build libsoil_cuda.so in-tree for sm_100a with nvcc.

    python -m soil_b200.build [--force]

Flags: -gencode arch=compute_100a,code=sm_100a, -O3, -lineinfo, and
-fmad=false so that no a*b+c is contracted into an FMA — the reference's Rust
arithmetic never contracts, and every explicit mul_add of the reference is an
explicit fma() in the kernels.  The CUDA runtime is linked statically so the
library has no dependency beyond the driver.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libsoil_cuda.so")
BUILD_DIR = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + \
        [os.path.join(ROOT, "include", "soil_cuda.h")]


def _stale(obj, src):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + headers())


def build(force=False, verbose=False, jobs=8):
    os.makedirs(BUILD_DIR, exist_ok=True)
    objs, procs = [], []
    for src in sources():
        obj = os.path.join(BUILD_DIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                stderr=subprocess.STDOUT)))
            if len(procs) >= jobs:
                _wait(procs, verbose)
                procs = []
    _wait(procs, verbose)
    if force or not os.path.exists(OUT) or \
            any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", OUT] + objs
        subprocess.check_call(cmd)
    return OUT


def _wait(procs, verbose):
    for src, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            sys.stderr.write(text)
            raise RuntimeError(f"nvcc failed on {src}")
        if verbose and text.strip():
            sys.stderr.write(text)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
