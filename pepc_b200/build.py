"""Build libpepcg.so in-tree for sm_100a.

Usage: python -m pepc_b200.build   (or pepc_b200.build.build())

Every .cu under pepc_b200/csrc is compiled with
  nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3
The FP64 translation units that must reproduce the reference's IEEE
arithmetic bit for bit are compiled with --fmad=false (no contraction of
a*b+c into fma); the mixed-precision walk keeps contraction on.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpepcg.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-Xptxas", "-v"] + ARCH
EXACT_FP64 = {"grow.cu", "walk_plain.cu", "direct.cu", "scalar.cu", "lattice.cu", "timeloop.cu"}


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def _flags(name):
    f = list(COMMON)
    if name in EXACT_FP64:
        f += ["--fmad=false"]
    return f


def _stale(src, obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def build(verbose=False, jobs=8):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    deps.append(os.path.join(HERE, "..", "include", "pepcg.h"))
    objs = []
    jobs_list = []
    for s in srcs:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s[:-3] + ".o")
        objs.append(obj)
        if _stale(src, obj, deps):
            jobs_list.append([nvcc()] + _flags(s) + ["-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with ThreadPoolExecutor(max_workers=jobs) as ex:
        for cmd, r in ex.map(run, jobs_list):
            if r.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
                raise RuntimeError("nvcc failed for " + cmd[-3])
            if verbose:
                sys.stdout.write(r.stderr)
            with open(cmd[-1] + ".ptxas.txt", "w") as fh:
                fh.write(r.stderr)
    if jobs_list or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
