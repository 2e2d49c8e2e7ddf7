"""Builds libcqfock.so (the C-ABI library with the sm_100a kernels) in-tree.

    python -m chronusq_public_b200.build

Each .cu file under csrc/ is compiled separately (in parallel) with
``-gencode arch=compute_100a,code=sm_100a`` and linked into
chronusq_public_b200/_lib/libcqfock.so.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libcqfock.so")
PEAK_SRC = os.path.join(HERE, "peaks", "fma_peak.cu")
PEAK_LIB = os.path.join(OUT_DIR, "libcqf_peaks.so")
OBJ_DIR = os.path.join(ROOT, "_build", "obj")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
                "-Xcompiler", "-O3", "--expt-relaxed-constexpr",
                "-ccbin", "/usr/bin/g++"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(CSRC, "gen", "*.cuh")) +
                  glob.glob(os.path.join(CSRC, "*.hpp")) +
                  glob.glob(os.path.join(ROOT, "include", "*.h")))


def _compile(src, verbose):
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    newest_dep = max([os.path.getmtime(src)] +
                     [os.path.getmtime(d) for d in _deps()])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj
    cmd = [NVCC] + FLAGS + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return obj


def generate(verbose: bool = False):
    """Runs the kernel generators (csrc/gen_*.py -> csrc/gen/*.cuh)."""
    for gen in sorted(glob.glob(os.path.join(CSRC, "gen_*.py"))):
        out = os.path.join(CSRC, "gen", "cqf_" + os.path.basename(gen)[:-3] + ".cuh")
        if (not os.path.exists(out)
                or os.path.getmtime(out) < os.path.getmtime(gen)):
            if verbose:
                print("generate", out, flush=True)
            subprocess.check_call([sys.executable, gen, out])


def build(verbose: bool = False) -> str:
    generate(verbose)
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
            os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-ccbin", "/usr/bin/g++",
                               "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    if not os.path.exists(PEAK_LIB) or os.path.getmtime(PEAK_LIB) < os.path.getmtime(PEAK_SRC):
        cmd = [NVCC] + FLAGS + ["-shared", "-cudart", "static", PEAK_SRC, "-o", PEAK_LIB]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
