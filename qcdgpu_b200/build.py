"""Builds the native parts in-tree with nvcc / g++ (no JIT, no setuptools):

  qcdgpu_b200/lib/libqg_sun.so   CUDA kernels + C-ABI (include/qcdgpu_b200.h)
  qcdgpu_b200/bin/qcdgpu         C++ host driver (init.dat run setup + output)

Every CUDA object is compiled for sm_100a only.  Objects are rebuilt when a
source or header is newer; translation units compile in parallel.
"""
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "lib")
BIN = os.path.join(PKG, "bin")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: every fused multiply-add in the kernels is an explicit fma()
# in a fixed order, so results do not depend on the compiler's contraction
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC", "-I" + INCLUDE]
CUDA_SOURCES = ["qg_update_f32.cu", "qg_update_f64.cu", "qg_fields.cu", "qg_ranlux.cu", "qg_capi.cu",
                "qg_noalloc.cu", "qg_batch.cu",
                "qg_learned.cu"]
LIB_HOST_SOURCES = ["qg_host.cpp", "qg_state.cpp", "qg_results.cpp"]          # C++ host code linked into the library
CLI_SOURCES = ["qcdgpu_main.cpp"]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def cuda_home():
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc())))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def build(verbose=False, ptxas_info=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    hdrs = _headers()
    jobs = []
    objs = []
    for src in CUDA_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs) or ptxas_info:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([nvcc()] + NVCC_FLAGS + extra + ["-c", s, "-o", o])
    for src in LIB_HOST_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", "-I" + INCLUDE, "-c", s, "-o", o])
    logs = []
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            logs = list(ex.map(lambda c: _run(c, verbose), jobs))
    lib = os.path.join(LIB, "libqg_sun.so")
    if _stale(lib, objs):
        _run([nvcc()] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"], verbose)
    cli = [os.path.join(CSRC, s) for s in CLI_SOURCES]
    exe = os.path.join(BIN, "qcdgpu")
    if _stale(exe, cli + hdrs + [lib]):
        _run(["g++", "-O2", "-std=c++17", "-I" + INCLUDE, "-o", exe] + cli +
             ["-L" + LIB, "-lqg_sun", "-Wl,-rpath,$ORIGIN/../lib", "-lm"], verbose)
    return "\n".join(logs)


if __name__ == "__main__":
    out = build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    if "--ptxas" in sys.argv:
        print(out)
