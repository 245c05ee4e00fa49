"""Build recipe of libcfdb.so (sm_100a) and the C++ facade example.

Compiles every CUDA source with nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a), the host sources with the system
g++, and links them into cfdarcov2_b200/_lib/libcfdb.so.  Objects are rebuilt
only when a source or header is newer.  Run ``python -m cfdarcov2_b200.build``.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(PKG, "_build", "obj")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libcfdb.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# Sources whose arithmetic must round every operation separately (the FP64
# plain path is compared bit for bit with the CPU oracle).
NO_FMA = {"plain_ops.cu", "euler_plain.cu", "geometry_dev.cu"}


def host_cxx() -> str:
    """The image exports CXX pointing at a compiler without libgomp; prefer the system g++."""
    for cand in (os.environ.get("CFDB_CXX"), "/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("no g++ found")


def _newer(src_deps, target) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_deps)


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.hpp")) + glob.glob(os.path.join(CSRC, "*.cuh"))
            + glob.glob(os.path.join(INCLUDE, "*.h")))


def _compile_cmd(src: str, obj: str):
    name = os.path.basename(src)
    common_inc = ["-I", INCLUDE, "-I", CSRC]
    if name.endswith(".cu"):
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
               "--expt-relaxed-constexpr", "-ccbin", host_cxx(), *common_inc, "-c", src, "-o", obj]
        if name in NO_FMA:
            cmd[3:3] = ["--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
        return cmd
    return [host_cxx(), "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-Wall",
            "-I", os.path.join(CUDA_HOME, "include"), *common_inc, "-c", src, "-o", obj]


FACADE_LIB = os.path.join(LIBDIR, "libcfdb_fvm.so")
EXAMPLE_BIN = os.path.join(LIBDIR, "fvm_example")


def build_facade(verbose: bool = False) -> str:
    """The drop-in C++ facade (include/cfdb/) over the C ABI, and its example."""
    srcs = sorted(glob.glob(os.path.join(CSRC, "facade", "*.cpp")))
    hdrs = glob.glob(os.path.join(INCLUDE, "cfdb", "*.hpp")) + [os.path.join(INCLUDE, "cfdb.h")]
    cxx = host_cxx()
    if _newer(srcs + hdrs + [LIB], FACADE_LIB):
        cmd = [cxx, "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-I", INCLUDE, *srcs, "-o", FACADE_LIB,
               "-L", LIBDIR, "-lcfdb", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    ex = os.path.join(PKG, "examples", "fvm_example.cpp")
    if _newer([ex, FACADE_LIB] + hdrs, EXAMPLE_BIN):
        cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-I", INCLUDE, ex, "-o", EXAMPLE_BIN, "-L", LIBDIR, "-lcfdb_fvm",
               "-lcfdb", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return FACADE_LIB


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    headers = _headers()
    todo, objs = [], []
    for s in sources:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if _newer([s, *headers, __file__], o):
            todo.append((s, o))

    def run(pair):
        cmd = _compile_cmd(*pair)
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {pair[0]}\n{r.stdout}\n{r.stderr}")
        return pair[0]

    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        for _ in ex.map(run, todo):
            pass
    if todo or _newer(objs, LIB):
        # NVRTC for the run-time compiled equation kernels (jit.cpp), found via rpath
        cudalib = os.path.join(CUDA_HOME, "lib64")
        cmd = [NVCC, *ARCH, "-shared", "-ccbin", host_cxx(), "-o", LIB, *objs, "-Xcompiler", "-fopenmp", "-lgomp",
               "-L", cudalib, "-lnvrtc", "-Xlinker", f"-rpath,{cudalib}"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    build_facade(verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
