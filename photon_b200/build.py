"""Builds photon_b200/libphoton_wavefront.so (the C ABI of include/photon_wavefront.h) in-tree.

Device code: nvcc for sm_100a only, with -fmad=false and IEEE division / square root so that the
integrator's arithmetic rounds like the host reference (see csrc/pt_math.cuh). Host code: g++
-std=c++20 -O3 for baseline x86-64 (no FMA contraction either). Incremental: an object is rebuilt
when its source or any header in csrc/ or include/ is newer.

    python -m photon_b200.build [--force] [-j N]
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libphoton_wavefront.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", *GENCODE]
CXX_FLAGS = ["-std=c++20", "-O3", "-fPIC", "-pthread", "-Wall", "-Wno-missing-field-initializers"]


def _headers():
    hs = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                hs.append(os.path.join(d, f))
    return hs


def _stale(obj, src, headers):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or any(os.path.getmtime(h) > t for h in headers)


def _compile(src, obj):
    inc = ["-I", INCLUDE, "-I", CSRC]
    if src.endswith(".cu"):
        cmd = [NVCC, *NVCC_FLAGS, *inc, "-c", src, "-o", obj]
    else:
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, *CXX_FLAGS, *inc, "-I", os.path.join(CUDA_HOME, "include"), "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force=False, jobs=None, verbose=False):
    """Compiles every source in csrc/ and links the shared library; returns its path."""
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))
    objs, todo = [], []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(o, s, headers):
            todo.append((s, o))
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for o in ex.map(lambda so: _compile(*so), todo):
            if verbose:
                print("built", os.path.relpath(o, ROOT))
    if todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, "-shared", *GENCODE, "-o", LIB, *objs, "-cudart", "static", "-Xcompiler", "-pthread", "-lz"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    a = ap.parse_args()
    try:
        print(build(a.force, a.j, verbose=True))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
