"""Build libbh.so (the sm_100a tracer and its C-ABI) in place.

    python black-hole_b200/build.py [--verbose]

CUDA sources are compiled by nvcc for sm_100a only; host C++ by g++ without
FMA contraction (the host-side derivation is float arithmetic that must
match the reference's host build bit for bit).  Objects go to _build/, the
library to black-hole_b200/libbh.so, which the Python front end loads.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libbh.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
HOSTCXX = shutil.which("g++", path="/usr/bin:/bin") or "g++"
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCS = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", *GENCODE, "-Xcompiler", "-fPIC",
           "-Xcompiler", "-ffp-contract=off", "--ptxas-options=-v", *INCS]
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-I" + os.path.join(CUDA, "include"), *INCS]


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    return hs


def _stale(src, obj, newest_header):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or newest_header > t


def _compile(src, verbose):
    obj = os.path.join(OUT, os.path.basename(src) + ".o")
    if src.endswith(".cu"):
        cmd = [NVCC, *NVFLAGS, "-c", src, "-o", obj]
    else:
        cmd = [HOSTCXX, *CXXFLAGS, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(r.stderr, end="")
    return obj


def build(verbose=False, force=False):
    os.makedirs(OUT, exist_ok=True)
    newest = max(os.path.getmtime(h) for h in _headers())
    srcs = [os.path.join(CSRC, f) for f in _sources()]
    objs = [os.path.join(OUT, os.path.basename(s) + ".o") for s in srcs]
    todo = [s for s, o in zip(srcs, objs) if force or _stale(s, o, newest)]
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
        list(ex.map(lambda s: _compile(s, verbose), todo))
    if todo or not os.path.exists(LIB) or force:
        cmd = [NVCC, "-shared", *GENCODE, "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force="--force" in sys.argv))
