"""Build the package's native libraries in-tree (nextgen_b200/lib/).

  libcgx.so          CUDA kernels + C ABI (include/cgx.h, include/cgx_ops.h), sm_100a only
  libcgx_meshgen.so  host mesh/operator generator and .mles reader
                     (include/cgx_meshgen.h, include/cgx_mles.h)

`python -m nextgen_b200.build` rebuilds whatever is out of date.
"""
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
INC = os.path.join(ROOT, "include")

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _cxx():
    # the system g++ (an environment CXX may lack libgomp)
    for c in ("/usr/bin/g++", "g++"):
        if shutil.which(c):
            return c
    raise RuntimeError("no g++ found")


def _nvcc():
    for c in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if shutil.which(c):
            return c
    raise RuntimeError("no nvcc found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build failed: %s" % " ".join(cmd))
    return r.stdout


def build_meshgen(force=False):
    out = os.path.join(LIB, "libcgx_meshgen.so")
    srcs = [os.path.join(CSRC, f) for f in ("meshgen.cpp", "mles.cpp")]
    deps = srcs + [os.path.join(CSRC, "svd33.h"), os.path.join(INC, "cgx_meshgen.h"), os.path.join(INC, "cgx_mles.h")]
    if force or _stale(out, deps):
        os.makedirs(LIB, exist_ok=True)
        _run([_cxx(), "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", out] + srcs)
    return out


def build_cgx(force=False, verbose=False):
    out = os.path.join(LIB, "libcgx.so")
    ops_obj = os.path.join(LIB, "cgx_ops.o")
    srcs = [os.path.join(CSRC, f) for f in ("cgx.cu", "cgx_kernels.cuh", "cgx_mixed.cuh", "cgx_ops.cu", "svd33.h")] + \
        [os.path.join(INC, h) for h in ("cgx.h", "cgx_ops.h", "cgx_meshgen.h")]
    if force or _stale(out, srcs):
        os.makedirs(LIB, exist_ok=True)
        common = [_nvcc(), "-O3", "-std=c++17"] + NVCC_ARCH + ["-lineinfo", "-ccbin", _cxx()]
        if verbose:
            common.insert(1, "-Xptxas=-v")
        # the operator build reproduces the host generator's arithmetic bit
        # for bit, so it is compiled without multiply-add contraction
        log = _run(common + ["-fmad=false", "-Xcompiler", "-fPIC,-fopenmp", "-c", "-o", ops_obj,
                             os.path.join(CSRC, "cgx_ops.cu")])
        log += _run(common + ["-Xcompiler", "-fPIC,-fopenmp", "-shared", "-o", out,
                              os.path.join(CSRC, "cgx.cu"), ops_obj, "-lgomp"])
        os.remove(ops_obj)
        if verbose:
            sys.stdout.write(log)
    return out


def build_all(force=False, verbose=False):
    return [build_meshgen(force), build_cgx(force, verbose)]


if __name__ == "__main__":
    for p in build_all(force="--force" in sys.argv, verbose="-v" in sys.argv):
        print(p)
