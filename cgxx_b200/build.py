"""Builds the native parts of cgxx_b200 in-tree.

  libcgb200.so   CUDA kernels (sm_100a) + C ABI (include/cgx.h) + MatrixMarket
                 I/O, compiled with nvcc for `-gencode arch=compute_100a,
                 code=sm_100a` only.
  cg_b200        the `<binary> <matrix.mtx> [<repetitions>]` executable: the
                 C++ CG class (host/) over libcgb200.so.

Usage: python -m cgxx_b200.build [--force]
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libcgb200.so")
EXE = os.path.join(HERE, "cg_b200")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
              "--expt-relaxed-constexpr"]
CU_SOURCES = ["csrc/api.cu", "csrc/noalloc.cu"]
CPP_SOURCES = ["csrc/mtx_io.cpp"]
HOST_SOURCES = ["host/CG.cpp", "host/Matrix.cpp", "host/CGB200.cpp"]


def _host_cxx():
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("no g++ found")


def _nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("no nvcc found")


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _deps(patterns):
    out = []
    for d, exts in patterns:
        full = os.path.join(HERE, d)
        for f in sorted(os.listdir(full)):
            if f.endswith(exts):
                out.append(os.path.join(full, f))
    return out


def _run(cmd):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, cwd=HERE, check=True)


def build(force=False):
    nvcc = _nvcc()
    cxx = _host_cxx()
    inc = ["-I" + os.path.join(REPO, "include"), "-I" + os.path.join(HERE, "csrc")]
    lib_deps = _deps([("csrc", (".cu", ".cuh", ".cpp", ".h"))]) + \
        [os.path.join(REPO, "include", "cgx.h")]
    if force or _stale(LIB, lib_deps):
        objs = []
        os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
        for src in CU_SOURCES:
            obj = os.path.join(HERE, "_build", os.path.basename(src) + ".o")
            _run([nvcc, *ARCH, *NVCC_FLAGS, *inc, "-ccbin", cxx, "-c", src, "-o", obj])
            objs.append(obj)
        for src in CPP_SOURCES:
            obj = os.path.join(HERE, "_build", os.path.basename(src) + ".o")
            _run([cxx, "-O3", "-std=c++17", "-fPIC", "-Wall", *inc, "-c", src, "-o", obj])
            objs.append(obj)
        tmp = LIB + ".tmp"
        _run([nvcc, *ARCH, "-shared", "-ccbin", cxx, "-o", tmp, *objs, "-lpthread"])
        os.replace(tmp, LIB)
    host_srcs = [os.path.join(HERE, s) for s in HOST_SOURCES]
    host_deps = _deps([("host", (".cpp", ".h"))]) + [LIB]
    if all(os.path.exists(s) for s in host_srcs) and (force or _stale(EXE, host_deps)):
        _run([cxx, "-O3", "-std=c++17", "-Wall", *inc, "-I" + os.path.join(HERE, "host"),
              "-o", EXE, *host_srcs, "-L" + HERE, "-lcgb200",
              "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
