"""Builds the racon_b200 native library and CLI in-tree for sm_100a.

Outputs (git-ignored, shipped with the working tree):
  racon_b200/lib/libracon_b200.so   CUDA kernels + C ABI + racon C++ API
  racon_b200/bin/racon_b200         command-line front end
Objects go to racon_b200/_build/. Rebuilds only what changed.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libracon_b200.so")
BIN = os.path.join(HERE, "bin", "racon_b200")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                   "-Wno-deprecated-gpu-targets"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-pthread",
             "-I/usr/local/cuda/include"]

CU_SOURCES = ["nw_align.cu", "poa_consensus.cu", "layers.cu"]
CXX_SOURCES = ["rb_capi.cpp", "ring_service.cpp", "host/polisher.cpp", "host/server.cpp"]
HEADERS = ["rb_internal.hpp", "ring_queue.cuh", "host/racon.hpp", os.path.join("..", "..", "include", "racon_b200.h")]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r.stdout


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace("/", "_") + ".o")
        if _newer(o, [s] + headers):
            out = _run([NVCC] + CU_FLAGS + ["-c", s, "-o", o])
            if verbose and out:
                print(out)
        objs.append(o)
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace("/", "_") + ".o")
        if _newer(o, [s] + headers):
            _run(["g++"] + CXX_FLAGS + ["-c", s, "-o", o])
        objs.append(o)
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs +
             ["-lz", "-cudart", "static", "-Xlinker", "-rpath,$ORIGIN"])
    main_src = os.path.join(CSRC, "host", "main.cpp")
    if _newer(BIN, [main_src, LIB] + headers):
        _run(["g++"] + CXX_FLAGS + [main_src, "-o", BIN, "-L" + os.path.dirname(LIB), "-lracon_b200",
              "-Wl,-rpath,$ORIGIN/../lib", "-lz"])
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
