"""Build recipe for the in-tree shared library ``libalenka_b200.so``.

CUDA sources are compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``),
host sources with g++; the CUDA runtime is linked statically so the library does not
depend on which libcudart a host process already loaded.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libalenka_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SRCS = ["csrc/kernels.cu", "csrc/pipeline.cu", "csrc/card.cu", "csrc/batch.cu", "csrc/gen.cu",
            "csrc/encode.cu", "csrc/strings.cu", "csrc/frontend_state.cu", "csrc/load.cu",
            "csrc/star.cu"]
CPP_SRCS = ["host/format.cpp", "host/script.cpp", "host/engine.cpp", "host/engine_ops.cpp",
            "host/capi.cpp", "host/gen.cpp", "host/card.cpp", "host/resident.cpp", "host/frontend_abi.cpp",
            "host/frontend_embed.cpp", "host/star.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    return r.stdout


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(ROOT, "include", "alenka_b200.h")]
    for d in ("csrc", "host"):
        for f in os.listdir(os.path.join(HERE, d)):
            if f.endswith((".h", ".cuh")):
                headers.append(os.path.join(HERE, d, f))
    objs = []
    for src in CU_SRCS:
        s = os.path.join(HERE, src)
        if not os.path.exists(s):
            continue
        o = os.path.join(BUILD, os.path.basename(src) + ".o")
        if _stale(o, [s] + headers):
            _run([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                  "-I" + os.path.join(ROOT, "include"), "-c", s, "-o", o])
        objs.append(o)
    for src in CPP_SRCS:
        s = os.path.join(HERE, src)
        o = os.path.join(BUILD, os.path.basename(src) + ".o")
        if _stale(o, [s] + headers):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function",
                  "-I" + os.path.join(CUDA, "include"), "-I" + os.path.join(ROOT, "include"),
                  "-c", s, "-o", o])
        objs.append(o)
    if _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs,
              "-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"])
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
