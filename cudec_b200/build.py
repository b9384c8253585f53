"""Build recipe for the in-tree native libraries.

    libcudec_b200.so      the decode library: C ABI (include/cudec.h) over
                          hand-written sm_100a kernels; CUDA runtime linked
                          statically so the .so carries no runtime-version
                          dependency
    libcudec_workload.so  host-only synthetic-content generator for the
                          benchmark and tests (not part of the decode ABI)

Run `python -m cudec_b200.build` (or __graft_entry__.build()). Objects go to
cudec_b200/_build/; the .so files land next to this file so the package finds
them and they travel with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
INC = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libcudec_b200.so")
WORKLOAD = os.path.join(HERE, "libcudec_workload.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-I" + INC, "-I" + CSRC, "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-I" + INC, "-I" + CSRC,
             "-I/usr/local/cuda/include", "-Wall", "-Wextra"]
CC_FLAGS = ["-O2", "-std=c11", "-fPIC", "-I" + INC, "-Wall", "-Wextra"]

LIB_SOURCES = ["batch.cu", "zstd.cu", "mixed.cu", "gdeflate.cu", "serve.cpp", "frame.cpp", "stream.cpp", "host_util.cpp", "version.c"]


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)
            if f.endswith((".cuh", ".h"))] + [os.path.join(INC, "cudec.h")]


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose=False, extra_nvcc=()):
    os.makedirs(OBJ, exist_ok=True)
    hdrs = _headers()
    objs = []
    for src in LIB_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if not _stale(obj, [path] + hdrs + [__file__]):
            continue
        if src.endswith(".cu"):
            cmd = [NVCC] + NVCC_FLAGS + list(extra_nvcc) + ["-c", path, "-o", obj]
        elif src.endswith(".cpp"):
            cmd = ["g++"] + CXX_FLAGS + ["-c", path, "-o", obj]
        else:
            cmd = ["gcc"] + CC_FLAGS + ["-c", path, "-o", obj]
        _run(cmd, verbose)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs +
             ["-lpthread", "-ldl", "-lrt"], verbose)
    wsrc = [os.path.join(CSRC, "workload.c"), os.path.join(CSRC, "gdeflate_enc.c")]
    if _stale(WORKLOAD, wsrc):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-pthread", "-o",
              WORKLOAD] + wsrc + ["-lm"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra_nvcc=sys.argv[1:])
