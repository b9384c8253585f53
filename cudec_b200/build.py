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

`python -m cudec_b200.build install --prefix P` installs the decode library
for other builds to link: P/lib/libcudec_b200.so, P/include/cudec.h, a CMake
package config (find_package(cudec) gives the imported target cudec::cudec,
the name the reference's own package exports) and P/lib/pkgconfig/cudec.pc.
Both configs locate the prefix from their own position, so the tree can be
moved after installation.
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
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-Xlinker",
                              "-soname=" + os.path.basename(LIB), "-o", LIB] + objs +
             ["-lpthread", "-ldl", "-lrt"], verbose)
    wsrc = [os.path.join(CSRC, "workload.c"), os.path.join(CSRC, "gdeflate_enc.c")]
    if _stale(WORKLOAD, wsrc):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-pthread", "-o",
              WORKLOAD] + wsrc + ["-lm"], verbose)
    return LIB


def version():
    """(major, minor, patch) from the CUDEC_VERSION_* macros of cudec.h."""
    import re
    text = open(os.path.join(INC, "cudec.h")).read()
    return tuple(int(re.search(r"#define CUDEC_VERSION_%s (\d+)" % k, text).group(1))
                 for k in ("MAJOR", "MINOR", "PATCH"))


# find_package(cudec): the imported target over this prefix's library and
# header. The CUDA runtime is inside the library (linked statically), so the
# consumer needs no CUDA toolkit.
_CMAKE_CONFIG = """\
# cudec package config: the imported target cudec::cudec (libcudec_b200.so and
# cudec.h of this prefix, found from this file's own position).
get_filename_component(_cudec_prefix "${CMAKE_CURRENT_LIST_DIR}/../../.." ABSOLUTE)
if(NOT TARGET cudec::cudec)
  add_library(cudec::cudec SHARED IMPORTED)
  set_target_properties(cudec::cudec PROPERTIES
    IMPORTED_LOCATION "${_cudec_prefix}/lib/libcudec_b200.so"
    IMPORTED_SONAME "libcudec_b200.so"
    INTERFACE_INCLUDE_DIRECTORIES "${_cudec_prefix}/include")
endif()
unset(_cudec_prefix)
"""

# Version policy: at 0.x a minor release may break the ABI, so a request is
# met only by the same major.minor at a patch level at or above it (CMake's
# SameMinorVersion rule; a version range is met by its lower end's rule).
_CMAKE_VERSION = """\
set(PACKAGE_VERSION "@V@")
if(PACKAGE_FIND_VERSION_RANGE)
  set(_cudec_want "${PACKAGE_FIND_VERSION_MIN}")
else()
  set(_cudec_want "${PACKAGE_FIND_VERSION}")
endif()
if(NOT _cudec_want)
  set(PACKAGE_VERSION_COMPATIBLE TRUE)
else()
  string(REGEX MATCH "^[0-9]+\\.[0-9]+" _cudec_want_mm "${_cudec_want}.0")
  if(_cudec_want_mm STREQUAL "@MM@" AND NOT _cudec_want VERSION_GREATER PACKAGE_VERSION)
    set(PACKAGE_VERSION_COMPATIBLE TRUE)
    if(_cudec_want VERSION_EQUAL PACKAGE_VERSION)
      set(PACKAGE_VERSION_EXACT TRUE)
    endif()
  else()
    set(PACKAGE_VERSION_COMPATIBLE FALSE)
  endif()
endif()
unset(_cudec_want)
unset(_cudec_want_mm)
"""

_PKGCONFIG = """\
prefix=${pcfiledir}/../..
libdir=${prefix}/lib
includedir=${prefix}/include

Name: cudec
Description: batch LZ4, Snappy, Zstd and GDeflate decode on B200 behind the cudec C ABI
Version: @V@
Libs: -L${libdir} -lcudec_b200
Cflags: -I${includedir}
"""


def install(prefix, verbose=False):
    """Build if needed, then install the library, header and package
    configs under `prefix`."""
    import shutil
    build(verbose=verbose)
    ver = "%d.%d.%d" % version()
    mm = ".".join(ver.split(".")[:2])
    lib_dir = os.path.join(prefix, "lib")
    cmake_dir = os.path.join(lib_dir, "cmake", "cudec")
    pc_dir = os.path.join(lib_dir, "pkgconfig")
    inc_dir = os.path.join(prefix, "include")
    for d in (cmake_dir, pc_dir, inc_dir):
        os.makedirs(d, exist_ok=True)
    shutil.copy2(LIB, os.path.join(lib_dir, os.path.basename(LIB)))
    shutil.copy2(os.path.join(INC, "cudec.h"), os.path.join(inc_dir, "cudec.h"))
    with open(os.path.join(cmake_dir, "cudec-config.cmake"), "w") as f:
        f.write(_CMAKE_CONFIG)
    with open(os.path.join(cmake_dir, "cudec-config-version.cmake"), "w") as f:
        f.write(_CMAKE_VERSION.replace("@V@", ver).replace("@MM@", mm))
    with open(os.path.join(pc_dir, "cudec.pc"), "w") as f:
        f.write(_PKGCONFIG.replace("@V@", ver))
    if verbose:
        print("installed cudec %s under %s" % (ver, prefix))
    return prefix


if __name__ == "__main__":
    if sys.argv[1:2] == ["install"]:
        import argparse
        ap = argparse.ArgumentParser(prog="python -m cudec_b200.build install")
        ap.add_argument("--prefix", required=True)
        install(os.path.abspath(ap.parse_args(sys.argv[2:]).prefix), verbose=True)
    else:
        build(verbose=True, extra_nvcc=sys.argv[1:])
