"""Build recipe for libwukong_b200.so (CUDA for sm_100a + C++ host) and the oracle.

Compiles in-tree so the shared objects travel with the repository snapshot:
  wukong-cube_b200/libwukong_b200.so   the product: kernels + C ABI (include/wukong_b200.h)
  wukong-cube_b200/libwk_synth.so      the synthetic-graph generator alone (wk_synth.cpp), for
                                       callers that need the workload without the product
                                       (the bench's CPU reference arm)
  oracle/liboracle.so                  the CPU checker (test infrastructure only)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwukong_b200.so")
ORACLE_DIR = os.path.join(ROOT, "oracle")

NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["wk_kernels.cu", "wk_explore.cu", "wk_batch.cu", "wk_serve.cu", "wk_noalloc.cu", "wk_flat.cu",
              "wk_final.cu", "wk_versatile.cu", "wk_gbuild.cu"]
CPP_SOURCES = ["wk_ctx.cpp", "wk_gstore.cpp", "wk_synth.cpp", "wk_tune.cpp", "wk_loader.cpp"]
HEADERS = ["wk_format.h", "wk_internal.h", "wk_kernels.h", "wk_ctx.h", "wk_batch.h",
           "wk_device.cuh", "wk_explore.h", "wk_flat.h", "wk_versatile.h"]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout)
        raise RuntimeError("build step failed: " + cmd[0])
    return r.stdout


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def build_lib(verbose=False, force=False, variant=None, defines=()):
    """Build the library; `variant` names an extra build (objects in _build/<variant>, library
    libwukong_b200_<variant>.so) compiled with the given -D defines."""
    obj = os.path.join(OBJ, variant) if variant else OBJ
    lib = os.path.join(HERE, "libwukong_b200_%s.so" % variant) if variant else LIB
    dflags = ["-D" + d for d in defines]
    os.makedirs(obj, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "wukong_b200.h")]
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(obj, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            out = _run([NVCC] + ARCH + dflags + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                                                 "-Xcompiler", "-fopenmp", "-Xptxas", "-v", "-c", s, "-o", o])
            if verbose:
                print(out)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(obj, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            _run([CXX] + dflags + ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall",
                                   "-Wno-unused-function", "-I" + os.path.join(CUDA_HOME, "include"),
                                   "-c", s, "-o", o])
    if force or _stale(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"])
    return lib


SYNTH_LIB = os.path.join(HERE, "libwk_synth.so")


def build_synth(force=False):
    """The generator on its own: the same wk_synth.cpp the product links, as a small library."""
    src = os.path.join(CSRC, "wk_synth.cpp")
    deps = [src] + [os.path.join(CSRC, h) for h in ("wk_format.h", "wk_internal.h")] + \
        [os.path.join(ROOT, "include", "wukong_b200.h")]
    if force or _stale(SYNTH_LIB, deps):
        _run([CXX, "-O3", "-std=c++17", "-fPIC", "-shared", "-Wall", "-o", SYNTH_LIB, src])
    return SYNTH_LIB


REFERENCE_TREE = "/root/reference"


def build_oracle():
    """The oracle, and where the reference tree is present the reference's own engine
    (oracle/_ref/libwkref.so, the oracle's checker); elsewhere a copy built before travels."""
    _run(["make", "-s", "-C", ORACLE_DIR])
    if os.path.isdir(os.path.join(REFERENCE_TREE, "src")):
        _run(["make", "-s", "-C", ORACLE_DIR, "ref", "REF=" + REFERENCE_TREE])
    return os.path.join(ORACLE_DIR, "liboracle.so")


if __name__ == "__main__":
    print(build_lib(verbose="-v" in sys.argv, force="-f" in sys.argv))
    print(build_synth(force="-f" in sys.argv))
    print(build_oracle())
