"""In-tree build of the B200-native DTC-SpMM path (sm_100a only).

Produces, inside this directory:
  lib/libdtcspmm.so          CUDA kernels + C ABI (include/dtc_spmm.h)
  lib/libdtcgen.so           seeded synthetic matrix generators (host C++)
  DTCSpMM<ext-suffix>.so     PyTorch extension mirroring the reference API

Usage: python dtc-spmm_asplos24_b200/build.py [--force]
"""
import concurrent.futures as cf
import os
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
EXT_SUFFIX = sysconfig.get_config_var("EXT_SUFFIX")

CU_SOURCES = ["abi.cu", "convert.cu", "spmm_tc.cu", "spmm_split.cu", "spmm_mma.cu", "formats.cu",
              "noalloc.cu", "tune.cu",
              "relabel.cu", "tca.cu", "features.cu", "mlp.cu"]
GEN_SOURCES = ["gen.cpp"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", f"-I{INC}", f"-I{CSRC}"]

LIBDTC = os.path.join(LIB, "libdtcspmm.so")
LIBGEN = os.path.join(LIB, "libdtcgen.so")
EXT = os.path.join(PKG, "DTCSpMM" + EXT_SUFFIX)


def _headers():
    hs = [os.path.join(INC, f) for f in os.listdir(INC) if f.endswith(".h")]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _compile_cu(src, force):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if force or _stale(obj, [src] + _headers()):
        _run([NVCC, "-c", src, "-o", obj] + NVCC_FLAGS)
    return obj


def build_libdtc(force=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile_cu(s, force), srcs))
    if force or _stale(LIBDTC, objs):
        _run([NVCC, "-shared", "-o", LIBDTC] + objs +
             ["-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "shared"])
    return LIBDTC


def build_libgen(force=False):
    os.makedirs(LIB, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in GEN_SOURCES]
    if force or _stale(LIBGEN, srcs):
        _run(["g++", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", "-std=c++17"] +
             srcs + ["-o", LIBGEN])
    return LIBGEN


def build_ext(force=False):
    import torch
    tdir = os.path.dirname(torch.__file__)
    src = os.path.join(CSRC, "ext.cpp")
    if not (force or _stale(EXT, [src, LIBDTC] + _headers())):
        return EXT
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    pyinc = sysconfig.get_paths()["include"]
    tlib = os.path.join(tdir, "lib")
    cmd = ["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-w", src, "-o", EXT,
           "-DTORCH_EXTENSION_NAME=DTCSpMM", "-DTORCH_API_INCLUDE_EXTENSION_H",
           f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           f"-I{os.path.join(tdir, 'include')}",
           f"-I{os.path.join(tdir, 'include', 'torch', 'csrc', 'api', 'include')}",
           f"-I{pyinc}", f"-I{os.path.join(CUDA, 'include')}", f"-I{INC}",
           f"-L{tlib}", f"-Wl,-rpath,{tlib}", "-lc10", "-ltorch", "-ltorch_cpu",
           "-ltorch_python", "-lc10_cuda", "-ltorch_cuda",
           f"-L{LIB}", "-Wl,-rpath,$ORIGIN/lib", "-ldtcspmm",
           f"-L{os.path.join(CUDA, 'lib64')}", "-lcudart"]
    _run(cmd)
    return EXT


def build(force=False, ext=True):
    out = [build_libdtc(force), build_libgen(force)]
    if ext:
        out.append(build_ext(force))
    return out


if __name__ == "__main__":
    for p in build(force="--force" in sys.argv, ext="--no-ext" not in sys.argv):
        print(p)
