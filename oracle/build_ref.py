"""Build recipe for the UNMODIFIED reference extension (test infrastructure).

Compiles the reference's two translation units, where they lie in the
reference checkout (its DTC-SpMM/ folder; the checkout's root is taken from the
DTC_REFERENCE_ROOT environment variable, default /root/reference), into
``oracle/_ref/DTCSpMM*.so`` for sm_100a. Nothing is
copied out of the reference tree; the only addition is the sputnik stub header
under ``oracle/sputnik_stub`` (sputnik is an un-vendored submodule of the
reference; only its competitor-baseline entry point needs it).

The product never loads this library. It is used only

* by ``tests/golden/make_golden.py`` to produce golden ME-TCF vectors from the
  reference's own ``preprocess`` (CPU) and ``preprocess_gpu`` (GPU) entry points,
* by ``-m gpu`` tests, when present, as a second bit-exactness check,
* by ``bench.py --impl reference`` to time the reference's own conversion and
  kernels rebuilt for sm_100a.

Usage: ``python oracle/build_ref.py`` (no-op when the reference tree is absent,
e.g. on a GPU box that received the prebuilt ``oracle/_ref``).
"""
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("DTC_REFERENCE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "DTC-SpMM")
OUT = os.path.join(HERE, "_ref")
EXT_SUFFIX = sysconfig.get_config_var("EXT_SUFFIX")
TARGET = os.path.join(OUT, "DTCSpMM" + EXT_SUFFIX)


def _torch_paths():
    import torch
    tdir = os.path.dirname(torch.__file__)
    inc = [os.path.join(tdir, "include"),
           os.path.join(tdir, "include", "torch", "csrc", "api", "include")]
    lib = os.path.join(tdir, "lib")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    return inc, lib, abi


def build(force=False):
    if not os.path.isdir(REF_SRC):
        return None
    srcs = [os.path.join(REF_SRC, "DTCSpMM.cpp"),
            os.path.join(REF_SRC, "DTCSpMM_kernel.cu")]
    if (not force and os.path.exists(TARGET)
            and all(os.path.getmtime(TARGET) > os.path.getmtime(s) for s in srcs)):
        return TARGET
    os.makedirs(OUT, exist_ok=True)
    inc, lib, abi = _torch_paths()
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    pyinc = sysconfig.get_paths()["include"]
    defs = ["-DTORCH_EXTENSION_NAME=DTCSpMM", "-DTORCH_API_INCLUDE_EXTENSION_H",
            f"-D_GLIBCXX_USE_CXX11_ABI={abi}"]
    incs = [f"-I{p}" for p in inc + [pyinc, os.path.join(cuda, "include"),
                                      os.path.join(HERE, "sputnik_stub"), REF_SRC]]
    obj_cpp = os.path.join(OUT, "DTCSpMM.o")
    obj_cu = os.path.join(OUT, "DTCSpMM_kernel.o")
    cmds = [
        ["g++", "-c", srcs[0], "-o", obj_cpp, "-O2", "-fPIC", "-std=c++17", "-fopenmp", "-w"]
        + defs + incs,
        [os.path.join(cuda, "bin", "nvcc"), "-c", srcs[1], "-o", obj_cu, "-O3",
         "-std=c++17", "-Xcompiler", "-fPIC", "-w",
         "-gencode", "arch=compute_100a,code=sm_100a",
         "--expt-relaxed-constexpr", "-D__CUDA_NO_HALF_OPERATORS__",
         "-D__CUDA_NO_HALF_CONVERSIONS__", "-D__CUDA_NO_BFLOAT16_CONVERSIONS__",
         "-D__CUDA_NO_HALF2_OPERATORS__"] + defs + incs,
        ["g++", "-shared", obj_cpp, obj_cu, "-o", TARGET, "-fopenmp",
         f"-L{lib}", f"-Wl,-rpath,{lib}", "-lc10", "-ltorch", "-ltorch_cpu",
         "-ltorch_python", "-lc10_cuda", "-ltorch_cuda",
         f"-L{os.path.join(cuda, 'lib64')}", "-lcudart", "-lcusparse"],
    ]
    for c in cmds:
        print(" ".join(c), flush=True)
        subprocess.check_call(c)
    for o in (obj_cpp, obj_cu):
        os.remove(o)
    return TARGET


if __name__ == "__main__":
    t = build(force="--force" in sys.argv)
    print(t if t else "reference tree absent; nothing built")
