"""Build recipe for the CPU oracle (test infrastructure only).

``gcc -O2 -fopenmp -shared`` of ``oracle/metcf_oracle.c`` into
``oracle/_build/libmetcf_oracle.so``. Only tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg load it.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "metcf_oracle.c")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libmetcf_oracle.so")


def build(force=False):
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) > os.path.getmtime(SRC)):
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["gcc", "-O2", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared",
           "-std=c11", "-Wall", SRC, "-o", LIB, "-lm"]
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
