"""Build the CPU oracle (test infrastructure) into oracle/libscarl_oracle.so.

The oracle is the parity checker and the CPU baseline; the product never
links it.  Plain gcc, OpenMP, no fused multiply-add contraction so the
restated arithmetic rounds like the reference's scalar code.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libscarl_oracle.so")
SRC = os.path.join(HERE, "scarl_oracle.c")


def build(force: bool = False) -> str:
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(SRC),
                                             os.path.getmtime(os.path.join(HERE, "scarl_oracle.h")))):
        return LIB
    cmd = ["gcc", "-std=gnu11", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           "-Wall", "-Wno-unused-variable", "-o", LIB, SRC, "-lm"]
    subprocess.check_call(cmd, cwd=HERE)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
