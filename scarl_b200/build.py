"""Build libscarl_b200.so in-tree: every CUDA source for sm_100a with nvcc,
the host sources with the same compiler driver, static CUDA runtime.

Run `python scarl_b200/build.py [--force]` (a plain script: importing the
package would load the library it builds).
"""
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libscarl_b200.so")
OBJ = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

CUDA_SOURCES = ["gen_padded.cu", "gen_f32.cu", "gen_f64.cu", "dct_literal.cu", "post.cu", "stats.cu",
                "noalloc.cu"]
HOST_SOURCES = ["api.cpp", "host_maps.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-I", CSRC, "-I", INCLUDE]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _digest():
    h = hashlib.sha256()
    for d in (CSRC, INCLUDE):
        for f in sorted(os.listdir(d)):
            p = os.path.join(d, f)
            if os.path.isfile(p):
                h.update(f.encode())
                with open(p, "rb") as fh:
                    h.update(fh.read())
    h.update(" ".join(ARCH + COMMON).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> str:
    stamp = os.path.join(OBJ, "stamp")
    dig = _digest()
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as fh:
            if fh.read().strip() == dig:
                return LIB
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    objs = []
    procs = []
    for src in CUDA_SOURCES + HOST_SOURCES:
        obj = os.path.join(OBJ, src + ".o")
        cmd = [nvcc] + COMMON + ["-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu"):
            cmd[1:1] = ARCH + ["-lineinfo"]
        else:
            cmd[1:1] = ["-x", "cu"] + ARCH
        if verbose:
            print(" ".join(cmd))
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    rcs = [p.wait() for p in procs]
    if any(rcs):
        raise RuntimeError("nvcc failed for " + ", ".join(
            s for s, r in zip(CUDA_SOURCES + HOST_SOURCES, rcs) if r))
    link = [nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
    subprocess.check_call(link)
    with open(stamp, "w") as fh:
        fh.write(dig)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
