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

CUDA_SOURCES = ["gen_padded.cu", "gen_tc.cu", "c2r_tc.cu", "dct_literal.cu", "post.cu", "stats.cu", "cov.cu",
                "mlp.cu", "noalloc.cu"]
# gen_inst.cu once per (precision, line-length group): the generator pass
# instantiations compile in parallel
# (0: power-of-two lengths 4..128, -1 / -2: mixed lengths 24..112 / 160..224)
INSTANCES = [(dt, n) for dt in (4, 8)
             for n in (0, -1, -2, 256, 320, 384, 448, 512, 640, 768, 896, 1024, 1280, 1536, 1792,
                       2048)]
HOST_SOURCES = ["api.cpp", "host_maps.cpp", "h5io.cpp"]
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
    hdr = hashlib.sha256()
    for d in (CSRC, INCLUDE):
        for f in sorted(os.listdir(d)):
            if f.endswith((".h", ".cuh", ".hpp")):
                with open(os.path.join(d, f), "rb") as fh:
                    hdr.update(f.encode() + fh.read())

    def job_digest(cmd, src):
        # an object is rebuilt when its command, its source or any header changes
        h = hashlib.sha256(hdr.digest())
        h.update(" ".join(cmd).encode())
        with open(src, "rb") as fh:
            h.update(fh.read())
        return h.hexdigest()

    jobs = []  # (label, command, object)
    for dt, n in INSTANCES:
        obj = os.path.join(OBJ, f"gen_inst_{dt}_{n}.o")
        jobs.append((f"gen_inst.cu[{dt},{n}]", [nvcc] + ARCH + ["-lineinfo"] + COMMON + [
            f"-DSCARL_INST_DT={dt}", f"-DSCARL_INST_N={n}", "-c", os.path.join(CSRC, "gen_inst.cu"),
            "-o", obj], obj))
    for src in CUDA_SOURCES + HOST_SOURCES:
        obj = os.path.join(OBJ, src + ".o")
        cmd = [nvcc] + COMMON + ["-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu"):
            cmd[1:1] = ARCH + ["-lineinfo"]
        else:
            cmd[1:1] = ["-x", "cu"] + ARCH
        jobs.append((src, cmd, obj))
    # longest jobs first, at most one per core; up-to-date objects are kept
    pending = []
    for label, cmd, obj in jobs:
        src = cmd[cmd.index("-c") + 1]
        dg = job_digest(cmd, src)
        st = obj + ".stamp"
        if not force and os.path.exists(obj) and os.path.exists(st):
            with open(st) as fh:
                if fh.read().strip() == dg:
                    continue
        if os.path.exists(st):
            os.remove(st)
        pending.append((label, cmd, obj, st, dg))
    running, failed = [], []
    width = max(1, os.cpu_count() or 1)
    while pending or running:
        while pending and len(running) < width:
            label, cmd, _, st, dg = pending.pop(0)
            if verbose:
                print(" ".join(cmd))
            running.append((label, subprocess.Popen(cmd), st, dg))
        label, p, st, dg = running.pop(0)
        if p.wait() != 0:
            failed.append(label)
        else:
            with open(st, "w") as fh:
                fh.write(dg)
    if failed:
        raise RuntimeError("nvcc failed for " + ", ".join(failed))
    objs = [j[2] for j in jobs]
    link = [nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
    subprocess.check_call(link)
    with open(stamp, "w") as fh:
        fh.write(dig)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
