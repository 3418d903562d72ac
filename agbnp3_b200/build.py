"""Builds the in-tree shared libraries of the package:

- libagbnp3_b200.so : the engine (C host layer + sm_100a CUDA kernels)
- libagbnp3_b200_sp.so : the same engine with the reference's float interface
  (its entry points built with SINGLE_PREC_INTERFACE: float_i = float)
- libagbnp3_globule.so : the seeded synthetic-globule generator

Usage: python -m agbnp3_b200.build  (or __graft_entry__.build()).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libagbnp3_b200.so")
LIB_SP = os.path.join(HERE, "libagbnp3_b200_sp.so")
GLOBULE = os.path.join(HERE, "libagbnp3_globule.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SRC = ["agbnp3_dev.cu", "agbnp3_prim.cu", "agbnp3_static.cu", "agbnp3_peaks.cu", "agbnp3_mlp.cu"]
C_SRC = ["agbnp3_host.c", "nblist.c"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} (rc={r.returncode})")
    return r.stdout + r.stderr


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hdrs += [os.path.join(INC, f) for f in os.listdir(INC)]
    objs = []
    log = []
    for f in CUDA_SRC:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            log.append(_run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xptxas", "-v", "-Xcompiler", "-fPIC",
                             "-I", CSRC, "-I", INC, "-c", src, "-o", obj]))
    for f in C_SRC:
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            log.append(_run(["gcc", "-O2", "-fPIC", "-std=c11", "-Wall", "-I", CSRC, "-I", INC,
                             "-I", "/usr/local/cuda/include", "-c", src, "-o", obj]))
    if force or _stale(LIB, objs):
        log.append(_run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs, "-ldl"]))
    # the float-interface library: the host layer again with float_i = float
    src = os.path.join(CSRC, "agbnp3_host.c")
    obj_sp = os.path.join(BUILD, "agbnp3_host_sp.c.o")
    if force or _stale(obj_sp, [src] + hdrs):
        log.append(_run(["gcc", "-O2", "-fPIC", "-std=c11", "-Wall", "-DSINGLE_PREC_INTERFACE", "-I", CSRC, "-I", INC,
                         "-I", "/usr/local/cuda/include", "-c", src, "-o", obj_sp]))
    objs_sp = [obj_sp if o.endswith("agbnp3_host.c.o") else o for o in objs]
    if force or _stale(LIB_SP, objs_sp):
        log.append(_run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB_SP, *objs_sp, "-ldl"]))
    gsrc = os.path.join(CSRC, "globule.c")
    if force or _stale(GLOBULE, [gsrc]):
        log.append(_run(["gcc", "-O2", "-shared", "-fPIC", "-o", GLOBULE, gsrc, "-lm"]))
    if verbose:
        print("\n".join(x for x in log if x.strip()))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
