"""Build libjurassic_b200.so: C host code (gcc) + CUDA kernels for sm_100a
(nvcc), linked into one shared library under lib/.

    python build.py [--force]

The library exports the drop-in formod()/brightness()/planck() and the
jsc_* C-ABI declared in include/jurassic_b200.h.  Device code is compiled
with --fmad=false: no multiply-add contraction, so floating-point results
follow the reference's operation order.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib")
OBJ = os.path.join(OUT, "obj")
LIB = os.path.join(OUT, "libjurassic_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

C_SRCS = ["model_host.c", "formod.c", "optprop.c", "compat.c"]
CU_SRCS = ["model_dev.cu", "batch.cu", "ega_g2.cu", "ega_g4.cu", "ega_g8.cu",
           "ega_gmax.cu", "ega_lane_s.cu", "ega_lane_l.cu", "ega_ray.cu", "noalloc.cu", "surrogate.cu",
           "surrogate_tc.cu", "mie.cu"]
HEADERS = ["jsc_internal.h", "physics.h", "ckd_tables.h", "jsc_model.h",
           "cuda_util.cuh", "device_common.cuh", "kernels.cuh", "ega_kernel.cuh",
           "ega_lane.cuh", "scatter.cuh", "surrogate.h", "surrogate_tc.h"]

INC = ["-I" + os.path.join(REPO, "include"), "-I" + CSRC]
CFLAGS = ["-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-std=gnu11",
          "-Wall", "-Wextra", "-Wno-unused-parameter"]
NVFLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
           "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
           "-Xptxas", "-v"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, log=None):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        with open(log, "w") as f:
            f.write(res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
        raise RuntimeError("build step failed: %s" % cmd[0])


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    hdrs.append(os.path.join(REPO, "include", "jurassic_b200.h"))
    objs = []
    jobs = []
    for s in C_SRCS:
        src = os.path.join(CSRC, s)
        o = os.path.join(OBJ, s + ".o")
        if force or _newer(o, [src] + hdrs):
            jobs.append((["gcc"] + CFLAGS + INC + ["-c", src, "-o", o], None))
        objs.append(o)
    for s in CU_SRCS:
        src = os.path.join(CSRC, s)
        o = os.path.join(OBJ, s + ".o")
        if force or _newer(o, [src] + hdrs):
            jobs.append(([NVCC] + NVFLAGS + INC + ["-c", src, "-o", o],
                         os.path.join(OBJ, s + ".ptxas.txt")))
        objs.append(o)
    # the translation units compile independently: run them in parallel
    with cf.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        for f in [ex.submit(_run, cmd, log) for cmd, log in jobs]:
            f.result()
    if force or _newer(LIB, objs):
        _run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
              "-o", LIB] + objs + ["-Xcompiler", "-fopenmp", "-lgomp",
                                   "-lpthread", "-lm"])
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(force=a.force, verbose=True)
