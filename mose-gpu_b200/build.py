"""Builds the engine's shared library in-tree: mose-gpu_b200/mosegpu/libmose_b200.so (sm_100a).

  mb_f64.cu, mb_api.cu   --fmad=false  (the FP64 form rounds statement by statement as written)
  mb_f32.cu              --fmad=true   (the mixed form: FP32 flux arithmetic with FMA)

Usage: python mose-gpu_b200/build.py [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "mosegpu", "libmose_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo", "-Xptxas", "-v"]
UNITS = [("mb_f64.cu", ["--fmad=false"]), ("mb_f32.cu", ["--fmad=true"]), ("mb_api.cu", ["--fmad=false"]),
         ("mb_noalloc.cu", ["--fmad=false"])]
DEPS = ["mb_physics.cuh", "mb_engine.cuh", "mb_launch.h", os.path.join("..", "..", "include", "mose_b200.h")]


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    dep_t = max(_mtime(os.path.join(CSRC, d)) for d in DEPS)
    objs = []
    logs = []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _mtime(o) < max(_mtime(s), dep_t):
            cmd = [NVCC] + ARCH + COMMON + flags + ["-c", s, "-o", o]
            r = subprocess.run(cmd, capture_output=True, text=True)
            logs.append(r.stderr)
            if r.returncode != 0:
                sys.stderr.write(r.stderr)
                raise RuntimeError("nvcc failed on %s" % src)
    if force or _mtime(OUT) < max(_mtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", OUT] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stderr)
            raise RuntimeError("link failed")
    if verbose:
        for l in logs:
            sys.stdout.write(l)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
