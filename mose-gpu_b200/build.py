"""Builds the engine's shared library in-tree: mose-gpu_b200/mosegpu/libmose_b200.so (sm_100a).

  mb_f64.cu, mb_irs.cu, mb_prec.cu, mb_api.cu, mb_noalloc.cu, mb_sweep_f64_*.cu   --fmad=false
      (the FP64 form rounds statement by statement as written)
  mb_sweep_f64f_*.cu  --fmad=true
      (the FP64 production form: FMA contraction; FP64 division and square root stay IEEE)
  mb_sweep_f32_*.cu   --fmad=true -prec-div=false -prec-sqrt=false -ftz=true
      (the mixed form: FP32 flux arithmetic with FMA and the fast FP32 divide / square root; the FP64 state
       arithmetic in those units is unaffected by these single-precision options)

Units compile in parallel. Usage: python mose-gpu_b200/build.py [--force] [-v]
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "mosegpu", "libmose_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo", "-Xptxas", "-v"]
F64 = ["--fmad=false"]
F64F = ["--fmad=true"]
F32 = ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
UNITS = [("mb_f64.cu", F64), ("mb_irs.cu", F64), ("mb_prec.cu", F64), ("mb_api.cu", F64), ("mb_noalloc.cu", F64)] + \
        [("mb_sweep_f64_rs%d.cu" % r, F64) for r in (0, 1, 4, 12)] + \
        [("mb_sweep_f64f_rs%d.cu" % r, F64F) for r in (0, 1, 4, 12)] + \
        [("mb_sweep_f32_rs%d.cu" % r, F32) for r in (0, 1, 4, 12)]
DEPS = ["mb_physics.cuh", "mb_engine.cuh", "mb_launch.h", "mb_sweep_inst.inc",
        os.path.join("..", "..", "include", "mose_b200.h")]


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    dep_t = max(_mtime(os.path.join(CSRC, d)) for d in DEPS)
    jobs = []
    objs = []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _mtime(o) < max(_mtime(s), dep_t):
            jobs.append((src, [NVCC] + ARCH + COMMON + flags + ["-c", s, "-o", o]))

    def run(job):
        src, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, r

    logs = []
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        for src, r in ex.map(run, jobs):
            logs.append((src, r.stderr))
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
        for src, l in logs:
            sys.stdout.write("== %s\n%s" % (src, l))
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
