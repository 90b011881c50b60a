"""In-tree build of the native libraries.

    python -m ucns3d_b200.build

* ``ucns3d_b200/lib/libucns3d_gpu.so``  - CUDA engine, sm_100a (nvcc)
* ``ucns3d_b200/lib/libucns3d_prep.so`` - host set-up library (g++, OpenMP)

nvcc cross-compiles for sm_100a without a GPU.  The libraries are built
in-tree so that they travel with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "lib")
INC = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_prep(force=False):
    src = os.path.join(PKG, "csrc", "prep", "prep.cpp")
    out = os.path.join(LIB, "libucns3d_prep.so")
    deps = [src, os.path.join(INC, "ucns3d_prep.h"), os.path.join(INC, "ucns3d_gpu.h"),
            os.path.join(PKG, "csrc", "common", "rules.h")]
    if force or _stale(out, deps):
        os.makedirs(LIB, exist_ok=True)
        # the system g++ (the environment's CXX wrapper has no OpenMP runtime);
        # no contracted multiply-adds, like the device set-up (setup.cu), so
        # both give the same tables bit for bit
        _run(["g++", "-O3", "-march=x86-64-v2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
              "-I", INC, src, "-o", out])
    return out


# translation units of the engine, compiled in parallel and linked together;
# the reconstruction kernels are split by precision and order because the
# IORDER 4 instantiations dominate the compile time
ENGINE_TUS = ("recon_char_p4.cu", "recon_f64_p4.cu", "recon_f32_p4.cu", "recon_char.cu", "recon_f64.cu", "recon_f32.cu",
              "adjoint_weno.cu", "adjoint.cu", "engine.cu", "static_scratch.cu", "setup.cu", "implicit.cu",
              "halo.cu")
ENGINE_HDRS = ("kernels.cuh", "recon2.cuh", "device.cuh", "ad.cuh", "engine_internal.h", "expand.cuh", "../common/rules.h")
# per-unit flags: the device set-up evaluates the host set-up's operations
# one by one (no fused multiply-adds), so its tables match bit for bit
ENGINE_TU_FLAGS = {"setup.cu": ["-fmad=false"]}


def build_engine(force=False, extra=()):
    d = os.path.join(PKG, "csrc", "engine")
    srcs = [os.path.join(d, f) for f in ENGINE_TUS + ENGINE_HDRS]
    srcs.append(os.path.join(INC, "ucns3d_gpu.h"))
    out = os.path.join(LIB, "libucns3d_gpu.so")
    if force or _stale(out, srcs):
        os.makedirs(LIB, exist_ok=True)
        objdir = os.path.join(PKG, "_build")
        os.makedirs(objdir, exist_ok=True)
        procs, objs = [], []
        for tu in ENGINE_TUS:
            obj = os.path.join(objdir, tu.replace(".cu", ".o"))
            cmd = [NVCC, *GENCODE, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INC, *extra,
                   *ENGINE_TU_FLAGS.get(tu, []), "-c", os.path.join(d, tu), "-o", obj]
            print(" ".join(cmd), flush=True)
            procs.append((subprocess.Popen(cmd), cmd))
            objs.append(obj)
        failed = None
        for proc, cmd in procs:
            if proc.wait() != 0 and failed is None:
                failed = subprocess.CalledProcessError(proc.returncode, cmd)
        if failed is not None:
            raise failed
        _run([NVCC, *GENCODE, "-shared", *objs, "-o", out])
    return out


def build_all(force=False):
    return build_prep(force), build_engine(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
