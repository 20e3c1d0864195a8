"""Builds the native core in-tree: lightmetrica_b200/_lib/liblmgpu.so.

CUDA sources are compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a); the host BVH builder is compiled by
the system g++ with -ffp-contract=off so that its float arithmetic rounds
each operation separately, like the reference's float SSE build. Device code
is compiled with --fmad=false for the same reason: no multiply-add is fused
behind the source's back, so a kernel instantiated in two contexts (one
scene, a scene batch) computes every path bit for bit the same. Plain `/`
and sqrtf compile to the approximate forms (-prec-div=false
-prec-sqrt=false; deterministic, so the contexts still agree): the shading,
camera and light code renders the reference's expected image, not its
bits, and the exact intersection path spells every operation with an
explicit round-to-nearest intrinsic (__fdiv_rn, __frcp_rn, ...), which
these flags do not touch. Measured: the adjoint pair 15.5 / 27.3 ms ->
13.6 / 23.8 ms, the one-scene megakernel 1,883 -> 1,777 ms, the 1080p
frame 166.7 -> 165.1 ms.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OUT = os.path.join(OUT_DIR, "liblmgpu.so")
BUILD_DIR = os.path.join(HERE, "_build")

CU_SOURCES = ["api.cu", "pathtrace.cu", "adjoint.cu", "noalloc.cu", "batch.cu", "eval.cu"]
CPP_SOURCES = ["builder.cpp"]
HEADERS = ["layout.h", "builder.h", "internal.h", "scene.cuh", "trace.cuh", "trace4.cuh",
           "shading.cuh", "rng.cuh", "pathtrace.cuh", "trace_kernels.cuh", "pt_kernels.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(cuda, "bin", "nvcc")
    return p if os.path.exists(p) else (shutil.which("nvcc") or "nvcc")


def _cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


# Libraries built from the same sources: the product and the bounds-checked
# build (tree references checked at scene build, every wavefront queue
# append checked against its capacity; see LMGPU_BOUNDS_CHECK in
# csrc/scene.cuh). The host builder object is shared.
VARIANTS = [(OUT, BUILD_DIR, []),
            (os.path.join(OUT_DIR, "liblmgpu_check.so"), os.path.join(BUILD_DIR, "check"), ["-DLMGPU_BOUNDS_CHECK=1"])]
CHECK_OUT = VARIANTS[1][0]


def build(verbose: bool = False, ptxas_verbose: bool = False) -> str:
    """Compiles what is stale and links both libraries; returns the product's path."""
    os.makedirs(OUT_DIR, exist_ok=True)
    # This file's flags are a dependency of every object too.
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(os.path.dirname(HERE), "include", "lmgpu.h"),
                                                       os.path.abspath(__file__)]
    procs = []
    host_objs = []
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD_DIR, src + ".o")
        os.makedirs(BUILD_DIR, exist_ok=True)
        host_objs.append(o)
        if _stale(o, [s] + hdrs):
            cmd = [_cxx(), "-O2", "-std=c++17", "-fPIC", "-pthread", "-ffp-contract=off", "-fno-fast-math",
                   "-c", s, "-o", o]
            procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    links = []
    for out, bdir, defs in VARIANTS:
        os.makedirs(bdir, exist_ok=True)
        objs = []
        for src in CU_SOURCES:
            s = os.path.join(CSRC, src)
            if not os.path.exists(s):
                continue
            o = os.path.join(bdir, src + ".o")
            objs.append(o)
            if _stale(o, [s] + hdrs):
                cmd = [_nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                       "-Xcompiler", "-ffp-contract=off", "--fmad=false", "-prec-div=false", "-prec-sqrt=false",
                       "--expt-relaxed-constexpr", *defs,
                       "-ccbin", _cxx(), "-c", s, "-o", o]
                if ptxas_verbose and not defs:
                    cmd.insert(1, "-Xptxas=-v")
                procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        links.append((out, objs + host_objs))
    for cmd, p in procs:
        out, _ = p.communicate()
        if verbose or ptxas_verbose or p.returncode != 0:
            sys.stdout.write(out)
        if p.returncode != 0:
            raise RuntimeError("compile failed: " + " ".join(cmd))
    for out, objs in links:
        if _stale(out, objs):
            cmd = [_nvcc(), *ARCH, "-shared", "-ccbin", _cxx(), "-o", out, *objs, "-Xcompiler", "-pthread"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                sys.stdout.write(r.stdout + r.stderr)
                raise RuntimeError("link failed: " + out)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, ptxas_verbose="-v" in sys.argv))
