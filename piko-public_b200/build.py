"""Builds libpiko_b200.so in-tree with nvcc for sm_100a.

    python piko-public_b200/build.py [-v]

Every device file is compiled with --fmad=false: the raster and Reyes stages
must reproduce the reference CPU backend's individually rounded float
operations bit for bit, so no multiply-add may be contracted.  Division and
square root keep their IEEE defaults (no fast-math flags).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libpiko_b200.so")
SOURCES = ["csrc/runtime.cu", "csrc/raster_kernels.cu", "csrc/reyes_kernels.cu", "csrc/server.cu", "csrc/tuner.cu",
           "csrc/assets.cpp", "csrc/noalloc.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "-I", os.path.join(ROOT, "include"),
]


def sources():
    return [os.path.join(HERE, s) for s in SOURCES if os.path.exists(os.path.join(HERE, s))]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))]
    deps.append(os.path.join(ROOT, "include", "piko_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


SAMPLES_LIB = os.path.join(HERE, "libpiko_stage_samples.so")
SAMPLES_SRC = os.path.join(HERE, "samples", "stage_samples.cu")


def build_samples(verbose=False, force=False):
    """The stage-API sample pipelines (samples/stage_samples.cu against
    include/piko_stage.cuh)."""
    deps = [SAMPLES_SRC, os.path.join(ROOT, "include", "piko_stage.cuh")]
    if not force and os.path.exists(SAMPLES_LIB) and all(os.path.getmtime(d) <= os.path.getmtime(SAMPLES_LIB)
                                                         for d in deps):
        return SAMPLES_LIB
    cmd = [NVCC] + FLAGS + ["-o", SAMPLES_LIB + ".tmp", SAMPLES_SRC]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(SAMPLES_LIB + ".tmp", SAMPLES_LIB)
    return SAMPLES_LIB


def build(verbose=False, force=False, extra=()):
    if not force and not needs_build():
        return LIB
    cmd = [NVCC] + FLAGS + list(extra) + ["-o", LIB + ".tmp"] + sources()
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(verbose=v, force=True, extra=extra))
    print(build_samples(verbose=v, force=True))
