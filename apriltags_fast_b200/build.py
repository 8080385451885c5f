"""Build libapriltag_b200.so in-tree with nvcc for sm_100a.

    python -m apriltags_fast_b200.build [--force]

The built-in tag families come from csrc/families.bin (committed data),
turned into a C source under _build/ by csrc/gen_families.py.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libapriltag_b200.so")
SYNTH_JPEG_LIB = os.path.join(PKG, "libsynthjpeg.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# every floating point operation rounded on its own, as the reference
# (built with -ffp-contract=off) rounds it
FP = ["--fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
CUFLAGS = ARCH + FP + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                       "-I", os.path.join(ROOT, "include"), "-I", CSRC]
SOURCES = ["at_kernels.cu", "at_cluster.cu", "at_order.cu", "at_detector.cu", "at_noalloc.cu", "at_server.cu", "at_pose.cu", "at_jpeg.cu"]
C_SOURCES = ["at_upstream.c"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in ("at_gpu.h", "at_kernels.h", "at_device.cuh")] + [
        os.path.join(ROOT, "include", "apriltag_fast.h")]
    objs = []
    fam_c = os.path.join(BUILD, "at_families_data.c")
    fam_bin = os.path.join(CSRC, "families.bin")
    if force or _newer(fam_c, [fam_bin, os.path.join(CSRC, "gen_families.py")]):
        _run([sys.executable, os.path.join(CSRC, "gen_families.py"), "csource", fam_c])
    fam_o = os.path.join(BUILD, "at_families_data.o")
    if force or _newer(fam_o, [fam_c]):
        _run(["gcc", "-O1", "-fPIC", "-I", os.path.join(ROOT, "include"), "-c", fam_c, "-o", fam_o])
    objs.append(fam_o)
    # the upstream API shim (plain C over the native API)
    for src in C_SOURCES:
        c = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".c", ".o"))
        if force or _newer(o, [c] + [os.path.join(ROOT, "include", "apriltag.h"), os.path.join(ROOT, "include", "apriltag_fast.h")]):
            _run(["gcc", "-O2", "-fPIC", "-std=gnu11", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
                  "-c", c, "-o", o])
        objs.append(o)
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        if force or _newer(o, [s] + headers):
            _run([NVCC] + CUFLAGS + ["-c", s, "-o", o])
        objs.append(o)
    if force or _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lm"])
    # the synthetic-input JPEG encoder (bench and tests; not the detector)
    sj = os.path.join(CSRC, "synth_jpeg.c")
    if force or _newer(SYNTH_JPEG_LIB, [sj]):
        _run(["gcc", "-O2", "-fPIC", "-std=gnu11", "-shared", "-o", SYNTH_JPEG_LIB, sj, "-lm"])
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.force))
